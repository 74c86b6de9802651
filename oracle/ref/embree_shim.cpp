// Test infrastructure only: stands in for the Embree 3.5.2 library when the
// reference's own renderer code is compiled for the oracle (oracle/_ref).
//
// Embree's sources are vendored with the reference but need cmake and
// generated configuration to build, so the library is not built here. The
// reference's EmbreeAccel (src/accel/embreeaccel.h) is compiled unchanged
// against Embree's public headers (dependencies/embree/include/embree3), and
// this file implements the subset of that C API it calls, answering the ray
// queries with the oracle's restatement of Embree's triangle test
// (oracle/oracle_raycast.h). Alpha filter callbacks are not invoked: the
// scenes carry no alpha textures, for which the reference's filters
// (embreeaccel.h:182-220) accept every hit.
//
// User geometries (RTC_GEOMETRY_TYPE_USER; the reference's Phong tessellation
// patches, embreeaccel.h:242-257) are supported as Embree 3 runs them: the
// bounds callback is asked once per primitive at commit, the boxes go into the
// caster's user-primitive BVH, and a ray that reaches a primitive's box calls the
// geometry's intersect (occluded) callback with the ray's current tfar, through
// the same argument structs Embree passes. rtcFilterIntersection /
// rtcFilterOcclusion do nothing: the reference sets no filter on user geometry.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "embree3/rtcore.h"
#include "../oracle_raycast.h"

struct ShimGeometry {
    RTCGeometryType type;
    std::vector<float> vertices;     // float3 per vertex (stride may be larger in Embree; here 12)
    std::vector<unsigned> indices;   // uint3 per triangle
    std::vector<float> attribs;      // float2 texture coordinates
    unsigned geom_id = RTC_INVALID_GEOMETRY_ID;
    int refs = 1;
    // user geometry
    void *user_data = nullptr;
    unsigned prim_count = 0;
    RTCBoundsFunction bounds = nullptr;
    RTCIntersectFunctionN intersect = nullptr;
    RTCOccludedFunctionN occluded = nullptr;
};

struct ShimScene {
    std::vector<ShimGeometry *> geoms;
    oracle::RayCaster rc;
};

// the context of the query in flight on this thread (the callbacks read it)
static thread_local RTCIntersectContext *g_context = nullptr;

struct ShimDevice { RTCErrorFunction err = nullptr; void *user = nullptr; };

static void shim_fail(const char *what) {
    fprintf(stderr, "embree shim: unsupported call %s\n", what);
    abort();
}

extern "C" {

RTCDevice rtcNewDevice(const char *) { return reinterpret_cast<RTCDevice>(new ShimDevice()); }

void rtcSetDeviceErrorFunction(RTCDevice d, RTCErrorFunction f, void *u) {
    reinterpret_cast<ShimDevice *>(d)->err = f;
    reinterpret_cast<ShimDevice *>(d)->user = u;
}

RTCScene rtcNewScene(RTCDevice) { return reinterpret_cast<RTCScene>(new ShimScene()); }

RTCGeometry rtcNewGeometry(RTCDevice, enum RTCGeometryType type) {
    if (type != RTC_GEOMETRY_TYPE_TRIANGLE && type != RTC_GEOMETRY_TYPE_USER) shim_fail("rtcNewGeometry(type)");
    ShimGeometry *g = new ShimGeometry();
    g->type = type;
    return reinterpret_cast<RTCGeometry>(g);
}

unsigned int rtcAttachGeometry(RTCScene s, RTCGeometry g) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    ShimGeometry *sg = reinterpret_cast<ShimGeometry *>(g);
    sg->geom_id = unsigned(sc->geoms.size());
    sg->refs++;
    sc->geoms.push_back(sg);
    return sg->geom_id;
}

RTCGeometry rtcGetGeometry(RTCScene s, unsigned int id) {
    return reinterpret_cast<RTCGeometry>(reinterpret_cast<ShimScene *>(s)->geoms.at(id));
}

void *rtcSetNewGeometryBuffer(RTCGeometry g, enum RTCBufferType type, unsigned int slot, enum RTCFormat format,
                              size_t byteStride, size_t itemCount) {
    ShimGeometry *sg = reinterpret_cast<ShimGeometry *>(g);
    if (slot != 0) shim_fail("buffer slot");
    if (type == RTC_BUFFER_TYPE_VERTEX && format == RTC_FORMAT_FLOAT3 && byteStride == 12) {
        sg->vertices.assign(itemCount * 3 + 1, 0.f);   // Embree asks for readable padding past the end
        return sg->vertices.data();
    }
    if (type == RTC_BUFFER_TYPE_INDEX && format == RTC_FORMAT_UINT3 && byteStride == 12) {
        sg->indices.assign(itemCount * 3, 0u);
        return sg->indices.data();
    }
    if (type == RTC_BUFFER_TYPE_VERTEX_ATTRIBUTE && format == RTC_FORMAT_FLOAT2 && byteStride == 8) {
        sg->attribs.assign(itemCount * 2 + 2, 0.f);
        return sg->attribs.data();
    }
    shim_fail("rtcSetNewGeometryBuffer(type/format)");
    return nullptr;
}

void rtcSetGeometryVertexAttributeCount(RTCGeometry, unsigned int) {}
void rtcSetGeometryUserData(RTCGeometry g, void *ptr) { reinterpret_cast<ShimGeometry *>(g)->user_data = ptr; }
void rtcSetGeometryIntersectFilterFunction(RTCGeometry, RTCFilterFunctionN) {}
void rtcSetGeometryOccludedFilterFunction(RTCGeometry, RTCFilterFunctionN) {}
void rtcSetGeometryUserPrimitiveCount(RTCGeometry g, unsigned int n) {
    ShimGeometry *sg = reinterpret_cast<ShimGeometry *>(g);
    if (sg->type != RTC_GEOMETRY_TYPE_USER) shim_fail("rtcSetGeometryUserPrimitiveCount on a non-user geometry");
    sg->prim_count = n;
}
void rtcSetGeometryBoundsFunction(RTCGeometry g, RTCBoundsFunction f, void *) { reinterpret_cast<ShimGeometry *>(g)->bounds = f; }
void rtcSetGeometryIntersectFunction(RTCGeometry g, RTCIntersectFunctionN f) { reinterpret_cast<ShimGeometry *>(g)->intersect = f; }
void rtcSetGeometryOccludedFunction(RTCGeometry g, RTCOccludedFunctionN f) { reinterpret_cast<ShimGeometry *>(g)->occluded = f; }
void rtcFilterIntersection(const RTCIntersectFunctionNArguments *, const RTCFilterFunctionNArguments *) {}
void rtcFilterOcclusion(const RTCOccludedFunctionNArguments *, const RTCFilterFunctionNArguments *) {}
void rtcCommitGeometry(RTCGeometry) {}

void rtcReleaseGeometry(RTCGeometry g) {
    ShimGeometry *sg = reinterpret_cast<ShimGeometry *>(g);
    if (--sg->refs == 0) delete sg;
}

void rtcCommitScene(RTCScene s) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    sc->rc = oracle::RayCaster();
    for (ShimGeometry *g : sc->geoms) {
        if (g->type == RTC_GEOMETRY_TYPE_USER) {
            if (!g->bounds || !g->intersect || !g->occluded) shim_fail("user geometry without callbacks");
            for (unsigned p = 0; p < g->prim_count; ++p) {
                RTCBounds b;
                RTCBoundsFunctionArguments a;
                a.geometryUserPtr = g->user_data;
                a.primID = p;
                a.timeStep = 0;
                a.bounds_o = &b;
                g->bounds(&a);
                oracle::RcUser u;
                u.lo[0] = b.lower_x; u.lo[1] = b.lower_y; u.lo[2] = b.lower_z;
                u.hi[0] = b.upper_x; u.hi[1] = b.upper_y; u.hi[2] = b.upper_z;
                u.geom = int(g->geom_id);
                u.prim = int(p);
                u.ref = int(g->geom_id);
                sc->rc.add_user(u);
            }
            continue;
        }
        std::vector<int> tri(g->indices.begin(), g->indices.end());
        sc->rc.add_mesh(g->vertices.data(), tri.data(), int(tri.size() / 3), int(g->geom_id));
    }
    sc->rc.user_closest = [sc](const oracle::RcUser &u, const float o[3], const float d[3], float tnear, float tfar,
                               oracle::RcHit *h) {
        ShimGeometry *g = sc->geoms[size_t(u.ref)];
        RTCRayHit rh;
        rh.ray.org_x = o[0]; rh.ray.org_y = o[1]; rh.ray.org_z = o[2];
        rh.ray.dir_x = d[0]; rh.ray.dir_y = d[1]; rh.ray.dir_z = d[2];
        rh.ray.tnear = tnear; rh.ray.tfar = tfar;
        rh.ray.time = 0.f; rh.ray.mask = ~0u; rh.ray.id = 0; rh.ray.flags = 0;
        rh.hit.geomID = RTC_INVALID_GEOMETRY_ID;
        rh.hit.primID = RTC_INVALID_GEOMETRY_ID;
        int valid = -1;
        RTCIntersectFunctionNArguments a;
        a.valid = &valid;
        a.geometryUserPtr = g->user_data;
        a.primID = unsigned(u.prim);
        a.context = g_context;
        a.rayhit = reinterpret_cast<RTCRayHitN *>(&rh);
        a.N = 1;
        g->intersect(&a);
        if (rh.hit.geomID == RTC_INVALID_GEOMETRY_ID) return false;
        h->t = rh.ray.tfar;
        h->u = rh.hit.u; h->v = rh.hit.v;
        h->ng[0] = rh.hit.Ng_x; h->ng[1] = rh.hit.Ng_y; h->ng[2] = rh.hit.Ng_z;
        h->geom = int(rh.hit.geomID);
        h->prim = int(rh.hit.primID);
        return true;
    };
    sc->rc.user_any = [sc](const oracle::RcUser &u, const float o[3], const float d[3], float tnear, float tfar) {
        ShimGeometry *g = sc->geoms[size_t(u.ref)];
        RTCRay r;
        r.org_x = o[0]; r.org_y = o[1]; r.org_z = o[2];
        r.dir_x = d[0]; r.dir_y = d[1]; r.dir_z = d[2];
        r.tnear = tnear; r.tfar = tfar;
        r.time = 0.f; r.mask = ~0u; r.id = 0; r.flags = 0;
        int valid = -1;
        RTCOccludedFunctionNArguments a;
        a.valid = &valid;
        a.geometryUserPtr = g->user_data;
        a.primID = unsigned(u.prim);
        a.context = g_context;
        a.ray = reinterpret_cast<RTCRayN *>(&r);
        a.N = 1;
        g->occluded(&a);
        return r.tfar == -INFINITY;
    };
    sc->rc.build();
}

void rtcGetSceneBounds(RTCScene s, struct RTCBounds *b) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    b->lower_x = sc->rc.scene_lo[0]; b->lower_y = sc->rc.scene_lo[1]; b->lower_z = sc->rc.scene_lo[2];
    b->upper_x = sc->rc.scene_hi[0]; b->upper_y = sc->rc.scene_hi[1]; b->upper_z = sc->rc.scene_hi[2];
    b->align0 = b->align1 = 0.f;
}

void rtcIntersect1(RTCScene s, struct RTCIntersectContext *ctx, struct RTCRayHit *rh) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    g_context = ctx;
    const float o[3] = {rh->ray.org_x, rh->ray.org_y, rh->ray.org_z};
    const float d[3] = {rh->ray.dir_x, rh->ray.dir_y, rh->ray.dir_z};
    oracle::RcHit h;
    if (sc->rc.closest(o, d, rh->ray.tnear, rh->ray.tfar, &h)) {
        rh->ray.tfar = h.t;
        rh->hit.geomID = unsigned(h.geom);
        rh->hit.primID = unsigned(h.prim);
        rh->hit.u = h.u; rh->hit.v = h.v;
        rh->hit.Ng_x = h.ng[0]; rh->hit.Ng_y = h.ng[1]; rh->hit.Ng_z = h.ng[2];
        rh->hit.instID[0] = RTC_INVALID_GEOMETRY_ID;
    }
}

void rtcOccluded1(RTCScene s, struct RTCIntersectContext *ctx, struct RTCRay *r) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    g_context = ctx;
    const float o[3] = {r->org_x, r->org_y, r->org_z};
    const float d[3] = {r->dir_x, r->dir_y, r->dir_z};
    if (sc->rc.occluded(o, d, r->tnear, r->tfar)) r->tfar = -INFINITY;
}

void rtcInterpolate(const struct RTCInterpolateArguments *a) {
    ShimGeometry *sg = reinterpret_cast<ShimGeometry *>(a->geometry);
    if (a->bufferType != RTC_BUFFER_TYPE_VERTEX_ATTRIBUTE || a->valueCount != 2) shim_fail("rtcInterpolate");
    const unsigned *t = &sg->indices[3 * size_t(a->primID)];
    for (unsigned k = 0; k < 2; ++k)
        a->P[k] = (1.f - a->u - a->v) * sg->attribs[2 * t[0] + k] + a->u * sg->attribs[2 * t[1] + k] +
                  a->v * sg->attribs[2 * t[2] + k];
}

}  // extern "C"
