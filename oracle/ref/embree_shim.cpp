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
// (embreeaccel.h:182-220) accept every hit. User geometries (phong
// tessellation, analytic cubes and planes) are out of scope and rejected.

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
};

struct ShimScene {
    std::vector<ShimGeometry *> geoms;
    oracle::RayCaster rc;
};

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
    if (sg->type != RTC_GEOMETRY_TYPE_TRIANGLE) shim_fail("user geometry");
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
void rtcSetGeometryUserData(RTCGeometry, void *) {}
void rtcSetGeometryIntersectFilterFunction(RTCGeometry, RTCFilterFunctionN) {}
void rtcSetGeometryOccludedFilterFunction(RTCGeometry, RTCFilterFunctionN) {}
void rtcSetGeometryUserPrimitiveCount(RTCGeometry, unsigned int) { shim_fail("rtcSetGeometryUserPrimitiveCount"); }
void rtcSetGeometryBoundsFunction(RTCGeometry, RTCBoundsFunction, void *) { shim_fail("rtcSetGeometryBoundsFunction"); }
void rtcSetGeometryIntersectFunction(RTCGeometry, RTCIntersectFunctionN) { shim_fail("rtcSetGeometryIntersectFunction"); }
void rtcSetGeometryOccludedFunction(RTCGeometry, RTCOccludedFunctionN) { shim_fail("rtcSetGeometryOccludedFunction"); }
void rtcFilterIntersection(const RTCIntersectFunctionNArguments *, const RTCFilterFunctionNArguments *) { shim_fail("rtcFilterIntersection"); }
void rtcFilterOcclusion(const RTCOccludedFunctionNArguments *, const RTCFilterFunctionNArguments *) { shim_fail("rtcFilterOcclusion"); }
void rtcCommitGeometry(RTCGeometry) {}

void rtcReleaseGeometry(RTCGeometry g) {
    ShimGeometry *sg = reinterpret_cast<ShimGeometry *>(g);
    if (--sg->refs == 0) delete sg;
}

void rtcCommitScene(RTCScene s) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    sc->rc = oracle::RayCaster();
    for (ShimGeometry *g : sc->geoms) {
        std::vector<int> tri(g->indices.begin(), g->indices.end());
        sc->rc.add_mesh(g->vertices.data(), tri.data(), int(tri.size() / 3), int(g->geom_id));
    }
    sc->rc.build();
}

void rtcGetSceneBounds(RTCScene s, struct RTCBounds *b) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
    b->lower_x = sc->rc.scene_lo[0]; b->lower_y = sc->rc.scene_lo[1]; b->lower_z = sc->rc.scene_lo[2];
    b->upper_x = sc->rc.scene_hi[0]; b->upper_y = sc->rc.scene_hi[1]; b->upper_z = sc->rc.scene_hi[2];
    b->align0 = b->align1 = 0.f;
}

void rtcIntersect1(RTCScene s, struct RTCIntersectContext *, struct RTCRayHit *rh) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
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

void rtcOccluded1(RTCScene s, struct RTCIntersectContext *, struct RTCRay *r) {
    ShimScene *sc = reinterpret_cast<ShimScene *>(s);
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
