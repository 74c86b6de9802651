// Ray / BVH traversal for the B200 renderer: closest hit (the query of
// EmbreeAccel::intersect, src/accel/embreeaccel.h:353-422) and any hit (the
// occlusion query of EmbreeAccel::isIntersect, :336-351).
//
// * Binary BVH, both child boxes of a node in one 64-byte record fetched as four
//   16-byte vector loads through the read-only path (__ldg).
// * Near-child-first descent; the far child is pushed on a per-ray stack whose
//   first kSmemStack entries live in shared memory (one column per thread, so a
//   warp's pushes hit 32 different banks) and whose rare deeper entries spill to
//   a small local array. The builder bounds the tree depth by kMaxStack.
// * Watertight ray/triangle test in FP32 (Woop, Benthin, Wald, "Watertight
//   Ray/Triangle Intersection", JCGT 2013): per-ray shear to a frame where the
//   ray is +z, 2-D edge functions evaluated without contraction so that the two
//   triangles sharing an edge see exactly opposite values, FP64 re-evaluation
//   when an edge function is exactly zero. Hits are accepted on (tmin, tmax] as
//   Embree's |den|*tnear < T <= |den|*tfar, with no back-face culling. The
//   barycentrics returned are Embree's (u, v) = weights of v1 and v2.
//
// Scenes with Phong tessellation patches use the PHONG instantiation: a leaf primitive whose
// record carries wrp::kPatchFlag is tested first against its own box, then with the FP64
// patch test of wr_phong.cuh; an accepted patch hit stores its unit normal, octahedrally
// encoded, in the two barycentric slots. Triangle-only scenes never compile that code in.
#pragma once

#include "wr_device.cuh"
#include "wr_phong.cuh"

namespace wrd {

struct RayPre {
    float ox, oy, oz;          // origin
    float ix, iy, iz;          // 1 / direction (finite)
    float oix, oiy, oiz;       // origin / direction
    int kx, ky, kz;            // watertight axis permutation
    float sx, sy, sz;          // shear constants
};

__device__ __forceinline__ float comp(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ RayPre ray_setup(f3 o, f3 d) {
    RayPre r;
    r.ox = o.x; r.oy = o.y; r.oz = o.z;
    const float eps = 1e-30f;
    const float dx = fabsf(d.x) > eps ? d.x : copysignf(eps, d.x);
    const float dy = fabsf(d.y) > eps ? d.y : copysignf(eps, d.y);
    const float dz = fabsf(d.z) > eps ? d.z : copysignf(eps, d.z);
    r.ix = 1.0f / dx; r.iy = 1.0f / dy; r.iz = 1.0f / dz;
    r.oix = o.x * r.ix; r.oiy = o.y * r.iy; r.oiz = o.z * r.iz;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    r.kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    r.kx = r.kz == 2 ? 0 : r.kz + 1;
    r.ky = r.kx == 2 ? 0 : r.kx + 1;
    if (comp(d, r.kz) < 0.f) { int t = r.kx; r.kx = r.ky; r.ky = t; }
    const float dkz = comp(d, r.kz);
    r.sx = comp(d, r.kx) / dkz;
    r.sy = comp(d, r.ky) / dkz;
    r.sz = 1.0f / dkz;
    return r;
}

// slab test of one child box; returns entry distance, or +inf when missed
__device__ __forceinline__ float box_entry(const RayPre &r, float lox, float hix, float loy, float hiy, float loz,
                                           float hiz, float tmin, float tmax) {
    const float t0x = fmaf(lox, r.ix, -r.oix), t1x = fmaf(hix, r.ix, -r.oix);
    const float t0y = fmaf(loy, r.iy, -r.oiy), t1y = fmaf(hiy, r.iy, -r.oiy);
    const float t0z = fmaf(loz, r.iz, -r.oiz), t1z = fmaf(hiz, r.iz, -r.oiz);
    const float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), tmin));
    const float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), tmax));
    // 1 + 2*gamma(3) widening keeps the slab test conservative (Ize 2013)
    return tn <= tf * 1.00000024f ? tn : __int_as_float(0x7f800000);
}

// watertight test; on hit writes t and Embree-style barycentrics (u, v)
__device__ __forceinline__ bool tri_test(const RayPre &r, float4 a, float4 b, float4 c, float tmin, float tmax,
                                         float &t_out, float &u_out, float &v_out) {
    const f3 A0 = mk(a.x - r.ox, a.y - r.oy, a.z - r.oz);
    const f3 B0 = mk(b.x - r.ox, b.y - r.oy, b.z - r.oz);
    const f3 C0 = mk(c.x - r.ox, c.y - r.oy, c.z - r.oz);
    const float Akx = comp(A0, r.kx), Aky = comp(A0, r.ky), Akz = comp(A0, r.kz);
    const float Bkx = comp(B0, r.kx), Bky = comp(B0, r.ky), Bkz = comp(B0, r.kz);
    const float Ckx = comp(C0, r.kx), Cky = comp(C0, r.ky), Ckz = comp(C0, r.kz);
    const float Ax = Akx - r.sx * Akz, Ay = Aky - r.sy * Akz;
    const float Bx = Bkx - r.sx * Bkz, By = Bky - r.sy * Bkz;
    const float Cx = Ckx - r.sx * Ckz, Cy = Cky - r.sy * Ckz;
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.f || V == 0.f || W == 0.f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    const float det = U + V + W;
    if (det == 0.f) return false;
    const float Az = r.sz * Akz, Bz = r.sz * Bkz, Cz = r.sz * Ckz;
    const float T = U * Az + V * Bz + W * Cz;
    const float sgn = det < 0.f ? -1.f : 1.f;
    const float Ts = T * sgn, ad = det * sgn;
    if (!(Ts > tmin * ad && Ts <= tmax * ad)) return false;
    const float rcp = 1.0f / det;
    t_out = T * rcp;
    u_out = V * rcp;
    v_out = W * rcp;
    return true;
}

// the float ray as the patch test takes it (PHONG instantiations only)
struct PatchRay {
    float ox, oy, oz, dx, dy, dz;
};

// leaf primitive i is a patch: its own box, then the FP64 test against (tmin, t]; on a hit
// lowers t and stores the encoded normal in (bu, bv)
__device__ __forceinline__ bool patch_leaf_test(const RayPre &r, const PatchRay &pr, const double *patches, uint32_t i,
                                                float4 a, float4 b, float4 c, float tmin, float &t, float &bu,
                                                float &bv) {
    float lo[3], hi[3];
    wrp::load_patch_box(patches, i, lo, hi);
    if (box_entry(r, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], tmin, t) == __int_as_float(0x7f800000)) return false;
    const wrp::Patch<wrp::Rd> P = wrp::load_patch(patches, i, a, b, c);
    wrp::Rd tm = wrp::Rd(double(t));
    wrp::V<wrp::Rd> n;
    if (!wrp::patch_intersect(P, pr.ox, pr.oy, pr.oz, pr.dx, pr.dy, pr.dz, tmin, tm, n)) return false;
    const float2 e = wrp::oct_encode(float(n.x.v), float(n.y.v), float(n.z.v));
    t = float(tm.v);
    bu = e.x;
    bv = e.y;
    return true;
}

// unit geometry normal of a hit on leaf primitive (a, b, c): the triangle's face normal,
// or the patch normal the traversal stored (encoded) in the barycentric slots
__device__ __forceinline__ f3 surface_normal(float4 a, float4 b, float4 c, float bu, float bv) {
    if (__float_as_uint(a.w) & wrp::kPatchFlag) {
        const float3 n = wrp::oct_decode(bu, bv);
        return mk(n.x, n.y, n.z);
    }
    return normalize(cross(xyz(b) - xyz(a), xyz(c) - xyz(a)));
}

struct TraceStack {
    uint32_t *smem;   // kSmemStack x blockDim.x words, column = threadIdx.x
    int stride;
    int local[kMaxStack - kSmemStack];
    int sp;
    __device__ __forceinline__ void push(int v) {
        if (sp < kSmemStack) smem[sp * stride] = uint32_t(v);
        else local[sp - kSmemStack] = v;
        ++sp;
    }
    __device__ __forceinline__ int pop() {
        --sp;
        return sp < kSmemStack ? int(smem[sp * stride]) : local[sp - kSmemStack];
    }
};

// Traverses the BVH. ANY_HIT: returns at the first accepted hit.
// On return `t` holds the closest accepted distance; `tri` the leaf-order triangle (or MISS).
//
// Loop structure after Aila & Laine ("Understanding the Efficiency of Ray
// Traversal on GPUs", HPG 2009): inner nodes and leaves are handled in two
// separate loops, and a lane that reaches a leaf postpones it and keeps
// descending inner nodes until every converged lane of the warp holds a leaf,
// so that the triangle tests run with most lanes active. The warp vote only
// steers scheduling; each lane's result does not depend on other lanes.
template <bool ANY_HIT, bool PHONG = false>
__device__ __forceinline__ bool traverse(const float4 *__restrict__ nodes, const float4 *__restrict__ tris, f3 o,
                                         f3 d, float tmin, float tmax, uint32_t *smem_stack, float &t, uint32_t &tri,
                                         float &bu, float &bv, uint32_t *node_visits = nullptr,
                                         uint32_t *tri_tests = nullptr, const double *patches = nullptr) {
    constexpr int kDone = 0x7fffffff;   // traversal finished (stack empty)
    const RayPre r = ray_setup(o, d);
    const PatchRay pr{o.x, o.y, o.z, d.x, d.y, d.z};
    TraceStack st;
    st.smem = smem_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.sp = 0;
    tri = MISS;
    t = tmax;
    int node = 0;    // next inner node (>= 0), a leaf code (< 0) or kDone
    int leaf = 0;    // postponed leaf code (< 0), 0 when none
    uint32_t nv = 0, nt = 0;
    while (node != kDone) {
        while (node >= 0 && node != kDone) {
            const float4 n0 = __ldg(nodes + 4 * node + 0);
            const float4 n1 = __ldg(nodes + 4 * node + 1);
            const float4 n2 = __ldg(nodes + 4 * node + 2);
            const float4 n3 = __ldg(nodes + 4 * node + 3);
            ++nv;
            const float e0 = box_entry(r, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, tmin, t);
            const float e1 = box_entry(r, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, tmin, t);
            const int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            const bool h0 = e0 != __int_as_float(0x7f800000), h1 = e1 != __int_as_float(0x7f800000);
            if (h0 && h1) {
                int near = c0, far = c1;
                if (e1 < e0) { near = c1; far = c0; }
                st.push(far);
                node = near;
            } else if (h0) {
                node = c0;
            } else if (h1) {
                node = c1;
            } else {
                node = st.sp ? st.pop() : kDone;
            }
            if (node < 0 && leaf == 0) {   // postpone the first leaf found, keep descending
                leaf = node;
                node = st.sp ? st.pop() : kDone;
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;
        }
        while (leaf < 0) {
            const uint32_t code = uint32_t(leaf);
            const uint32_t first = code & 0x07ffffffu;
            const uint32_t count = ((code >> 27) & 0xfu) + 1u;
            for (uint32_t i = first; i < first + count; ++i) {
                const float4 a = __ldg(tris + 3 * i + 0);
                const float4 b = __ldg(tris + 3 * i + 1);
                const float4 c = __ldg(tris + 3 * i + 2);
                ++nt;
                if (PHONG && (__float_as_uint(a.w) & wrp::kPatchFlag)) {
                    if (patch_leaf_test(r, pr, patches, i, a, b, c, tmin, t, bu, bv)) {
                        tri = i;
                        if (ANY_HIT) {
                            if (node_visits) { *node_visits += nv; *tri_tests += nt; }
                            return true;
                        }
                    }
                    continue;
                }
                float th, uh, vh;
                if (tri_test(r, a, b, c, tmin, t, th, uh, vh)) {
                    if (ANY_HIT) {
                        t = th; tri = i; bu = uh; bv = vh;
                        if (node_visits) { *node_visits += nv; *tri_tests += nt; }
                        return true;
                    }
                    if (th < t || tri == MISS) { t = th; tri = i; bu = uh; bv = vh; }
                }
            }
            leaf = 0;
            if (node < 0 && node != kDone) {   // the traversal is sitting on another leaf
                leaf = node;
                node = st.sp ? st.pop() : kDone;
            }
        }
    }
    if (node_visits) { *node_visits += nv; *tri_tests += nt; }
    return tri != MISS;
}

// Resumable form of `traverse` for persistent kernels with dynamic ray fetching (Aila &
// Laine 2009, "replace terminated rays"): the per-ray state (node, postponed leaf, stack,
// best hit) lives in the caller and survives between calls. The while-while loop runs as in
// `traverse`, but after each leaf pass the warp leaves it when fewer than `min_active` of its
// lanes are still traversing, so that the caller can hand new rays to the finished lanes.
// Returns true when this lane's ray is finished (any hit found for ANY_HIT, or the tree
// exhausted); the result is the same as `traverse`'s, only the schedule differs.
constexpr int kTraceDone = 0x7fffffff;

template <bool ANY_HIT, bool PHONG = false>
__device__ __forceinline__ bool traverse_steps(const float4 *__restrict__ nodes, const float4 *__restrict__ tris,
                                               const RayPre &r, float tmin, float &t, uint32_t &tri, float &bu,
                                               float &bv, int &node, int &leaf, TraceStack &st, uint32_t &nv,
                                               uint32_t &nt, int min_active, const double *patches = nullptr,
                                               const PatchRay &pr = PatchRay{}) {
    while (node != kTraceDone) {
        while (node >= 0 && node != kTraceDone) {
            const float4 n0 = __ldg(nodes + 4 * node + 0);
            const float4 n1 = __ldg(nodes + 4 * node + 1);
            const float4 n2 = __ldg(nodes + 4 * node + 2);
            const float4 n3 = __ldg(nodes + 4 * node + 3);
            ++nv;
            const float e0 = box_entry(r, n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, tmin, t);
            const float e1 = box_entry(r, n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, tmin, t);
            const int c0 = __float_as_int(n3.x), c1 = __float_as_int(n3.y);
            const bool h0 = e0 != __int_as_float(0x7f800000), h1 = e1 != __int_as_float(0x7f800000);
            if (h0 && h1) {
                int near = c0, far = c1;
                if (e1 < e0) { near = c1; far = c0; }
                st.push(far);
                node = near;
            } else if (h0) {
                node = c0;
            } else if (h1) {
                node = c1;
            } else {
                node = st.sp ? st.pop() : kTraceDone;
            }
            if (node < 0 && leaf == 0) {   // postpone the first leaf found, keep descending
                leaf = node;
                node = st.sp ? st.pop() : kTraceDone;
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;
        }
        while (leaf < 0) {
            const uint32_t code = uint32_t(leaf);
            const uint32_t first = code & 0x07ffffffu;
            const uint32_t count = ((code >> 27) & 0xfu) + 1u;
            for (uint32_t i = first; i < first + count; ++i) {
                const float4 a = __ldg(tris + 3 * i + 0);
                const float4 b = __ldg(tris + 3 * i + 1);
                const float4 c = __ldg(tris + 3 * i + 2);
                ++nt;
                if (PHONG && (__float_as_uint(a.w) & wrp::kPatchFlag)) {
                    if (patch_leaf_test(r, pr, patches, i, a, b, c, tmin, t, bu, bv)) {
                        tri = i;
                        if (ANY_HIT) {
                            node = kTraceDone;
                            leaf = 0;
                            return true;
                        }
                    }
                    continue;
                }
                float th, uh, vh;
                if (tri_test(r, a, b, c, tmin, t, th, uh, vh)) {
                    if (ANY_HIT) {
                        t = th; tri = i; bu = uh; bv = vh;
                        node = kTraceDone;
                        leaf = 0;
                        return true;
                    }
                    if (th < t || tri == MISS) { t = th; tri = i; bu = uh; bv = vh; }
                }
            }
            leaf = 0;
            if (node < 0 && node != kTraceDone) {   // the traversal is sitting on another leaf
                leaf = node;
                node = st.sp ? st.pop() : kTraceDone;
            }
        }
        if (node != kTraceDone && __popc(__activemask()) < min_active) return false;
    }
    return true;
}

}  // namespace wrd
