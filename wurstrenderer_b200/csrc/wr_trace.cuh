// Ray / BVH traversal for the B200 renderer: closest hit (the query of
// EmbreeAccel::intersect, src/accel/embreeaccel.h:353-422) and any hit (the
// occlusion query of EmbreeAccel::isIntersect, :336-351).
//
// * Binary BVH, both child boxes of a node in one 64-byte record fetched as two
//   32-byte vector loads through the read-only path (ld.global.nc.v8.f32; four 16-byte
//   loads measured 4.7 % slower on the 1M-triangle workload).
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

// one 64-byte BVH node as two 256-bit read-only loads (nodes are 64-byte aligned)
__device__ __forceinline__ void ld_node(const float4 *p, float4 &a, float4 &b, float4 &c, float4 &d) {
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
    asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
        : "=f"(c.x), "=f"(c.y), "=f"(c.z), "=f"(c.w), "=f"(d.x), "=f"(d.y), "=f"(d.z), "=f"(d.w)
        : "l"(p + 2));
}

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
            float4 n0, n1, n2, n3;
            ld_node(nodes + 4 * node, n0, n1, n2, n3);
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
            float4 n0, n1, n2, n3;
            ld_node(nodes + 4 * node, n0, n1, n2, n3);
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

// ------------------------------------------------------------------------
// Traversal of the compressed 8-wide BVH (layout in wr_bvh.cpp: 80-byte nodes, child boxes
// quantised to 8 bits on a per-node power-of-two grid, octant-ordered slots).
//
// Per node: the 8 child boxes are decoded in ray space, t = q * (scale / d) + (p - o) / d (one
// FMA per plane), and slab-tested against (tmin, t]; the triangles of the hit leaf slots are
// tested at once; the hit inner slots form a group visited in order slot ^ octant. The current
// group is (node << 8 | remaining hit positions) with that node's first-child index and inner
// mask in registers; a group with hits left is pushed when its first child is entered, and
// re-read from its node when popped. Resumable like traverse_steps (state: next node, group,
// stack), leaving after any node once fewer than `min_active` lanes of the warp are busy.
struct WideState {
    int node;            // next node to intersect, -1 when none
    uint32_t grp;        // current group: node << 8 | hit positions left
    uint32_t gbase;      // first inner child of the group's node
    uint32_t gimask;     // inner slots of the group's node
};

// quantised byte k of an 8-byte lane (two words) as an exact float: the byte is placed in the
// mantissa of 2^23 by one byte permute, and 2^23 is subtracted (exact for integers < 2^23)
__device__ __forceinline__ float wq_byte(uint32_t lo, uint32_t hi, int k) {
    return __uint_as_float(__byte_perm(k < 4 ? lo : hi, 0x4B000000u, 0x7540u | uint32_t(k & 3))) - 8388608.0f;
}

template <bool ANY_HIT, bool PHONG = false>
__device__ __forceinline__ bool traverse_steps_w8(const uint4 *__restrict__ wnodes, const float4 *__restrict__ tris,
                                                  const RayPre &r, uint32_t oct, float tmin, float &t, uint32_t &tri,
                                                  float &bu, float &bv, WideState &ws, TraceStack &st, uint32_t &nv,
                                                  uint32_t &nt, int min_active, const double *patches = nullptr,
                                                  const PatchRay &pr = PatchRay{}) {
    const bool negx = r.ix < 0.f, negy = r.iy < 0.f, negz = r.iz < 0.f;
    while (true) {
        if (ws.node >= 0) {
            const uint4 n0 = __ldg(wnodes + 5 * ws.node + 0);
            const uint4 n1 = __ldg(wnodes + 5 * ws.node + 1);
            const uint4 n2 = __ldg(wnodes + 5 * ws.node + 2);
            const uint4 n3 = __ldg(wnodes + 5 * ws.node + 3);
            const uint4 n4 = __ldg(wnodes + 5 * ws.node + 4);
            ++nv;
            const float sx = __uint_as_float((n0.w & 0xffu) << 23) * r.ix;
            const float sy = __uint_as_float(((n0.w >> 8) & 0xffu) << 23) * r.iy;
            const float sz = __uint_as_float(((n0.w >> 16) & 0xffu) << 23) * r.iz;
            const float ox = fmaf(__uint_as_float(n0.x), r.ix, -r.oix);
            const float oy = fmaf(__uint_as_float(n0.y), r.iy, -r.oiy);
            const float oz = fmaf(__uint_as_float(n0.z), r.iz, -r.oiz);
            const uint32_t imask = n0.w >> 24;
            // near / far quantised planes per axis (lo words: 8 bytes x, y, z; hi words likewise)
            const uint32_t xnl = negx ? n3.z : n2.x, xnh = negx ? n3.w : n2.y;
            const uint32_t xfl = negx ? n2.x : n3.z, xfh = negx ? n2.y : n3.w;
            const uint32_t ynl = negy ? n4.x : n2.z, ynh = negy ? n4.y : n2.w;
            const uint32_t yfl = negy ? n2.z : n4.x, yfh = negy ? n2.w : n4.y;
            const uint32_t znl = negz ? n4.z : n3.x, znh = negz ? n4.w : n3.y;
            const uint32_t zfl = negz ? n3.x : n4.z, zfh = negz ? n3.y : n4.w;
            uint32_t hits = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float txn = fmaf(wq_byte(xnl, xnh, k), sx, ox), txf = fmaf(wq_byte(xfl, xfh, k), sx, ox);
                const float tyn = fmaf(wq_byte(ynl, ynh, k), sy, oy), tyf = fmaf(wq_byte(yfl, yfh, k), sy, oy);
                const float tzn = fmaf(wq_byte(znl, znh, k), sz, oz), tzf = fmaf(wq_byte(zfl, zfh, k), sz, oz);
                const float tn = fmaxf(fmaxf(txn, tyn), fmaxf(tzn, tmin));
                const float tf = fminf(fminf(txf, tyf), fminf(tzf, t));
                if (tn <= tf * 1.0000005f) hits |= 1u << k;
            }
            // triangles of the hit leaf slots
            uint32_t tmask = 0, inner = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                if (!(hits & (1u << k))) continue;
                if (imask & (1u << k)) {
                    inner |= 1u << (uint32_t(k) ^ oct);
                } else {
                    const uint32_t m = ((k < 4 ? n1.z : n1.w) >> (8 * (k & 3))) & 0xffu;
                    tmask |= ((1u << (m >> 5)) - 1u) << (m & 31u);
                }
            }
            const uint32_t base_tri = n1.y;
            while (tmask) {
                const uint32_t i = base_tri + uint32_t(__ffs(tmask) - 1);
                tmask &= tmask - 1u;
                const float4 a = __ldg(tris + 3 * i + 0);
                const float4 b = __ldg(tris + 3 * i + 1);
                const float4 c = __ldg(tris + 3 * i + 2);
                ++nt;
                if (PHONG && (__float_as_uint(a.w) & wrp::kPatchFlag)) {
                    if (patch_leaf_test(r, pr, patches, i, a, b, c, tmin, t, bu, bv)) {
                        tri = i;
                        if (ANY_HIT) {
                            ws.node = -1;
                            ws.grp = 0;
                            st.sp = 0;
                            return true;
                        }
                    }
                    continue;
                }
                float th, uh, vh;
                if (tri_test(r, a, b, c, tmin, t, th, uh, vh)) {
                    if (ANY_HIT) {
                        t = th; tri = i; bu = uh; bv = vh;
                        ws.node = -1;
                        ws.grp = 0;
                        st.sp = 0;
                        return true;
                    }
                    if (th < t || tri == MISS) { t = th; tri = i; bu = uh; bv = vh; }
                }
            }
            if (inner) {
                if (ws.grp & 0xffu) st.push(int(ws.grp));
                ws.grp = uint32_t(ws.node) << 8 | inner;
                ws.gbase = n1.x;
                ws.gimask = imask;
            }
            ws.node = -1;
        }
        // next child: the lowest hit position of the current group, else a popped group
        if (!(ws.grp & 0xffu)) {
            if (!st.sp) return true;
            ws.grp = uint32_t(st.pop());
            const uint32_t pn = ws.grp >> 8;
            const uint32_t *pw = reinterpret_cast<const uint32_t *>(wnodes + 5 * pn);
            ws.gbase = __ldg(pw + 4);
            ws.gimask = __ldg(pw + 3) >> 24;
        }
        const uint32_t pos = uint32_t(__ffs(ws.grp & 0xffu) - 1);
        ws.grp &= ~(1u << pos);
        const uint32_t slot = pos ^ oct;
        ws.node = int(ws.gbase + __popc(ws.gimask & ((1u << slot) - 1u)));
        if (__popc(__activemask()) < min_active) return false;
    }
}

__device__ __forceinline__ uint32_t ray_octant(f3 d) {
    return (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
}

// one whole query on the compressed 8-wide BVH (the k_trace_batch path)
template <bool ANY_HIT, bool PHONG = false>
__device__ __forceinline__ bool traverse_w8(const uint4 *__restrict__ wnodes, const float4 *__restrict__ tris, f3 o,
                                            f3 d, float tmin, float tmax, uint32_t *smem_stack, float &t,
                                            uint32_t &tri, float &bu, float &bv, uint32_t *node_visits = nullptr,
                                            uint32_t *tri_tests = nullptr, const double *patches = nullptr) {
    const RayPre r = ray_setup(o, d);
    const PatchRay pr{o.x, o.y, o.z, d.x, d.y, d.z};
    TraceStack st;
    st.smem = smem_stack + threadIdx.x;
    st.stride = blockDim.x;
    st.sp = 0;
    WideState ws{0, 0u, 0u, 0u};
    tri = MISS;
    t = tmax;
    uint32_t nv = 0, nt = 0;
    traverse_steps_w8<ANY_HIT, PHONG>(wnodes, tris, r, ray_octant(d), tmin, t, tri, bu, bv, ws, st, nv, nt, 0,
                                      patches, pr);
    if (node_visits) { *node_visits += nv; *tri_tests += nt; }
    return tri != MISS;
}

}  // namespace wrd
