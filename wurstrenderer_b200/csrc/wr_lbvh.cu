// On-device BVH build: linear BVH over 62-bit keys (30-bit Morton code of the
// triangle centroid, then the triangle index), after Karras, "Maximizing
// Parallelism in the Construction of BVHs, Octrees, and k-d Trees" (HPG 2012).
//
//   k_lbvh_keys     centroid -> Morton code on a cubic grid -> key (Morton << 32 | index)
//   radix sort      CUB DeviceRadixSort on (key, triangle) pairs
//   k_lbvh_topology one thread per inner node: key range, split, children, parents
//   k_lbvh_refit    one thread per leaf walking to the root; the second thread to
//                   reach an inner node unions its two children's boxes
//   k_lbvh_emit     writes the traversal layout (wr_bvh.cpp: 4 x float4 per node,
//                   both child boxes + child codes) and the leaf-order triangles; an inner
//                   node over two one-triangle leaves becomes a two-triangle leaf where the
//                   SAH rule of the host builder prefers it (566 against 550 Mpaths/s on the
//                   1M-triangle workload)
//
// Leaves hold one or two triangles. Every inner node splits at the first differing key bit
// of its range, so the depth is at most 63 (key bits + 1) and the 64-entry
// traversal stack always suffices. The result replaces Embree's BVH build
// (src/accel/embreeaccel.h:466-469) when a scene is created with the device builder;
// the default remains the host binned-SAH build, whose trees traverse faster.

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include "wr_host.h"

namespace {

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {   // 10 bits -> every third bit
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__device__ __forceinline__ void tri_box(const float *v, uint32_t t, float lo[3], float hi[3]) {
    const float *p = v + 9 * size_t(t);
    for (int k = 0; k < 3; ++k) {
        lo[k] = fminf(p[k], fminf(p[3 + k], p[6 + k]));
        hi[k] = fmaxf(p[k], fmaxf(p[3 + k], p[6 + k]));
    }
}

__global__ void k_lbvh_keys(const float *verts, uint32_t n, float3 lo, float3 inv_ext, unsigned long long *keys,
                            uint32_t *ids) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float bl[3], bh[3];
        tri_box(verts, i, bl, bh);
        const float cx = (0.5f * (bl[0] + bh[0]) - lo.x) * inv_ext.x;
        const float cy = (0.5f * (bl[1] + bh[1]) - lo.y) * inv_ext.y;
        const float cz = (0.5f * (bl[2] + bh[2]) - lo.z) * inv_ext.z;
        const uint32_t x = min(max(int(cx * 1024.f), 0), 1023), y = min(max(int(cy * 1024.f), 0), 1023),
                       z = min(max(int(cz * 1024.f), 0), 1023);
        const uint32_t m = (expand_bits(x) << 2) | (expand_bits(y) << 1) | expand_bits(z);
        keys[i] = ((unsigned long long)m << 32) | i;
        ids[i] = i;
    }
}

__device__ __forceinline__ int delta(const unsigned long long *k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    return __clzll(k[i] ^ k[j]);   // keys are unique (index in the low bits)
}

// inner node i in [0, n-2]; child codes: >= 0 inner node, ~leaf (< 0) leaf position
__global__ void k_lbvh_topology(const unsigned long long *k, int n, int2 *child, int *parent_inner,
                                int *parent_leaf) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
        const int dmin = delta(k, n, i, i - d);
        int lmax = 2;
        while (delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(k, n, i, j);
        int s = 0;
        for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
            if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int g = i + s * d + min(d, 0);
        const int lo = min(i, j), hi = max(i, j);
        int2 c;
        c.x = (lo == g) ? ~g : g;
        c.y = (hi == g + 1) ? ~(g + 1) : (g + 1);
        child[i] = c;
        if (c.x < 0) parent_leaf[~c.x] = i; else parent_inner[c.x] = i;
        if (c.y < 0) parent_leaf[~c.y] = i; else parent_inner[c.y] = i;
    }
}

__global__ void k_lbvh_refit(const float *verts, const uint32_t *ids, int n, const int2 *child,
                             const int *parent_inner, const int *parent_leaf, float *box, int *flag) {
    for (int leaf = blockIdx.x * blockDim.x + threadIdx.x; leaf < n; leaf += gridDim.x * blockDim.x) {
        int node = parent_leaf[leaf];
        while (node >= 0) {
            __threadfence();
            if (atomicAdd(&flag[node], 1) == 0) break;   // the sibling subtree is not finished yet
            __threadfence();
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            const int2 c = child[node];
            for (int s = 0; s < 2; ++s) {
                const int code = s ? c.y : c.x;
                float bl[3], bh[3];
                if (code < 0) {
                    tri_box(verts, ids[~code], bl, bh);
                } else {
                    const volatile float *b = box + 6 * size_t(code);
                    for (int k = 0; k < 3; ++k) { bl[k] = b[k]; bh[k] = b[3 + k]; }
                }
                for (int k = 0; k < 3; ++k) { lo[k] = fminf(lo[k], bl[k]); hi[k] = fmaxf(hi[k], bh[k]); }
            }
            volatile float *b = box + 6 * size_t(node);
            for (int k = 0; k < 3; ++k) { b[k] = lo[k]; b[3 + k] = hi[k]; }
            node = node == 0 ? -1 : parent_inner[node];
        }
    }
}

__device__ __forceinline__ float half_area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_lbvh_emit(const float *verts, const uint32_t *ids, int n, const int2 *child, const float *box,
                            float4 *nodes) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int2 c = child[i];
        float cb[2][6];
        int code[2];
        for (int s = 0; s < 2; ++s) {
            const int ch = s ? c.y : c.x;
            float bl[3], bh[3];
            if (ch < 0) {
                tri_box(verts, ids[~ch], bl, bh);
                code[s] = int(0x80000000u | uint32_t(~ch));   // one-triangle leaf at sorted position ~ch
            } else {
                for (int k = 0; k < 3; ++k) { bl[k] = box[6 * size_t(ch) + k]; bh[k] = box[6 * size_t(ch) + 3 + k]; }
                code[s] = ch;
                // an inner child over two one-triangle leaves (consecutive sorted positions) becomes
                // a two-triangle leaf when that is the cheaper choice by the host builder's SAH
                // rule: 2 triangle tests <= 1 traversal step + the two leaves' relative areas
                const int2 gc = child[ch];
                if (gc.x < 0 && gc.y < 0) {
                    float l0[3], h0[3], l1[3], h1[3];
                    tri_box(verts, ids[~gc.x], l0, h0);
                    tri_box(verts, ids[~gc.y], l1, h1);
                    const float ap = half_area(bl, bh);
                    if (ap > 0.f && 2.f * ap <= ap + half_area(l0, h0) + half_area(l1, h1))
                        code[s] = int(0x80000000u | (1u << 27) | uint32_t(min(~gc.x, ~gc.y)));
                }
            }
            for (int k = 0; k < 3; ++k) { cb[s][k] = bl[k]; cb[s][3 + k] = bh[k]; }
        }
        float4 *o = nodes + 4 * size_t(i);
        o[0] = make_float4(cb[0][0], cb[0][3], cb[0][1], cb[0][4]);
        o[1] = make_float4(cb[1][0], cb[1][3], cb[1][1], cb[1][4]);
        o[2] = make_float4(cb[0][2], cb[0][5], cb[1][2], cb[1][5]);
        o[3] = make_float4(__int_as_float(code[0]), __int_as_float(code[1]), 0.f, 0.f);
    }
}

#define LB_CUDA(call)                                                                                     \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) throw wr::Error(WR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct Tmp {
    void *p = nullptr;
    ~Tmp() { if (p) cudaFree(p); }
    void alloc(size_t n) { LB_CUDA(cudaMalloc(&p, n < 16 ? 16 : n)); }
    template <typename T> T *as() { return static_cast<T *>(p); }
};

}  // namespace

namespace wr {

// Builds on the device; returns nodes (16 floats each, device layout) and the leaf order.
BvhBuildResult build_bvh_lbvh(const std::vector<float> &tri_vertices, cudaStream_t st, double *device_ms) {
    BvhBuildResult res;
    const int n = int(tri_vertices.size() / 9);
    if (n == 0) return res;
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            // centroid bounds
            float cen = (tri_vertices[9 * size_t(i) + c] + tri_vertices[9 * size_t(i) + 3 + c] +
                         tri_vertices[9 * size_t(i) + 6 + c]) / 3.f;
            lo[c] = std::min(lo[c], cen);
            hi[c] = std::max(hi[c], cen);
        }
    float3 lo3 = make_float3(lo[0], lo[1], lo[2]);
    // one scale for the three axes (the Morton grid's cells are cubes over the centroid box's
    // longest side): on a flat scene, a grid stretched to the box per axis would split the thin
    // axis as often as the long ones (600 against 568 Mpaths/s on the 1M-triangle workload)
    const float ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    const float iext = ext > 0.f ? 1.f / ext : 0.f;
    float3 inv = make_float3(iext, iext, iext);
    Tmp verts, keys, keys2, ids, ids2, child, pin, pleaf, box, flag, nodes, temp;
    verts.alloc(tri_vertices.size() * 4);
    keys.alloc(size_t(n) * 8);
    keys2.alloc(size_t(n) * 8);
    ids.alloc(size_t(n) * 4);
    ids2.alloc(size_t(n) * 4);
    const int ni = std::max(n - 1, 1);
    child.alloc(size_t(ni) * 8);
    pin.alloc(size_t(ni) * 4);
    pleaf.alloc(size_t(n) * 4);
    box.alloc(size_t(ni) * 24);
    flag.alloc(size_t(ni) * 4);
    nodes.alloc(size_t(ni) * 64);
    cudaEvent_t e0, e1;
    LB_CUDA(cudaEventCreate(&e0));
    LB_CUDA(cudaEventCreate(&e1));
    LB_CUDA(cudaMemcpyAsync(verts.p, tri_vertices.data(), tri_vertices.size() * 4, cudaMemcpyHostToDevice, st));
    LB_CUDA(cudaEventRecord(e0, st));
    const int grid = std::min(4096, (n + 255) / 256);
    k_lbvh_keys<<<grid, 256, 0, st>>>(verts.as<float>(), uint32_t(n), lo3, inv, keys.as<unsigned long long>(),
                                      ids.as<uint32_t>());
    size_t temp_bytes = 0;
    LB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.as<unsigned long long>(),
                                            keys2.as<unsigned long long>(), ids.as<uint32_t>(), ids2.as<uint32_t>(),
                                            n, 0, 64, st));
    temp.alloc(temp_bytes);
    LB_CUDA(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, keys.as<unsigned long long>(),
                                            keys2.as<unsigned long long>(), ids.as<uint32_t>(), ids2.as<uint32_t>(),
                                            n, 0, 64, st));
    LB_CUDA(cudaMemsetAsync(flag.p, 0, size_t(ni) * 4, st));
    LB_CUDA(cudaMemsetAsync(pin.p, 0xff, size_t(ni) * 4, st));
    if (n > 1) {
        k_lbvh_topology<<<grid, 256, 0, st>>>(keys2.as<unsigned long long>(), n, child.as<int2>(), pin.as<int>(),
                                              pleaf.as<int>());
        k_lbvh_refit<<<grid, 256, 0, st>>>(verts.as<float>(), ids2.as<uint32_t>(), n, child.as<int2>(), pin.as<int>(),
                                           pleaf.as<int>(), box.as<float>(), flag.as<int>());
        k_lbvh_emit<<<grid, 256, 0, st>>>(verts.as<float>(), ids2.as<uint32_t>(), n, child.as<int2>(),
                                          box.as<float>(), nodes.as<float4>());
    }
    LB_CUDA(cudaGetLastError());
    LB_CUDA(cudaEventRecord(e1, st));
    res.tri_order.resize(size_t(n));
    LB_CUDA(cudaMemcpyAsync(res.tri_order.data(), ids2.p, size_t(n) * 4, cudaMemcpyDeviceToHost, st));
    if (n > 1) {
        res.nodes.resize(size_t(n - 1) * 16);
        LB_CUDA(cudaMemcpyAsync(res.nodes.data(), nodes.p, size_t(n - 1) * 64, cudaMemcpyDeviceToHost, st));
    }
    LB_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    LB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (device_ms) *device_ms = ms;
    if (n == 1) {
        // a single triangle: root with the leaf and an empty child (box at +infinity)
        res.nodes.assign(16, 0.f);
        const float *p = tri_vertices.data();
        float bl[3], bh[3];
        for (int k = 0; k < 3; ++k) {
            bl[k] = std::min(p[k], std::min(p[3 + k], p[6 + k]));
            bh[k] = std::max(p[k], std::max(p[3 + k], p[6 + k]));
        }
        float *o = res.nodes.data();
        o[0] = bl[0]; o[1] = bh[0]; o[2] = bl[1]; o[3] = bh[1];
        o[4] = o[5] = o[6] = o[7] = INFINITY;
        o[8] = bl[2]; o[9] = bh[2]; o[10] = INFINITY; o[11] = INFINITY;
        const int32_t c0 = int32_t(0x80000000u), c1 = int32_t(0x80000000u);
        memcpy(&o[12], &c0, 4);
        memcpy(&o[13], &c1, 4);
    }
    // depth and SAH cost of the tree (host walk; the tree is small next to the triangles)
    const size_t nn = res.nodes.size() / 16;
    if (nn) {
        res.sah_cost = 1.0;   // the root
        std::vector<std::pair<int, int>> stack{{0, 1}};
        double root_area = 0.0;
        auto area = [](const float *b) {
            if (!(b[1] >= b[0])) return 0.0;
            const double dx = double(b[1]) - b[0], dy = double(b[3]) - b[2], dz = double(b[5]) - b[4];
            return dx * dy + dy * dz + dz * dx;
        };
        {
            const float *o = &res.nodes[0];
            float u[6] = {std::min(o[0], o[4]), std::max(o[1], o[5]), std::min(o[2], o[6]), std::max(o[3], o[7]),
                          std::min(o[8], o[10]), std::max(o[9], o[11])};
            root_area = std::max(area(u), 1e-30);
        }
        while (!stack.empty()) {
            auto [ni2, dep] = stack.back();
            stack.pop_back();
            res.depth = std::max(res.depth, dep);
            const float *o = &res.nodes[16 * size_t(ni2)];
            int32_t cc[2];
            memcpy(&cc[0], &o[12], 4);
            memcpy(&cc[1], &o[13], 4);
            for (int s = 0; s < 2; ++s) {
                const float b[6] = {o[4 * s + 0], o[4 * s + 1], o[4 * s + 2], o[4 * s + 3], o[8 + 2 * s], o[9 + 2 * s]};
                const double a = area(b) / root_area;
                if (cc[s] >= 0) { res.sah_cost += a; stack.push_back({cc[s], dep + 1}); }
                else if (b[0] != INFINITY) res.sah_cost += a * double(((uint32_t(cc[s]) >> 27) & 0xfu) + 1u);
            }
        }
    }
    return res;
}

}  // namespace wr
