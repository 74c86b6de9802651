// Host binned-SAH BVH builder for the B200 traversal kernels (the role of
// Embree's BVH8Triangle4 SAH build behind EmbreeAccel::commit,
// src/accel/embreeaccel.h:466-469; the reference never exposes its tree, so
// only the query results -- not the tree -- are part of the drop-in contract).
//
// Output layout (one node = 64 bytes = 4 x float4, loaded with 16-byte vector
// loads on the device):
//   float4 a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   float4 b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   float4 c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   float4 d = (child0, child1, 0, 0) as int bits
// A child >= 0 is an inner node index; a child with bit 31 set is a leaf:
// bits 0-26 first triangle (leaf order), bits 27-30 count - 1. An empty child
// carries a box at +infinity so that it is never entered. Nodes are stored in
// depth-first order (left child right after its parent) so that a traversal
// descending to the near child mostly touches adjacent cache lines.
// Top levels are built in parallel with std::thread, and the bounds and bins of long ranges are
// gathered by several threads.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <new>
#include <thread>
#include <type_traits>

#include "wr_host.h"

namespace wr {
namespace {

struct Aabb {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const Aabb &b) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
    }
    void grow(const float *p) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    double half_area() const {
        if (!(hi[0] >= lo[0])) return 0.0;
        const double dx = double(hi[0]) - lo[0], dy = double(hi[1]) - lo[1], dz = double(hi[2]) - lo[2];
        return dx * dy + dy * dz + dz * dx;
    }
};

struct TmpNode {
    Aabb box;
    int child[2] = {-1, -1};
    uint32_t start = 0, count = 0;   // leaf when child[0] < 0
    int depth = 0;
};

constexpr int kBins = 32;
constexpr uint32_t kMaxLeafHard = 16;   // 4-bit count field
constexpr int kDepthBudget = 60;         // traversal stack holds 64 entries
constexpr uint32_t kParallelRange = 1u << 18;   // ranges at least this long are binned by several threads
constexpr uint32_t kChunk = 1u << 16;           // primitives per thread at least
constexpr uint32_t kSpawnRange = 1u << 13;      // subtrees at least this large may get a thread

// SAH bins of one range for all three axes. Merging two bin sets gives exactly the bins of the
// union (box min / max; counts; weights that are small integers in the scenes built here), so the
// tree does not depend on how a range was split between threads.
struct BinSet {
    Aabb box[3][kBins];
    uint32_t cnt[3][kBins] = {};
    double w[3][kBins] = {};
    void merge(const BinSet &o) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < kBins; ++b) {
                box[a][b].grow(o.box[a][b]);
                cnt[a][b] += o.cnt[a][b];
                w[a][b] += o.w[a][b];
            }
    }
};

// splits [start, start + count) into up to `threads` chunks run in parallel; f(a, b, chunk)
template <class F>
int for_chunks(uint32_t start, uint32_t count, int threads, F &&f) {
    const int parts = count >= kParallelRange ? int(std::min<uint32_t>(uint32_t(std::max(threads, 1)), count / kChunk)) : 1;
    if (parts <= 1) {
        f(start, start + count, 0);
        return 1;
    }
    const uint32_t step = (count + uint32_t(parts) - 1) / uint32_t(parts);
    std::vector<std::future<void>> fut;
    for (int p = 1; p < parts; ++p) {
        const uint32_t a = start + std::min(count, uint32_t(p) * step), b = start + std::min(count, uint32_t(p + 1) * step);
        fut.push_back(std::async(std::launch::async, [&f, a, b, p] { f(a, b, p); }));
    }
    f(start, start + std::min(count, step), 0);
    for (auto &x : fut) x.get();
    return parts;
}

// one primitive's build record; the records are partitioned in place, so every pass over a
// node's range reads contiguous memory
struct Prim {
    Aabb box;
    float c[3];      // centroid of the box
    uint32_t id;     // input order
    float w;         // SAH cost of its test
};

// Array of trivially destructible objects whose storage is not initialised on allocation: the
// builder constructs its elements in parallel (hundreds of MB for 10M primitives).
template <class T>
struct RawArray {
    static_assert(std::is_trivially_destructible<T>::value, "RawArray holds trivially destructible types");
    T *p = nullptr;
    size_t n = 0;
    RawArray() = default;
    RawArray(const RawArray &) = delete;
    RawArray &operator=(const RawArray &) = delete;
    ~RawArray() { ::operator delete(p); }
    void allocate(size_t count) {
        p = static_cast<T *>(::operator new(std::max<size_t>(count, 1) * sizeof(T)));
        n = count;
    }
    T &operator[](size_t i) { return p[i]; }
    const T &operator[](size_t i) const { return p[i]; }
    T *begin() { return p; }
    size_t size() const { return n; }
};

struct Builder {
    const std::vector<float> &v;       // 9 floats per triangle
    RawArray<Prim> prims;
    RawArray<TmpNode> nodes;
    int max_leaf;
    double trav_cost;                  // SAH cost of a traversal step, relative to a triangle test
    const std::vector<float> *prim_cost;   // SAH cost of each primitive's test (null: 1 each)
    int nthreads;
    std::atomic<int> spawned{0};       // subtree threads running besides the caller's

    Builder(const std::vector<float> &verts, int ml, int threads, double ct, const std::vector<float> *pc)
        : v(verts), max_leaf(ml), trav_cost(ct), prim_cost(pc), nthreads(threads) {
        const size_t n = v.size() / 9;
        const size_t nn = std::max<size_t>(2 * n + 1, 3);
        prims.allocate(n);
        nodes.allocate(nn);
        auto prep = [&](size_t a, size_t b) {
            for (size_t i = a; i < b; ++i) {
                Prim *q = new (&prims[i]) Prim();
                Aabb bb;
                for (int c = 0; c < 3; ++c) bb.grow(&v[9 * i + 3 * c]);
                q->box = bb;
                for (int k = 0; k < 3; ++k) q->c[k] = 0.5f * (bb.lo[k] + bb.hi[k]);
                q->id = uint32_t(i);
                q->w = prim_cost ? (*prim_cost)[i] : 1.f;
            }
            // the node slots, 2 per primitive
            for (size_t i = 2 * a; i < std::min(2 * b, nn); ++i) new (&nodes[i]) TmpNode();
            if (b == n)
                for (size_t i = 2 * b; i < nn; ++i) new (&nodes[i]) TmpNode();
        };
        std::vector<std::thread> th;
        const size_t chunk = (n + threads - 1) / std::max(threads, 1);
        for (int t = 0; t < threads; ++t) {
            size_t a = std::min(n, t * chunk), b = std::min(n, a + chunk);
            if (a < b) th.emplace_back(prep, a, b);
        }
        for (auto &x : th) x.join();
        if (n == 0)
            for (size_t i = 0; i < nn; ++i) new (&nodes[i]) TmpNode();
    }

    // Node slots without a shared counter: a subtree over c primitives has at most 2c - 1 nodes,
    // so the node of a range owns the 2c - 1 slots from its own index; its left child takes the
    // next slot (and 2 nl - 1 slots), its right child the slots after those.

    // builds the subtree over prims[start, start+count) into node `ni`
    void build(int ni, uint32_t start, uint32_t count, int depth) {
        TmpNode &nd = nodes[ni];
        nd.depth = depth;
        Aabb box, cb;   // node box and centroid box
        auto bound = [&](uint32_t a, uint32_t b, Aabb &bb_out, Aabb &cc_out) {
            Aabb bb, cc;   // local: the per-thread outputs sit next to each other
            for (uint32_t i = a; i < b; ++i) {
                bb.grow(prims[i].box);
                cc.grow(prims[i].c);
            }
            bb_out = bb;
            cc_out = cc;
        };
        if (count < kParallelRange) {
            bound(start, start + count, box, cb);
        } else {
            std::vector<Aabb> pb(size_t(std::min(nthreads, 64))), pc(pb.size());
            const int parts = for_chunks(start, count, int(pb.size()), [&](uint32_t a, uint32_t b, int p) {
                bound(a, b, pb[size_t(p)], pc[size_t(p)]);
            });
            for (int p = 0; p < parts; ++p) { box.grow(pb[size_t(p)]); cb.grow(pc[size_t(p)]); }
        }
        nd.box = box;
        if (count <= 1) { nd.start = start; nd.count = count; return; }

        // binned SAH over the three axes: one pass over the primitives fills the bins of all three
        float scale[3];
        bool axis_ok[3];
        for (int ax = 0; ax < 3; ++ax) {
            const float ext = cb.hi[ax] - cb.lo[ax];
            axis_ok[ax] = ext > 0.f;
            scale[ax] = axis_ok[ax] ? kBins / ext : 0.f;
        }
        auto fill = [&](uint32_t a, uint32_t b, BinSet &bs) {
            for (uint32_t i = a; i < b; ++i) {
                const Prim &q = prims[i];
                const Aabb &tb = q.box;
                const double wt = double(q.w);
                for (int ax = 0; ax < 3; ++ax) {
                    if (!axis_ok[ax]) continue;
                    int bi = int((q.c[ax] - cb.lo[ax]) * scale[ax]);
                    bi = std::min(std::max(bi, 0), kBins - 1);
                    bs.box[ax][bi].grow(tb);
                    bs.cnt[ax][bi]++;
                    bs.w[ax][bi] += wt;
                }
            }
        };
        BinSet bins;
        if (count < kParallelRange) {
            fill(start, start + count, bins);
        } else {
            std::vector<BinSet> part(size_t(std::min(nthreads, 64)));
            const int parts = for_chunks(start, count, int(part.size()), [&](uint32_t a, uint32_t b, int p) {
                fill(a, b, part[size_t(p)]);
            });
            for (int p = 0; p < parts; ++p) bins.merge(part[size_t(p)]);
        }
        int best_axis = -1, best_split = -1;
        double best_cost = INFINITY;
        double total_w = -1.0;   // summed primitive costs (from the bins of any binned axis)
        for (int ax = 0; ax < 3; ++ax) {
            if (!axis_ok[ax]) continue;
            const Aabb *binb = bins.box[ax];
            const uint32_t *cnt = bins.cnt[ax];
            const double *wsum = bins.w[ax];
            if (total_w < 0.0) {
                total_w = 0.0;
                for (int b = 0; b < kBins; ++b) total_w += wsum[b];
            }
            double right_area[kBins], right_w[kBins];
            uint32_t right_cnt[kBins];
            Aabb acc;
            uint32_t c = 0;
            double w = 0.0;
            for (int b = kBins - 1; b > 0; --b) {
                acc.grow(binb[b]);
                c += cnt[b];
                w += wsum[b];
                right_area[b] = acc.half_area();
                right_cnt[b] = c;
                right_w[b] = w;
            }
            acc = Aabb();
            c = 0;
            w = 0.0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc.grow(binb[b]);
                c += cnt[b];
                w += wsum[b];
                if (c == 0 || right_cnt[b + 1] == 0) continue;
                const double cost = acc.half_area() * w + right_area[b + 1] * right_w[b + 1];
                if (cost < best_cost) { best_cost = cost; best_axis = ax; best_split = b; }
            }
        }
        const double parent_area = box.half_area();
        // SAH with traversal cost trav_cost and each primitive's test cost (relative to the parent's area)
        double leaf_cost = total_w;
        if (leaf_cost < 0.0) {   // no axis was binned (coincident centroids)
            leaf_cost = 0.0;
            for (uint32_t i = start; i < start + count; ++i) leaf_cost += double(prims[i].w);
        }
        const double split_cost = trav_cost + (parent_area > 0 ? best_cost / parent_area : leaf_cost);
        if (count <= uint32_t(max_leaf) && (best_axis < 0 || leaf_cost <= split_cost)) {
            nd.start = start; nd.count = count; return;
        }
        uint32_t nl;
        int log2c = 0;
        while ((1u << log2c) < count) ++log2c;
        if (best_axis >= 0 && depth + log2c >= kDepthBudget) {
            // keep the tree shallower than the traversal stack: object median on the widest axis
            int ax = 0;
            for (int k = 1; k < 3; ++k) if (cb.hi[k] - cb.lo[k] > cb.hi[ax] - cb.lo[ax]) ax = k;
            nl = count / 2;
            std::nth_element(prims.begin() + start, prims.begin() + start + nl, prims.begin() + start + count,
                             [ax](const Prim &a, const Prim &b2) { return a.c[ax] < b2.c[ax]; });
        } else if (best_axis < 0) {
            nl = count / 2;   // coincident centroids: split the range
        } else {
            const float ext = cb.hi[best_axis] - cb.lo[best_axis];
            const float scale = kBins / ext;
            auto mid = std::partition(prims.begin() + start, prims.begin() + start + count, [&](const Prim &q) {
                int b = int((q.c[best_axis] - cb.lo[best_axis]) * scale);
                b = std::min(std::max(b, 0), kBins - 1);
                return b <= best_split;
            });
            nl = uint32_t(mid - (prims.begin() + start));
            if (nl == 0 || nl == count) nl = count / 2;
        }
        const int l = ni + 1, r = ni + 2 * int(nl);
        nd.child[0] = l;
        nd.child[1] = r;
        // subtrees of more than kSpawnRange primitives go to their own thread while fewer than
        // 2 x nthreads such threads run: SAH splits are uneven, so threads are handed out as the
        // tree unfolds rather than by depth
        bool spawn = false;
        if (nl > kSpawnRange && count - nl > kSpawnRange) {
            spawn = spawned.fetch_add(1) < 2 * nthreads;
            if (!spawn) spawned.fetch_sub(1);
        }
        if (spawn) {
            auto fut = std::async(std::launch::async, [&, l, start, nl, depth] {
                build(l, start, nl, depth + 1);
                spawned.fetch_sub(1);
            });
            build(r, start + nl, count - nl, depth + 1);
            fut.get();
        } else {
            build(l, start, nl, depth + 1);
            build(r, start + nl, count - nl, depth + 1);
        }
    }
};

void put_child_box(float *out, int slot, const Aabb &b, bool empty) {
    // slot 0 -> a.xyzw + c.xy, slot 1 -> b.xyzw + c.zw
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = empty ? INFINITY : b.lo[k];   // a box at +inf is missed by every ray
        hi[k] = empty ? INFINITY : b.hi[k];
    }
    float *xy = out + (slot == 0 ? 0 : 4);
    xy[0] = lo[0]; xy[1] = hi[0]; xy[2] = lo[1]; xy[3] = hi[1];
    out[8 + 2 * slot] = lo[2];
    out[9 + 2 * slot] = hi[2];
}

}  // namespace

BvhBuildResult build_bvh_sah(const std::vector<float> &tri_vertices, int max_leaf, int threads, double trav_cost,
                             const std::vector<float> *prim_cost) {
    BvhBuildResult res;
    const uint32_t n = uint32_t(tri_vertices.size() / 9);
    if (threads <= 0) threads = std::max(1u, std::thread::hardware_concurrency());
    max_leaf = std::max(1, std::min(max_leaf, int(kMaxLeafHard)));
    if (n >= (1u << 27)) throw Error(WR_ERR_UNSUPPORTED, "more than 2^27 triangles");
    if (prim_cost && prim_cost->size() != n) throw Error(WR_ERR_INVALID_ARGUMENT, "prim_cost size");
    Builder b(tri_vertices, max_leaf, threads, trav_cost, prim_cost);
    const int root = 0;
    if (n > 0) b.build(root, 0, n, 0);
    else b.nodes[root].count = 0;

    // Depth-first linearisation; the device root is always an inner node. A node's left child
    // sits in the next slot and its right subtree after the whole left subtree, so depth-first
    // preorder is the order of the slots: device indices and triangle offsets are prefix sums
    // over the slots, computed in parallel chunks.
    const size_t nn = b.nodes.size();
    auto inner = [&](size_t i) { return i == size_t(root) || b.nodes[i].child[0] >= 0; };
    auto leaf_tris = [&](size_t i) -> uint32_t {   // triangles of the leaf children of inner slot i
        const TmpNode &nd = b.nodes[i];
        if (nd.child[0] < 0) return nd.count;       // the whole scene is one leaf
        uint32_t c = 0;
        for (int s = 0; s < 2; ++s) {
            const TmpNode &ch = b.nodes[size_t(nd.child[s])];
            if (ch.child[0] < 0) c += ch.count;
        }
        return c;
    };
    const int parts = int(std::max<size_t>(1, std::min<size_t>(size_t(threads), nn / kChunk)));
    const size_t step = (nn + size_t(parts) - 1) / size_t(parts);
    std::vector<size_t> inner_base(size_t(parts) + 1, 0), tri_base(size_t(parts) + 1, 0);
    std::vector<int> part_depth(size_t(parts), 0);
    auto run_parts = [&](auto &&fn) {
        std::vector<std::future<void>> fut;
        for (int p = 1; p < parts; ++p) fut.push_back(std::async(std::launch::async, [&fn, p] { fn(p); }));
        fn(0);
        for (auto &x : fut) x.get();
    };
    run_parts([&](int p) {
        size_t ci = 0, ct = 0;
        int d = 0;
        for (size_t i = size_t(p) * step; i < std::min(nn, size_t(p + 1) * step); ++i)
            if (inner(i)) {
                ++ci;
                ct += leaf_tris(i);
                d = std::max(d, b.nodes[i].depth + 1);
            }
        inner_base[size_t(p) + 1] = ci;
        tri_base[size_t(p) + 1] = ct;
        part_depth[size_t(p)] = d;
    });
    for (int p = 0; p < parts; ++p) {
        inner_base[size_t(p) + 1] += inner_base[size_t(p)];
        tri_base[size_t(p) + 1] += tri_base[size_t(p)];
        res.depth = std::max(res.depth, part_depth[size_t(p)]);
    }
    const size_t n_inner = inner_base[size_t(parts)];
    RawArray<int> dev_of;
    dev_of.allocate(nn);
    run_parts([&](int p) {
        int di = int(inner_base[size_t(p)]);
        for (size_t i = size_t(p) * step; i < std::min(nn, size_t(p + 1) * step); ++i)
            if (inner(i)) dev_of[i] = di++;
    });
    std::vector<float> &out = res.nodes;
    out.assign(n_inner * 16, 0.f);
    res.tri_order.resize(tri_base[size_t(parts)]);
    run_parts([&](int p) {
        size_t di = inner_base[size_t(p)];
        uint32_t first = uint32_t(tri_base[size_t(p)]);
        for (size_t i = size_t(p) * step; i < std::min(nn, size_t(p + 1) * step); ++i) {
            if (!inner(i)) continue;
            const TmpNode &nd = b.nodes[i];
            float *o = &out[di++ * 16];
            int32_t child_code[2];
            if (nd.child[0] < 0) {
                // the whole scene is one leaf: child 0 holds it, child 1 is empty
                for (uint32_t k = 0; k < nd.count; ++k) res.tri_order[first + k] = b.prims[nd.start + k].id;
                put_child_box(o, 0, nd.box, nd.count == 0);
                put_child_box(o, 1, nd.box, true);
                child_code[0] = int32_t(0x80000000u | (uint32_t(std::max<uint32_t>(nd.count, 1) - 1) << 27) | first);
                child_code[1] = int32_t(0x80000000u);
                first += nd.count;
            } else {
                for (int s = 0; s < 2; ++s) {
                    const TmpNode &c = b.nodes[size_t(nd.child[s])];
                    put_child_box(o, s, c.box, false);
                    if (c.child[0] >= 0) {
                        child_code[s] = dev_of[size_t(nd.child[s])];
                    } else {
                        for (uint32_t k = 0; k < c.count; ++k) res.tri_order[first + k] = b.prims[c.start + k].id;
                        child_code[s] = int32_t(0x80000000u | ((c.count - 1) << 27) | first);
                        first += c.count;
                    }
                }
            }
            memcpy(&o[12], &child_code[0], 4);
            memcpy(&o[13], &child_code[1], 4);
        }
    });
    // SAH cost of the tree, summed in device order
    const double root_area = std::max(b.nodes[root].box.half_area(), 1e-30);
    for (size_t i = 0; i < nn; ++i) {
        if (!inner(i)) continue;
        const TmpNode &nd = b.nodes[i];
        if (nd.child[0] < 0) {
            res.sah_cost += nd.box.half_area() / root_area * nd.count;
            continue;
        }
        res.sah_cost += nd.box.half_area() / root_area;
        for (int s = 0; s < 2; ++s) {
            const TmpNode &c = b.nodes[size_t(nd.child[s])];
            if (c.child[0] < 0) res.sah_cost += c.box.half_area() / root_area * c.count;
        }
    }
    return res;
}

// ------------------------------------------------------------------------
// Compressed 8-wide BVH (after Ylitie, Karras and Laine, "Efficient incoherent ray traversal on
// GPUs through compressed wide BVHs", HPG 2017), collapsed from the binary tree above.
//
// Node = 80 bytes = 5 x uint4 (words):
//   0-2  p.xyz: origin of the child-box grid (the node box's lower corner), float
//   3    e.x | e.y << 8 | e.z << 16 | imask << 24: grid scale 2^(e-127) per axis (biased
//        float exponents); imask bit s: slot s holds an inner node
//   4    first inner child (inner children are stored contiguously in slot order)
//   5    first triangle (leaf triangles of all leaf slots are stored contiguously)
//   6-7  meta byte per slot: leaf = count (1..3) << 5 | offset from word 5; else 0
//   8-13 quantised lower bounds: 8 bytes x, 8 bytes y, 8 bytes z
//   14-19 quantised upper bounds: 8 bytes x, 8 bytes y, 8 bytes z
// Child box along x: [p.x + lo_q * 2^(e.x-127), p.x + hi_q * 2^(e.x-127)], rounded outward; empty
// slots carry lo_q = 255 > hi_q = 0 and are never entered.
// Slot s holds the child that a ray of direction octant s (bit k: negative component k) should
// visit first: children are assigned greedily by the least dot(child centre - node centre,
// octant direction). A ray of octant o then visits its hit inner children in order of slot ^ o.
namespace {

struct WChild {
    Aabb box;
    int32_t code;   // binary inner node (>= 0) or leaf code (bit 31 set)
};

Aabb binary_child_box(const float *o, int slot) {
    Aabb b;
    const float *xy = o + (slot == 0 ? 0 : 4);
    b.lo[0] = xy[0]; b.hi[0] = xy[1]; b.lo[1] = xy[2]; b.hi[1] = xy[3];
    b.lo[2] = o[8 + 2 * slot]; b.hi[2] = o[9 + 2 * slot];
    return b;
}

}  // namespace

WideBvh build_wide8(const BvhBuildResult &bin) {
    WideBvh w;
    const size_t nbin = bin.nodes.size() / 16;
    if (nbin == 0) return w;
    struct Work { int bnode; uint32_t wnode; int depth; };
    std::vector<Work> work{{0, 0u, 1}};
    w.nodes.assign(20, 0u);
    auto children_of = [&](int b, std::vector<WChild> &out) {
        const float *o = &bin.nodes[size_t(b) * 16];
        int32_t code[2];
        memcpy(&code[0], &o[12], 4);
        memcpy(&code[1], &o[13], 4);
        for (int s = 0; s < 2; ++s) {
            const Aabb bx = binary_child_box(o, s);
            if (!(bx.lo[0] <= bx.hi[0]) || bx.lo[0] == INFINITY) continue;   // empty slot
            out.push_back(WChild{bx, code[s]});
        }
    };
    while (!work.empty()) {
        const Work it = work.back();
        work.pop_back();
        w.depth = std::max(w.depth, it.depth);
        std::vector<WChild> ch;
        children_of(it.bnode, ch);
        // open the inner child of largest area until 8 children
        while (ch.size() < 8) {
            int best = -1;
            double best_area = -1.0;
            for (size_t i = 0; i < ch.size(); ++i)
                if (ch[i].code >= 0 && ch[i].box.half_area() > best_area) {
                    best = int(i);
                    best_area = ch[i].box.half_area();
                }
            if (best < 0) break;
            std::vector<WChild> sub;
            children_of(ch[size_t(best)].code, sub);
            if (ch.size() - 1 + sub.size() > 8) break;
            ch.erase(ch.begin() + best);
            ch.insert(ch.end(), sub.begin(), sub.end());
        }
        Aabb nb;
        for (const WChild &c : ch) nb.grow(c.box);
        // slot assignment by octant
        int slot_of[8], child_in[8];
        for (int i = 0; i < 8; ++i) { slot_of[i] = -1; child_in[i] = -1; }
        {
            double cost[8][8];
            for (size_t i = 0; i < ch.size(); ++i) {
                double v[3];
                for (int k = 0; k < 3; ++k)
                    v[k] = 0.5 * (double(ch[i].box.lo[k]) + ch[i].box.hi[k]) - 0.5 * (double(nb.lo[k]) + nb.hi[k]);
                for (int s = 0; s < 8; ++s)
                    cost[i][s] = ((s & 1) ? -v[0] : v[0]) + ((s & 2) ? -v[1] : v[1]) + ((s & 4) ? -v[2] : v[2]);
            }
            for (size_t n = 0; n < ch.size(); ++n) {
                double bc = INFINITY;
                int bi = -1, bs = -1;
                for (size_t i = 0; i < ch.size(); ++i) {
                    if (slot_of[i] >= 0) continue;
                    for (int s = 0; s < 8; ++s)
                        if (child_in[s] < 0 && cost[i][s] < bc) { bc = cost[i][s]; bi = int(i); bs = s; }
                }
                if (bi < 0) {   // NaN costs: any free slot
                    for (size_t i = 0; i < ch.size() && bi < 0; ++i)
                        if (slot_of[i] < 0) bi = int(i);
                    for (int s = 0; s < 8 && bs < 0; ++s)
                        if (child_in[s] < 0) bs = s;
                }
                slot_of[bi] = bs;
                child_in[bs] = bi;
            }
        }
        uint32_t *o = &w.nodes[size_t(it.wnode) * 20];
        // grid: origin at the node's lower corner, per-axis power-of-two scale with 255 steps
        int e[3];
        for (int k = 0; k < 3; ++k) {
            const double ext = double(nb.hi[k]) - double(nb.lo[k]);
            int ex = -126;
            if (ext > 0.0) {
                frexp(ext / 255.0, &ex);   // ext / 255 < 2^ex
                ex = std::max(ex, -126);
            }
            e[k] = ex + 127;
            if (e[k] > 254) throw Error(WR_ERR_UNSUPPORTED, "scene extent too large for the compressed BVH");
            memcpy(&o[k], &nb.lo[k], 4);
        }
        uint32_t imask = 0, n_inner = 0;
        for (int s = 0; s < 8; ++s)
            if (child_in[s] >= 0 && ch[size_t(child_in[s])].code >= 0) { imask |= 1u << s; ++n_inner; }
        o[3] = uint32_t(e[0]) | uint32_t(e[1]) << 8 | uint32_t(e[2]) << 16 | imask << 24;
        const uint32_t base_child = uint32_t(w.nodes.size() / 20);
        const uint32_t base_tri = uint32_t(w.order.size());
        o[4] = base_child;
        o[5] = base_tri;
        uint8_t meta[8] = {0, 0, 0, 0, 0, 0, 0, 0}, qlo[3][8], qhi[3][8];
        for (int s = 0; s < 8; ++s)
            for (int k = 0; k < 3; ++k) { qlo[k][s] = 255; qhi[k][s] = 0; }
        uint32_t next_inner = 0;
        std::vector<Work> pushes;
        for (int s = 0; s < 8; ++s) {
            if (child_in[s] < 0) continue;
            const WChild &c = ch[size_t(child_in[s])];
            for (int k = 0; k < 3; ++k) {
                const double scale = std::ldexp(1.0, e[k] - 127);
                const double p = double(nb.lo[k]);
                double ql = std::floor((double(c.box.lo[k]) - p) / scale);
                double qh = std::ceil((double(c.box.hi[k]) - p) / scale);
                ql = std::min(std::max(ql, 0.0), 255.0);
                qh = std::min(std::max(qh, 0.0), 255.0);
                while (ql > 0.0 && p + ql * scale > double(c.box.lo[k])) ql -= 1.0;
                while (qh < 255.0 && p + qh * scale < double(c.box.hi[k])) qh += 1.0;
                qlo[k][s] = uint8_t(ql);
                qhi[k][s] = uint8_t(qh);
            }
            if (c.code >= 0) {
                pushes.push_back(Work{c.code, base_child + next_inner, it.depth + 1});
                ++next_inner;
            } else {
                const uint32_t code = uint32_t(c.code);
                const uint32_t first = code & 0x07ffffffu, count = ((code >> 27) & 0xfu) + 1u;
                if (count > 3) throw Error(WR_ERR_UNSUPPORTED, "compressed BVH leaves hold at most 3 triangles");
                const uint32_t off = uint32_t(w.order.size()) - base_tri;
                for (uint32_t t = first; t < first + count; ++t) w.order.push_back(bin.tri_order[t]);
                meta[s] = uint8_t(count << 5 | off);
            }
        }
        uint32_t *on = &w.nodes[size_t(it.wnode) * 20];   // (o may be stale after the resize below)
        memcpy(&on[6], meta, 8);
        for (int k = 0; k < 3; ++k) {
            memcpy(&on[8 + 2 * k], qlo[k], 8);
            memcpy(&on[14 + 2 * k], qhi[k], 8);
        }
        w.nodes.resize(w.nodes.size() + size_t(n_inner) * 20, 0u);
        for (auto pw = pushes.rbegin(); pw != pushes.rend(); ++pw) work.push_back(*pw);
    }
    if (w.nodes.size() / 20 >= (1u << 24)) throw Error(WR_ERR_UNSUPPORTED, "more than 2^24 compressed BVH nodes");
    return w;
}

}  // namespace wr
