// Test infrastructure only: the CPU oracle's ray caster.
//
// Restates the ray queries the reference obtains from Embree 3.5.2 (vendored
// under dependencies/embree; it needs cmake and generated code to build, so it
// is not compiled here):
//   * closest hit  EmbreeAccel::intersect -> rtcIntersect1   (src/accel/embreeaccel.h:353-422)
//   * occlusion    EmbreeAccel::isIntersect -> rtcOccluded1  (src/accel/embreeaccel.h:336-351)
// with Embree's default FAST triangle test, the single-precision
// Moeller-Trumbore variant of dependencies/embree/kernels/geometry/
// triangle_intersector_moeller.h:78-111 (edge e1 = v0-v1, e2 = v2-v0,
// Ng = cross(e2, e1), hit accepted when U >= 0, V >= 0, U+V <= |den| and
// |den|*tnear < T <= |den|*tfar, no back-face culling), returning
// t = T/|den|, u = U/|den|, v = V/|den| and the unnormalised Ng.
// Embree finishes with an approximate reciprocal; this restatement divides
// exactly, so hit distances agree to a few float ulps and triangle ids agree
// except on distance ties.
//
// The acceleration structure is a plain binary BVH (binned SAH, <= 4
// triangles per leaf) built on the host: it changes only the speed of the
// query, never its result (other than which of two exactly tied hits wins).
//
// User primitives (Embree's RTC_GEOMETRY_TYPE_USER, which the reference uses for
// Phong tessellation patches, src/accel/embreeaccel.h:242-257) are held as float
// boxes in a second BVH; a ray that enters a primitive's box calls the owner's
// test with the closest distance found so far as its far limit, as Embree calls
// the user intersect / occluded function.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <functional>
#include <vector>

namespace oracle {

struct RcTri {           // precomputed triangle in Embree's Moeller form
    float v0[3], e1[3], e2[3], ng[3];
    int geom, prim;      // Embree geomID / primID
};

struct RcNode {
    float lo[3], hi[3];
    int left = -1, right = -1;   // inner: child node indices; leaf: left = -1
    int first = 0, count = 0;    // leaf triangle range
};

struct RcHit {
    float t = INFINITY, u = 0.f, v = 0.f, ng[3] = {0.f, 0.f, 0.f};
    int geom = -1, prim = -1;
};

struct RcUser {          // a user primitive: its float box and the owner's handle
    float lo[3], hi[3];
    int geom, prim;
    int ref;             // index into the owner's primitive store
};

// closest: on a hit with t <= tfar fills *hit (t, ng, u, v, geom, prim) and returns true
using RcUserClosest = std::function<bool(const RcUser &, const float o[3], const float d[3], float tnear, float tfar, RcHit *hit)>;
// any hit in [tnear, tfar]
using RcUserAny = std::function<bool(const RcUser &, const float o[3], const float d[3], float tnear, float tfar)>;

struct RayCaster {
    std::vector<RcTri> tris;
    std::vector<RcNode> nodes;
    std::vector<RcUser> users;
    std::vector<RcNode> unodes;
    RcUserClosest user_closest;
    RcUserAny user_any;
    float scene_lo[3] = {INFINITY, INFINITY, INFINITY}, scene_hi[3] = {-INFINITY, -INFINITY, -INFINITY};

    void add_user(const RcUser &u) {
        users.push_back(u);
        for (int k = 0; k < 3; ++k) {
            scene_lo[k] = std::min(scene_lo[k], u.lo[k]);
            scene_hi[k] = std::max(scene_hi[k], u.hi[k]);
        }
    }

    // positions: float xyz per vertex; triangles: 3 indices per triangle
    void add_mesh(const float *positions, const int *triangles, int ntri, int geom_id) {
        for (int i = 0; i < ntri; ++i) {
            const float *p0 = positions + 3 * triangles[3 * i + 0];
            const float *p1 = positions + 3 * triangles[3 * i + 1];
            const float *p2 = positions + 3 * triangles[3 * i + 2];
            RcTri t;
            for (int k = 0; k < 3; ++k) {
                t.v0[k] = p0[k];
                t.e1[k] = p0[k] - p1[k];
                t.e2[k] = p2[k] - p0[k];
            }
            t.ng[0] = t.e2[1] * t.e1[2] - t.e2[2] * t.e1[1];
            t.ng[1] = t.e2[2] * t.e1[0] - t.e2[0] * t.e1[2];
            t.ng[2] = t.e2[0] * t.e1[1] - t.e2[1] * t.e1[0];
            t.geom = geom_id;
            t.prim = i;
            tris.push_back(t);
            for (const float *p : {p0, p1, p2})
                for (int k = 0; k < 3; ++k) {
                    scene_lo[k] = std::min(scene_lo[k], p[k]);
                    scene_hi[k] = std::max(scene_hi[k], p[k]);
                }
        }
    }

    static void tri_bounds(const RcTri &t, float lo[3], float hi[3]) {
        for (int k = 0; k < 3; ++k) {
            float a = t.v0[k], b = t.v0[k] - t.e1[k], c = t.v0[k] + t.e2[k];
            lo[k] = std::min(a, std::min(b, c));
            hi[k] = std::max(a, std::max(b, c));
        }
    }

    void build() {
        {
            const int n = int(tris.size());
            std::vector<float> clo(3 * size_t(n)), chi(3 * size_t(n));
            for (int i = 0; i < n; ++i) tri_bounds(tris[i], &clo[3 * i], &chi[3 * i]);
            std::vector<int> idx;
            build_nodes(clo, chi, n, nodes, idx);
            std::vector<RcTri> sorted(n);
            for (int i = 0; i < n; ++i) sorted[i] = tris[idx[i]];
            tris.swap(sorted);
        }
        {
            const int n = int(users.size());
            std::vector<float> clo(3 * size_t(n)), chi(3 * size_t(n));
            for (int i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) { clo[3 * i + k] = users[i].lo[k]; chi[3 * i + k] = users[i].hi[k]; }
            std::vector<int> idx;
            build_nodes(clo, chi, n, unodes, idx);
            std::vector<RcUser> sorted(n);
            for (int i = 0; i < n; ++i) sorted[i] = users[idx[i]];
            users.swap(sorted);
        }
    }

    // binned-SAH BVH over n boxes; idx receives the leaf order of the boxes
    static void build_nodes(const std::vector<float> &clo, const std::vector<float> &chi, int n,
                            std::vector<RcNode> &nodes, std::vector<int> &idx) {
        nodes.clear();
        idx.assign(n, 0);
        if (n == 0) return;
        std::vector<float> cen(3 * size_t(n));
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) cen[3 * i + k] = 0.5f * (clo[3 * i + k] + chi[3 * i + k]);
        for (int i = 0; i < n; ++i) idx[i] = i;
        nodes.reserve(2 * size_t(n) / 2 + 1);
        struct Job { int node, first, count; };
        std::vector<Job> stack;
        nodes.push_back(RcNode());
        stack.push_back({0, 0, n});
        const int B = 16;
        while (!stack.empty()) {
            Job j = stack.back(); stack.pop_back();
            RcNode nd;
            float clo_[3] = {INFINITY, INFINITY, INFINITY}, chi_[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int k = 0; k < 3; ++k) { nd.lo[k] = INFINITY; nd.hi[k] = -INFINITY; }
            for (int i = j.first; i < j.first + j.count; ++i) {
                int t = idx[i];
                for (int k = 0; k < 3; ++k) {
                    nd.lo[k] = std::min(nd.lo[k], clo[3 * t + k]);
                    nd.hi[k] = std::max(nd.hi[k], chi[3 * t + k]);
                    clo_[k] = std::min(clo_[k], cen[3 * t + k]);
                    chi_[k] = std::max(chi_[k], cen[3 * t + k]);
                }
            }
            int best_axis = -1, best_bin = -1;
            double best_cost = INFINITY;
            if (j.count > 4) {
                for (int ax = 0; ax < 3; ++ax) {
                    float ext = chi_[ax] - clo_[ax];
                    if (!(ext > 0.f)) continue;
                    int cnt[B] = {0};
                    float blo[B][3], bhi[B][3];
                    for (int b = 0; b < B; ++b)
                        for (int k = 0; k < 3; ++k) { blo[b][k] = INFINITY; bhi[b][k] = -INFINITY; }
                    for (int i = j.first; i < j.first + j.count; ++i) {
                        int t = idx[i];
                        int b = std::min(B - 1, int((cen[3 * t + ax] - clo_[ax]) / ext * B));
                        cnt[b]++;
                        for (int k = 0; k < 3; ++k) {
                            blo[b][k] = std::min(blo[b][k], clo[3 * t + k]);
                            bhi[b][k] = std::max(bhi[b][k], chi[3 * t + k]);
                        }
                    }
                    double rarea[B]; int rcnt[B];
                    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
                    int c = 0;
                    for (int b = B - 1; b > 0; --b) {
                        c += cnt[b];
                        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], blo[b][k]); hi[k] = std::max(hi[k], bhi[b][k]); }
                        rcnt[b] = c;
                        double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
                        rarea[b] = c ? dx * dy + dy * dz + dz * dx : 0.0;
                    }
                    for (int k = 0; k < 3; ++k) { lo[k] = INFINITY; hi[k] = -INFINITY; }
                    c = 0;
                    for (int b = 0; b < B - 1; ++b) {
                        c += cnt[b];
                        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], blo[b][k]); hi[k] = std::max(hi[k], bhi[b][k]); }
                        double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
                        double la = c ? dx * dy + dy * dz + dz * dx : 0.0;
                        double cost = la * c + rarea[b + 1] * rcnt[b + 1];
                        if (c > 0 && rcnt[b + 1] > 0 && cost < best_cost) { best_cost = cost; best_axis = ax; best_bin = b; }
                    }
                }
            }
            if (best_axis < 0) {
                if (j.count <= 4) {
                    nd.first = j.first; nd.count = j.count;
                    nodes[j.node] = nd;
                    continue;
                }
                // degenerate centroids: split in the middle of the index range
                int half = j.count / 2;
                nd.left = int(nodes.size()); nodes.push_back(RcNode());
                nd.right = int(nodes.size()); nodes.push_back(RcNode());
                nodes[j.node] = nd;
                stack.push_back({nd.left, j.first, half});
                stack.push_back({nd.right, j.first + half, j.count - half});
                continue;
            }
            float ext = chi_[best_axis] - clo_[best_axis];
            auto mid = std::partition(idx.begin() + j.first, idx.begin() + j.first + j.count, [&](int t) {
                int b = std::min(B - 1, int((cen[3 * t + best_axis] - clo_[best_axis]) / ext * B));
                return b <= best_bin;
            });
            int nl = int(mid - (idx.begin() + j.first));
            if (nl == 0 || nl == j.count) nl = j.count / 2;
            nd.left = int(nodes.size()); nodes.push_back(RcNode());
            nd.right = int(nodes.size()); nodes.push_back(RcNode());
            nodes[j.node] = nd;
            stack.push_back({nd.left, j.first, nl});
            stack.push_back({nd.right, j.first + nl, j.count - nl});
        }
    }

    // Moeller-Trumbore as in triangle_intersector_moeller.h:78-111.
    static inline bool test(const RcTri &tr, const float o[3], const float d[3], float tnear, float tfar,
                            float *T_out, float *U_out, float *V_out, float *absden_out) {
        const float C[3] = {tr.v0[0] - o[0], tr.v0[1] - o[1], tr.v0[2] - o[2]};
        const float R[3] = {C[1] * d[2] - C[2] * d[1], C[2] * d[0] - C[0] * d[2], C[0] * d[1] - C[1] * d[0]};
        const float den = tr.ng[0] * d[0] + tr.ng[1] * d[1] + tr.ng[2] * d[2];
        const float absden = std::fabs(den);
        const float sgn = den < 0.f ? -1.f : 1.f;   // signmsk(den) xor: flips the sign of U, V, T
        const float U = (R[0] * tr.e2[0] + R[1] * tr.e2[1] + R[2] * tr.e2[2]) * sgn;
        const float V = (R[0] * tr.e1[0] + R[1] * tr.e1[1] + R[2] * tr.e1[2]) * sgn;
        if (!(den != 0.f && U >= 0.f && V >= 0.f && U + V <= absden)) return false;
        const float T = (tr.ng[0] * C[0] + tr.ng[1] * C[1] + tr.ng[2] * C[2]) * sgn;
        if (!(absden * tnear < T && T <= absden * tfar)) return false;
        *T_out = T; *U_out = U; *V_out = V; *absden_out = absden;
        return true;
    }

    static inline bool box_hit(const RcNode &nd, const float o[3], const float inv[3], float tnear, float tfar, float *tentry) {
        float t0 = tnear, t1 = tfar;
        for (int k = 0; k < 3; ++k) {
            float a = (nd.lo[k] - o[k]) * inv[k], b = (nd.hi[k] - o[k]) * inv[k];
            if (a > b) std::swap(a, b);
            if (!(a != a)) t0 = std::max(t0, a);
            if (!(b != b)) t1 = std::min(t1, b);
        }
        *tentry = t0;
        // a little slack so that boxes of flat triangles are never culled by rounding
        return t0 <= t1 * 1.0000005f + 1e-30f;
    }

    static inline bool user_box_hit(const RcUser &u, const float o[3], const float inv[3], float tnear, float tfar) {
        RcNode nd;
        for (int k = 0; k < 3; ++k) { nd.lo[k] = u.lo[k]; nd.hi[k] = u.hi[k]; }
        float te;
        return box_hit(nd, o, inv, tnear, tfar, &te);
    }

    bool closest(const float o[3], const float d[3], float tnear, float tfar, RcHit *hit) const {
        bool found = closest_tris(o, d, tnear, tfar, hit);
        if (found) tfar = hit->t;
        if (unodes.empty() || !user_closest) return found;
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
        int stack[128]; int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const RcNode &nd = unodes[stack[--sp]];
            float te;
            if (!box_hit(nd, o, inv, tnear, tfar, &te)) continue;
            if (nd.left < 0) {
                for (int i = nd.first; i < nd.first + nd.count; ++i) {
                    if (!user_box_hit(users[i], o, inv, tnear, tfar)) continue;
                    RcHit h;
                    if (user_closest(users[i], o, d, tnear, tfar, &h)) {
                        *hit = h;
                        tfar = h.t;
                        found = true;
                    }
                }
            } else {
                stack[sp++] = nd.right;
                stack[sp++] = nd.left;
            }
        }
        return found;
    }

    bool closest_tris(const float o[3], const float d[3], float tnear, float tfar, RcHit *hit) const {
        if (nodes.empty()) return false;
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
        int stack[128]; int sp = 0;
        stack[sp++] = 0;
        bool found = false;
        while (sp) {
            const RcNode &nd = nodes[stack[--sp]];
            float te;
            if (!box_hit(nd, o, inv, tnear, tfar, &te)) continue;
            if (nd.left < 0) {
                for (int i = nd.first; i < nd.first + nd.count; ++i) {
                    float T, U, V, ad;
                    if (test(tris[i], o, d, tnear, tfar, &T, &U, &V, &ad)) {
                        float t = T / ad;
                        if (t < hit->t || !found) {
                            hit->t = t; hit->u = U / ad; hit->v = V / ad;
                            for (int k = 0; k < 3; ++k) hit->ng[k] = tris[i].ng[k];
                            hit->geom = tris[i].geom; hit->prim = tris[i].prim;
                            tfar = t;
                            found = true;
                        }
                    }
                }
            } else {
                float tl, tr;
                bool hl = box_hit(nodes[nd.left], o, inv, tnear, tfar, &tl);
                bool hr = box_hit(nodes[nd.right], o, inv, tnear, tfar, &tr);
                if (hl && hr) {
                    if (tl <= tr) { stack[sp++] = nd.right; stack[sp++] = nd.left; }
                    else { stack[sp++] = nd.left; stack[sp++] = nd.right; }
                } else if (hl) stack[sp++] = nd.left;
                else if (hr) stack[sp++] = nd.right;
            }
        }
        return found;
    }

    bool occluded(const float o[3], const float d[3], float tnear, float tfar) const {
        if (occluded_tris(o, d, tnear, tfar)) return true;
        if (unodes.empty() || !user_any) return false;
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
        int stack[128]; int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const RcNode &nd = unodes[stack[--sp]];
            float te;
            if (!box_hit(nd, o, inv, tnear, tfar, &te)) continue;
            if (nd.left < 0) {
                for (int i = nd.first; i < nd.first + nd.count; ++i)
                    if (user_box_hit(users[i], o, inv, tnear, tfar) && user_any(users[i], o, d, tnear, tfar)) return true;
            } else {
                stack[sp++] = nd.right;
                stack[sp++] = nd.left;
            }
        }
        return false;
    }

    // Occlusion bounds for checking another ray caster's any-hit answers. Each triangle is tested
    // in FP64 from its float vertices: *hi = the segment may be blocked (a triangle grown by eps in
    // barycentric coordinates, or a hit within eps * max(|t|, 1) outside either end of the segment),
    // *lo = it is blocked beyond doubt (a triangle shrunk by eps, the segment shortened by the same
    // tolerance, and a ray not grazing the plane: |cos| >= 1e-4). Two correct FP32 tests of the same
    // ray -- Embree's and a watertight one -- answer between *lo and *hi. User primitives count for
    // both bounds through user_any on the shortened / lengthened segment.
    void occluded_bracket(const float o[3], const float d[3], float tnear, float tfar, double eps,
                          bool *lo, bool *hi) const {
        *lo = false;
        *hi = false;
        const double tol_n = eps * std::max(std::fabs(double(tnear)), 1.0);
        const bool far_inf = std::isinf(tfar);
        const double tol_f = far_inf ? 0.0 : eps * std::max(std::fabs(double(tfar)), 1.0);
        const double n_hi = double(tnear) - tol_n, f_hi = double(tfar) + tol_f;   // lengthened
        const double n_lo = double(tnear) + tol_n, f_lo = double(tfar) - tol_f;   // shortened
        double diag = 0.0;
        for (int k = 0; k < 3; ++k) diag = std::max(diag, double(scene_hi[k]) - double(scene_lo[k]));
        const float margin = float(4.0 * eps * diag) + 1e-6f;
        const double dd[3] = {d[0], d[1], d[2]};
        const double dlen = std::sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
        if (!nodes.empty()) {
            int stack[128]; int sp = 0;
            stack[sp++] = 0;
            while (sp && !*lo) {
                RcNode nd = nodes[stack[--sp]];
                for (int k = 0; k < 3; ++k) { nd.lo[k] -= margin; nd.hi[k] += margin; }
                float te;
                if (!box_hit(nd, o, inv, float(n_hi), float(f_hi) * 1.0001f, &te)) continue;
                if (nd.left >= 0) {
                    stack[sp++] = nd.right;
                    stack[sp++] = nd.left;
                    continue;
                }
                for (int i = nd.first; i < nd.first + nd.count; ++i) {
                    const RcTri &tr = tris[i];
                    double e1[3], e2[3], C[3];
                    for (int k = 0; k < 3; ++k) {
                        e1[k] = double(tr.e1[k]);
                        e2[k] = double(tr.e2[k]);
                        C[k] = double(tr.v0[k]) - double(o[k]);
                    }
                    const double ng[3] = {e2[1] * e1[2] - e2[2] * e1[1], e2[2] * e1[0] - e2[0] * e1[2],
                                          e2[0] * e1[1] - e2[1] * e1[0]};
                    const double R[3] = {C[1] * dd[2] - C[2] * dd[1], C[2] * dd[0] - C[0] * dd[2],
                                         C[0] * dd[1] - C[1] * dd[0]};
                    const double den = ng[0] * dd[0] + ng[1] * dd[1] + ng[2] * dd[2];
                    const double absden = std::fabs(den);
                    if (!(absden > 0.0)) continue;
                    const double sgn = den < 0.0 ? -1.0 : 1.0;
                    const double u = (R[0] * e2[0] + R[1] * e2[1] + R[2] * e2[2]) * sgn / absden;
                    const double v = (R[0] * e1[0] + R[1] * e1[1] + R[2] * e1[2]) * sgn / absden;
                    const double t = (ng[0] * C[0] + ng[1] * C[1] + ng[2] * C[2]) * sgn / absden;
                    const double nlen = std::sqrt(ng[0] * ng[0] + ng[1] * ng[1] + ng[2] * ng[2]);
                    const double cosv = absden / (nlen * dlen);
                    if (u >= -eps && v >= -eps && u + v <= 1.0 + eps && t > n_hi && (far_inf || t <= f_hi))
                        *hi = true;
                    if (cosv >= 1e-4 && u >= eps && v >= eps && u + v <= 1.0 - eps && t > n_lo && (far_inf || t <= f_lo)) {
                        *lo = true;
                        break;
                    }
                }
            }
        }
        if (!*lo && !unodes.empty() && user_any) {
            if (occluded_users(o, d, float(n_lo), far_inf ? tfar : float(f_lo))) *lo = true;
            if (occluded_users(o, d, float(n_hi), far_inf ? tfar : float(f_hi))) *hi = true;
        }
        if (*lo) *hi = true;
    }

    bool occluded_users(const float o[3], const float d[3], float tnear, float tfar) const {
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
        int stack[128]; int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const RcNode &nd = unodes[stack[--sp]];
            float te;
            if (!box_hit(nd, o, inv, tnear, tfar, &te)) continue;
            if (nd.left < 0) {
                for (int i = nd.first; i < nd.first + nd.count; ++i)
                    if (user_box_hit(users[i], o, inv, tnear, tfar) && user_any(users[i], o, d, tnear, tfar)) return true;
            } else {
                stack[sp++] = nd.right;
                stack[sp++] = nd.left;
            }
        }
        return false;
    }

    bool occluded_tris(const float o[3], const float d[3], float tnear, float tfar) const {
        if (nodes.empty()) return false;
        float inv[3];
        for (int k = 0; k < 3; ++k) inv[k] = 1.0f / d[k];
        int stack[128]; int sp = 0;
        stack[sp++] = 0;
        while (sp) {
            const RcNode &nd = nodes[stack[--sp]];
            float te;
            if (!box_hit(nd, o, inv, tnear, tfar, &te)) continue;
            if (nd.left < 0) {
                for (int i = nd.first; i < nd.first + nd.count; ++i) {
                    float T, U, V, ad;
                    if (test(tris[i], o, d, tnear, tfar, &T, &U, &V, &ad)) return true;
                }
            } else {
                stack[sp++] = nd.right;
                stack[sp++] = nd.left;
            }
        }
        return false;
    }
};

}  // namespace oracle
