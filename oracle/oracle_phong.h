// Test infrastructure only: the oracle's FP64 restatement of the reference's
// Phong tessellation patches (src/geometry/phongmesh.h), the geometry a simple2
// mesh entry with "phong_tessellation": true becomes
// (src/sceneio/simple2parser.h:37-55).
//
// A patch is one triangle (p1, p2, p3) with unit vertex normals (n1, n2, n3) and
// the shape factor alpha = 3/4 (phongmesh.h:46). The surface is Boubekeur and
// Alexa's Phong tessellation
//     p*(u, v) = (1 - alpha) p(u, v) + alpha sum_i w_i pi_i(p(u, v)),
// with p(u, v) = u p1 + v p2 + w p3 the flat point and pi_i the projection onto
// the tangent plane of vertex i (phongmesh.h:24-33). The ray test is the
// algebraic one of the reference (phongmesh.h:178-368): the ray is written as
// the intersection of two planes, each plane meets the patch in a conic in
// (u, v), a cubic in the pencil parameter x picks a degenerate member of the
// pencil (a line pair), and each line is substituted back into the first conic,
// leaving a quadratic. The patch bound is the reference's (phongmesh.h:61-164):
// the flat triangle thickened along its normal by the patch height at the
// extremum (u^, v^) of eq. 21-22, and pushed out across each edge by the
// "side drop" of eq. 23.
//
// The arithmetic is written out operation by operation in the order the
// reference's expressions evaluate (left to right, with its vector helpers'
// component-wise products and left-to-right dot sums), so that, compiled
// without floating-point contraction, every double matches the reference's.
// One deliberate difference: when no root of the cubic has a finite selection
// cost (all candidate costs NaN, which happens for a flat patch whose vertex
// normals all equal the face normal), the reference goes on with an
// uninitialised root; this restatement reports no intersection.
#pragma once

#include <algorithm>
#include <cmath>
#include <limits>

namespace oracle {
namespace phong {

struct D3 { double x = 0.0, y = 0.0, z = 0.0; };

inline D3 d3(double x, double y, double z) { D3 r; r.x = x; r.y = y; r.z = z; return r; }
inline D3 add(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline D3 sub(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline D3 scl(double s, D3 a) { return d3(s * a.x, s * a.y, s * a.z); }
inline D3 scr(D3 a, double s) { return d3(a.x * s, a.y * s, a.z * s); }   // vec * scalar
inline double dot(D3 a, D3 b) { double s = a.x * b.x; s += a.y * b.y; s += a.z * b.z; return s; }
inline D3 cross(D3 u, D3 v) { return d3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x); }
inline double length(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 normalize(D3 a) { const double l = length(a); return d3(a.x / l, a.y / l, a.z / l); }
inline double comp(D3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
inline double dmax(double a, double b) { return a < b ? b : a; }   // std::max

constexpr double kPi = 3.141592653589793238462643383279502884197169399375105820974;
constexpr double kSmall = 1e-12;
constexpr double kAlpha = 3.0 / 4.0;

// Math::IsApprox(a, 0.0) (src/common/math/scalarmath.h:112-119)
inline bool is_approx_zero(double a) {
    const double absA = std::abs(a), absB = 0.0;
    const double larger = absA < absB ? absB : absA;
    return std::abs(a - 0.0) <= dmax(larger * kSmall, kSmall);
}

// Math::SolveQuadratic (scalarmath.h:144-162)
inline bool solve_quadratic(double *x0, double *x1, double a, double b, double c) {
    if (is_approx_zero(a)) {
        const double ans = -c / b;
        *x0 = ans; *x1 = ans;
        return true;
    }
    const double disc = b * b - 4.0 * a * c;
    if (disc < 0) return false;
    const double sq = std::sqrt(disc);
    const double q = (b > 0) ? -0.5 * (b + sq) : -0.5 * (b - sq);
    *x0 = q / a;
    *x1 = c / q;
    return true;
}

// Math::SolveRealCubic (scalarmath.h:167-207): roots of ua x^3 + ub x^2 + uc x + ud
inline int solve_real_cubic(double *xs, double ua, double ub, double uc, double ud) {
    if (is_approx_zero(ua)) return solve_quadratic(&xs[0], &xs[1], ub, uc, ud) ? 2 : 0;
    const double b = ub / ua, c = uc / ua, d = ud / ua;
    const double b2 = b * b;
    const double bBy3 = b / 3.0;
    const double q = (3.0 * c - b2) / 9.0;
    const double q3 = q * q * q;
    const double r = -d * 0.5 + b * (9.0 * c - 2.0 * b2) / 54.0;
    const double disc = q3 + r * r;
    if (disc > 0) {
        const double sqrtDisc = std::sqrt(disc);
        xs[0] = -bBy3 + std::cbrt(r + sqrtDisc) + std::cbrt(r - sqrtDisc);
        return 1;
    } else if (disc == 0) {
        const double r13 = std::cbrt(r);
        xs[0] = -bBy3 + 2.0 * r13;
        xs[1] = -(r13 + bBy3);
        return 2;
    }
    const double dum1 = std::acos(r / std::sqrt(-q3));
    const double r13 = 2.0 * std::sqrt(-q);
    xs[0] = -bBy3 + r13 * std::cos(dum1 / 3.0);
    xs[1] = -bBy3 + r13 * std::cos((dum1 + 2.0 * kPi) / 3.0);
    xs[2] = -bBy3 + r13 * std::cos((dum1 + 4.0 * kPi) / 3.0);
    return 3;
}

struct Patch {
    D3 p[3], n[3];   // positions (from float) and unit normals, vertex order of the triangle
};

// the per-patch edge (e) and normal-curvature (c) vectors of phongmesh.h:80-91, 1-based as there
struct Coeffs {
    D3 e12, e23, e31, c12, c23, c31;
};

inline D3 c_of(const D3 &ni, const D3 &nj, const D3 &eij) {
    // alpha * (Dot(n_j, e_ij) n_j - Dot(n_i, e_ij) n_i)
    return scl(kAlpha, sub(scl(dot(nj, eij), nj), scl(dot(ni, eij), ni)));
}

inline Coeffs coeffs(const Patch &P) {
    Coeffs k;
    k.e12 = sub(P.p[1], P.p[0]);
    k.e23 = sub(P.p[2], P.p[1]);
    k.e31 = sub(P.p[0], P.p[2]);
    k.c12 = c_of(P.n[0], P.n[1], k.e12);
    k.c23 = c_of(P.n[1], P.n[2], k.e23);
    k.c31 = c_of(P.n[2], P.n[0], k.e31);
    return k;
}

// EvalPhongTessellationPosition (phongmesh.h:24-33); weights u, v, 1 - u - v on p1, p2, p3
inline D3 eval_position(const Patch &P, double u, double v) {
    const double w = 1.0 - u - v;
    const D3 puv = add(add(scl(u, P.p[0]), scl(v, P.p[1])), scl(w, P.p[2]));
    D3 pi[3];
    for (int i = 0; i < 3; ++i) pi[i] = sub(puv, scl(dot(sub(puv, P.p[i]), P.n[i]), P.n[i]));
    const D3 pStar = add(add(scl(u, pi[0]), scl(v, pi[1])), scl(w, pi[2]));
    return add(scl(1.0 - kAlpha, puv), scl(kAlpha, pStar));
}

// EvalPhongTessellationNormal (phongmesh.h:35-44, eq. 29)
inline D3 eval_normal(const Coeffs &k, double u, double v) {
    const double w = 1.0 - u - v;
    const D3 dpdu = add(add(scl(w - u, k.c31), scl(v, sub(k.c12, k.c23))), k.e31);
    const D3 dpdv = sub(add(scl(w - v, k.c23), scl(u, sub(k.c12, k.c31))), k.e23);
    return normalize(cross(dpdu, dpdv));
}

// PhongMeshGeometry::bound(primitiveIndex) (phongmesh.h:61-164)
inline void bound(const Patch &P, double lo[3], double hi[3]) {
    const Coeffs k = coeffs(P);
    const D3 ng = normalize(cross(sub(P.p[1], P.p[0]), sub(P.p[2], P.p[0])));
    const D3 c31e31 = add(k.c31, k.e31);
    const D3 c23e23 = sub(k.c23, k.e23);
    const D3 c122331 = sub(sub(k.c12, k.c23), k.c31);
    const double den = 4.0 * dot(ng, k.c23) * dot(ng, k.c31) - dot(ng, c122331);
    const double kk = 1.0 / (den * den);
    const double uhat = kk * (2.0 * dot(ng, k.c23) * dot(ng, c31e31) + dot(ng, c23e23) * dot(ng, c122331));
    const double vhat = kk * (2.0 * dot(ng, k.c31) * dot(ng, c23e23) + dot(ng, c31e31) * dot(ng, c122331));
    auto height = [&](double u, double v) { return dot(ng, sub(eval_position(P, u, v), P.p[0])); };
    double thickness = 0.0;
    const bool uok = uhat >= 0.0 && uhat <= 1.0;
    const bool vok = vhat >= 0.0 && vhat <= 1.0;
    if (uok && vok && uhat + vhat <= 1.0) {
        thickness = height(uhat, vhat);
    } else {
        const double a = uok ? height(uhat, 0.0) : 0.0;
        const double b = vok ? height(0.0, vhat) : 0.0;
        thickness = dmax(a, b);
    }
    for (int c = 0; c < 3; ++c) {
        lo[c] = std::numeric_limits<double>::max();
        hi[c] = std::numeric_limits<double>::lowest();
    }
    auto grow = [&](const D3 &q) {
        for (int c = 0; c < 3; ++c) {
            lo[c] = std::min(lo[c], comp(q, c));
            hi[c] = std::max(hi[c], comp(q, c));
        }
    };
    if (thickness == 0.0) {
        for (int i = 0; i < 3; ++i) grow(P.p[i]);
        return;
    }
    // eq. 23: distance of the patch point at each edge midpoint from each edge line
    double sidedrops[3] = {0.0, 0.0, 0.0};
    const double uvws[3][2] = {{0.0, 0.5}, {0.5, 0.0}, {0.5, 0.5}};
    for (int m = 0; m < 3; ++m) {
        const D3 pa = eval_position(P, uvws[m][0], uvws[m][1]);
        for (int e = 0; e < 3; ++e) {
            const D3 &pi = P.p[e], &pj = P.p[(e + 1) % 3];
            const double s = length(cross(sub(pj, pa), sub(pi, pa))) / length(sub(pj, pi));
            sidedrops[e] = dmax(s, sidedrops[e]);
        }
    }
    for (int e = 0; e < 3; ++e) {
        const D3 &pi = P.p[e], &pj = P.p[(e + 1) % 3];
        const D3 x = normalize(sub(pj, pi));
        const D3 z = cross(x, ng);
        const D3 vi = add(scr(z, sidedrops[e]), pi);
        const D3 vj = add(scr(z, sidedrops[e]), pj);
        grow(vi);
        grow(vj);
        grow(add(vi, scr(ng, thickness)));
        grow(add(vj, scr(ng, thickness)));
    }
}

// PhongMeshGeometry::intersect (phongmesh.h:178-368) for a ray given in float,
// as Embree hands it to the user-geometry callback (embreeaccel.h:77-99).
// On a hit in [tmin, *tmax] updates *tmax and the unit normal; returns whether it did.
inline bool intersect(const Patch &P, const float of[3], const float df[3], float tminf, double *tmax, D3 *normal) {
    const D3 org = d3(of[0], of[1], of[2]);
    const D3 dir = d3(df[0], df[1], df[2]);
    const double tmin = tminf;
    // Math::MaxDimension: first index of the largest (signed) component
    int axis = 0;
    double mx = dir.x;
    if (dir.y > mx) { axis = 1; mx = dir.y; }
    if (dir.z > mx) { axis = 2; mx = dir.z; }
    // TwoPlanesFromRay with CoordFrame3(direction) (coordframe.h:50-60)
    const double sign = std::copysign(1.0, dir.y);
    const double fa = -1.0 / (sign + dir.y);
    const double fb = dir.z * dir.x * fa;
    const D3 fx = d3(sign + dir.x * dir.x * fa, -dir.x, fb);
    const D3 fz = d3(sign * fb, -sign * dir.z, 1.0 + sign * dir.z * dir.z * fa);
    const D3 d1 = cross(fx, dir);
    const double o1 = -dot(org, d1);
    const D3 d2 = cross(fz, dir);
    const double o2 = -dot(org, d2);

    const Coeffs k = coeffs(P);
    const D3 c123 = sub(sub(k.c12, k.c23), k.c31);
    const D3 ce31 = add(k.c31, k.e31);
    const D3 ce23 = sub(k.c23, k.e23);
    // eq. 5-6
    const double a = -dot(d1, k.c31);
    const double b = -dot(d1, k.c23);
    const double c = dot(d1, P.p[2]) + o1;
    const double d = dot(d1, c123);
    const double e = dot(d1, ce31);
    const double f = dot(d1, ce23);
    const double l = -dot(d2, k.c31);
    const double m = -dot(d2, k.c23);
    const double n = dot(d2, P.p[2]) + o2;
    const double o = dot(d2, c123);
    const double p = dot(d2, ce31);
    const double q = dot(d2, ce23);
    // eq. 16
    const double a3 = a * b * c + (d * e * f - a * f * f - b * e * e - c * d * d) * 0.25;
    const double a2 = a * b * n + a * m * c + l * b * c - (a * f * q + b * e * p + c * d * o) * 0.5 +
                      (o * e * f + d * e * q + d * p * f - l * f * f - m * e * e - n * d * d) * 0.25;
    const double a1 = a * m * n + l * b * n + l * m * c - (l * f * q + m * e * p + n * d * o) * 0.5 +
                      (d * p * q + o * e * q + o * p * f - a * q * q - b * p * p - c * o * o) * 0.25;
    const double a0 = l * m * n + (o * p * q - l * q * q - m * p * p - n * o * o) * 0.25;

    double xs[3] = {0.0, 0.0, 0.0};
    const int numXs = solve_real_cubic(xs, a3, a2, a1, a0);
    if (numXs == 0) return false;
    // the root with the smallest M12^2 - M11 M22 (section 3.2)
    double x = 0.0, minCost = std::numeric_limits<double>::infinity();
    bool chosen = false;
    for (int i = 0; i < numXs; ++i) {
        const double m11 = xs[i] * a + l;
        const double m22 = xs[i] * b + m;
        const double m12 = (xs[i] * d + o) * 0.5;
        const double cost = m12 * m12 - m11 * m22;
        if (cost < minCost) { x = xs[i]; minCost = cost; chosen = true; }
    }
    if (minCost < 0) return false;
    if (!chosen) return false;   // the reference reads an uninitialised root here

    const double m11 = x * a + l;
    const double m22 = x * b + m;
    const bool greater = std::abs(m11) > std::abs(m22);
    double albeta[2], gamma[2];
    if (greater) {
        const double inv = 1.0 / m11;
        const double mp22 = m22 * inv;
        const double mp33 = (x * c + n) * inv;
        const double mp12 = (x * d + o) * 0.5 * inv;
        const double mp13 = (x * e + p) * 0.5 * inv;
        const double mp23 = (x * f + q) * 0.5 * inv;
        const double bs = std::sqrt(mp12 * mp12 - mp22);
        const double gs = std::sqrt(mp13 * mp13 - mp33);
        albeta[0] = mp12 + bs; albeta[1] = mp12 - bs;
        gamma[0] = mp13 + gs; gamma[1] = mp13 - gs;
        const double diffA = std::abs((2.0 * mp23) - (albeta[0] * gamma[0] + albeta[1] * gamma[1]));
        const double diffB = std::abs((2.0 * mp23) - (albeta[0] * gamma[1] + albeta[1] * gamma[0]));
        if (diffA < diffB) std::swap(gamma[0], gamma[1]);
    } else {
        const double inv = 1.0 / m22;
        const double mp11 = m11 * inv;
        const double mp12 = (x * d + o) * 0.5 * inv;
        const double mp13 = (x * e + p) * 0.5 * inv;
        const double mp23 = (x * f + q) * 0.5 * inv;
        const double mp33 = (x * c + n) * inv;
        const double as = std::sqrt(mp12 * mp12 - mp11);
        const double gs = std::sqrt(mp23 * mp23 - mp33);
        albeta[0] = mp12 + as; albeta[1] = mp12 - as;
        gamma[0] = mp23 + gs; gamma[1] = mp23 - gs;
        const double diffA = std::abs((2.0 * mp13) - (albeta[0] * gamma[0] + albeta[1] * gamma[1]));
        const double diffB = std::abs((2.0 * mp13) - (albeta[0] * gamma[1] + albeta[1] * gamma[0]));
        if (diffA < diffB) std::swap(gamma[0], gamma[1]);
    }
    bool hit = false;
    for (int i = 0; i < 2; ++i) {
        const double g = -albeta[i];
        const double h = -gamma[i];
        double k2, k1, k0;
        if (greater) {   // u = g v + h
            k2 = a * g * g + b + d * g;
            k1 = 2.0 * a * g * h + d * h + e * g + f;
            k0 = a * h * h + c + e * h;
        } else {         // v = g u + h
            k2 = a + b * g * g + d * g;
            k1 = 2.0 * b * g * h + d * h + e + f * g;
            k0 = b * h * h + c + f * h;
        }
        double ans[2];
        if (!solve_quadratic(&ans[0], &ans[1], k2, k1, k0)) continue;
        for (int j = 0; j < 2; ++j) {
            double u, v;
            if (greater) { v = ans[j]; u = g * v + h; }
            else { u = ans[j]; v = g * u + h; }
            const double w = 1.0 - u - v;
            if (!(v >= 0.0 && u >= 0.0 && w >= 0.0)) continue;
            const D3 pos = eval_position(P, u, v);
            const double t = (comp(pos, axis) - comp(org, axis)) / comp(dir, axis);
            if (*tmax >= t && tmin <= t) {
                hit = true;
                *tmax = t;
                *normal = eval_normal(k, u, v);
            }
        }
    }
    return hit;
}

}  // namespace phong
}  // namespace oracle
