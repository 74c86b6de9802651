// Phong tessellation patches: the surface a simple2 mesh entry with
// "phong_tessellation": true turns its (non-emitting) triangles into
// (PhongMeshGeometry, src/geometry/phongmesh.h; src/sceneio/simple2parser.h:37-55).
//
// A patch is a triangle p1 p2 p3 with unit vertex normals n1 n2 n3 and shape factor
// alpha = 3/4. Its surface is Boubekeur and Alexa's Phong tessellation: the flat point
// p(u, v) = u p1 + v p2 + w p3 blended with the barycentric combination of its
// projections onto the three vertex tangent planes,
//     p*(u, v) = (1 - alpha) p(u, v) + alpha sum_i w_i (p - ((p - p_i) . n_i) n_i).
// The ray test is the reference's algebraic one (phongmesh.h:178-368): the ray is the
// intersection of two planes through it; each plane cuts the patch in a conic in (u, v);
// the cubic of eq. 16 picks the degenerate member of the pencil of the two conics (a
// line pair); each line, substituted back into the first conic, leaves a quadratic whose
// roots inside the triangle are the candidate hits, with t measured along the ray's
// largest (signed) direction component. The bound is the reference's (phongmesh.h:61-164):
// the flat triangle, thickened along its normal by the patch height at the extremum of
// eq. 21-22, pushed out across each edge by the side drop of eq. 23.
//
// Everything runs in FP64. The code is templated on the scalar: the host instantiates it
// with double (the bound, at scene build), the device with `Rd`, a double whose
// operators are the explicitly rounded __dadd_rn / __dmul_rn / ... so that no multiply-add
// is contracted into an FMA. Each expression is written in the reference's evaluation
// order (left to right, component-wise vector products, left-to-right dot sums), so every
// add, multiply, divide and square root rounds exactly as the reference's do; only cbrt,
// acos and cos come from CUDA's library instead of the host's.
//
// Where the reference reads an uninitialised root (no root of the cubic has a finite
// selection cost -- a flat patch whose vertex normals all equal its face normal) this code
// reports no intersection.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>

#ifdef __CUDACC__
#define WRP_HD __host__ __device__ __forceinline__
#else
#define WRP_HD inline
#endif

namespace wrp {

constexpr uint32_t kPatchFlag = 0x80000000u;   // set in the leaf record's first .w word
constexpr int kPatchDoubles = 12;               // n1 n2 n3 (9 doubles) + float box lo/hi (6 floats)
constexpr double kAlpha = 3.0 / 4.0;
constexpr double kPi = 3.141592653589793238462643383279502884197169399375105820974;
constexpr double kSmall = 1e-12;                // Math::SmallValue

#ifdef __CUDACC__
// FP64 scalar with explicitly rounded device operations (no contraction); the host side of
// these operators (never used for rendering) is plain double arithmetic
#ifdef __CUDA_ARCH__
#define WRP_OP(dev, host) return Rd(dev)
#else
#define WRP_OP(dev, host) return Rd(host)
#endif
struct Rd {
    double v;
    Rd() = default;
    __host__ __device__ __forceinline__ constexpr Rd(double x) : v(x) {}
};
__host__ __device__ __forceinline__ Rd operator+(Rd a, Rd b) { WRP_OP(__dadd_rn(a.v, b.v), a.v + b.v); }
__host__ __device__ __forceinline__ Rd operator-(Rd a, Rd b) { WRP_OP(__dsub_rn(a.v, b.v), a.v - b.v); }
__host__ __device__ __forceinline__ Rd operator*(Rd a, Rd b) { WRP_OP(__dmul_rn(a.v, b.v), a.v * b.v); }
__host__ __device__ __forceinline__ Rd operator/(Rd a, Rd b) { WRP_OP(__ddiv_rn(a.v, b.v), a.v / b.v); }
__host__ __device__ __forceinline__ Rd sqrt_(Rd a) { WRP_OP(__dsqrt_rn(a.v), std::sqrt(a.v)); }
#undef WRP_OP
__host__ __device__ __forceinline__ Rd operator-(Rd a) { return Rd(-a.v); }
__host__ __device__ __forceinline__ bool operator<(Rd a, Rd b) { return a.v < b.v; }
__host__ __device__ __forceinline__ bool operator>(Rd a, Rd b) { return a.v > b.v; }
__host__ __device__ __forceinline__ bool operator<=(Rd a, Rd b) { return a.v <= b.v; }
__host__ __device__ __forceinline__ bool operator>=(Rd a, Rd b) { return a.v >= b.v; }
__host__ __device__ __forceinline__ bool operator==(Rd a, Rd b) { return a.v == b.v; }
__host__ __device__ __forceinline__ Rd cbrt_(Rd a) { return Rd(cbrt(a.v)); }
__host__ __device__ __forceinline__ Rd acos_(Rd a) { return Rd(acos(a.v)); }
__host__ __device__ __forceinline__ Rd cos_(Rd a) { return Rd(cos(a.v)); }
__host__ __device__ __forceinline__ Rd abs_(Rd a) { return Rd(fabs(a.v)); }
__host__ __device__ __forceinline__ Rd copysign_(Rd a, Rd b) { return Rd(copysign(a.v, b.v)); }
#endif

WRP_HD double sqrt_(double a) { return sqrt(a); }
WRP_HD double cbrt_(double a) { return cbrt(a); }
WRP_HD double acos_(double a) { return acos(a); }
WRP_HD double cos_(double a) { return cos(a); }
WRP_HD double abs_(double a) { return fabs(a); }
WRP_HD double copysign_(double a, double b) { return copysign(a, b); }

template <class T> struct V {
    T x, y, z;
};
template <class T> WRP_HD V<T> v3(T x, T y, T z) { return V<T>{x, y, z}; }
template <class T> WRP_HD V<T> operator+(V<T> a, V<T> b) { return v3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> WRP_HD V<T> operator-(V<T> a, V<T> b) { return v3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> WRP_HD V<T> operator*(T s, V<T> a) { return v3<T>(s * a.x, s * a.y, s * a.z); }
template <class T> WRP_HD V<T> operator*(V<T> a, T s) { return v3<T>(a.x * s, a.y * s, a.z * s); }
template <class T> WRP_HD T dot(V<T> a, V<T> b) {
    T s = a.x * b.x;
    s = s + a.y * b.y;
    s = s + a.z * b.z;
    return s;
}
template <class T> WRP_HD V<T> cross(V<T> u, V<T> v) {
    return v3<T>(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
}
template <class T> WRP_HD T length(V<T> a) { return sqrt_(dot(a, a)); }
template <class T> WRP_HD V<T> normalize(V<T> a) {
    const T l = length(a);
    return v3<T>(a.x / l, a.y / l, a.z / l);
}
template <class T> WRP_HD T comp(V<T> a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
template <class T> WRP_HD T tmax_(T a, T b) { return a < b ? b : a; }   // std::max

// Math::IsApprox(a, 0) (src/common/math/scalarmath.h:112-119)
template <class T> WRP_HD bool is_approx_zero(T a) {
    const T absA = abs_(a), absB = T(0.0);
    const T larger = absA < absB ? absB : absA;
    return abs_(a - T(0.0)) <= tmax_(larger * T(kSmall), T(kSmall));
}

// Math::SolveQuadratic (scalarmath.h:144-162)
template <class T> WRP_HD bool solve_quadratic(T &x0, T &x1, T a, T b, T c) {
    if (is_approx_zero(a)) {
        const T ans = -c / b;
        x0 = ans;
        x1 = ans;
        return true;
    }
    const T disc = b * b - T(4.0) * a * c;
    if (disc < T(0.0)) return false;
    const T sq = sqrt_(disc);
    const T q = (b > T(0.0)) ? T(-0.5) * (b + sq) : T(-0.5) * (b - sq);
    x0 = q / a;
    x1 = c / q;
    return true;
}

// Math::SolveRealCubic (scalarmath.h:167-207): real roots of ua x^3 + ub x^2 + uc x + ud
template <class T> WRP_HD int solve_real_cubic(T xs[3], T ua, T ub, T uc, T ud) {
    if (is_approx_zero(ua)) return solve_quadratic(xs[0], xs[1], ub, uc, ud) ? 2 : 0;
    const T b = ub / ua, c = uc / ua, d = ud / ua;
    const T b2 = b * b;
    const T bBy3 = b / T(3.0);
    const T q = (T(3.0) * c - b2) / T(9.0);
    const T q3 = q * q * q;
    const T r = -d * T(0.5) + b * (T(9.0) * c - T(2.0) * b2) / T(54.0);
    const T disc = q3 + r * r;
    if (disc > T(0.0)) {
        const T sd = sqrt_(disc);
        xs[0] = -bBy3 + cbrt_(r + sd) + cbrt_(r - sd);
        return 1;
    }
    if (disc == T(0.0)) {
        const T r13 = cbrt_(r);
        xs[0] = -bBy3 + T(2.0) * r13;
        xs[1] = -(r13 + bBy3);
        return 2;
    }
    const T dum1 = acos_(r / sqrt_(-q3));
    const T r13 = T(2.0) * sqrt_(-q);
    xs[0] = -bBy3 + r13 * cos_(dum1 / T(3.0));
    xs[1] = -bBy3 + r13 * cos_((dum1 + T(2.0) * T(kPi)) / T(3.0));
    xs[2] = -bBy3 + r13 * cos_((dum1 + T(4.0) * T(kPi)) / T(3.0));
    return 3;
}

template <class T> struct Patch {
    V<T> p[3], n[3];
};

// edge vectors e_ij = p_j - p_i and curvature vectors c_ij of phongmesh.h:80-91
template <class T> struct Coeffs {
    V<T> e12, e23, e31, c12, c23, c31;
};

template <class T> WRP_HD V<T> curvature(V<T> ni, V<T> nj, V<T> eij) {
    return T(kAlpha) * (dot(nj, eij) * nj - dot(ni, eij) * ni);
}

template <class T> WRP_HD Coeffs<T> coeffs(const Patch<T> &P) {
    Coeffs<T> k;
    k.e12 = P.p[1] - P.p[0];
    k.e23 = P.p[2] - P.p[1];
    k.e31 = P.p[0] - P.p[2];
    k.c12 = curvature(P.n[0], P.n[1], k.e12);
    k.c23 = curvature(P.n[1], P.n[2], k.e23);
    k.c31 = curvature(P.n[2], P.n[0], k.e31);
    return k;
}

// p*(u, v), weights u, v, 1 - u - v on p1, p2, p3 (phongmesh.h:24-33)
template <class T> WRP_HD V<T> eval_position(const Patch<T> &P, T u, T v) {
    const T w = T(1.0) - u - v;
    const V<T> puv = u * P.p[0] + v * P.p[1] + w * P.p[2];
    const V<T> pi0 = puv - dot(puv - P.p[0], P.n[0]) * P.n[0];
    const V<T> pi1 = puv - dot(puv - P.p[1], P.n[1]) * P.n[1];
    const V<T> pi2 = puv - dot(puv - P.p[2], P.n[2]) * P.n[2];
    const V<T> ps = u * pi0 + v * pi1 + w * pi2;
    return T(1.0 - kAlpha) * puv + T(kAlpha) * ps;
}

// unit normal dp/du x dp/dv (phongmesh.h:35-44, eq. 29)
template <class T> WRP_HD V<T> eval_normal(const Coeffs<T> &k, T u, T v) {
    const T w = T(1.0) - u - v;
    const V<T> dpdu = (w - u) * k.c31 + v * (k.c12 - k.c23) + k.e31;
    const V<T> dpdv = (w - v) * k.c23 + u * (k.c12 - k.c31) - k.e23;
    return normalize(cross(dpdu, dpdv));
}

// PhongMeshGeometry::bound(primitiveIndex) (phongmesh.h:61-164), in double
inline void patch_bound(const Patch<double> &P, double lo[3], double hi[3]) {
    typedef double T;
    const Coeffs<T> k = coeffs(P);
    const V<T> ng = normalize(cross(P.p[1] - P.p[0], P.p[2] - P.p[0]));
    const V<T> c31e31 = k.c31 + k.e31;
    const V<T> c23e23 = k.c23 - k.e23;
    const V<T> c122331 = k.c12 - k.c23 - k.c31;
    const T den = 4.0 * dot(ng, k.c23) * dot(ng, k.c31) - dot(ng, c122331);
    const T kk = 1.0 / (den * den);
    const T uhat = kk * (2.0 * dot(ng, k.c23) * dot(ng, c31e31) + dot(ng, c23e23) * dot(ng, c122331));
    const T vhat = kk * (2.0 * dot(ng, k.c31) * dot(ng, c23e23) + dot(ng, c31e31) * dot(ng, c122331));
    auto height = [&](T u, T v) { return dot(ng, eval_position(P, u, v) - P.p[0]); };
    T thickness = 0.0;
    const bool uok = uhat >= 0.0 && uhat <= 1.0;
    const bool vok = vhat >= 0.0 && vhat <= 1.0;
    if (uok && vok && uhat + vhat <= 1.0) {
        thickness = height(uhat, vhat);
    } else {
        const T a = uok ? height(uhat, 0.0) : 0.0;
        const T b = vok ? height(0.0, vhat) : 0.0;
        thickness = tmax_(a, b);
    }
    for (int c = 0; c < 3; ++c) {
        lo[c] = std::numeric_limits<double>::max();
        hi[c] = std::numeric_limits<double>::lowest();
    }
    auto grow = [&](const V<T> &q) {
        for (int c = 0; c < 3; ++c) {
            const T x = comp(q, c);
            lo[c] = x < lo[c] ? x : lo[c];
            hi[c] = x > hi[c] ? x : hi[c];
        }
    };
    if (thickness == 0.0) {
        for (int i = 0; i < 3; ++i) grow(P.p[i]);
        return;
    }
    // eq. 23: the patch point at each edge midpoint, distance from each edge line
    T drop[3] = {0.0, 0.0, 0.0};
    const T mid[3][2] = {{0.0, 0.5}, {0.5, 0.0}, {0.5, 0.5}};
    for (int m = 0; m < 3; ++m) {
        const V<T> pa = eval_position(P, mid[m][0], mid[m][1]);
        for (int e = 0; e < 3; ++e) {
            const V<T> pi = P.p[e], pj = P.p[(e + 1) % 3];
            const T s = length(cross(pj - pa, pi - pa)) / length(pj - pi);
            drop[e] = tmax_(s, drop[e]);
        }
    }
    for (int e = 0; e < 3; ++e) {
        const V<T> pi = P.p[e], pj = P.p[(e + 1) % 3];
        const V<T> x = normalize(pj - pi);
        const V<T> z = cross(x, ng);
        const V<T> vi = z * drop[e] + pi;
        const V<T> vj = z * drop[e] + pj;
        grow(vi);
        grow(vj);
        grow(vi + ng * thickness);
        grow(vj + ng * thickness);
    }
}

// PhongMeshGeometry::intersect (phongmesh.h:178-368) for a float ray as Embree passes it
// (embreeaccel.h:77-99). Accepts a candidate with tmin <= t <= tmax, lowering tmax each
// time, and returns whether any was accepted; `normal` is the unit patch normal there.
template <class T>
WRP_HD bool patch_intersect(const Patch<T> &P, float ox, float oy, float oz, float dx, float dy, float dz, float tminf,
                            T &tmax, V<T> &normal) {
    const V<T> org = v3<T>(T(double(ox)), T(double(oy)), T(double(oz)));
    const V<T> dir = v3<T>(T(double(dx)), T(double(dy)), T(double(dz)));
    const T tmin = T(double(tminf));
    int axis = 0;   // Math::MaxDimension: first index of the largest signed component
    T mx = dir.x;
    if (dir.y > mx) { axis = 1; mx = dir.y; }
    if (dir.z > mx) { axis = 2; }
    // TwoPlanesFromRay over CoordFrame3(direction) (coordframe.h:50-60)
    const T sign = copysign_(T(1.0), dir.y);
    const T fa = T(-1.0) / (sign + dir.y);
    const T fb = dir.z * dir.x * fa;
    const V<T> fx = v3<T>(sign + dir.x * dir.x * fa, -dir.x, fb);
    const V<T> fz = v3<T>(sign * fb, -sign * dir.z, T(1.0) + sign * dir.z * dir.z * fa);
    const V<T> d1 = cross(fx, dir);
    const T o1 = -dot(org, d1);
    const V<T> d2 = cross(fz, dir);
    const T o2 = -dot(org, d2);

    const Coeffs<T> k = coeffs(P);
    const V<T> c123 = k.c12 - k.c23 - k.c31;
    const V<T> ce31 = k.c31 + k.e31;
    const V<T> ce23 = k.c23 - k.e23;
    // eq. 5-6
    const T a = -dot(d1, k.c31);
    const T b = -dot(d1, k.c23);
    const T c = dot(d1, P.p[2]) + o1;
    const T d = dot(d1, c123);
    const T e = dot(d1, ce31);
    const T f = dot(d1, ce23);
    const T l = -dot(d2, k.c31);
    const T m = -dot(d2, k.c23);
    const T n = dot(d2, P.p[2]) + o2;
    const T o = dot(d2, c123);
    const T p = dot(d2, ce31);
    const T q = dot(d2, ce23);
    // eq. 16
    const T a3 = a * b * c + (d * e * f - a * f * f - b * e * e - c * d * d) * T(0.25);
    const T a2 = a * b * n + a * m * c + l * b * c - (a * f * q + b * e * p + c * d * o) * T(0.5) +
                 (o * e * f + d * e * q + d * p * f - l * f * f - m * e * e - n * d * d) * T(0.25);
    const T a1 = a * m * n + l * b * n + l * m * c - (l * f * q + m * e * p + n * d * o) * T(0.5) +
                 (d * p * q + o * e * q + o * p * f - a * q * q - b * p * p - c * o * o) * T(0.25);
    const T a0 = l * m * n + (o * p * q - l * q * q - m * p * p - n * o * o) * T(0.25);

    T xs[3] = {T(0.0), T(0.0), T(0.0)};
    const int nx = solve_real_cubic(xs, a3, a2, a1, a0);
    if (nx == 0) return false;
    // the root with the least M12^2 - M11 M22 (section 3.2)
    T x = T(0.0), best = T(std::numeric_limits<double>::infinity());
    bool chosen = false;
    for (int i = 0; i < nx; ++i) {
        const T m11 = xs[i] * a + l;
        const T m22 = xs[i] * b + m;
        const T m12 = (xs[i] * d + o) * T(0.5);
        const T cost = m12 * m12 - m11 * m22;
        if (cost < best) {
            x = xs[i];
            best = cost;
            chosen = true;
        }
    }
    if (best < T(0.0) || !chosen) return false;

    const T m11 = x * a + l;
    const T m22 = x * b + m;
    const bool greater = abs_(m11) > abs_(m22);
    T al[2], ga[2];
    if (greater) {
        const T inv = T(1.0) / m11;
        const T mp22 = m22 * inv;
        const T mp33 = (x * c + n) * inv;
        const T mp12 = (x * d + o) * T(0.5) * inv;
        const T mp13 = (x * e + p) * T(0.5) * inv;
        const T mp23 = (x * f + q) * T(0.5) * inv;
        const T bs = sqrt_(mp12 * mp12 - mp22);
        const T gs = sqrt_(mp13 * mp13 - mp33);
        al[0] = mp12 + bs;
        al[1] = mp12 - bs;
        ga[0] = mp13 + gs;
        ga[1] = mp13 - gs;
        const T dA = abs_((T(2.0) * mp23) - (al[0] * ga[0] + al[1] * ga[1]));
        const T dB = abs_((T(2.0) * mp23) - (al[0] * ga[1] + al[1] * ga[0]));
        if (dA < dB) { const T tg = ga[0]; ga[0] = ga[1]; ga[1] = tg; }
    } else {
        const T inv = T(1.0) / m22;
        const T mp11 = m11 * inv;
        const T mp12 = (x * d + o) * T(0.5) * inv;
        const T mp13 = (x * e + p) * T(0.5) * inv;
        const T mp23 = (x * f + q) * T(0.5) * inv;
        const T mp33 = (x * c + n) * inv;
        const T as = sqrt_(mp12 * mp12 - mp11);
        const T gs = sqrt_(mp23 * mp23 - mp33);
        al[0] = mp12 + as;
        al[1] = mp12 - as;
        ga[0] = mp23 + gs;
        ga[1] = mp23 - gs;
        const T dA = abs_((T(2.0) * mp13) - (al[0] * ga[0] + al[1] * ga[1]));
        const T dB = abs_((T(2.0) * mp13) - (al[0] * ga[1] + al[1] * ga[0]));
        if (dA < dB) { const T tg = ga[0]; ga[0] = ga[1]; ga[1] = tg; }
    }
    bool hit = false;
    for (int i = 0; i < 2; ++i) {
        const T g = -al[i];
        const T h = -ga[i];
        T k2, k1, k0;
        if (greater) {   // u = g v + h
            k2 = a * g * g + b + d * g;
            k1 = T(2.0) * a * g * h + d * h + e * g + f;
            k0 = a * h * h + c + e * h;
        } else {         // v = g u + h
            k2 = a + b * g * g + d * g;
            k1 = T(2.0) * b * g * h + d * h + e + f * g;
            k0 = b * h * h + c + f * h;
        }
        T ans[2];
        if (!solve_quadratic(ans[0], ans[1], k2, k1, k0)) continue;
        for (int j = 0; j < 2; ++j) {
            T u, v;
            if (greater) { v = ans[j]; u = g * v + h; }
            else { u = ans[j]; v = g * u + h; }
            const T w = T(1.0) - u - v;
            if (!(v >= T(0.0) && u >= T(0.0) && w >= T(0.0))) continue;
            const V<T> pos = eval_position(P, u, v);
            const T t = (comp(pos, axis) - comp(org, axis)) / comp(dir, axis);
            if (tmax >= t && tmin <= t) {
                hit = true;
                tmax = t;
                normal = eval_normal(k, u, v);
            }
        }
    }
    return hit;
}

// ------------------------------------------------------------------ device ----
#ifdef __CUDACC__
// Octahedral unit-vector encoding (Meyer et al., "On floating-point normal vectors",
// EGSR 2010): a patch hit stores its normal in the two barycentric slots of the hit record.
__device__ __forceinline__ float2 oct_encode(float x, float y, float z) {
    const float s = fabsf(x) + fabsf(y) + fabsf(z);
    float px = x / s, py = y / s;
    if (z < 0.f) {
        const float qx = (1.f - fabsf(py)) * (px >= 0.f ? 1.f : -1.f);
        const float qy = (1.f - fabsf(px)) * (py >= 0.f ? 1.f : -1.f);
        px = qx;
        py = qy;
    }
    return make_float2(px, py);
}

__device__ __forceinline__ float3 oct_decode(float px, float py) {
    float x = px, y = py;
    const float z = 1.f - fabsf(px) - fabsf(py);
    if (z < 0.f) {
        x = (1.f - fabsf(py)) * (px >= 0.f ? 1.f : -1.f);
        y = (1.f - fabsf(px)) * (py >= 0.f ? 1.f : -1.f);
    }
    const float inv = rsqrtf(x * x + y * y + z * z);
    return make_float3(x * inv, y * inv, z * inv);
}

// the patch of leaf primitive `i`: positions from its float leaf record, normals (FP64) from
// the patch array
__device__ __forceinline__ Patch<Rd> load_patch(const double *patches, uint32_t i, float4 a, float4 b, float4 c) {
    const double2 *q = reinterpret_cast<const double2 *>(patches + size_t(kPatchDoubles) * i);
    const double2 n01 = __ldg(q + 0), n23 = __ldg(q + 1), n45 = __ldg(q + 2), n67 = __ldg(q + 3), n8x = __ldg(q + 4);
    Patch<Rd> P;
    P.p[0] = v3<Rd>(double(a.x), double(a.y), double(a.z));
    P.p[1] = v3<Rd>(double(b.x), double(b.y), double(b.z));
    P.p[2] = v3<Rd>(double(c.x), double(c.y), double(c.z));
    P.n[0] = v3<Rd>(n01.x, n01.y, n23.x);
    P.n[1] = v3<Rd>(n23.y, n45.x, n45.y);
    P.n[2] = v3<Rd>(n67.x, n67.y, n8x.x);
    return P;
}

// the patch's own (float, outward-rounded) box: words 9..11 of its record as 6 floats
__device__ __forceinline__ void load_patch_box(const double *patches, uint32_t i, float lo[3], float hi[3]) {
    const float2 *q = reinterpret_cast<const float2 *>(patches + size_t(kPatchDoubles) * i + 9);
    const float2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    lo[0] = a.x; lo[1] = a.y; lo[2] = b.x;
    hi[0] = b.y; hi[1] = c.x; hi[2] = c.y;
}
#endif

}  // namespace wrp
