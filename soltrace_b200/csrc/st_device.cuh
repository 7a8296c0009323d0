// Device-side geometry and optics of the B200 trace.
//
// Every function here restates, for one ray held in registers, a step of the
// reference's per-ray state machine (coretrace/raytrace.cpp:582-1040); the
// citation on each gives the reference routine whose results it reproduces.
// FP64 paths keep the reference's arithmetic order where it matters for
// agreement to 1e-9 m.  In MIXED mode the geometry that fixes hit positions
// (transforms, closed-form roots, the torus quartic, Newton refinement,
// reflection and refraction directions) stays in double, which is what holds
// explicit-ray positions within 1e-5 m at km scale; aperture tests, property
// tables, Fresnel coefficients, error sampling and flux binning run in float.
#pragma once
#include <cstdint>
#include <cmath>
#include "st_scene.h"

namespace stb {

constexpr double kPiD = 3.141592653589793238462643;
constexpr double kDeg = 0.017453292519943295;
constexpr double kSlope60 = 1.7320508075688767;
// cos/sin(30 * acos(-1)/180) as glibc rounds them (the reference evaluates them at run time)
constexpr double kCos30 = 0.8660254037844387;
constexpr double kSin30 = 0.49999999999999994;

__device__ __forceinline__ void sincos_t(double x, double &s, double &c) { sincos(x, &s, &c); }
__device__ __forceinline__ void sincos_t(float x, float &s, float &c) { sincosf(x, &s, &c); }

// ------------------------------------------------------------------------------------
// Per-ray counter-based random stream: Philox4x32-10 (Salmon et al., SC'11).
// Draw k of ray s: block k/2 of counter {k/2, s_lo, s_hi, 0x5B200}, key
// {seed, 0x50C7A5E1}; even k takes words 0,1, odd k words 2,3; 53-bit doubles.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void philox10(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t &c3, uint32_t k0,
                                         uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__device__ __forceinline__ double words_to_unit(uint32_t a, uint32_t b) {
    // (a >> 5) * 2^26 + (b >> 6), times 2^-53; both products are exact in double
    return fma(double(a >> 5), 67108864.0, double(b >> 6)) * (1.0 / 9007199254740992.0);
}

struct RayRng {
    uint32_t seed;
    uint32_t s_lo, s_hi;
    uint32_t k;
    uint32_t w0, w1, w2, w3;
    uint32_t blk;  // block held in w*, 0xffffffff when none

    __device__ void init(uint32_t sd, uint64_t sid, uint32_t k0) {
        seed = sd;
        s_lo = uint32_t(sid);
        s_hi = uint32_t(sid >> 32);
        k = k0;
        blk = 0xffffffffu;
    }
    __device__ __forceinline__ double u() {
        const uint32_t b = k >> 1;
        if (b != blk) {
            w0 = b;
            w1 = s_lo;
            w2 = s_hi;
            w3 = 0x0005B200u;
            philox10(w0, w1, w2, w3, seed, 0x50C7A5E1u);
            blk = b;
        }
        const double r = (k & 1u) ? words_to_unit(w2, w3) : words_to_unit(w0, w1);
        ++k;
        return r;
    }
};

// ------------------------------------------------------------------------------------
// Transforms (mathproc.cpp:115-173): local = R (ref - origin), ref = R^T local + origin
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void to_local(const double *R, const double *o, const double p[3], const double d[3],
                                         double pl[3], double dl[3]) {
    const double x = p[0] - o[0], y = p[1] - o[1], z = p[2] - o[2];
    pl[0] = R[0] * x + R[1] * y + R[2] * z;
    pl[1] = R[3] * x + R[4] * y + R[5] * z;
    pl[2] = R[6] * x + R[7] * y + R[8] * z;
    dl[0] = R[0] * d[0] + R[1] * d[1] + R[2] * d[2];
    dl[1] = R[3] * d[0] + R[4] * d[1] + R[5] * d[2];
    dl[2] = R[6] * d[0] + R[7] * d[1] + R[8] * d[2];
}
__device__ __forceinline__ void to_ref(const double *R, const double *o, const double pl[3], const double dl[3],
                                       double p[3], double d[3]) {
    const double x = R[0] * pl[0] + R[3] * pl[1] + R[6] * pl[2];
    const double y = R[1] * pl[0] + R[4] * pl[1] + R[7] * pl[2];
    const double z = R[2] * pl[0] + R[5] * pl[1] + R[8] * pl[2];
    d[0] = R[0] * dl[0] + R[3] * dl[1] + R[6] * dl[2];
    d[1] = R[1] * dl[0] + R[4] * dl[1] + R[7] * dl[2];
    d[2] = R[2] * dl[0] + R[5] * dl[1] + R[8] * dl[2];
    p[0] = x + o[0];
    p[1] = y + o[1];
    p[2] = z + o[2];
}
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// ------------------------------------------------------------------------------------
// Aperture membership (determineelementintersectionnew.cpp:109-624; the start-plane
// variant of intersect.cpp:270-547 differs for rectangles, whose test there can
// never fail, and for the torus annulus, whose radial test it keeps).
// Returns 1 inside, 0 outside, -1 when no hexagon/triangle section matched.
// ------------------------------------------------------------------------------------
template <typename T>
__device__ inline int aperture_in(const ElemRec &e, T x, T y, bool start_plane) {
    const T r = sqrt(x * x + y * y);
    const T A = T(e.ap[0]);
    switch (e.shape) {
        case 'c':
            return r > A / T(2) ? 0 : 1;
        case 'h': {
            const T ro = A / T(2);
            if (r > ro) return 0;
            const T ri = ro * T(kCos30);  // cos 30 deg
            if (r <= ri) return 1;
            const T xl = sqrt(ro * ro - ri * ri);
            if (x <= ro && x > xl) {
                const T y1 = T(kSlope60) * (x - ro);
                return (y >= y1 && y <= -y1) ? 1 : 0;
            }
            if (x <= xl && x >= -xl) return (y >= -ri && y <= ri) ? 1 : 0;
            if (x < -xl && x >= -ro) {
                const T y3 = T(kSlope60) * (x + ro);
                return (y >= -y3 && y <= y3) ? 1 : 0;
            }
            return -1;
        }
        case 't': {
            const T ro = A / T(2);
            if (r > ro) return 0;
            const T ri = ro * T(kSin30);  // sin 30 deg as the reference evaluates it
            if (r <= ri) return 1;
            if (x <= ro && x > T(0)) {
                const T y1 = -T(kSlope60) * (x - ri / T(kCos30));
                return (y <= y1 && y >= -ri) ? 1 : 0;
            }
            if (x >= -ro && x <= T(0)) {
                const T y3 = T(kSlope60) * (x + ri / T(kCos30));
                return (y >= -ri && y <= y3) ? 1 : 0;
            }
            return -1;
        }
        case 'r':
            if (start_plane) return 1;
            if (x > A / T(2) || x < -A / T(2)) return 0;
            if (y > T(e.ap[1]) / T(2) || y < -T(e.ap[1]) / T(2)) return 0;
            return 1;
        case 'a': {
            if (start_plane || !(e.ap[0] == 0.0 && e.ap[1] == 0.0))
                if (r < T(e.ap[0]) || r > T(e.ap[1])) return 0;
            const T half = T(e.ap[2]) * T(kDeg) / T(2);
            if (x >= T(0)) return (asin(y / r) > half || asin(y / r) < -half) ? 0 : 1;
            if (y >= T(0) && (acos(y / r) + T(kPiD / 2.0)) > half) return 0;
            if (y < T(0) && (-acos(-y / r) - T(kPiD / 2.0)) < -half) return 0;
            return 1;
        }
        case 'l':
            if (!(e.ap[0] == 0.0 && e.ap[1] == 0.0))
                if (x < T(e.ap[0]) || x > T(e.ap[1])) return 0;
            if (y < -T(e.ap[2]) / T(2) || y > T(e.ap[2]) / T(2)) return 0;
            return 1;
        case 'i':
        case 'q': {
            // cross-product sign agreement per triangle (intersect.cpp:119-138)
            auto tri = [&](int a, int b, int c) {
                const T x1 = T(e.ap[a]), y1 = T(e.ap[a + 1]), x2 = T(e.ap[b]), y2 = T(e.ap[b + 1]);
                const T x3 = T(e.ap[c]), y3 = T(e.ap[c + 1]);
                const T s1 = (x1 - x) * (y2 - y) - (x2 - x) * (y1 - y);
                const T s2 = (x2 - x) * (y3 - y) - (x3 - x) * (y2 - y);
                const T s3 = (x3 - x) * (y1 - y) - (x1 - x) * (y3 - y);
                return (s1 >= T(0)) == (s2 >= T(0)) && (s2 >= T(0)) == (s3 >= T(0));
            };
            if (e.shape == 'i') return tri(0, 2, 4) ? 1 : 0;
            return (tri(0, 2, 4) || tri(0, 4, 6)) ? 1 : 0;
        }
        default:
            return -1;
    }
}

// ------------------------------------------------------------------------------------
// Quadric closed forms: sphere, paraboloid, hyperboloid/ellipsoid, cylinder
// (quadricsurfaceclosedform.cpp:58-308).  Returns 0 and (out, n, t) on success.
// ------------------------------------------------------------------------------------
__device__ inline int quadric_hit(const ElemRec &e, const double P[3], const double D[3], double out[3], double n[3],
                           double &t) {
    double zc = 0, kx = 1, ky = 1, kz = 1, a2 = 1, b2 = 1, c2 = 1, A, B, C;
    const int s = e.surf | 0x20;
    const double xd = P[0], yd = P[1];
    if (s == 'p') {
        a2 = 2.0 / e.vcx;
        b2 = e.vcy > 0.0 ? 2.0 / e.vcy : 1e10;
        ky = (e.stype == kSurfSingleAxis) ? 0.0 : 1.0;
        kz = 0.0;
        A = D[0] * D[0] * kx / a2 + D[1] * D[1] * ky / b2;
        B = 2.0 * (kx * xd * D[0] / a2 + ky * yd * D[1] / b2) - D[2] / c2;
        C = kx * xd * xd / a2 + ky * yd * yd / b2 - P[2] / c2;
    } else {
        double rhs;
        if (s == 's') {
            ky = (e.stype == kSurfSingleAxis) ? 0.0 : 1.0;
            const double r = 1.0 / e.vcx;
            zc = r;
            rhs = r * r;
        } else if (s == 'o') {
            kz = e.kappa;
            zc = 1.0 / e.kappa / e.vcx;
            rhs = 1.0 / e.kappa / (e.vcx * e.vcx);
        } else {  // 't'
            ky = 0.0;
            const double r = 1.0 / e.curv_rev;
            zc = r;
            rhs = r * r;
        }
        const double zd = P[2] - zc;
        A = D[0] * D[0] * kx / a2 + D[1] * D[1] * ky / b2 + D[2] * D[2] * kz / c2;
        B = 2.0 * (kx * xd * D[0] / a2 + ky * yd * D[1] / b2 + kz * zd * D[2] / c2);
        C = kx * xd * xd / a2 + ky * yd * yd / b2 + kz * zd * zd / c2 - rhs;
    }
    if (fabs(A) < 1e-12) {
        const double t1 = -C / B;
        if (!(t1 > 0)) return 1;
        t = t1;
    } else if (B * B > 4.0 * A * C) {
        const double q = sqrt(B * B - 4.0 * A * C);
        const double t1 = (-B + q) / (2.0 * A);
        const double t2 = (-B - q) / (2.0 * A);
        if (t2 > 0) {
            t = t2;
            if (P[2] + t2 * D[2] > e.zap) t = t1;
            const bool finite_len = (s == 't') || (s == 's' && e.stype == kSurfSingleAxis);
            if (finite_len) {
                const double yt = P[1] + t * D[1];
                if (yt < -e.ap[2] / 2.0 || yt > e.ap[2] / 2.0) t = t1;
            }
        } else if (t2 == 0 || (t2 < 0 && t1 > 0)) {
            t = t1;
        } else {
            return 1;
        }
    } else {
        return 1;
    }
    out[0] = P[0] + t * D[0];
    out[1] = P[1] + t * D[1];
    out[2] = P[2] + t * D[2];
    // the reference squares each gradient term as ((((2 K d)/a2) * 2) * K * d)/a2
    const double gx = 2.0 * kx * out[0] / a2, gy = 2.0 * ky * out[1] / b2;
    const double sx = (gx * 2.0 * kx * out[0]) / a2, sy = (gy * 2.0 * ky * out[1]) / b2;
    if (s == 'p') {
        const double m = sqrt(sx + sy + 1.0);
        n[0] = -gx / m;
        n[1] = -gy / m;
        n[2] = 1.0 / m;
    } else {
        const double gz = 2.0 * kz * (out[2] - zc) / c2;
        const double sz = (gz * 2.0 * kz * (out[2] - zc)) / c2;
        const double m = sqrt(sx + sy + sz);
        n[0] = -gx / m;
        n[1] = -gy / m;
        n[2] = -gz / m;
    }
    return 0;
}

// ------------------------------------------------------------------------------------
// Torus: quartic in t, Ferrari reduction with a bisected resolvent cubic
// (torusclosedform.cpp:57-188, root432.cpp:53-284, piksrt mathproc.cpp:333-348).
// Kept in FP64 in every precision mode.
// ------------------------------------------------------------------------------------
struct QuarticSolver {
    double a20, a21;        // quadratic x^2 + a21 x + a20
    double a30, a31, a32;   // cubic x^3 + a32 x^2 + a31 x + a30
    double r1, r2, r3, r4, im, ii;
    __device__ void root2() {
        const double w = a21 * a21 - 4 * a20;
        const double q1 = -a21 / 2.0;
        if (w < 0) {
            im = sqrt(-w) / 2.0;
            r1 = q1;
            r2 = q1;
        } else if (w == 0) {
            r1 = q1;
            r2 = q1;
            im = 0.0;
        } else if (w > 0) {
            const double q2 = sqrt(w) / 2.0;
            im = 0.0;
            r1 = q1 + q2;
            r2 = q1 - q2;
        }
    }
    __device__ double cubic(double x) const { return x * x * x + a32 * x * x + a31 * x + a30; }
    __device__ double cubic_root() const {  // one real root by bisection to 1e-6
        if (a30 == 0) return 0.0;
        double am = fabs(a30);
        am = fmax(am, fabs(a31));
        am = fmax(am, fabs(a32));  // the reference also scans a[3][3], which is 0
        double xa, xb;
        if (a30 > 0) {
            xa = -am - 1;
            xb = 0;
        } else {
            xa = 0;
            xb = am + 1;
        }
        if (cubic(xa) == 0) return xa;
        if (cubic(xb) == 0) return xb;
        double xc;
        for (int it = 0; it < 200; ++it) {
            xc = (xa + xb) / 2.0;
            const double te = cubic(xc);
            if (te == 0) break;
            if (xb - xa < 0.000001) break;
            if (cubic(xa) * te > 0)
                xa = xc;
            else
                xb = xc;
        }
        return xc;
    }
    // normalised quartic x^4 + a x^3 + b x^2 + c x + d
    __device__ void solve(double aa, double b, double c, double d) {
        double q = b - (3.0 * aa * aa / 8.0);
        double rr = c - (aa * b / 2) + (aa * aa * aa / 8.0);
        const double s = d - (aa * c / 4) + (aa * aa * b / 16.0) - (3 * aa * aa * aa * aa / 256.0);
        a32 = q / 2.0;
        a31 = (q * q - 4 * s) / 16.0;
        a30 = -(rr * rr / 64.0);
        im = 0.0;
        r1 = r2 = 0.0;
        double r3v;
        if ((rr != 0) || (a31 >= 0)) {
            r3v = cubic_root();
        } else {
            a21 = a32;
            a20 = a31;
            root2();
            r3v = r1;
        }
        const double k = sqrt(r3v);
        if (k == 0) {
            rr = sqrt(q * q - 4 * s);
        } else {
            q = q + (4 * r3v);
            rr = rr / (2 * k);
        }
        const double l = (q - rr) / 2.0, m = (q + rr) / 2.0;
        a21 = 2 * k;
        a20 = l;
        root2();
        r3 = r1 - (aa / 4);
        r4 = r2 - (aa / 4.0);
        ii = im;
        a21 = -2 * k;
        a20 = m;
        root2();
        r2 = r2 - (aa / 4.0);
        r1 = r1 - (aa / 4.0);
    }
};

__device__ inline int torus_hit(const ElemRec &e, const double P[3], const double D[3], double out[3], double n[3],
                         double &t) {
    const double Rs = e.rs, Ra = e.ra;
    const double Xo = P[0], Yo = P[1], Zo = P[2];
    const double Ep = D[0], Et = D[1], Rh = D[2];
    const double c4 = pow(Ep, 4) + 2.0 * Ep * Ep * (Et * Et + Rh * Rh) + pow(Et, 4) + 2.0 * Et * Et * Rh * Rh + pow(Rh, 4);
    const double c3 = 4.0 * (Ep * Ep + Et * Et + Rh * Rh) * (Ep * Xo + Et * Yo + Rh * Zo - Rh * Rs);
    const double c2 = Xo * Xo * (6.0 * Ep * Ep + 2.0 * Et * Et + 2.0 * Rh * Rh) + 8.0 * Ep * Xo * (Et * Yo + Rh * Zo - Rh * Rs) +
                      2.0 * Yo * Yo * (Ep * Ep + 3.0 * Et * Et + Rh * Rh) + 8.0 * Et * Rh * Yo * (Zo - Rs) +
                      (Ep * Ep + Et * Et + 3.0 * Rh * Rh) * (2.0 * Zo * Zo - 4.0 * Rs * Zo) -
                      2.0 * Ra * Ra * (Ep * Ep + Et * Et - Rh * Rh) + 4.0 * Rh * Rh * Rs * Rs;
    const double c1 = 4.0 * (Xo * Xo * (Ep * Xo + Et * Yo + Rh * Zo - Rh * Rs) + Yo * Yo * (Ep * Xo + Et * Yo + Rh * Zo - Rh * Rs) +
                             Zo * Zo * (Ep * Xo + Et * Yo + Rh * Zo - 3.0 * Rh * Rs) - 2.0 * Ep * Rs * Xo * Zo -
                             Ep * Ra * Ra * Xo - 2.0 * Et * Rs * Yo * Zo - Et * Ra * Ra * Yo + Rh * Ra * Ra * (Zo - Rs) +
                             2.0 * Rh * Rs * Rs * Zo);
    const double c0 = pow(Xo, 4) + 2.0 * Xo * Xo * (Yo * Yo + Zo * Zo - 2.0 * Rs * Zo - Ra * Ra) + pow(Yo, 4) +
                      2.0 * Yo * Yo * (Zo * Zo - 2.0 * Rs * Zo - Ra * Ra) + pow(Zo, 4) - 4.0 * Rs * Zo * Zo * Zo +
                      2.0 * Ra * Ra * Zo * Zo + 4.0 * Rs * Rs * Zo * Zo - 4.0 * Ra * Ra * Rs * Zo + pow(Ra, 4);
    QuarticSolver qs;
    qs.solve(c3 / c4, c2 / c4, c1 / c4, c0 / c4);
    double pl;
    if (qs.im == 0.0 && qs.ii == 0.0) {
        // the reference sorts entries 0..3 of {0, r1, r2, r3, r4} with its insertion sort
        double v[5] = {0.0, qs.r1, qs.r2, qs.r3, qs.r4};
        for (int j = 1; j < 4; ++j) {
            const double a = v[j];
            int i = j - 1;
            while (i >= 0 && !(v[i] <= a)) {
                v[i + 1] = v[i];
                --i;
            }
            if (i < 0) i = 0;
            v[i + 1] = a;
        }
        if (v[4] <= 0.0) return 1;
        pl = v[4];
        if (v[3] > 0.0) {
            pl = v[3];
            if (v[2] > 0.0) {
                pl = v[2];
                if (v[1] > 0.0) pl = v[1];
            }
        }
    } else if (qs.im == 0.0) {
        pl = (qs.r1 <= qs.r2) ? qs.r1 : qs.r2;
    } else if (qs.ii == 0.0) {
        pl = (qs.r3 <= qs.r4) ? qs.r3 : qs.r4;
    } else {
        pl = 0.0;
    }
    if (pl == 0.0) return 1;
    t = pl;
    const double X = Xo + pl * Ep, Y = Yo + pl * Et, Z = Zo + pl * Rh;
    const double rho = sqrt(X * X + Y * Y);
    out[0] = X;
    out[1] = Y;
    out[2] = Z;
    n[0] = 2.0 * X * (Ra - rho) / rho;
    n[1] = 2.0 * Y * (Ra - rho) / rho;
    n[2] = -(2.0 * (Z - Rs));
    return 0;
}

// ------------------------------------------------------------------------------------
// Implicit surfaces for the Newton path (surface.cpp:57-413, surfacezatxypair.cpp:56-280,
// vshot.cpp:59-139,290-367, mathproc.cpp:220-283).  Kept in FP64 in every mode.
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double ipow(double x, int n) {
    // the reference evaluates pow(x, n) for integer n
    return pow(x, double(n));
}
__device__ inline double eval_mono(const ElemRec &e, const double *B, double x, double y) {
    const int o = e.fit_order, w = o + 1;
    double z = 0.0;
    for (int i = 0; i <= o; ++i)
        for (int j = 0; j <= i; ++j) {
            const double xx = (j == 0) ? 1.0 : ipow(x, j);
            const double yy = (i - j == 0) ? 1.0 : ipow(y, i - j);
            z = z + B[i * w + j] * xx * yy;
        }
    return z;
}
__device__ inline void mono_slope(const ElemRec &e, const double *B, double sx, double sy, double &dx, double &dy) {
    const int o = e.fit_order, w = o + 1;
    if (sx == 0.0) sx = sx + 1.0e-10;
    if (sy == 0.0) sy = sy + 1.0e-10;
    dx = 0.0;
    dy = 0.0;
    for (int i = 1; i <= o; ++i)
        for (int j = 0; j <= i; ++j) {
            dx = dx + j * B[i * w + j] * ipow(sx, j - 1) * ipow(sy, i - j);
            dy = dy + (i - j) * B[i * w + j] * ipow(sx, j) * ipow(sy, i - j - 1);
        }
}
__device__ inline double eval_poly(const double *c, int order, double x, double y) {
    double z = 0.0;
    const double r = sqrt(x * x + y * y);
    for (int i = 0; i <= order; ++i) z = z + c[i] * ipow(r, i);
    return z;
}
__device__ inline void poly_slope(const double *c, int order, double x, double y, double &dx, double &dy) {
    double dzdr = 0.0;
    const double r = sqrt(x * x + y * y);
    const double drdx = x / r, drdy = y / r;
    for (int i = 1; i <= order; ++i) dzdr = dzdr + i * c[i] * ipow(r, i - 1);
    dx = dzdr * drdx;
    dy = dzdr * drdy;
}
__device__ inline bool splint(const double *xa, const double *ya, const double *y2a, int n, double x, double &y,
                       double &dydx) {
    int klo = 0, khi = n - 1;
    while (khi - klo > 1) {
        const int k = (khi + klo) / 2;
        if (xa[k] > x)
            khi = k;
        else
            klo = k;
    }
    const double h = xa[khi] - xa[klo];
    if (h == 0.0) return false;
    const double a = (xa[khi] - x) / h, b = (x - xa[klo]) / h;
    y = a * ya[klo] + b * ya[khi] + ((a * a * a - a) * y2a[klo] + (b * b * b - b) * y2a[khi]) * (h * h) / 6.0;
    dydx = (ya[khi] - ya[klo]) / (xa[khi] - xa[klo]) - (3.0 * a * a - 1.0) * (xa[khi] - xa[klo]) * y2a[klo] / 6.0 +
           (3.0 * b * b - 1.0) * (xa[khi] - xa[klo]) * y2a[khi] / 6.0;
    return true;
}

// ------------------------------------------------------------------------------------
// Finite-element surface (vshot.cpp:166-242): kriging with a power-law variogram on the 7
// nearest nodes among a query zone's candidates (Numerical Recipes 3rd ed. 3.7.4, Krig with
// Powvargram; LU decomposition with implicit partial pivoting, 2.3), arithmetic in the
// reference's order (interpolate.cpp:5-238).  Table layout: st_host.cpp fe_table.
// ------------------------------------------------------------------------------------
static __device__ unsigned int g_fe_fail = 0;  // a query found fewer than 3 candidate nodes

struct FeKriging {
    int n;
    double x[7][2], alph;
    double lu[8][8], yvi[8];
    __device__ double pvg(double r) const { return 0.0 + alph * pow(r, 1.999); }
    __device__ static double dist(double ax, double ay, double bx, double by) {
        double d = 0.;
        d += (ax - bx) * (ax - bx);
        d += (ay - by) * (ay - by);
        return sqrt(d);
    }
    __device__ void setup(const double *py) {
        double num = 0., den = 0.;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) {
                double rb = 0.;
                rb += (x[i][0] - x[j][0]) * (x[i][0] - x[j][0]);
                rb += (x[i][1] - x[j][1]) * (x[i][1] - x[j][1]);
                rb = pow(rb, 0.5 * 1.999);
                num += rb * (0.5 * ((py[i] - py[j]) * (py[i] - py[j])) - 0.0);
                den += rb * rb;
            }
        alph = num / den;
        const int m = n + 1;
        for (int i = 0; i < n; i++) {
            for (int j = i; j < n; j++) lu[i][j] = lu[j][i] = pvg(dist(x[i][0], x[i][1], x[j][0], x[j][1]));
            lu[i][n] = lu[n][i] = 1.;
        }
        lu[n][n] = 0.;
        double vv[8];
        int indx[8];
        for (int i = 0; i < m; i++) {
            double big = 0.0;
            for (int j = 0; j < m; j++) big = fabs(lu[i][j]) > big ? fabs(lu[i][j]) : big;
            vv[i] = 1.0 / big;
        }
        for (int k = 0; k < m; k++) {
            double big = 0.0;
            int imax = k;
            for (int i = k; i < m; i++) {
                const double t = vv[i] * fabs(lu[i][k]);
                if (t > big) {
                    big = t;
                    imax = i;
                }
            }
            if (k != imax) {
                for (int j = 0; j < m; j++) {
                    const double t = lu[imax][j];
                    lu[imax][j] = lu[k][j];
                    lu[k][j] = t;
                }
                vv[imax] = vv[k];
            }
            indx[k] = imax;
            if (lu[k][k] == 0.0) lu[k][k] = 1.0e-40;
            for (int i = k + 1; i < m; i++) {
                const double t = lu[i][k] /= lu[k][k];
                for (int j = k + 1; j < m; j++) lu[i][j] -= t * lu[k][j];
            }
        }
        for (int i = 0; i < n; i++) yvi[i] = py[i];
        yvi[n] = 0.;
        int ii = 0;
        for (int i = 0; i < m; i++) {
            const int ip = indx[i];
            double sum = yvi[ip];
            yvi[ip] = yvi[i];
            if (ii != 0)
                for (int j = ii - 1; j < i; j++) sum -= lu[i][j] * yvi[j];
            else if (sum != 0.0)
                ii = i + 1;
            yvi[i] = sum;
        }
        for (int i = m - 1; i >= 0; i--) {
            double sum = yvi[i];
            for (int j = i + 1; j < m; j++) sum -= lu[i][j] * yvi[j];
            yvi[i] = sum / lu[i][i];
        }
    }
    __device__ double interp(double qx, double qy) const {
        double v = 0.;
        for (int i = 0; i < n; i++) v += yvi[i] * pvg(dist(qx, qy, x[i][0], x[i][1]));
        v += yvi[n] * 1.;
        return v;
    }
};

// surface z at (X, Y) and the slopes of F = z_local - z (finite differences of step
// 0.001/sqrt(nodes per aperture area)); 1 when the query zone has fewer than 3 candidates
static __device__ __noinline__ int fe_eval(const ElemRec &e, const double *sd, double X, double Y, double &zr, double &fx,
                                    double &fy) {
    const double *h = sd + e.data_off;
    const int nn = int(h[0]), lx = int(h[1]), ly = int(h[2]), nz = int(h[7]);
    const double *starts = h + 8, *items = starts + nz + 1, *nodes = items + int(starts[nz]);
    double x0 = h[3], x1 = h[4], y0 = h[5], y1 = h[6];
    int ix = 0, iy = 0;
    for (int k = 0; k < lx; ++k) {
        const double c = (x0 + x1) * 0.5;
        if (X > c) {
            x0 = c;
            ix = 2 * ix + 1;
        } else {
            x1 = c;
            ix = 2 * ix;
        }
    }
    for (int k = 0; k < ly; ++k) {
        const double c = (y0 + y1) * 0.5;
        if (Y > c) {
            y0 = c;
            iy = 2 * iy + 1;
        } else {
            y1 = c;
            iy = 2 * iy;
        }
    }
    const int zone = iy * (1 << lx) + ix;
    const int a = int(starts[zone]), b = int(starts[zone + 1]);
    if (b - a < 3) {
        atomicOr(&g_fe_fail, 1u);
        return 1;
    }
    // the 7 nearest candidates, nearest first (earlier candidates first on ties)
    double br[7];
    int bi[7], m = 0;
    for (int k = a; k < b; ++k) {
        const int j = int(items[k]);
        const double dx = X - nodes[3 * j], dy = Y - nodes[3 * j + 1];
        const double r = sqrt(dx * dx + dy * dy);
        int p;
        if (m < 7)
            p = m++;
        else if (r < br[6])
            p = 6;
        else
            continue;
        while (p > 0 && br[p - 1] > r) {
            br[p] = br[p - 1];
            bi[p] = bi[p - 1];
            --p;
        }
        br[p] = r;
        bi[p] = j;
    }
    (void)nn;
    FeKriging g;
    g.n = m;
    double py[7];
    for (int i = 0; i < m; ++i) {
        g.x[i][0] = nodes[3 * bi[i]];
        g.x[i][1] = nodes[3 * bi[i] + 1];
        py[i] = nodes[3 * bi[i] + 2];
    }
    g.setup(py);
    const double step = 0.001 / sqrt(double(nn) / e.area);
    zr = g.interp(X, Y);
    const double xa = X + step;
    const double za = g.interp(xa, Y);
    const double zb = g.interp(xa - step, Y + step);
    fx = (zr - za) / step;
    fy = (zr - zb) / step;
    return 0;
}

// F and grad F; may replace pos[2] by the surface z for data surfaces.  0 = ok.
__device__ inline int surface_eval(const ElemRec &e, const double *sd, double pos[3], double &F, double dF[3]) {
    const double X = pos[0], Y = pos[1], Z = pos[2];
    switch (e.stype) {
        case kSurfConic:
        case kSurfSingleAxis: {
            if (e.cone_deg != 0.0) {
                const double rho2 = (e.stype == kSurfConic) ? X * X + Y * Y : X * X;
                const double tc = tan(e.cone_deg * kDeg);
                F = Z - sqrt(rho2) / tc;
                dF[0] = -X / (sqrt(rho2) * tc);
                dF[1] = -Y / (sqrt(rho2) * tc);
                dF[2] = 1.0;
                return 0;
            }
            const double q = e.vcx * e.vcx * X * X + e.vcy * e.vcy * Y * Y;
            const int err = (1.0 - e.kappa * q < 0) ? 1 : 0;
            const double term = sqrt(1.0 - e.kappa * q);
            F = Z - (e.vcx * X * X + e.vcy * Y * Y) / (1.0 + term) - 0.0;
            dF[0] = -X * (e.vcx / term + 2.0 * 0.0);
            dF[1] = -Y * (e.vcy / term + 2.0 * 0.0);
            dF[2] = 1.0;
            return err;
        }
        case kSurfFlat:
            F = Z;
            dF[0] = 0.0;
            dF[1] = 0.0;
            dF[2] = 1.0;
            return 0;
        case kSurfFE: {  // surface.cpp:217-241
            if (X * X + Y * Y == 0.0) {
                F = Z;
                dF[0] = dF[1] = 0.0;
                dF[2] = 1.0;
                return 0;
            }
            double zr, fx, fy;
            if (fe_eval(e, sd, X, Y, zr, fx, fy)) return 1;
            pos[2] = zr;
            F = Z - zr;
            dF[0] = fx;
            dF[1] = fy;
            dF[2] = 1.0;
            return 0;
        }
        case kSurfVshot: {
            if (X * X + Y * Y == 0.0) {
                F = Z;
                dF[0] = dF[1] = 0.0;
                dF[2] = 1.0;
                return 0;
            }
            const double *B = sd + e.data_off;
            const int nb = (e.fit_order + 1) * (e.fit_order + 1);
            const double zm = eval_mono(e, B, X, Y);
            const double density = e.data_n / e.area;
            const double roi2 = 30.0 / density / 3.14159;
            const double *V = B + nb;
            double s = 0.0, wx = 0.0, wy = 0.0, zx = 0.0, zy = 0.0;
            bool exact = false;
            for (int i = 0; i < e.data_n; ++i) {
                const double *v = V + 5 * i;
                const double xx = v[0] - X, yy = v[1] - Y;
                if (xx == 0.0 && yy == 0.0) {
                    zx = v[2];
                    zy = v[3];
                    exact = true;
                    break;
                }
                const double r2 = xx * xx + yy * yy;
                if (r2 < roi2) {
                    s = s + 1.0 / r2;
                    wx = wx + v[2] / r2;
                    wy = wy + v[3] / r2;
                }
            }
            if (!exact && s != 0.0) {
                zx = wx / s;
                zy = wy / s;
            }
            pos[2] = zm;
            F = Z - zm;
            dF[0] = -tan(zx);
            dF[1] = -tan(zy);
            dF[2] = 1.0;
            return 0;
        }
        case kSurfZernike: {
            const double *B = sd + e.data_off;
            const double zz = eval_mono(e, B, X, Y);
            double sx, sy;
            mono_slope(e, B, X, Y, sx, sy);
            pos[2] = zz;
            F = Z - zz;
            dF[0] = -sx;
            dF[1] = -sy;
            dF[2] = 1.0;
            return 0;
        }
        case kSurfPoly: {
            const double *c = sd + e.data_off;
            const double yv = (e.shape == 'l') ? 0.0 : Y;
            const double zz = eval_poly(c, e.fit_order, X, yv);
            double sx, sy;
            poly_slope(c, e.fit_order, X, yv, sx, sy);
            pos[2] = zz;
            F = Z - zz;
            dF[0] = -sx;
            dF[1] = -sy;
            dF[2] = 1.0;
            return 0;
        }
        case kSurfSpline: {
            const double *xs = sd + e.data_off, *ys = xs + e.spl_n, *y2 = ys + e.spl_n;
            double rho = sqrt(X * X + Y * Y), drx = X / rho, dry = Y / rho;
            if (e.shape == 'l') {
                rho = X;
                drx = 1.0;
                dry = 0.0;
            }
            double zz, dz;
            if (!splint(xs, ys, y2, e.spl_n, rho, zz, dz)) return 3;
            pos[2] = zz;
            F = Z - zz;
            dF[0] = -(dz * drx);
            dF[1] = -(dz * dry);
            dF[2] = 1.0;
            return 0;
        }
        default:
            return 4;
    }
}

__device__ inline double surface_z_at(const ElemRec &e, const double *sd, double X, double Y) {
    switch (e.stype) {
        case kSurfConic:
        case kSurfSingleAxis: {
            if (e.cone_deg != 0.0) {
                const double rho2 = (e.stype == kSurfConic) ? X * X + Y * Y : X * X;
                return sqrt(rho2) / tan(e.cone_deg * kDeg);
            }
            const double q = e.vcx * e.vcx * X * X + e.vcy * e.vcy * Y * Y;
            if (e.kappa * q > 1.0) return 0.0;
            return (e.vcx * X * X + e.vcy * Y * Y) / (1.0 + sqrt(1.0 - e.kappa * q));
        }
        case kSurfVshot:
            if (X * X + Y * Y == 0.0) return 0.0;
            return eval_mono(e, sd + e.data_off, X, Y);
        case kSurfZernike:
            return eval_mono(e, sd + e.data_off, X, Y);
        case kSurfPoly:
            return eval_poly(sd + e.data_off, e.fit_order, X, (e.shape == 'l') ? 0.0 : Y);
        default:
            return 0.0;
    }
}

// start plane from a virtual cylinder/plane at the spline data limit
// (newzstartforcubicsplinesurf.cpp:57-142); returns false if the ray misses it
__device__ inline bool spline_cyl_z(double cr, const double P[3], const double D[3], int ap, double &z) {
    if (ap == 'a') {
        const double A = D[0] * D[0] + D[1] * D[1];
        const double B = 2.0 * (P[0] * D[0] + P[1] * D[1]);
        const double C = P[0] * P[0] + P[1] * P[1] - cr * cr;
        if (!(B * B > 4.0 * A * C)) return false;
        const double q = sqrt(B * B - 4.0 * A * C);
        const double t1 = (-B + q) / (2.0 * A), t2 = (-B - q) / (2.0 * A);
        if (t2 > 0) {
            z = P[2] + t2 * D[2];
            return true;
        }
        if (t2 == 0 || (t2 < 0 && t1 > 0)) {
            z = P[2] + t1 * D[2];
            return true;
        }
        return false;
    }
    if (ap == 'l') {
        const double t1 = (cr - P[0]) / D[0];
        if (t1 >= 0.0) {
            z = P[2] + t1 * D[2];
            return true;
        }
        return false;
    }
    return true;
}

// Newton starting plane for spline surfaces (intersect.cpp:597-945)
__device__ inline double spline_start(const ElemRec &e, const double *sd, const double P[3], const double D[3], int &err) {
    const double *xs = sd + e.data_off, *ys = xs + e.spl_n, *y2 = ys + e.spl_n;
    const int n = e.spl_n;
    const double outer = xs[n - 1], inner = xs[0], ZA = ys[n - 1];
    const int ap = e.shape;
    const bool an = (ap == 'a'), ln = (ap == 'l');
    const double s00 = -P[2] / (D[2] + 0.00000000001);
    const double X10 = P[0] + D[0] * s00, Y10 = P[1] + D[1] * s00, R10 = sqrt(X10 * X10 + Y10 * Y10);
    const double s0a = (ZA - P[2]) / (D[2] + 0.00000000001);
    const double X1A = P[0] + D[0] * s0a, Y1A = P[1] + D[1] * s0a, R1A = sqrt(X1A * X1A + Y1A * Y1A);
    auto gt_out = [&](double R, double X) { return (an && R > outer) || (ln && X > outer); };
    auto ge_out = [&](double R, double X) { return (an && R >= outer) || (ln && X >= outer); };
    auto le_out = [&](double R, double X) { return (an && R <= outer) || (ln && X <= outer); };
    auto lt_out = [&](double R, double X) { return (an && R < outer) || (ln && X < outer); };
    auto le_in = [&](double R, double X) { return (an && R <= inner) || (ln && X <= inner); };
    auto inside = [&](double R, double X) { return (an && R < outer && R > inner) || (ln && X < outer && X > inner); };
    double z = 0.0, zc;
    if (P[2] >= ZA && D[2] < 0.0) {
        const double PA[3] = {X1A, Y1A, ZA};
        if (gt_out(R1A, X1A)) return spline_cyl_z(outer * 0.999999, PA, D, ap, zc) ? zc : 0.0;
        if (le_out(R1A, X1A)) {
            if (ge_out(R10, X10)) return spline_cyl_z(outer * 0.999999, PA, D, ap, zc) ? zc : 0.0;
            return 0.0;
        }
    }
    if (P[2] <= 0.0 && D[2] > 0.0) {
        const double P0[3] = {X10, Y10, 0.0};
        if (ge_out(R10, X10)) return spline_cyl_z(outer * 0.999999, P0, D, ap, zc) ? zc : 0.0;
        if (inside(R10, X10)) return 0.0;
        if (le_in(R10, X10)) return spline_cyl_z(inner / 0.999999, P0, D, ap, zc) ? zc : 0.0;
    }
    const double R1 = sqrt(P[0] * P[0] + P[1] * P[1]);
    if (P[2] < ZA && P[2] > 0.0 && D[2] < 0.0) {
        if (ge_out(R1, P[0])) return spline_cyl_z(outer * 0.999999, P, D, ap, zc) ? zc : 0.0;
        if (inside(R1, P[0])) {
            double z1, dz;
            if (!splint(xs, ys, y2, n, an ? R1 : P[0], z1, dz)) {
                err = 3;
                return 0.0;
            }
            if (z1 < P[2]) {
                if (ge_out(R10, X10)) return spline_cyl_z(outer * 0.999999, P, D, ap, zc) ? zc : 0.0;
                return 0.0;
            }
            return P[2];
        }
        if (le_in(R1, P[0])) return spline_cyl_z(inner / 0.999999, P, D, ap, zc) ? zc : 0.0;
    }
    if (P[2] < ZA && P[2] > 0.0 && D[2] > 0.0) {
        if (ge_out(R1, P[0])) return spline_cyl_z(outer * 0.999999, P, D, ap, zc) ? zc : 0.0;
        if (inside(R1, P[0])) {
            double z1, dz;
            if (!splint(xs, ys, y2, n, an ? R1 : P[0], z1, dz)) {
                err = 3;
                return 0.0;
            }
            if (z1 < P[2]) {
                if (ge_out(R1A, X1A)) return spline_cyl_z(outer * 0.999999, P, D, ap, zc) ? zc : 0.0;
                return 0.0;
            }
            if (lt_out(R10, X10)) return 0.0;
            if (ge_out(R10, X10)) {
                const double PD[3] = {X10, Y10, 0.0};
                return spline_cyl_z(outer * 0.999999, PD, D, ap, zc) ? zc : 0.0;
            }
        }
        if (le_in(R1, P[0])) return spline_cyl_z(outer * 0.999999, P, D, ap, zc) ? zc : 0.0;
    }
    return z;
}

// Start plane + Newton-Raphson on F(p + s d) = 0 (intersect.cpp:272-1007).  0 = converged.
__device__ inline int newton_hit(const ElemRec &e, const double *sd, const double P[3], const double D[3], double out[3],
                         double n[3], double &plen) {
    int err = 0;
    const int st = e.stype;
    double zstart = 0.0;
    if (st != kSurfFlat && st != kSurfFE && st != kSurfSpline) {
        double s0a = 0.0;
        if (e.zap - P[2] != 0.0) s0a = (e.zap - P[2]) / (D[2] + 0.00000000001);
        const bool za_in = aperture_in<double>(e, P[0] + D[0] * s0a, P[1] + D[1] * s0a, true) == 1;
        const double fxy = surface_z_at(e, sd, P[0], P[1]);
        if (P[2] <= 0.0 && D[2] > 0.0)
            zstart = 0.0;
        else if (P[2] <= fxy && D[2] > 0.0)
            zstart = 0.0;
        else if (P[2] <= fxy && D[2] < 0.0 && P[2] > e.zap && za_in)
            zstart = 0.0;
        else if (P[2] <= fxy && D[2] < 0.0)
            zstart = e.zap;
        else if (P[2] > fxy && D[2] < 0.0)
            zstart = 0.0;
        else if (P[2] > fxy && D[2] > 0.0)
            zstart = e.zap;
    } else if (st == kSurfSpline) {
        zstart = spline_start(e, sd, P, D, err);
        if (err) return err;
    }
    double s0 = 0.0;
    if (zstart - P[2] != 0.0) s0 = (zstart - P[2]) / (D[2] + 0.00000000001);
    const double x1 = P[0] + D[0] * s0, y1 = P[1] + D[1] * s0;
    double lo = -1e10, hi = 1e10;
    if (st == kSurfSpline) {
        const double *xs = sd + e.data_off;
        const double sa = (xs[0] - x1) / (D[0] + 0.00000000001);
        const double sb = (xs[e.spl_n - 1] - x1) / (D[0] + 0.00000000001);
        lo = fmin(sa, sb);
        hi = fmax(sa, sb);
    }
    double sj = 0.0, sj1 = 0.0;
    for (int it = 0; it < 20; ++it) {
        sj = sj1;
        out[0] = x1 + D[0] * sj;
        out[1] = y1 + D[1] * sj;
        out[2] = zstart + D[2] * sj;
        double F;
        if (surface_eval(e, sd, out, F, n) != 0) {
            plen = s0 + sj;
            return 2;
        }
        const double dfd = n[0] * D[0] + n[1] * D[1] + n[2] * D[2];
        if (fabs(F) <= 0.000001 * fabs(dfd)) {
            plen = s0 + sj;
            return 0;
        }
        sj1 = sj - F / dfd;
        if (st == kSurfSpline) {
            if ((F < 0 && D[2] > 0) || (F > 0 && D[2] < 0))
                lo = fmax(sj, lo);
            else if ((F < 0 && D[2] < 0) || (F > 0 && D[2] > 0))
                hi = fmin(sj, hi);
            if (sj1 < lo || sj1 > hi) sj1 = 0.5 * (lo + hi);
            if (hi <= lo) break;
        }
    }
    plen = s0 + sj;
    return 1;
}

// ------------------------------------------------------------------------------------
// One candidate element (raytrace.cpp:716-769 + determineelementintersectionnew.cpp):
// transform to the element, nudge by 1e-5 along the ray, intersect, test the
// aperture, accept if z <= ZAperture (or a Zernike/polynomial surface).
// Returns true with plen (and, if full, the element-local hit, direction, normal
// and backside flag).
// ------------------------------------------------------------------------------------
struct Hit {
    double pe[3];  // hit point, element frame
    double ce[3];  // incoming direction, element frame
    double n[3];   // surface normal (flipped when hit from behind)
    double plen;
    int back;
};

// Surfaces that are rare in large fields (torus quartic, Newton-iterated conics,
// cones and file-defined surfaces) stay out of line so that the hot flat and
// closed-form quadric paths inline without call-saved registers.
static __device__ __noinline__ int cold_intersect(const SceneDev &S, const ElemRec &e, const double pe[3],
                                           const double ce[3], double out[3], double n[3], double &t) {
    if (e.stype == kSurfTorus) return torus_hit(e, pe, ce, out, n, t);
    return newton_hit(e, S.surf_data, pe, ce, out, n, t);
}

// CLOSED: the element is known to have a closed-form surface (closed_form_surface), so the
// out-of-line path is left out of the caller
template <int MIXED, int CLOSED = 0>
__device__ __forceinline__ bool element_test(const SceneDev &S, const ElemRec &e, const double ps[3],
                                             const double cs[3], double &plen, Hit *full) {
    double pe[3], ce[3];
    to_local(e.R, e.o, ps, cs, pe, ce);
    pe[0] = pe[0] + 1.0e-5 * ce[0];
    pe[1] = pe[1] + 1.0e-5 * ce[1];
    pe[2] = pe[2] + 1.0e-5 * ce[2];
    double out[3], n[3] = {0.0, 0.0, 1.0}, t = 0.0;
    int err;
    switch (e.stype) {
        case kSurfFlat: {
            // the Newton iteration on z = 0 converges at its first step (intersect.cpp:948-1007)
            t = (0.0 - pe[2] != 0.0) ? (0.0 - pe[2]) / (ce[2] + 0.00000000001) : 0.0;
            out[0] = pe[0] + ce[0] * t;
            out[1] = pe[1] + ce[1] * t;
            out[2] = 0.0;
            err = 0;
            break;
        }
        case kSurfCylinder:
            err = quadric_hit(e, pe, ce, out, n, t);
            break;
        case kSurfTorus:
            err = CLOSED ? 1 : cold_intersect(S, e, pe, ce, out, n, t);
            break;
        default: {
            const int s = e.surf | 0x20;
            const bool closed = (s == 'p') || (s == 's' && (e.stype == kSurfConic || e.stype == kSurfSingleAxis)) ||
                                (s == 'o' && e.stype == kSurfConic);
            if (closed)
                err = quadric_hit(e, pe, ce, out, n, t);
            else
                err = CLOSED ? 1 : cold_intersect(S, e, pe, ce, out, n, t);
        }
    }
    if (err > 0 || t < 0) return false;
    int in;
    if (MIXED)
        in = aperture_in<float>(e, float(out[0]), float(out[1]), false);
    else
        in = aperture_in<double>(e, out[0], out[1], false);
    if (in != 1) return false;
    const int s = e.surf | 0x20;
    if (!(out[2] <= e.zap || s == 'm' || s == 'r')) return false;
    plen = t;
    if (full) {
        const int back = (ce[0] * n[0] + ce[1] * n[1] + ce[2] * n[2] < 0) ? 0 : 1;
        for (int q = 0; q < 3; ++q) {
            full->pe[q] = out[q];
            full->ce[q] = ce[q];
            full->n[q] = back ? -n[q] : n[q];
        }
        full->plen = t;
        full->back = back;
    }
    return true;
}

// element_test for a flat element (surface type 3), without the other surfaces' code: the
// same arithmetic as element_test's flat branch, for kernels that only meet flat elements
template <int MIXED>
__device__ __forceinline__ bool element_test_flat(const ElemRec &e, const double ps[3], const double cs[3],
                                                  double &plen, Hit *full = nullptr) {
    double pe[3], ce[3];
    to_local(e.R, e.o, ps, cs, pe, ce);
    pe[0] = pe[0] + 1.0e-5 * ce[0];
    pe[1] = pe[1] + 1.0e-5 * ce[1];
    pe[2] = pe[2] + 1.0e-5 * ce[2];
    const double t = (0.0 - pe[2] != 0.0) ? (0.0 - pe[2]) / (ce[2] + 0.00000000001) : 0.0;
    if (t < 0) return false;
    const double ox = pe[0] + ce[0] * t, oy = pe[1] + ce[1] * t;
    const int in = MIXED ? aperture_in<float>(e, float(ox), float(oy), false) : aperture_in<double>(e, ox, oy, false);
    if (in != 1) return false;
    const int s = e.surf | 0x20;
    if (!(0.0 <= e.zap || s == 'm' || s == 'r')) return false;
    plen = t;
    if (full) {
        const int back = (ce[2] < 0) ? 0 : 1;
        full->pe[0] = ox;
        full->pe[1] = oy;
        full->pe[2] = 0.0;
        for (int q = 0; q < 3; ++q) full->ce[q] = ce[q];
        full->n[0] = back ? -0.0 : 0.0;  // the flipped normal of element_test, signed zeros included
        full->n[1] = back ? -0.0 : 0.0;
        full->n[2] = back ? -1.0 : 1.0;
        full->plen = t;
        full->back = back;
    }
    return true;
}

// ------------------------------------------------------------------------------------
// Error sampling (errors.cpp:60-226, surfacenormalerrors.cpp:58-167) with per-ray
// inverse-CDF samplers: |theta| of a 2-D Gaussian is Rayleigh, a pillbox disc is
// delta*sqrt(u), a table sunshape inverts the CDF of theta*I(theta), the diffuse
// distribution is asin(sqrt(u)); phi is an independent uniform as in the reference.
// ------------------------------------------------------------------------------------
// table sunshape: theta(u) tabulated at u = j / kSunInvCells, linear in between (mrad -> rad)
__device__ __forceinline__ double sample_table(const SunDev &sun, double u) {
    if (sun.inv_cdf == nullptr) return 0.0;  // no table was given (st_sun_userdata)
    const double x = u * kSunInvCells;
    const int j = min(int(x), kSunInvCells - 1);
    const double f = x - j;
    return (sun.inv_cdf[j] + f * (sun.inv_cdf[j + 1] - sun.inv_cdf[j])) / 1000.0;
}

__device__ __forceinline__ double sample_theta(int dist, double delop, double u, const SunDev &sun) {
    switch (dist) {
        case 'g':
        case 'G':
            return delop * sqrt(-2.0 * log(1.0 - u));
        case 'p':
        case 'P':
            return delop * sqrt(u);
        case 'd':
        case 'D':
            return sample_table(sun, u);
        case 'f':
        case 'F':
            return asin(sqrt(u));
        default:
            return 0.0;
    }
}

__device__ __forceinline__ float sample_theta_f(int dist, float delop, double u, const SunDev &sun) {
    switch (dist) {
        case 'g':
        case 'G':
            return delop * sqrtf(-2.f * __logf(float(1.0 - u)));  // 1 - u in double: never 0
        case 'p':
        case 'P':
            return delop * sqrtf(float(u));
        case 'd':
        case 'D':
            return float(sample_table(sun, u));
        case 'f':
        case 'F':
            return asinf(sqrtf(float(u)));
        default:
            return 0.f;
    }
}

// Rotate the local vector (sin t cos p, sin t sin p, cos t) out of the frame whose
// Euler angles are atan2(ax, az), atan2(ay, |(ax, az)|), 0 -- the reference's
// frame, including its choices when az == 0 -- without evaluating the angles.
template <typename T>
__device__ inline void perturb(const double axis[3], T theta, T phi, double out[3]) {
    const T ax = T(axis[0]), ay = T(axis[1]), az = T(axis[2]);
    T ca, sa, cb, sb;
    const T h = sqrt(ax * ax + az * az);
    if (az == T(0) && ax == T(0)) {
        ca = T(1);
        sa = T(0);
        cb = T(0);
        sb = T(1);
    } else {
        if (az == T(0)) {
            ca = T(0);
            sa = T(1);
        } else {
            ca = az / h;
            sa = ax / h;
        }
        const T m = sqrt(h * h + ay * ay);
        cb = h / m;
        sb = ay / m;
    }
    T st, ct, sp, cp;
    sincos_t(theta, st, ct);
    sincos_t(phi, sp, cp);
    const T lx = st * cp, ly = st * sp, lz = ct;
    out[0] = double(lx * ca - ly * sa * sb + lz * sa * cb);
    out[1] = double(ly * cb + lz * sb);
    out[2] = double(-lx * sa - ly * ca * sb + lz * ca * cb);
}

}  // namespace stb
