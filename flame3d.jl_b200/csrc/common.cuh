// common.cuh — shared device helpers for libflame3d_b200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "../../include/flame3d_b200.h"

#include <nvtx3/nvToolsExt.h>  // header-only; a no-op unless a profiler is attached

namespace flame {

constexpr double kEps = 2.220446049250313e-16;  // CUDA.eps(Float64), utils.jl:100
// Scheme constants, run.jl:51-57.
constexpr double kWenoEps = 1e-26;
constexpr double kHybrid1 = 1e-3;
constexpr double kHybrid2 = 0.1;
constexpr double kUP7_2 = 17.0 / 600, kUP7_3 = -23.0 / 120, kUP7_4 = 22.0 / 30, kUP7_5 = 0.5,
                 kUP7_6 = -0.075, kUP7_7 = 0.005;  // UP7[1] is 0 (run.jl:57)

// Extents of a ghosted grid; every array index is computed in 64-bit.
struct Dims {
    int nx, ny, nz, ng, ns;
    long long tx, ty, tz, np;
    __host__ __device__ long long P(long long i, long long j, long long k) const {
        return i + tx * (j + ty * k);
    }
};

inline Dims make_dims(const FlameGrid &g) {
    Dims d;
    d.nx = g.nx, d.ny = g.ny, d.nz = g.nz, d.ng = g.ng, d.ns = g.ns;
    d.tx = g.nx + 2LL * g.ng, d.ty = g.ny + 2LL * g.ng, d.tz = g.nz + 2LL * g.ng;
    d.np = d.tx * d.ty * d.tz;
    return d;
}

__device__ __forceinline__ double jmax(double a, double b) {  // Julia max: NaN-propagating
    if (a != a || b != b) return __longlong_as_double(0x7ff8000000000000LL);
    return a > b ? a : b;
}

__device__ __forceinline__ int64_t tag_at(const int64_t *tag, long long p) {
    return tag ? tag[p] : 0;
}

// ------------------------------------------------------------------ NASA-7 thermo (thermo.jl)
// h_specs, thermo.jl:107-133 (J/kg)
__device__ __forceinline__ double h_spec(const FlameThermo &th, int n, double T, double T2,
                                         double T3, double T4, double T5) {
    const double *lo = th.coeffs_lo + 7 * n;
    double h;
    if (T < th.coeffs_sep[n]) {
        h = lo[0] * T + lo[1] * T2 + lo[2] * T3 + lo[3] * T4 + lo[4] * T5;
    } else {
        const double *hc = th.coeffs_hi + 7 * n;
        h = hc[0] * T + hc[1] * T2 + hc[2] * T3 + hc[3] * T4 + hc[4] * T5 + (hc[5] - lo[5]);
    }
    return h * (th.Ru / th.mw[n]);
}

// cp_specs, thermo.jl:82-104 (dimensionless cp/R)
__device__ __forceinline__ double cp_spec(const FlameThermo &th, int n, double T, double T2,
                                          double T3, double T4) {
    const double *c = (T < th.coeffs_sep[n]) ? th.coeffs_lo + 7 * n : th.coeffs_hi + 7 * n;
    return c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4;
}

// ei_specs, thermo.jl:136-160 (dimensionless e/R)
__device__ __forceinline__ double ei_spec(const FlameThermo &th, int n, double T, double T2,
                                          double T3, double T4, double T5) {
    const double *lo = th.coeffs_lo + 7 * n;
    if (T < th.coeffs_sep[n])
        return (lo[0] - 1) * T + lo[1] * T2 + lo[2] * T3 + lo[3] * T4 + lo[4] * T5;
    const double *hc = th.coeffs_hi + 7 * n;
    return (hc[0] - 1) * T + hc[1] * T2 + hc[2] * T3 + hc[3] * T4 + hc[4] * T5 + (hc[5] - lo[5]);
}

// InternalEnergy, thermo.jl:219-228 (J/m^3)
template <int NS>
__device__ __forceinline__ double internal_energy(const FlameThermo &th, int ns, double T,
                                                  const double *rhoi) {
    double T2 = 0.5 * T * T;
    double T3 = 2.0 / 3.0 * T2 * T;
    double T4 = T2 * T2;
    double T5 = 0.8 * T4 * T;
    double r = 0;
    const int n_end = NS > 0 ? NS : ns;
#pragma unroll
    for (int n = 0; n < (NS > 0 ? NS : FLAME_MAX_NS); ++n) {
        if (n >= n_end) break;
        r += rhoi[n] * ei_spec(th, n, T, T2, T3, T4, T5) / th.mw[n];
    }
    return r * th.Ru;
}

// CV, thermo.jl:194-203 (J/(m^3 K))
template <int NS>
__device__ __forceinline__ double heat_cv(const FlameThermo &th, int ns, double T,
                                          const double *rhoi) {
    double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
    double r = 0;
    const int n_end = NS > 0 ? NS : ns;
#pragma unroll
    for (int n = 0; n < (NS > 0 ? NS : FLAME_MAX_NS); ++n) {
        if (n >= n_end) break;
        r += (cp_spec(th, n, T, T2, T3, T4) - 1) * rhoi[n] / th.mw[n];
    }
    return r * th.Ru;
}

// GetT, thermo.jl:231-282: Newton on e(T) with ±100 K step clamp and break-before-update.
template <int NS>
__device__ double get_T(const FlameThermo &th, int ns, double ein, const double *rhoi) {
    const double tol = 1e-3;
    const double tmin = th.min_temp, tmax = th.max_temp;
    const int n_end = NS > 0 ? NS : ns;
    double emin = internal_energy<NS>(th, ns, tmin, rhoi);
    double emax = internal_energy<NS>(th, ns, tmax, rhoi);
    if (ein < emin) return tmin - (emin - ein) / heat_cv<NS>(th, ns, tmin, rhoi);
    if (ein > emax) return tmax - (emax - ein) / heat_cv<NS>(th, ns, tmax, rhoi);
    double As = 0;
    for (int n = 0; n < n_end; ++n) As += (th.coeffs_lo[7 * n] - 1) * th.Ru / th.mw[n] * rhoi[n];
    double t1 = ein / As;
    if (t1 < tmin || t1 > tmax) t1 = tmin + (tmax - tmin) / (emax - emin) * (ein - emin);
    for (int it = 0; it < 30; ++it) {
        double e1 = internal_energy<NS>(th, ns, t1, rhoi);
        double cv = heat_cv<NS>(th, ns, t1, rhoi);
        double dt = (ein - e1) / cv;
        if (dt > 100.0)
            dt = 100.0;
        else if (dt < -100.0)
            dt = -100.0;
        else if (fabs(dt) < tol)
            break;
        else if (t1 + dt == t1)
            break;
        t1 += dt;
    }
    return t1;
}

// GetT for the fused stages: the same iteration as get_T (start, clamps, tolerance, break
// before the update), with e(T) and cv(T) of the mixture evaluated from its own polynomial.
// e/R and cv/R are linear in the species weights w_n = ρ_n / W_n, so the per-species NASA-7
// coefficients are summed once per cell into the mixture's coefficients for the low and the
// high range; an iteration then costs one polynomial instead of ns.  Where T lies between
// separators of different species the per-species sums are used.  The result differs from
// get_T by round-off only.
template <int NS>
struct MixPoly {
    double lo[5], hi[5], off, smin, smax;  // e/R = Σ_a c_a T_a (+ off in the high range)
    double wsum;                           // Σ_n w_n, so that Σ_n w_n cp_n = cv + Ru wsum
    const FlameThermo *th;
    const double *rhoi;
    __device__ __forceinline__ MixPoly(const FlameThermo &t, const double *r) : th(&t), rhoi(r) {
#pragma unroll
        for (int a = 0; a < 5; ++a) lo[a] = 0.0, hi[a] = 0.0;
        off = 0.0, wsum = 0.0;
        smin = smax = t.coeffs_sep[0];
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            const double w = r[n] / t.mw[n];
            wsum += w;
            const double *L = t.coeffs_lo + 7 * n, *H = t.coeffs_hi + 7 * n;
            lo[0] += w * (L[0] - 1), hi[0] += w * (H[0] - 1);
#pragma unroll
            for (int a = 1; a < 5; ++a) lo[a] += w * L[a], hi[a] += w * H[a];
            off += w * (H[5] - L[5]);
            smin = fmin(smin, t.coeffs_sep[n]), smax = fmax(smax, t.coeffs_sep[n]);
        }
    }
    __device__ __forceinline__ double e(double T) const {  // InternalEnergy, J/m^3
        if (T >= smin && T < smax) return internal_energy<NS>(*th, NS, T, rhoi);
        const double T2 = 0.5 * T * T, T3 = 2.0 / 3.0 * T2 * T, T4 = T2 * T2, T5 = 0.8 * T4 * T;
        const double *c = T < smin ? lo : hi;
        const double r = c[0] * T + c[1] * T2 + c[2] * T3 + c[3] * T4 + c[4] * T5;
        return (T < smin ? r : r + off) * th->Ru;
    }
    __device__ __forceinline__ double cv(double T) const {  // CV, J/(m^3 K)
        if (T >= smin && T < smax) return heat_cv<NS>(*th, NS, T, rhoi);
        const double *c = T < smin ? lo : hi;
        const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
        return (c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4) * th->Ru;
    }
};

template <int NS>
__device__ double get_T_mix(const MixPoly<NS> &M, const FlameThermo &th, double ein,
                            const double *rhoi) {
    const double tol = 1e-3;
    const double tmin = th.min_temp, tmax = th.max_temp;
    const double emin = M.e(tmin), emax = M.e(tmax);
    if (ein < emin) return tmin - (emin - ein) / M.cv(tmin);
    if (ein > emax) return tmax - (emax - ein) / M.cv(tmax);
    double As = 0;
    for (int n = 0; n < NS; ++n) As += (th.coeffs_lo[7 * n] - 1) * th.Ru / th.mw[n] * rhoi[n];
    double t1 = ein / As;
    if (t1 < tmin || t1 > tmax) t1 = tmin + (tmax - tmin) / (emax - emin) * (ein - emin);
    for (int it = 0; it < 30; ++it) {
        double dt = (ein - M.e(t1)) / M.cv(t1);
        if (dt > 100.0)
            dt = 100.0;
        else if (dt < -100.0)
            dt = -100.0;
        else if (fabs(dt) < tol)
            break;
        else if (t1 + dt == t1)
            break;
        t1 += dt;
    }
    return t1;
}

// Pmixture, thermo.jl:20-26
template <int NS>
__device__ __forceinline__ double p_mixture(const FlameThermo &th, int ns, double T,
                                            const double *rhoi) {
    double yow = 0;
    const int n_end = NS > 0 ? NS : ns;
#pragma unroll
    for (int n = 0; n < (NS > 0 ? NS : FLAME_MAX_NS); ++n) {
        if (n >= n_end) break;
        yow += rhoi[n] / th.mw[n];
    }
    return th.Ru * T * yow;
}

// ----------------------------------------------------------- hybrid reconstruction (schemes.jl)
template <typename T>
__device__ __forceinline__ T minmod(T a, T b) {  // schemes.jl:26-28
    return (a * b > 0) ? ((fabs(a) > fabs(b)) ? b : a) : T(0);
}

// WENO-Z weights and combination, schemes.jl:152-162, for the 1:1 kernels: the smoothness
// indicators come in the arithmetic type T and the weights are formed in FP64 in the reference's
// four-division form (in plain FP32, q = τ/(1e-26 + β) overflows when a one-sided split makes β
// exactly 0, and ∞·0 would poison the flux; wenoz_combine_fast<float> below avoids that).
template <typename T>
__device__ __forceinline__ T wenoz_combine(T s11_, T s22_, T s33_, T v1, T v2, T v3) {
    const double s11 = s11_, s22 = s22_, s33 = s33_;
    const double tau = fabs(s11 - s33);
    double q, a1, a2, a3;
    q = tau / (kWenoEps + s11), a1 = (1 + q * q) * 1;
    q = tau / (kWenoEps + s22), a2 = (1 + q * q) * 6;
    q = tau / (kWenoEps + s33), a3 = (1 + q * q) * 3;
    const double invsum = 1 / (a1 + a2 + a3);
    return T((1.0 / 6.0) * invsum * (a1 * double(v1) + a2 * double(v2) + a3 * double(v3)));
}

// WENO-Z5 positive-flux reconstruction from V1..V5 = F+[c-3..c+1], schemes.jl:139-162
template <typename T>
__device__ __forceinline__ T wenoz_plus(T V1, T V2, T V3, T V4, T V5) {
    const T tmp1 = T(13.0 / 12.0), q4 = T(0.25);
    T a, b;
    a = V1 - 2 * V2 + V3, b = V1 - 4 * V2 + 3 * V3;
    const T s11 = tmp1 * (a * a) + q4 * (b * b);
    a = V2 - 2 * V3 + V4, b = V2 - V4;
    const T s22 = tmp1 * (a * a) + q4 * (b * b);
    a = V3 - 2 * V4 + V5, b = 3 * V3 - 4 * V4 + V5;
    const T s33 = tmp1 * (a * a) + q4 * (b * b);
    return wenoz_combine<T>(s11, s22, s33, 2 * V1 - 7 * V2 + 11 * V3, -V2 + 5 * V3 + 2 * V4,
                            2 * V3 + 5 * V4 - V5);
}

// WENO-Z5 negative-flux reconstruction from V1..V5 = F-[c-2..c+2], schemes.jl:164-187
template <typename T>
__device__ __forceinline__ T wenoz_minus(T V1, T V2, T V3, T V4, T V5) {
    const T tmp1 = T(13.0 / 12.0), q4 = T(0.25);
    T a, b;
    a = V5 - 2 * V4 + V3, b = V5 - 4 * V4 + 3 * V3;
    const T s11 = tmp1 * (a * a) + q4 * (b * b);
    a = V2 - 2 * V3 + V4, b = V4 - V2;
    const T s22 = tmp1 * (a * a) + q4 * (b * b);
    a = V3 - 2 * V2 + V1, b = 3 * V3 - 4 * V2 + V1;
    const T s33 = tmp1 * (a * a) + q4 * (b * b);
    return wenoz_combine<T>(s11, s22, s33, 11 * V3 - 7 * V4 + 2 * V5, -V4 + 5 * V3 + 2 * V2,
                            2 * V3 + 5 * V2 - V1);
}

// The same WENO-Z combination with one division instead of four: with b_k = ε + β_k,
// α_k = d_k (1 + τ²/b_k²) and ω_k = α_k / Σα; multiplying every α_k by b_1² b_2² b_3² gives
// A_k = d_k (b_k² + τ²) Π_{j≠k} b_j² with the same ratios.  Exact in real arithmetic; in FP64 it
// differs from the reference's rounding by a few ulp (the products stay in range for |β| < 1e50).
template <typename T>
__device__ __forceinline__ T wenoz_combine_fast(T s11_, T s22_, T s33_, T v1, T v2, T v3) {
    const double b1 = kWenoEps + double(s11_), b2 = kWenoEps + double(s22_),
                 b3 = kWenoEps + double(s33_);
    const double tau = fabs(double(s11_) - double(s33_));
    const double t = tau * tau;
    const double p1 = b1 * b1, p2 = b2 * b2, p3 = b3 * b3;
    const double a1 = (p1 + t) * (p2 * p3);
    const double a2 = 6.0 * (p2 + t) * (p1 * p3);
    const double a3 = 3.0 * (p3 + t) * (p1 * p2);
    return T((a1 * double(v1) + a2 * double(v2) + a3 * double(v3)) / (6.0 * (a1 + a2 + a3)));
}

// FP32 form for the mixed-precision paths, in the reference's own shape α_k = d_k (1 + q_k²),
// q_k = τ / (ε + β_k), with every step kept inside FP32 range: q_k is capped at 1e15 (a stencil
// with q_k that large already carries weight 1 to FP32 precision; when two are capped their
// candidate values agree to far below FP32 resolution, since β_k < 1e-15 τ bounds their second
// differences), the α_k are normalised by their sum before they multiply the candidates, and
// the divisions are the fast approximate ones (2 ulp), ample for weights in FP32.
template <>
__device__ __forceinline__ float wenoz_combine_fast<float>(float s11, float s22, float s33,
                                                           float v1, float v2, float v3) {
    constexpr float eps = float(kWenoEps), qmax = 1e15f;
    const float tau = fabsf(s11 - s33);
    const float q1 = fminf(__fdividef(tau, eps + s11), qmax);
    const float q2 = fminf(__fdividef(tau, eps + s22), qmax);
    const float q3 = fminf(__fdividef(tau, eps + s33), qmax);
    const float a1 = 1.0f + q1 * q1, a2 = 6.0f * (1.0f + q2 * q2), a3 = 3.0f * (1.0f + q3 * q3);
    const float r = __fdividef(1.0f, a1 + a2 + a3);
    return (1.0f / 6.0f) * ((a1 * r) * v1 + (a2 * r) * v2 + (a3 * r) * v3);
}

// wenoz_combine_fast<double> as a fraction N / D (so two faces can share one division).
__device__ __forceinline__ void wenoz_fraction(double s11, double s22, double s33, double v1,
                                               double v2, double v3, double &N, double &D) {
    const double b1 = kWenoEps + s11, b2 = kWenoEps + s22, b3 = kWenoEps + s33;
    const double tau = fabs(s11 - s33);
    const double t = tau * tau;
    const double p1 = b1 * b1, p2 = b2 * b2, p3 = b3 * b3;
    const double a1 = (p1 + t) * (p2 * p3);
    const double a2 = 6.0 * (p2 + t) * (p1 * p3);
    const double a3 = 3.0 * (p3 + t) * (p1 * p2);
    N = a1 * v1 + a2 * v2 + a3 * v3;
    D = 6.0 * (a1 + a2 + a3);
}

__device__ __forceinline__ void wenoz_plus_fraction(double V1, double V2, double V3, double V4,
                                                    double V5, double &N, double &D) {
    const double tmp1 = 13.0 / 12.0, q4 = 0.25;
    double a, b;
    a = V1 - 2 * V2 + V3, b = V1 - 4 * V2 + 3 * V3;
    const double s11 = tmp1 * (a * a) + q4 * (b * b);
    a = V2 - 2 * V3 + V4, b = V2 - V4;
    const double s22 = tmp1 * (a * a) + q4 * (b * b);
    a = V3 - 2 * V4 + V5, b = 3 * V3 - 4 * V4 + V5;
    const double s33 = tmp1 * (a * a) + q4 * (b * b);
    wenoz_fraction(s11, s22, s33, 2 * V1 - 7 * V2 + 11 * V3, -V2 + 5 * V3 + 2 * V4,
                   2 * V3 + 5 * V4 - V5, N, D);
}

__device__ __forceinline__ void wenoz_minus_fraction(double V1, double V2, double V3, double V4,
                                                     double V5, double &N, double &D) {
    const double tmp1 = 13.0 / 12.0, q4 = 0.25;
    double a, b;
    a = V5 - 2 * V4 + V3, b = V5 - 4 * V4 + 3 * V3;
    const double s11 = tmp1 * (a * a) + q4 * (b * b);
    a = V2 - 2 * V3 + V4, b = V4 - V2;
    const double s22 = tmp1 * (a * a) + q4 * (b * b);
    a = V3 - 2 * V2 + V1, b = 3 * V3 - 4 * V2 + V1;
    const double s33 = tmp1 * (a * a) + q4 * (b * b);
    wenoz_fraction(s11, s22, s33, 11 * V3 - 7 * V4 + 2 * V5, -V4 + 5 * V3 + 2 * V2,
                   2 * V3 + 5 * V2 - V1, N, D);
}

template <typename T>
__device__ __forceinline__ T wenoz_plus_fast(T V1, T V2, T V3, T V4, T V5) {
    const T tmp1 = T(13.0 / 12.0), q4 = T(0.25);
    T a, b;
    a = V1 - 2 * V2 + V3, b = V1 - 4 * V2 + 3 * V3;
    const T s11 = tmp1 * (a * a) + q4 * (b * b);
    a = V2 - 2 * V3 + V4, b = V2 - V4;
    const T s22 = tmp1 * (a * a) + q4 * (b * b);
    a = V3 - 2 * V4 + V5, b = 3 * V3 - 4 * V4 + V5;
    const T s33 = tmp1 * (a * a) + q4 * (b * b);
    return wenoz_combine_fast<T>(s11, s22, s33, 2 * V1 - 7 * V2 + 11 * V3, -V2 + 5 * V3 + 2 * V4,
                                 2 * V3 + 5 * V4 - V5);
}

template <typename T>
__device__ __forceinline__ T wenoz_minus_fast(T V1, T V2, T V3, T V4, T V5) {
    const T tmp1 = T(13.0 / 12.0), q4 = T(0.25);
    T a, b;
    a = V5 - 2 * V4 + V3, b = V5 - 4 * V4 + 3 * V3;
    const T s11 = tmp1 * (a * a) + q4 * (b * b);
    a = V2 - 2 * V3 + V4, b = V4 - V2;
    const T s22 = tmp1 * (a * a) + q4 * (b * b);
    a = V3 - 2 * V2 + V1, b = 3 * V3 - 4 * V2 + V1;
    const T s33 = tmp1 * (a * a) + q4 * (b * b);
    return wenoz_combine_fast<T>(s11, s22, s33, 11 * V3 - 7 * V4 + 2 * V5, -V4 + 5 * V3 + 2 * V2,
                                 2 * V3 + 5 * V2 - V1);
}

// One face of the hybrid scheme for the fused paths: hybrid_face7 (below) with the
// one-division WENO-Z weights.
template <typename T>
__device__ __forceinline__ T hybrid_face_fast(const T *p, const T *m, T phif) {
    T fp, fm;
    if (phif < T(kHybrid1)) {
        fp = T(kUP7_2) * p[0] + T(kUP7_3) * p[1] + T(kUP7_4) * p[2] + T(kUP7_5) * p[3] +
             T(kUP7_6) * p[4] + T(kUP7_7) * p[5];
        fm = T(kUP7_7) * m[0] + T(kUP7_6) * m[1] + T(kUP7_5) * m[2] + T(kUP7_4) * m[3] +
             T(kUP7_3) * m[4] + T(kUP7_2) * m[5];
    } else if (phif < T(kHybrid2)) {
        if constexpr (sizeof(T) == 8) {
            // FP64: F+ and F- share one division, Np/Dp + Nm/Dm = (Np Dm + Nm Dp) / (Dp Dm),
            // while the product of the denominators stays inside the normal range
            double Np, Dp, Nm, Dm;
            wenoz_plus_fraction(p[0], p[1], p[2], p[3], p[4], Np, Dp);
            wenoz_minus_fraction(m[1], m[2], m[3], m[4], m[5], Nm, Dm);
            const double den = Dp * Dm;
            if (den > 1e-300 && den < 1e300) return (Np * Dm + Nm * Dp) / den;
            return Np / Dp + Nm / Dm;
        } else {
            fp = wenoz_plus_fast(p[0], p[1], p[2], p[3], p[4]);
            fm = wenoz_minus_fast(m[1], m[2], m[3], m[4], m[5]);
        }
    } else {
        fp = p[2] + T(0.5) * minmod(p[3] - p[2], p[2] - p[1]);
        fm = m[3] - T(0.5) * minmod(m[4] - m[3], m[3] - m[2]);
    }
    return fp + fm;
}

// One face of the hybrid scheme, schemes.jl:110-199.  p[0..6] = F+[c-3..c+3] (F+[c-4] has
// weight UP7[1] = 0 and is not read), m[0..6] = F-[c-3..c+3]; the face lies between c-1 and c.
template <typename T>
__device__ __forceinline__ T hybrid_face7(const T *p, const T *m, T phif) {
    T fp, fm;
    if (phif < T(kHybrid1)) {
        fp = T(kUP7_2) * p[0] + T(kUP7_3) * p[1] + T(kUP7_4) * p[2] + T(kUP7_5) * p[3] +
             T(kUP7_6) * p[4] + T(kUP7_7) * p[5];
        fm = T(kUP7_7) * m[0] + T(kUP7_6) * m[1] + T(kUP7_5) * m[2] + T(kUP7_4) * m[3] +
             T(kUP7_3) * m[4] + T(kUP7_2) * m[5];
    } else if (phif < T(kHybrid2)) {
        fp = wenoz_plus(p[0], p[1], p[2], p[3], p[4]);
        fm = wenoz_minus(m[1], m[2], m[3], m[4], m[5]);
    } else {
        fp = p[2] + T(0.5) * minmod(p[3] - p[2], p[2] - p[1]);
        fm = m[3] - T(0.5) * minmod(m[4] - m[3], m[3] - m[2]);
    }
    return fp + fm;
}

// ---- mixtureProperties, thermo.jl:284-369 (transport law 2) in the reference's order.
// dot5, thermo.jl:284-286
__device__ __forceinline__ double dot5(double l1, double l2, double l3, double l4,
                                       const double *p) {
    return p[0] + l1 * p[1] + l2 * p[2] + l3 * p[3] + l4 * p[4];
}

// X: mole fractions; poly: visc (5, ns) | conduct (5, ns) | binarydiff (5, ns, ns).  Writes the
// mixture-averaged D_k to Dk[n * stride] and returns λ, μ.  W is an ns*ns work array.
__device__ __forceinline__ void mixture_properties(double T, double P, const double *X,
                                                   const FlameThermo &th, const double *poly,
                                                   int ns, double *W, double *mui, double *Dk,
                                                   long long stride, double &lam, double &mu) {
    const double *visc = poly, *cond = poly + 5 * ns, *bin = poly + 10 * ns;
    const double sqT = sqrt(T), sqsqT = sqrt(sqT), lgT = log(T);
    const double lgT2 = lgT * lgT, lgT3 = lgT * lgT2, lgT4 = lgT2 * lgT2;
    for (int n = 0; n < ns; ++n) mui[n] = sqT * dot5(lgT, lgT2, lgT3, lgT4, cond + 5 * n);
    double sum1 = 0, sum2 = 0;
    for (int k = 0; k < ns; ++k) sum1 += X[k] * mui[k], sum2 += X[k] / mui[k];
    lam = 0.5 * (sum1 + 1 / sum2);
    for (int n = 0; n < ns; ++n) {
        const double s = sqsqT * dot5(lgT, lgT2, lgT3, lgT4, visc + 5 * n);
        mui[n] = s * s;
    }
    for (int n = 0; n < ns; ++n) {  // Wilke, W[n*ns + l] is the reference's D[(n-1)*Nspecs+l]
        const double tmp1 = 1 / th.mw[n], tmp2 = mui[n];
        for (int l = 0; l <= n; ++l) {
            const double wr = th.mw[l] * tmp1, vr = tmp2 / mui[l];
            const double f1 = 1 + sqrt(vr * sqrt(wr));
            const double t = f1 * f1 / sqrt(8 + 8 / wr);
            W[n * ns + l] = t;
            W[l * ns + n] = t / (vr * wr);
        }
        W[n * ns + n] = 1.0;
    }
    mu = 0;
    for (int n = 0; n < ns; ++n) {
        double t = 0.0;
        for (int l = 0; l < ns; ++l) t += X[l] * W[n * ns + l];
        mu += X[n] * mui[n] / t;
    }
    for (int n = 0; n < ns; ++n)
        for (int m = n; m < ns; ++m) {
            const double t = T * sqT * dot5(lgT, lgT2, lgT3, lgT4, bin + 5 * (m + ns * n));
            W[m * ns + n] = t;
            W[n * ns + m] = t;
        }
    for (int n = 0; n < ns; ++n) {
        double s = 0.0;
        for (int m = 0; m < ns; ++m) {
            if (m == n) continue;
            s += X[m] / W[n * ns + m];
        }
        s *= P;
        Dk[n * stride] = (1 - X[n]) / (s + kEps);
    }
}

// mixtureProperties (thermo.jl:289-369) for a compile-time species count, without the ns x ns
// work array of mixture_properties: the Wilke factors W[n][l] and W[l][n] come from the same
// pair terms, and the binary-diffusion matrix is symmetric, so each pair is evaluated once and
// added to both rows' sums.  Every row sum still takes its terms in the order l = 0 .. NS-1 of
// the reference's loops (row n's terms l < n arrive in iteration n, its terms l > n in the
// later iterations, in increasing order), and each term is the reference's expression.
//
// The block's MixTables hold the terms of the Wilke factors that depend on the molar masses
// alone (for the pair (n, l) at n * NS + l: 1 / wr with wr = W_l / W_n, sqrt(wr) and
// 1 / sqrt(8 + 8 / wr), each formed in FP64).  The per-point divisions of the reference's
// expressions become products with reciprocals (1 / μ_l once per species, 1 / D_nm once per
// pair): the same formulas, each term within a few ulps of the reference's, at a third of the
// divisions and square roots.  MT is the arithmetic type: double on the FP64 path; float on the
// mixed path, which stores μ, λ and D_k in FP32 anyway (the tables then also hold the
// polynomial fits rounded to FP32 once per block).
template <int NS, typename MT>
struct MixTables {
    MT pw[3 * NS * NS];
    MT poly[sizeof(MT) == 4 ? 10 * NS + 5 * NS * NS : 1];
};

template <int NS, typename MT>
__device__ __forceinline__ void mix_tables_fill(const FlameThermo &th, const FlameTransport &tr,
                                                MixTables<NS, MT> &t) {
    for (int i = threadIdx.x; i < NS * NS; i += blockDim.x) {
        const int n = i / NS, l = i % NS;
        const double tmp1 = 1 / th.mw[n];
        const double wr = th.mw[l] * tmp1;
        t.pw[i] = MT(1 / wr);
        t.pw[NS * NS + i] = MT(sqrt(wr));
        t.pw[2 * NS * NS + i] = MT(1 / sqrt(8 + 8 / wr));
    }
    if constexpr (sizeof(MT) == 4) {
        for (int i = threadIdx.x; i < 10 * NS + 5 * NS * NS; i += blockDim.x)
            t.poly[i] = MT(tr.poly[i]);
    }
}

template <typename MT>
__device__ __forceinline__ MT dot5t(MT l1, MT l2, MT l3, MT l4, const MT *p) {
    return p[0] + l1 * p[1] + l2 * p[2] + l3 * p[3] + l4 * p[4];
}

template <int NS, typename MT>
__device__ __forceinline__ void mixture_properties_pairs(MT T, MT P, const MT *X, const MT *pw,
                                                         const MT *poly, MT *Dk, MT &lam,
                                                         MT &mu) {
    const MT *visc = poly, *cond = poly + 5 * NS, *bin = poly + 10 * NS;
    const MT sqT = sqrt(T), sqsqT = sqrt(sqT), lgT = log(T);
    const MT lgT2 = lgT * lgT, lgT3 = lgT * lgT2, lgT4 = lgT2 * lgT2;
    MT mui[NS], row[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) mui[n] = sqT * dot5t<MT>(lgT, lgT2, lgT3, lgT4, cond + 5 * n);
    MT sum1 = 0, sum2 = 0;
#pragma unroll
    for (int k = 0; k < NS; ++k) sum1 += X[k] * mui[k], sum2 += X[k] / mui[k];
    lam = MT(0.5) * (sum1 + 1 / sum2);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        const MT s = sqsqT * dot5t<MT>(lgT, lgT2, lgT3, lgT4, visc + 5 * n);
        mui[n] = s * s;
        row[n] = 0;
    }
    MT rmu[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) rmu[n] = 1 / mui[n];
#pragma unroll
    for (int n = 0; n < NS; ++n) {  // Wilke: row[n] = Σ_l X[l] W[n][l]
#pragma unroll
        for (int l = 0; l < n; ++l) {
            const int i = n * NS + l;
            const MT vr = mui[n] * rmu[l];  // μ_n / μ_l
            const MT f1 = 1 + sqrt(vr * pw[NS * NS + i]);
            const MT t = f1 * f1 * pw[2 * NS * NS + i];
            row[n] += X[l] * t;                                 // W[n][l]
            row[l] += X[n] * (t * (mui[l] * rmu[n]) * pw[i]);  // W[l][n] = t / (vr wr)
        }
        row[n] += X[n] * MT(1);  // W[n][n]
    }
    mu = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n) mu += X[n] * mui[n] / row[n];
#pragma unroll
    for (int n = 0; n < NS; ++n) row[n] = 0;  // now Σ_{m≠n} X[m] / Dbin[n][m]
#pragma unroll
    for (int n = 0; n < NS; ++n)
#pragma unroll
        for (int m = n + 1; m < NS; ++m) {
            const MT t = T * sqT * dot5t<MT>(lgT, lgT2, lgT3, lgT4, bin + 5 * (m + NS * n));
            const MT rt = 1 / t;
            row[n] += X[m] * rt;
            row[m] += X[n] * rt;
        }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        const MT s = row[n] * P;
        Dk[n] = (1 - X[n]) / (s + MT(kEps));
    }
}

// The reference's mixture kernel at one point with law 2 (thermo.jl:371-403): Y = max(ρi/ρ, 0)
// with ρ = max(Q_ρ, eps), X from Y (Y2X, thermo.jl:38-52), then mixtureProperties in MT.  The
// fused stage stores the result as μ, λ, D_0 .. D_{NS-1}.  mt: the block's MixTables.
template <int NS, typename MT>
__device__ __forceinline__ void mixture_point(const FlameThermo &th, const FlameTransport &tr,
                                              const MixTables<NS, MT> &mt, double T, double P,
                                              double rho_raw, const double *r, double &mu,
                                              double &lam, double *Dk) {
    const double rhoinv = 1 / jmax(rho_raw, kEps);
    double X[NS];
    double yow = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n) X[n] = jmax(r[n] * rhoinv, 0.0), yow += X[n] / th.mw[n];
    const double yowinv = 1 / yow;
#pragma unroll
    for (int n = 0; n < NS; ++n) X[n] = X[n] / th.mw[n] * yowinv;
    if constexpr (sizeof(MT) == 8) {
        mixture_properties_pairs<NS, double>(T, P, X, mt.pw, tr.poly, Dk, lam, mu);
    } else {
        MT Xm[NS], Dm[NS], lm, mm;
#pragma unroll
        for (int n = 0; n < NS; ++n) Xm[n] = MT(X[n]);
        mixture_properties_pairs<NS, MT>(MT(T), MT(P), Xm, mt.pw, mt.poly, Dm, lm, mm);
        lam = lm, mu = mm;
#pragma unroll
        for (int n = 0; n < NS; ++n) Dk[n] = Dm[n];
    }
}

// An NVTX range over a host-side scope (stage launches show up by name in Nsight timelines).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

}  // namespace flame

// Error plumbing shared by every C entry point (defined in capi.cu).
int flame_fail(int code, const char *fmt, ...);
int flame_check_launch(const char *what);
int flame_check_grid(const FlameGrid *g, const char *what);
