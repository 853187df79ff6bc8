// flame_oracle.cpp — TEST INFRASTRUCTURE ONLY (the oracle).
//
// A CPU, FP64, strictly IEEE restatement of Flame3D.jl's per-stage right-hand side and RK3
// stage update.  It is the parity target of the sm_100a kernels and the timed CPU baseline.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm may load it;
// the product library never does.
//
// Parity status: the reference ships no golden vectors, no asserting tests and no CPU path
// (its RHS exists only as CUDA.jl kernel bodies and Julia is not installed), so this oracle is
// "parity unpinned" against the reference itself.  It is pinned by known-answer tests instead
// (UP7 constants regenerated from the reference's own Utils/FDMcoeffs.py, Steger-Warming
// F+ + F- = F, polynomial exactness, GetT round trip, free-stream preservation, conservation).
//
// Every function follows the reference kernel it names (file:line in the comment) in index
// range, masking, and floating point operation order (Julia evaluates a+b+c as (a+b)+c and
// x^2 as x*x).  Build with -ffp-contract=off so no multiply-add is fused.
//
// Layout: ghosted point (i,j,k,n), 0-based, at i + Tx*(j + Ty*(k + Tz*n)); face arrays are
// (N+1 on the swept axis) x (N on the others) x NV, unghosted.  Reference 1-based index r maps
// to 0-based r-1 throughout.

#include "../include/flame3d_b200.h"

#include <cmath>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <cstring>
#include <utility>
#include <vector>

namespace {

constexpr double kEps = 2.220446049250313e-16;  // CUDA.eps(Float64)
// run.jl:51-57
constexpr double kWenoEps = 1e-26;
constexpr double kHybrid1 = 1e-3;
constexpr double kHybrid2 = 0.1;
const double kUP7[7] = {0.0, 17.0 / 600, -23.0 / 120, 22.0 / 30, 0.5, -0.075, 0.005};

struct Dims {
    int nx, ny, nz, ng, ns;
    long tx, ty, tz, np;
    explicit Dims(const FlameGrid *g)
        : nx(g->nx), ny(g->ny), nz(g->nz), ng(g->ng), ns(g->ns), tx(g->nx + 2L * g->ng),
          ty(g->ny + 2L * g->ng), tz(g->nz + 2L * g->ng), np(tx * ty * tz) {}
    long P(long i, long j, long k) const { return i + tx * (j + ty * k); }
};

inline double jmax(double a, double b) {  // Julia max: NaN-propagating
    if (a != a || b != b) return NAN;
    return a > b ? a : b;
}
inline int64_t tagat(const int64_t *tag, long p) { return tag ? tag[p] : 0; }

// Face-array geometry for the swept direction d: extents and the ghosted "right cell" of face.
struct Faces {
    long fx, fy, fz;  // face array extents
    long sn;          // ghosted stride along the normal
    long st1, st2;    // ghosted strides of the two tangential directions (in xi, eta, zeta order)
    int d;
};
Faces faces_of(const Dims &D, int d) {
    Faces f;
    f.d = d;
    f.fx = D.nx + (d == 0);
    f.fy = D.ny + (d == 1);
    f.fz = D.nz + (d == 2);
    const long s[3] = {1, D.tx, D.tx * D.ty};
    f.sn = s[d];
    f.st1 = s[(d + 1) % 3];
    f.st2 = s[(d + 2) % 3];
    return f;
}

// ----------------------------------------------------------------------------------- thermo
// thermo.jl:107-133 h_specs
void h_specs(double *hi, double T, const FlameThermo *th, int ns) {
    double T2 = 0.5 * T * T;
    double T3 = 2.0 / 3.0 * T2 * T;
    double T4 = T2 * T2;
    double T5 = 0.8 * T4 * T;
    for (int n = 0; n < ns; ++n) {
        const double *lo = th->coeffs_lo + 7 * n, *hc = th->coeffs_hi + 7 * n;
        if (T < th->coeffs_sep[n])
            hi[n] = lo[0] * T + lo[1] * T2 + lo[2] * T3 + lo[3] * T4 + lo[4] * T5;
        else
            hi[n] = hc[0] * T + hc[1] * T2 + hc[2] * T3 + hc[3] * T4 + hc[4] * T5 +
                    (hc[5] - lo[5]);
        hi[n] *= th->Ru / th->mw[n];
    }
}
// thermo.jl:82-104 cp_specs
void cp_specs(double *cp, double T, const FlameThermo *th, int ns) {
    double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
    for (int n = 0; n < ns; ++n) {
        const double *c = (T < th->coeffs_sep[n]) ? th->coeffs_lo + 7 * n : th->coeffs_hi + 7 * n;
        cp[n] = c[0] + c[1] * T + c[2] * T2 + c[3] * T3 + c[4] * T4;
    }
}
// thermo.jl:136-160 ei_specs
void ei_specs(double *ei, double T, const FlameThermo *th, int ns) {
    double T2 = 0.5 * T * T;
    double T3 = 2.0 / 3.0 * T2 * T;
    double T4 = T2 * T2;
    double T5 = 0.8 * T4 * T;
    for (int n = 0; n < ns; ++n) {
        const double *lo = th->coeffs_lo + 7 * n, *hc = th->coeffs_hi + 7 * n;
        if (T < th->coeffs_sep[n])
            ei[n] = (lo[0] - 1) * T + lo[1] * T2 + lo[2] * T3 + lo[3] * T4 + lo[4] * T5;
        else
            ei[n] = (hc[0] - 1) * T + hc[1] * T2 + hc[2] * T3 + hc[3] * T4 + hc[4] * T5 +
                    (hc[5] - lo[5]);
    }
}
// thermo.jl:194-203 CV
double CV(double T, const double *rhoi, const FlameThermo *th, int ns) {
    double cp[FLAME_MAX_NS];
    cp_specs(cp, T, th, ns);
    double r = 0;
    for (int n = 0; n < ns; ++n) r += (cp[n] - 1) * rhoi[n] / th->mw[n];
    return r * th->Ru;
}
// thermo.jl:206-215 CP
double CPv(double T, const double *rhoi, const FlameThermo *th, int ns) {
    double cp[FLAME_MAX_NS];
    cp_specs(cp, T, th, ns);
    double r = 0;
    for (int n = 0; n < ns; ++n) r += cp[n] * rhoi[n] / th->mw[n];
    return r * th->Ru;
}
// thermo.jl:219-228 InternalEnergy
double InternalEnergy(double T, const double *rhoi, const FlameThermo *th, int ns) {
    double ei[FLAME_MAX_NS];
    ei_specs(ei, T, th, ns);
    double r = 0;
    for (int n = 0; n < ns; ++n) r += rhoi[n] * ei[n] / th->mw[n];
    return r * th->Ru;
}
// thermo.jl:20-26 Pmixture
double Pmixture(double T, const double *rhoi, const FlameThermo *th, int ns) {
    double yow = 0;
    for (int n = 0; n < ns; ++n) yow += rhoi[n] / th->mw[n];
    return th->Ru * T * yow;
}
// thermo.jl:231-282 GetT (Newton with break-before-update)
double GetT(double ein, const double *rhoi, const FlameThermo *th, int ns) {
    const int maxiter = 30;
    const double tol = 1e-3;
    const double tmin = th->min_temp, tmax = th->max_temp;
    double emin = InternalEnergy(tmin, rhoi, th, ns);
    double emax = InternalEnergy(tmax, rhoi, th, ns);
    if (ein < emin) {
        double cv = CV(tmin, rhoi, th, ns);
        return tmin - (emin - ein) / cv;
    }
    if (ein > emax) {
        double cv = CV(tmax, rhoi, th, ns);
        return tmax - (emax - ein) / cv;
    }
    double As = 0;
    for (int n = 0; n < ns; ++n) As += (th->coeffs_lo[7 * n] - 1) * th->Ru / th->mw[n] * rhoi[n];
    double t1 = ein / As;
    if (t1 < tmin || t1 > tmax) t1 = tmin + (tmax - tmin) / (emax - emin) * (ein - emin);
    for (int it = 0; it < maxiter; ++it) {
        double e1 = InternalEnergy(t1, rhoi, th, ns);
        double cv = CV(t1, rhoi, th, ns);
        double dt = (ein - e1) / cv;
        if (dt > 100.0)
            dt = 100.0;
        else if (dt < -100.0)
            dt = -100.0;
        else if (std::fabs(dt) < tol)
            break;
        else if (t1 + dt == t1)
            break;
        t1 += dt;
    }
    return t1;
}

// ------------------------------------------------------------------------------ reconstruction
inline double minmod(double a, double b) {  // schemes.jl:26-28
    return (a * b > 0) ? ((std::fabs(a) > std::fabs(b)) ? b : a) : 0.0;
}

// One face of WENO_x/y/z (schemes.jl:110-199) for one variable; p/m point at the ghosted
// "right cell" c of the face in Fp/Fm, s is the stride along the swept axis.
inline double hybrid_face(const double *p, const double *m, long s, double phif) {
    const double tmp1 = 13.0 / 12.0, tmp2 = 1.0 / 6.0;
    const double c1 = kUP7[0], c2 = kUP7[1], c3 = kUP7[2], c4 = kUP7[3], c5 = kUP7[4],
                 c6 = kUP7[5], c7 = kUP7[6];
    double fp, fm;
    if (phif < kHybrid1) {
        double V1 = p[-4 * s], V2 = p[-3 * s], V3 = p[-2 * s], V4 = p[-s], V5 = p[0], V6 = p[s],
               V7 = p[2 * s];
        fp = c1 * V1 + c2 * V2 + c3 * V3 + c4 * V4 + c5 * V5 + c6 * V6 + c7 * V7;
        V1 = m[-3 * s], V2 = m[-2 * s], V3 = m[-s], V4 = m[0], V5 = m[s], V6 = m[2 * s],
        V7 = m[3 * s];
        fm = c7 * V1 + c6 * V2 + c5 * V3 + c4 * V4 + c3 * V5 + c2 * V6 + c1 * V7;
    } else if (phif < kHybrid2) {
        double V1 = p[-3 * s], V2 = p[-2 * s], V3 = p[-s], V4 = p[0], V5 = p[s];
        double a, b;
        a = V1 - 2 * V2 + V3, b = V1 - 4 * V2 + 3 * V3;
        double s11 = tmp1 * (a * a) + 0.25 * (b * b);
        a = V2 - 2 * V3 + V4, b = V2 - V4;
        double s22 = tmp1 * (a * a) + 0.25 * (b * b);
        a = V3 - 2 * V4 + V5, b = 3 * V3 - 4 * V4 + V5;
        double s33 = tmp1 * (a * a) + 0.25 * (b * b);
        double tau = std::fabs(s11 - s33);
        double q;
        q = tau / (kWenoEps + s11), s11 = (1 + q * q) * 1;
        q = tau / (kWenoEps + s22), s22 = (1 + q * q) * 6;
        q = tau / (kWenoEps + s33), s33 = (1 + q * q) * 3;
        double invsum = 1 / (s11 + s22 + s33);
        double v1 = 2 * V1 - 7 * V2 + 11 * V3;
        double v2 = -V2 + 5 * V3 + 2 * V4;
        double v3 = 2 * V3 + 5 * V4 - V5;
        fp = tmp2 * invsum * (s11 * v1 + s22 * v2 + s33 * v3);

        V1 = m[-2 * s], V2 = m[-s], V3 = m[0], V4 = m[s], V5 = m[2 * s];
        a = V5 - 2 * V4 + V3, b = V5 - 4 * V4 + 3 * V3;
        s11 = tmp1 * (a * a) + 0.25 * (b * b);
        a = V2 - 2 * V3 + V4, b = V4 - V2;
        s22 = tmp1 * (a * a) + 0.25 * (b * b);
        a = V3 - 2 * V2 + V1, b = 3 * V3 - 4 * V2 + V1;
        s33 = tmp1 * (a * a) + 0.25 * (b * b);
        tau = std::fabs(s11 - s33);
        q = tau / (kWenoEps + s11), s11 = (1 + q * q) * 1;
        q = tau / (kWenoEps + s22), s22 = (1 + q * q) * 6;
        q = tau / (kWenoEps + s33), s33 = (1 + q * q) * 3;
        invsum = 1 / (s11 + s22 + s33);
        v1 = 11 * V3 - 7 * V4 + 2 * V5;
        v2 = -V4 + 5 * V3 + 2 * V2;
        v3 = 2 * V3 + 5 * V2 - V1;
        fm = tmp2 * invsum * (s11 * v1 + s22 * v2 + s33 * v3);
    } else {
        fp = p[-s] + 0.5 * minmod(p[0] - p[-s], p[-s] - p[-2 * s]);
        fm = m[0] - 0.5 * minmod(m[s] - m[0], m[0] - m[-s]);
    }
    return fp + fm;
}

}  // namespace

extern "C" {

// schemes.jl:1-24
void oracle_shockSensor(const FlameGrid *g, double *phi, const double *Q) {
    Dims D(g);
    const double *p = Q + 4 * D.np;
#pragma omp parallel for schedule(static)
    for (long k = 1; k < D.tz - 1; ++k)
        for (long j = 1; j < D.ty - 1; ++j)
            for (long i = 1; i < D.tx - 1; ++i) {
                long c = D.P(i, j, k);
                double Px1 = p[c - 1], Px2 = p[c], Px3 = p[c + 1];
                double Py1 = p[c - D.tx], Py2 = p[c], Py3 = p[c + D.tx];
                double Pz1 = p[c - D.tx * D.ty], Pz2 = p[c], Pz3 = p[c + D.tx * D.ty];
                double phx = std::fabs(-Px1 + 2 * Px2 - Px3) / (Px1 + 2 * Px2 + Px3);
                double phy = std::fabs(-Py1 + 2 * Py2 - Py3) / (Py1 + 2 * Py2 + Py3);
                double phz = std::fabs(-Pz1 + 2 * Pz2 - Pz3) / (Pz1 + 2 * Pz2 + Pz3);
                phi[c] = phx + phy + phz;
            }
}

// split.jl:17-89 (SWϵ2 = 0, run.jl:51)
void oracle_fluxSplit(const FlameGrid *g, const double *Q, double *Fp, double *Fm,
                      const double *Ax, const double *Ay, const double *Az, const int64_t *tag) {
    Dims D(g);
    const long np = D.np;
    const double SWeps2 = 0.0;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < D.tz; ++k)
        for (long j = 0; j < D.ty; ++j)
            for (long i = 0; i < D.tx; ++i) {
                long c = D.P(i, j, k);
                if (tagat(tag, c) == 1) continue;
                double rho = Q[c], u = Q[c + np], v = Q[c + 2 * np], w = Q[c + 3 * np],
                       p = Q[c + 4 * np], ei = Q[c + 6 * np];
                double A1 = Ax[c], A2 = Ay[c], A3 = Az[c];
                double gam = p / ei + 1;
                double cs = std::sqrt(gam * p / rho);
                double ss = std::sqrt(A1 * A1 + A2 * A2 + A3 * A3);
                double E1 = A1 * u + A2 * v + A3 * w;
                double E2 = E1 - cs * ss;
                double E3 = E1 + cs * ss;
                ss = 1 / ss;
                A1 *= ss;
                A2 *= ss;
                A3 *= ss;
                double E1P = (E1 + std::sqrt(E1 * E1 + SWeps2)) * 0.5;
                double E2P = (E2 + std::sqrt(E2 * E2 + SWeps2)) * 0.5;
                double E3P = (E3 + std::sqrt(E3 * E3 + SWeps2)) * 0.5;
                double E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
                double uc1 = u - cs * A1, uc2 = u + cs * A1;
                double vc1 = v - cs * A2, vc2 = v + cs * A2;
                double wc1 = w - cs * A3, wc2 = w + cs * A3;
                double vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.50;
                double vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.50;
                double vv = (gam - 1.0) * (u * u + v * v + w * w);
                double W2 = (3 - gam) / (2 * (gam - 1)) * (cs * cs);
                double tmp1 = rho / (2 * gam);
                double tmp2 = 2 * (gam - 1);
                Fp[c] = tmp1 * (tmp2 * E1P + E2P + E3P);
                Fp[c + np] = tmp1 * (tmp2 * E1P * u + E2P * uc1 + E3P * uc2);
                Fp[c + 2 * np] = tmp1 * (tmp2 * E1P * v + E2P * vc1 + E3P * vc2);
                Fp[c + 3 * np] = tmp1 * (tmp2 * E1P * w + E2P * wc1 + E3P * wc2);
                Fp[c + 4 * np] = tmp1 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
                Fm[c] = tmp1 * (tmp2 * E1M + E2M + E3M);
                Fm[c + np] = tmp1 * (tmp2 * E1M * u + E2M * uc1 + E3M * uc2);
                Fm[c + 2 * np] = tmp1 * (tmp2 * E1M * v + E2M * vc1 + E3M * vc2);
                Fm[c + 3 * np] = tmp1 * (tmp2 * E1M * w + E2M * wc1 + E3M * wc2);
                Fm[c + 4 * np] = tmp1 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
            }
}

// split.jl:101-130
void oracle_split(const FlameGrid *g, const double *rhoi, const double *Q, double *Fp, double *Fm,
                  const double *Ax, const double *Ay, const double *Az, const int64_t *tag) {
    Dims D(g);
    const long np = D.np;
#pragma omp parallel for schedule(static)
    for (long k = 0; k < D.tz; ++k)
        for (long j = 0; j < D.ty; ++j)
            for (long i = 0; i < D.tx; ++i) {
                long c = D.P(i, j, k);
                if (tagat(tag, c) == 1) continue;
                double u = Q[c + np], v = Q[c + 2 * np], w = Q[c + 3 * np];
                double un = Ax[c] * u + Ay[c] * v + Az[c] * w;
                double Ep = 0.5 * (un + std::fabs(un));
                double Em = 0.5 * (un - std::fabs(un));
                for (int n = 0; n < D.ns; ++n) {
                    Fp[c + n * np] = Ep * rhoi[c + n * np];
                    Fm[c + n * np] = Em * rhoi[c + n * np];
                }
            }
}

// schemes.jl:86-437 WENO_x / WENO_y / WENO_z; d = 0, 1, 2
void oracle_WENO(const FlameGrid *g, int d, double *F, const double *phi, const double *Fp,
                 const double *Fm, int NV, const int64_t *tag) {
    Dims D(g);
    Faces f = faces_of(D, d);
    const long nf = f.fx * f.fy * f.fz;
#pragma omp parallel for schedule(static)
    for (long fk = 0; fk < f.fz; ++fk)
        for (long fj = 0; fj < f.fy; ++fj)
            for (long fi = 0; fi < f.fx; ++fi) {
                long c = D.P(fi + D.ng, fj + D.ng, fk + D.ng);
                if (tagat(tag, c) == 1) continue;
                double phif = jmax(phi[c - f.sn], phi[c]);
                long fo = fi + f.fx * (fj + f.fy * fk);
                for (int n = 0; n < NV; ++n)
                    F[fo + n * nf] = hybrid_face(Fp + c + n * D.np, Fm + c + n * D.np, f.sn, phif);
            }
}

// viscous.jl:1-428 viscousFlux_x/y/z (LES branches compiled off, run.jl:7-8); d = 0, 1, 2
void oracle_viscousFlux(const FlameGrid *g, int d, double *Fv, const double *Q,
                        const FlameMetrics *m, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag) {
    Dims D(g);
    Faces f = faces_of(D, d);
    const long nf = f.fx * f.fy * f.fz, np = D.np;
    const double c23 = 2.0 / 3.0, c12 = 1.0 / 12.0;
    const double *M[9] = {m->dxidx,   m->dxidy,   m->dxidz,   m->detadx, m->detady,
                          m->detadz,  m->dzetadx, m->dzetady, m->dzetadz};
    // tangential directions in (xi, eta, zeta) order with their strides
    const int dir1 = (d + 1) % 3, dir2 = (d + 2) % 3;
#pragma omp parallel for schedule(static)
    for (long fk = 0; fk < f.fz; ++fk)
        for (long fj = 0; fj < f.fy; ++fj)
            for (long fi = 0; fi < f.fx; ++fi) {
                long c = D.P(fi + D.ng, fj + D.ng, fk + D.ng);
                if (tagat(tag, c) == 1) continue;
                const long sn = f.sn;
                double met[9];
                for (int a = 0; a < 9; ++a) met[a] = (M[a][c - sn] + M[a][c]) * 0.5;
                double Jac = (m->J[c - sn] + m->J[c]) * 0.5;
                double mui = (mu[c - sn] + mu[c]) * 0.5;
                double lami = (lambda[c - sn] + lambda[c]) * 0.5;
                // derivatives of (u, v, w, T) along (xi, eta, zeta)
                double dq[4][3];
                const int qv[4] = {1, 2, 3, 5};
                for (int a = 0; a < 4; ++a) {
                    const double *q = Q + qv[a] * np + c;
                    dq[a][d] = 1.25 * (q[0] - q[-sn]) - c12 * (q[sn] - q[-2 * sn]);
                    long st = (dir1 == 0) ? 1 : (dir1 == 1 ? D.tx : D.tx * D.ty);
                    dq[a][dir1] = 0.5 * (c23 * (q[st] + q[-sn + st] - q[-st] - q[-sn - st]) -
                                         c12 * (q[2 * st] + q[-sn + 2 * st] - q[-2 * st] -
                                                q[-sn - 2 * st]));
                    st = (dir2 == 0) ? 1 : (dir2 == 1 ? D.tx : D.tx * D.ty);
                    dq[a][dir2] = 0.5 * (c23 * (q[st] + q[-sn + st] - q[-st] - q[-sn - st]) -
                                         c12 * (q[2 * st] + q[-sn + 2 * st] - q[-2 * st] -
                                                q[-sn - 2 * st]));
                }
                double u = (Q[c - sn + np] + Q[c + np]) * 0.5;
                double v = (Q[c - sn + 2 * np] + Q[c + 2 * np]) * 0.5;
                double w = (Q[c - sn + 3 * np] + Q[c + 3 * np]) * 0.5;
                // met: [xi_x, xi_y, xi_z, eta_x, eta_y, eta_z, zeta_x, zeta_y, zeta_z]
                double gr[4][3];  // physical gradient of (u,v,w,T) along (x,y,z)
                for (int a = 0; a < 4; ++a)
                    for (int x = 0; x < 3; ++x)
                        gr[a][x] = (dq[a][0] * met[x] + dq[a][1] * met[3 + x] +
                                    dq[a][2] * met[6 + x]) *
                                   Jac;
                double dudx = gr[0][0], dudy = gr[0][1], dudz = gr[0][2];
                double dvdx = gr[1][0], dvdy = gr[1][1], dvdz = gr[1][2];
                double dwdx = gr[2][0], dwdy = gr[2][1], dwdz = gr[2][2];
                double dTdx = gr[3][0], dTdy = gr[3][1], dTdz = gr[3][2];
                double div = dudx + dvdy + dwdz;
                double t11 = mui * (2 * dudx - c23 * div);
                double t12 = mui * (dudy + dvdx);
                double t13 = mui * (dudz + dwdx);
                double t22 = mui * (2 * dvdy - c23 * div);
                double t23 = mui * (dwdy + dvdz);
                double t33 = mui * (2 * dwdz - c23 * div);
                long fo = fi + f.fx * (fj + f.fy * fk);
                double E1 = u * t11 + v * t12 + w * t13 + lami * dTdx + Fh[fo];
                double E2 = u * t12 + v * t22 + w * t23 + lami * dTdy + Fh[fo + nf];
                double E3 = u * t13 + v * t23 + w * t33 + lami * dTdz + Fh[fo + 2 * nf];
                const double *md = met + 3 * d;
                Fv[fo] = md[0] * t11 + md[1] * t12 + md[2] * t13;
                Fv[fo + nf] = md[0] * t12 + md[1] * t22 + md[2] * t23;
                Fv[fo + 2 * nf] = md[0] * t13 + md[1] * t23 + md[2] * t33;
                Fv[fo + 3 * nf] = md[0] * E1 + md[1] * E2 + md[2] * E3;
            }
}

// viscous.jl:430-665 specViscousFlux_x/y/z; d = 0, 1, 2
void oracle_specViscousFlux(const FlameGrid *g, int d, double *Fd, const double *Q,
                            const double *Yi, const FlameMetrics *m, const double *Dk, double *Fh,
                            const FlameThermo *th, const int64_t *tag) {
    Dims D(g);
    Faces f = faces_of(D, d);
    const long nf = f.fx * f.fy * f.fz, np = D.np;
    const double c12 = 1.0 / 12.0;
    const double *M[9] = {m->dxidx,   m->dxidy,   m->dxidz,   m->detadx, m->detady,
                          m->detadz,  m->dzetadx, m->dzetady, m->dzetadz};
    const int dir1 = (d + 1) % 3, dir2 = (d + 2) % 3;
    const int ns = D.ns;
#pragma omp parallel for schedule(static)
    for (long fk = 0; fk < f.fz; ++fk)
        for (long fj = 0; fj < f.fy; ++fj)
            for (long fi = 0; fi < f.fx; ++fi) {
                long c = D.P(fi + D.ng, fj + D.ng, fk + D.ng);
                if (tagat(tag, c) == 1) continue;
                const long sn = f.sn;
                double met[9];
                for (int a = 0; a < 9; ++a) met[a] = (M[a][c - sn] + M[a][c]) * 0.5;
                double Jac = (m->J[c - sn] + m->J[c]) * 0.5;
                double rho = (Q[c - sn] + Q[c]) * 0.5;
                double T = (Q[c - sn + 5 * np] + Q[c + 5 * np]) * 0.5;
                double Vk1[FLAME_MAX_NS], Vk2[FLAME_MAX_NS], Vk3[FLAME_MAX_NS], hi[FLAME_MAX_NS];
                h_specs(hi, T, th, ns);
                long fo = fi + f.fx * (fj + f.fy * fk);
                double fh1 = 0, fh2 = 0, fh3 = 0;
                double sum1 = 0, sum2 = 0, sum3 = 0;
                const long s1 = (dir1 == 0) ? 1 : (dir1 == 1 ? D.tx : D.tx * D.ty);
                const long s2 = (dir2 == 0) ? 1 : (dir2 == 1 ? D.tx : D.tx * D.ty);
                for (int n = 0; n < ns; ++n) {
                    const double *y = Yi + n * np + c;
                    double rhoDi = (Dk[c - sn + n * np] + Dk[c + n * np]) * rho;
                    double dY[3];
                    dY[d] = 1.25 * (y[0] - y[-sn]) - c12 * (y[sn] - y[-2 * sn]);
                    dY[dir1] = 0.25 * (y[s1] + y[-sn + s1] - y[-s1] - y[-sn - s1]);
                    dY[dir2] = 0.25 * (y[s2] + y[-sn + s2] - y[-s2] - y[-sn - s2]);
                    double Vx = (dY[0] * met[0] + dY[1] * met[3] + dY[2] * met[6]) * Jac * rhoDi;
                    double Vy = (dY[0] * met[1] + dY[1] * met[4] + dY[2] * met[7]) * Jac * rhoDi;
                    double Vz = (dY[0] * met[2] + dY[1] * met[5] + dY[2] * met[8]) * Jac * rhoDi;
                    Vk1[n] = Vx, Vk2[n] = Vy, Vk3[n] = Vz;
                    sum1 += Vx, sum2 += Vy, sum3 += Vz;
                }
                const double *md = met + 3 * d;
                for (int n = 0; n < ns; ++n) {
                    double Yn = 0.5 * (Yi[c - sn + n * np] + Yi[c + n * np]);
                    double hn = hi[n];
                    double V1 = Vk1[n] - sum1 * Yn;
                    double V2 = Vk2[n] - sum2 * Yn;
                    double V3 = Vk3[n] - sum3 * Yn;
                    Fd[fo + n * nf] = V1 * md[0] + V2 * md[1] + V3 * md[2];
                    fh1 += V1 * hn, fh2 += V2 * hn, fh3 += V3 * hn;
                }
                Fh[fo] = fh1, Fh[fo + nf] = fh2, Fh[fo + 2 * nf] = fh3;
            }
}

// div.jl:16-54
void oracle_div(const FlameGrid *g, double *U, const double *Fx, const double *Fy,
                const double *Fz, const double *Fvx, const double *Fvy, const double *Fvz,
                double dt, const double *J, const int64_t *tag) {
    Dims D(g);
    const long np = D.np;
    const long nfx = (D.nx + 1L) * D.ny * D.nz, nfy = D.nx * (D.ny + 1L) * D.nz,
               nfz = D.nx * (long)D.ny * (D.nz + 1L);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                long c = D.P(i + D.ng, j + D.ng, k + D.ng);
                if (tagat(tag, c) != 0) continue;
                double Jact = J[c] * dt;
                long x0 = i + (D.nx + 1L) * (j + D.ny * k), x1 = x0 + 1;
                long y0 = i + D.nx * (j + (D.ny + 1L) * k), y1 = y0 + D.nx;
                long z0 = i + D.nx * (j + (long)D.ny * k), z1 = z0 + (long)D.nx * D.ny;
                double dV[4];
                for (int a = 0; a < 4; ++a) {
                    double dx = Fvx[x1 + a * nfx] - Fvx[x0 + a * nfx];
                    double dy = Fvy[y1 + a * nfy] - Fvy[y0 + a * nfy];
                    double dz = Fvz[z1 + a * nfz] - Fvz[z0 + a * nfz];
                    dV[a] = dx + dy + dz;
                }
                for (int n = 0; n < 5; ++n)
                    U[c + n * np] += (Fx[x0 + n * nfx] - Fx[x1 + n * nfx] + Fy[y0 + n * nfy] -
                                      Fy[y1 + n * nfy] + Fz[z0 + n * nfz] - Fz[z1 + n * nfz]) *
                                     Jact;
                for (int a = 0; a < 4; ++a) U[c + (a + 1) * np] += dV[a] * Jact;
            }
}

// div.jl:61-84
void oracle_divSpecs(const FlameGrid *g, double *rhoi, const double *Fx, const double *Fy,
                     const double *Fz, const double *Fdx, const double *Fdy, const double *Fdz,
                     double dt, const double *J, const int64_t *tag) {
    Dims D(g);
    const long np = D.np;
    const long nfx = (D.nx + 1L) * D.ny * D.nz, nfy = D.nx * (D.ny + 1L) * D.nz,
               nfz = D.nx * (long)D.ny * (D.nz + 1L);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < D.nz; ++k)
        for (long j = 0; j < D.ny; ++j)
            for (long i = 0; i < D.nx; ++i) {
                long c = D.P(i + D.ng, j + D.ng, k + D.ng);
                if (tagat(tag, c) != 0) continue;
                double Jact = J[c] * dt;
                long x0 = i + (D.nx + 1L) * (j + D.ny * k), x1 = x0 + 1;
                long y0 = i + D.nx * (j + (D.ny + 1L) * k), y1 = y0 + D.nx;
                long z0 = i + D.nx * (j + (long)D.ny * k), z1 = z0 + (long)D.nx * D.ny;
                for (int n = 0; n < D.ns; ++n)
                    rhoi[c + n * np] +=
                        (Fx[x0 + n * nfx] - Fx[x1 + n * nfx] + Fy[y0 + n * nfy] -
                         Fy[y1 + n * nfy] + Fz[z0 + n * nfz] - Fz[z1 + n * nfz] +
                         Fdx[x1 + n * nfx] - Fdx[x0 + n * nfx] + Fdy[y1 + n * nfy] -
                         Fdy[y0 + n * nfy] + Fdz[z1 + n * nfz] - Fdz[z0 + n * nfz]) *
                        Jact;
            }
}

// utils.jl:95-112
void oracle_linComb(const FlameGrid *g, double *U, const double *Un, int NV, double a, double b,
                    const int64_t *tag) {
    Dims D(g);
#pragma omp parallel for schedule(static)
    for (long k = D.ng; k < D.nz + D.ng; ++k)
        for (long j = D.ng; j < D.ny + D.ng; ++j)
            for (long i = D.ng; i < D.nx + D.ng; ++i) {
                long c = D.P(i, j, k);
                if (tagat(tag, c) != 0) continue;
                for (int n = 0; n < NV; ++n)
                    U[c + n * D.np] = U[c + n * D.np] * a + Un[c + n * D.np] * b;
            }
}

// utils.jl:2-48
void oracle_c2Prim(const FlameGrid *g, const double *U, double *Q, double *rhoi,
                   const FlameThermo *th, const int64_t *tag) {
    Dims D(g);
    const long np = D.np;
    const int ns = D.ns;
#pragma omp parallel for schedule(static)
    for (long k = D.ng; k < D.nz + D.ng; ++k)
        for (long j = D.ng; j < D.ny + D.ng; ++j)
            for (long i = D.ng; i < D.nx + D.ng; ++i) {
                long c = D.P(i, j, k);
                if (tagat(tag, c) != 0) continue;
                double rho = jmax(U[c], kEps);
                double r[FLAME_MAX_NS];
                double rhoinv = 1 / rho;
                double sr = 0.0;
                for (int n = 0; n < ns; ++n) {
                    r[n] = jmax(rhoi[c + n * np], 0.0);
                    sr += r[n];
                }
                for (int n = 0; n < ns; ++n) r[n] *= rho / sr;
                double u = U[c + np] * rhoinv;
                double v = U[c + 2 * np] * rhoinv;
                double w = U[c + 3 * np] * rhoinv;
                double ei = jmax(U[c + 4 * np] - 0.5 * rho * (u * u + v * v + w * w), kEps);
                double T = jmax(GetT(ei, r, th, ns), kEps);
                double p = jmax(Pmixture(T, r, th, ns), kEps);
                for (int n = 0; n < ns; ++n) rhoi[c + n * np] = r[n];
                Q[c] = rho;
                Q[c + np] = u;
                Q[c + 2 * np] = v;
                Q[c + 3 * np] = w;
                Q[c + 4 * np] = p;
                Q[c + 5 * np] = T;
                Q[c + 6 * np] = ei;
            }
}

// utils.jl:71-92
void oracle_prim2c(const FlameGrid *g, double *U, const double *Q) {
    Dims D(g);
    const long np = D.np;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < np; ++c) {
        double rho = Q[c], u = Q[c + np], v = Q[c + 2 * np], w = Q[c + 3 * np],
               ei = Q[c + 6 * np];
        U[c] = rho;
        U[c + np] = u * rho;
        U[c + 2 * np] = v * rho;
        U[c + 3 * np] = w * rho;
        U[c + 4 * np] = ei + 0.5 * rho * (u * u + v * v + w * w);
    }
}

// thermo.jl:371-403 mixture(), with the FlameTransport law in place of Cantera's fits.
// mixtureProperties, thermo.jl:284-369 (transport law 2): Mathur λ, Wilke μ, mixture-averaged
// D_k from the log(T) fits; poly = visc (5, ns) | conduct (5, ns) | binarydiff (5, ns, ns).
static double dot5(double l1, double l2, double l3, double l4, const double *p) {
    return p[0] + l1 * p[1] + l2 * p[2] + l3 * p[3] + l4 * p[4];
}

void oracle_mixture_properties(double T, double P, const double *X, const FlameThermo *th,
                               const double *poly, int ns, double *Dk, double *lam_out,
                               double *mu_out) {
    const double *visc = poly, *cond = poly + 5 * ns, *bin = poly + 10 * ns;
    double mui[FLAME_MAX_NS], W[FLAME_MAX_NS * FLAME_MAX_NS];
    const double sqT = std::sqrt(T), sqsqT = std::sqrt(sqT), lgT = std::log(T);
    const double lgT2 = lgT * lgT, lgT3 = lgT * lgT2, lgT4 = lgT2 * lgT2;
    for (int n = 0; n < ns; ++n) mui[n] = sqT * dot5(lgT, lgT2, lgT3, lgT4, cond + 5 * n);
    double sum1 = 0, sum2 = 0;
    for (int k = 0; k < ns; ++k) sum1 += X[k] * mui[k], sum2 += X[k] / mui[k];
    *lam_out = 0.5 * (sum1 + 1 / sum2);
    for (int n = 0; n < ns; ++n) {
        const double sq = sqsqT * dot5(lgT, lgT2, lgT3, lgT4, visc + 5 * n);
        mui[n] = sq * sq;
    }
    for (int n = 0; n < ns; ++n) {  // Wilke, Poling et al. (2001) eq. 9-5.14
        const double tmp1 = 1 / th->mw[n], tmp2 = mui[n];
        for (int l = 0; l <= n; ++l) {
            const double wr = th->mw[l] * tmp1, vr = tmp2 / mui[l];
            const double f1 = 1 + std::sqrt(vr * std::sqrt(wr));
            const double t = f1 * f1 / std::sqrt(8 + 8 / wr);
            W[n * ns + l] = t;
            W[l * ns + n] = t / (vr * wr);
        }
        W[n * ns + n] = 1.0;
    }
    double mu = 0;
    for (int n = 0; n < ns; ++n) {
        double t = 0.0;
        for (int l = 0; l < ns; ++l) t += X[l] * W[n * ns + l];
        mu += X[n] * mui[n] / t;
    }
    *mu_out = mu;
    for (int n = 0; n < ns; ++n)
        for (int m = n; m < ns; ++m) {
            const double t = T * sqT * dot5(lgT, lgT2, lgT3, lgT4, bin + 5 * (m + ns * n));
            W[m * ns + n] = t;
            W[n * ns + m] = t;
        }
    for (int n = 0; n < ns; ++n) {
        double sm = 0.0;
        for (int m = 0; m < ns; ++m) {
            if (m == n) continue;
            sm += X[m] / W[n * ns + m];
        }
        sm *= P;
        Dk[n] = (1 - X[n]) / (sm + kEps);
    }
}

void oracle_mixture(const FlameGrid *g, const double *Q, const double *rhoi, double *Yi,
                    double *lambda, double *mu, double *Dk, const FlameThermo *th,
                    const FlameTransport *tr, const int64_t *tag) {
    Dims D(g);
    const long np = D.np;
    const int ns = D.ns;
#pragma omp parallel for schedule(static)
    for (long c = 0; c < np; ++c) {
        if (tagat(tag, c) == 1) continue;
        double T = Q[c + 5 * np];
        double rho = jmax(Q[c], kEps);
        double rhoinv = 1 / rho;
        double Y[FLAME_MAX_NS];
        for (int n = 0; n < ns; ++n) {
            Y[n] = jmax(rhoi[c + n * np] * rhoinv, 0.0);
            Yi[c + n * np] = Y[n];
        }
        double m, l, dd;
        if (tr->law == 2) {  // Y2X, thermo.jl:38-52
            double yow = 0;
            for (int n = 0; n < ns; ++n) yow += Y[n] / th->mw[n];
            const double yowinv = 1 / yow;
            double X[FLAME_MAX_NS], Dl[FLAME_MAX_NS];
            for (int n = 0; n < ns; ++n) X[n] = Y[n] / th->mw[n] * yowinv;
            oracle_mixture_properties(T, Q[c + 4 * np], X, th, tr->poly, ns, Dl, &l, &m);
            mu[c] = m;
            lambda[c] = l;
            for (int n = 0; n < ns; ++n) Dk[c + n * np] = Dl[n];
            continue;
        }
        if (tr->law == 0) {
            m = tr->mu_ref, l = tr->lambda_ref, dd = tr->D_ref;
        } else {
            double cp[FLAME_MAX_NS];
            cp_specs(cp, T, th, ns);
            double cpm = 0;
            for (int n = 0; n < ns; ++n) cpm += cp[n] * Y[n] / th->mw[n];
            cpm *= th->Ru;
            m = tr->mu_ref * std::pow(T / tr->T_ref, tr->exponent);
            l = cpm * m / tr->Pr;
            dd = l / (rho * cpm);
        }
        mu[c] = m;
        lambda[c] = l;
        for (int n = 0; n < ns; ++n) Dk[c + n * np] = dd;
    }
}

// Periodic ghost fill (new code: the reference has no periodic boundary, boundary.jl:1-191).
void oracle_fill_periodic(const FlameGrid *g, double *A, int nv) {
    Dims D(g);
    const int ng = D.ng;
    auto wrap = [ng](long i, long n, bool per) -> long {
        if (!per || (i >= ng && i < n + ng)) return i;
        return ng + (((i - ng) % n) + n) % n;
    };
    const bool px = g->periodic & 1, py = g->periodic & 2, pz = g->periodic & 4;
    for (int v = 0; v < nv; ++v) {
        double *a = A + v * D.np;
#pragma omp parallel for schedule(static)
        for (long k = 0; k < D.tz; ++k)
            for (long j = 0; j < D.ty; ++j)
                for (long i = 0; i < D.tx; ++i) {
                    long si = wrap(i, D.nx, px), sj = wrap(j, D.ny, py), sk = wrap(k, D.nz, pz);
                    if (si == i && sj == j && sk == k) continue;
                    a[D.P(i, j, k)] = a[D.P(si, sj, sk)];
                }
    }
}

// ---------------------------------------------------------------- boundary.jl:1-176 fills
// Reference 1-based planes map to 0-based ones: inflow i <= NG+1 -> i <= NG; outlet
// i >= Nxp+NG copying Nxp+NG-1 -> i >= nx+NG-1 copying nx+NG-2 (likewise in y and z).
static void set_inflow(const Dims &D, long p, double *Q, double *U, double *rhoi, double *Yi,
                       const FlameThermo *th, const FlameInflow *in) {
    const long np = D.np;
    const int ns = D.ns;
    for (int n = 0; n < ns; ++n) Yi[p + n * np] = 0.0, rhoi[p + n * np] = 0.0;
    for (int n = 0; n < ns; ++n) Yi[p + n * np] = in->Y[n];
    double yow = 0;  // ρmixture, thermo.jl:29-35
    for (int n = 0; n < ns; ++n) yow += Yi[p + n * np] / th->mw[n];
    const double rho = in->P / (th->Ru * in->T * yow);
    double r[FLAME_MAX_NS];
    for (int n = 0; n < ns; ++n) rhoi[p + n * np] = Yi[p + n * np] * rho, r[n] = rhoi[p + n * np];
    const double ei = InternalEnergy(in->T, r, th, ns);
    const double u = in->u, v = in->v, w = in->w;
    const double q[7] = {rho, u, v, w, in->P, in->T, ei};
    for (int n = 0; n < 7; ++n) Q[p + n * np] = q[n];
    U[p] = rho;
    U[p + np] = u * rho;
    U[p + 2 * np] = v * rho;
    U[p + 3 * np] = w * rho;
    U[p + 4 * np] = ei + 0.5 * rho * (u * u + v * v + w * w);
}

static void copy_point(const Dims &D, long dst, long src, double *Q, double *U, double *rhoi) {
    if (Q)
        for (int n = 0; n < 7; ++n) Q[dst + n * D.np] = Q[src + n * D.np];
    if (U)
        for (int n = 0; n < 5; ++n) U[dst + n * D.np] = U[src + n * D.np];
    if (rhoi)
        for (int n = 0; n < D.ns; ++n) rhoi[dst + n * D.np] = rhoi[src + n * D.np];
}

// boundary.jl:1-52
void oracle_fill_x(const FlameGrid *g, double *Q, double *U, double *rhoi, double *Yi,
                   const FlameThermo *th, const FlameInflow *in, int rank, int nprocs) {
    Dims D(g);
    for (long k = 0; k < D.tz; ++k)
        for (long j = 0; j < D.ty; ++j)
            for (long i = 0; i < D.tx; ++i) {
                const long p = D.P(i, j, k);
                if (rank == 0 && i <= D.ng) set_inflow(D, p, Q, U, rhoi, Yi, th, in);
                if (rank == nprocs - 1 && i >= D.nx + D.ng - 1)
                    copy_point(D, p, D.P(D.nx + D.ng - 2, j, k), Q, U, rhoi);
            }
}

// boundary.jl:54-80 (Q, U) and 139-158 (ρi alone: Q = U = null)
void oracle_fill_y(const FlameGrid *g, double *Q, double *U, double *rhoi) {
    Dims D(g);
    for (long k = 0; k < D.tz; ++k)
        for (long j = 0; j < D.ty; ++j)
            for (long i = 0; i < D.tx; ++i) {
                if (j <= D.ng)
                    copy_point(D, D.P(i, j, k), D.P(i, D.ng + 1, k), Q, U, rhoi);
                else if (j >= D.ny + D.ng - 1)
                    copy_point(D, D.P(i, j, k), D.P(i, D.ny + D.ng - 2, k), Q, U, rhoi);
            }
}

// boundary.jl:82-137
void oracle_fill_z(const FlameGrid *g, double *Q, double *U, double *rhoi, double *Yi,
                   const FlameThermo *th, const FlameInflow *in) {
    Dims D(g);
    for (long k = 0; k < D.tz; ++k)
        for (long j = 0; j < D.ty; ++j)
            for (long i = 0; i < D.tx; ++i) {
                const long p = D.P(i, j, k);
                if (k <= D.ng)
                    set_inflow(D, p, Q, U, rhoi, Yi, th, in);
                else if (k >= D.nz + D.ng - 1)
                    copy_point(D, p, D.P(i, j, D.nz + D.ng - 2), Q, U, nullptr);
            }
}

// boundary.jl:193-279 (fillIB; 15-point stencils with 1-based Julia indices)
void oracle_fill_ib(const FlameGrid *g, double *Q, double *U, double *rhoi, const int64_t *ni,
                    const int64_t *nj, const int64_t *nk, const double *cd, const double *cn,
                    const int64_t *tag, const FlameThermo *th, double Tw) {
    Dims D(g);
    const long np = D.np;
    const int ns = D.ns;
    const int NPT = 15;
    for (long p = 0; p < np; ++p) {
        if (tag[p] != 3) continue;
        long q[15];
        for (int m = 0; m < NPT; ++m)
            q[m] = D.P(ni[m + NPT * p] - 1, nj[m + NPT * p] - 1, nk[m + NPT * p] - 1);
        const double *cnp = cn + 16 * p, *cdp = cd + 16 * p;
        double Yg[FLAME_MAX_NS];
        for (int n = 0; n < ns; ++n) {
            double sum = 0.0;
            for (int m = 0; m < NPT; ++m) sum += cnp[m + 1] * (rhoi[q[m] + n * np] / Q[q[m]]);
            Yg[n] = -sum / cnp[0];
        }
        double sum = 0.0;
        for (int m = 0; m < NPT; ++m) sum += cnp[m + 1] * Q[q[m] + 4 * np];
        const double pg = -sum / cnp[0];
        double vel[3];
        for (int c = 0; c < 3; ++c) {
            sum = 0.0;
            for (int m = 0; m < NPT; ++m) sum += cdp[m + 1] * Q[q[m] + (1 + c) * np];
            vel[c] = -sum / cdp[0];
        }
        double yow = 0;
        for (int n = 0; n < ns; ++n) yow += Yg[n] / th->mw[n];
        const double rho = pg / (th->Ru * Tw * yow);
        double r[FLAME_MAX_NS];
        for (int n = 0; n < ns; ++n) r[n] = Yg[n] * rho, rhoi[p + n * np] = r[n];
        const double ei = InternalEnergy(Tw, r, th, ns);
        const double ug = vel[0], vg = vel[1], wg = vel[2];
        Q[p + 6 * np] = ei;
        Q[p] = rho;
        Q[p + np] = ug;
        Q[p + 2 * np] = vg;
        Q[p + 3 * np] = wg;
        Q[p + 4 * np] = pg;
        Q[p + 5 * np] = Tw;
        U[p] = rho;
        U[p + np] = rho * ug;
        U[p + 2 * np] = rho * vg;
        U[p + 3 * np] = rho * wg;
        U[p + 4 * np] = ei + 0.5 * rho * (ug * ug + vg * vg + wg * wg);
    }
}

// boundary.jl:160-176
void oracle_fill_z_s(const FlameGrid *g, double *rhoi) {
    Dims D(g);
    for (long k = D.nz + D.ng - 1; k < D.tz; ++k)
        for (long j = 0; j < D.ty; ++j)
            for (long i = 0; i < D.tx; ++i)
                copy_point(D, D.P(i, j, k), D.P(i, j, D.nz + D.ng - 2), nullptr, nullptr, rhoi);
}

// The CFL rate max over interior cells of Σ_d J (|m_d·u| + c |m_d|) (this project's dt rule;
// the reference runs a fixed dt, run.jl:30).
double oracle_cfl_max(const FlameGrid *g, const double *Q, const FlameMetrics *m) {
    Dims D(g);
    const long np = D.np;
    const double *rows[3][3] = {{m->dxidx, m->dxidy, m->dxidz},
                                {m->detadx, m->detady, m->detadz},
                                {m->dzetadx, m->dzetady, m->dzetadz}};
    double best = 0;
    for (long k = D.ng; k < D.nz + D.ng; ++k)
        for (long j = D.ng; j < D.ny + D.ng; ++j)
            for (long i = D.ng; i < D.nx + D.ng; ++i) {
                const long p = D.P(i, j, k);
                const double rho = Q[p], u = Q[p + np], v = Q[p + 2 * np], w = Q[p + 3 * np],
                             pr = Q[p + 4 * np], e = Q[p + 6 * np];
                const double gam = pr / e + 1;
                const double cs = std::sqrt(gam * pr / rho);
                const double J = m->J[p];
                double tot = 0;
                for (int d = 0; d < 3; ++d) {
                    const double mx = rows[d][0][p], my = rows[d][1][p], mz = rows[d][2][p];
                    tot += J * (std::fabs(mx * u + my * v + mz * w) +
                                cs * std::sqrt(mx * mx + my * my + mz * mz));
                }
                best = jmax(best, tot);
            }
    return best;
}

// ------------------------------------------------------------ reactions.jl finite-rate chemistry
static double ipow(double x, long k) {  // the stoichiometric integer powers
    double r = 1.0;
    const long m = k < 0 ? -k : k;
    for (long i = 0; i < m; ++i) r *= x;
    return k < 0 ? 1.0 / r : r;
}

// gibbs, thermo.jl:163-191
static void gibbs(double *gi, double T, double lgT, double invT, const FlameThermo *th, int ns) {
    const double mlogT = 1 - lgT;
    const double T1 = 0.5 * T;
    const double T2 = 1.0 / 6.0 * T * T;
    const double T3 = T1 * T2;
    const double T4 = 1.8 * T2 * T2;
    for (int n = 0; n < ns; ++n) {
        const double *c = T < th->coeffs_sep[n] ? th->coeffs_lo + 7 * n : th->coeffs_hi + 7 * n;
        gi[n] = c[0] * mlogT - c[1] * T1 - c[2] * T2 - c[3] * T3 - c[4] * T4 + c[5] * invT - c[6];
    }
}

// vproductionRate (reactions.jl:311-380); with A non-null also the Jacobian of
// vproductionRate_Jac (:383-462), A column-major ns x ns
void oracle_production_rate(double *wdot, const double *sc, double *A, double T,
                            const FlameThermo *th, const FlameReactions *M, int ns) {
    std::vector<double> gi(ns), kf(M->nreacs), Kc(M->nreacs);
    const double lgT = std::log(T);
    const double invT = 1.0 / T;
    for (int n = 0; n < M->nreacs; ++n)
        kf[n] = M->Arr[3 * n] * std::exp(M->Arr[3 * n + 1] * lgT - M->Arr[3 * n + 2] * invT);
    gibbs(gi.data(), T, lgT, invT, th, ns);
    const double RsT = th->Ru / M->atm * 1e6 * T;
    for (int n = 0; n < M->nreacs; ++n) {
        double dg = 0;
        for (int m = 0; m < ns; ++m) dg += gi[m] * double(M->vf[m + ns * n] - M->vr[m + ns * n]);
        Kc[n] = ipow(RsT, M->sgm[n]) * std::exp(dg);
    }
    for (int n = 0; n < M->nreacs; ++n) {
        double qf = kf[n];
        double qr = qf / Kc[n];
        for (int m = 0; m < ns; ++m) {
            const long vf = M->vf[m + ns * n], vr = M->vr[m + ns * n];
            if (vf != 0) qf *= ipow(sc[m], vf);
            if (vr != 0) qr *= ipow(sc[m], vr);
        }
        double mix = 0.0;
        if (M->reaction_type[n] == 2) {
            for (int m = 0; m < ns; ++m) mix += M->ef[m + ns * n] * sc[m];
            qf *= mix;
            qr *= mix;
        } else if (M->reaction_type[n] == 3) {
            for (int m = 0; m < ns; ++m) mix += M->ef[m + ns * n] * sc[m];
            const double *lo = M->loP + 3 * n, *tr = M->Troe + 4 * n;
            const double redP = mix / kf[n] * lo[0] * std::exp(lo[1] * lgT - lo[2] * invT);
            const double logPred = std::log10(redP);
            const double a = tr[0];
            const double logFcent = std::log10((1 - a) * std::exp(-T / tr[1]) +
                                               a * std::exp(-T / tr[2]) + std::exp(-tr[3] * invT));
            const double troe_c = -0.4 - 0.67 * logFcent;
            const double troe_n = 0.75 - 1.27 * logFcent;
            const double troe = (troe_c + logPred) / (troe_n - 0.14 * (troe_c + logPred));
            const double F = std::pow(10.0, logFcent / (1.0 + troe * troe));
            const double k1 = (redP / (1.0 + redP)) * F;
            qf *= k1;
            qr *= k1;
        }
        for (int m = 0; m < ns; ++m) {
            wdot[m] += (qf - qr) * double(M->vr[m + ns * n] - M->vf[m + ns * n]);
            if (A) {
                const double invsc = 1 / (sc[m] + kEps);
                const double Awf = double(M->vf[m + ns * n]) * qf * invsc;
                const double Awr = double(M->vr[m + ns * n]) * qr * invsc;
                for (int l = 0; l < ns; ++l)
                    A[l + ns * m] += (Awf - Awr) * double(M->vr[l + ns * n] - M->vf[l + ns * n]);
            }
        }
    }
}

// solve, reactions.jl:465-504 (a column-major ns x ns; a and b are overwritten)
void oracle_solve(double *x, double *a, double *b, int ns) {
    auto A = [a, ns](int i, int j) -> double & { return a[i + ns * j]; };
    for (int k = 0; k < ns - 1; ++k) {
        double fmax = std::fabs(A(k, k));
        int kk = k;
        for (int i = k + 1; i < ns; ++i) {
            const double absa = std::fabs(A(i, k));
            if (absa > fmax) fmax = absa, kk = i;
        }
        for (int j = k; j < ns; ++j) std::swap(A(k, j), A(kk, j));
        std::swap(b[k], b[kk]);
        for (int i = k + 1; i < ns; ++i) {
            const double f = -A(i, k) / A(k, k);
            for (int j = 0; j < ns; ++j) A(i, j) += f * A(k, j);
            b[i] += f * b[k];
        }
    }
    x[ns - 1] = b[ns - 1] / A(ns - 1, ns - 1);
    for (int i = ns - 2; i >= 0; --i) {
        x[i] = b[i];
        for (int j = i + 1; j < ns; ++j) x[i] -= A(i, j) * x[j];
        x[i] /= A(i, i);
    }
}

// eval_gpu (stiff 0, reactions.jl:187-232) and eval_gpu_stiff (stiff 1, :235-309)
void oracle_eval_chem(const FlameGrid *g, int stiff, double *U, double *Q, double *rhoi, double dt,
                      const FlameThermo *th, const FlameReactions *M, const int64_t *tag,
                      double Tcrit, int transposed) {
    Dims D(g);
    const long np = D.np;
    const int ns = D.ns;
#pragma omp parallel for schedule(static)
    for (long k = D.ng; k < D.nz + D.ng; ++k)
        for (long j = D.ng; j < D.ny + D.ng; ++j)
            for (long i = D.ng; i < D.nx + D.ng; ++i) {
                const long p = D.P(i, j, k);
                if (tagat(tag, p) != 0) continue;
                double T = Q[p + 5 * np];
                if (!(T > Tcrit)) continue;
                double sc[FLAME_MAX_NS], wdot[FLAME_MAX_NS], r[FLAME_MAX_NS], dr[FLAME_MAX_NS];
                for (int n = 0; n < ns; ++n) {
                    r[n] = rhoi[p + n * np];
                    sc[n] = r[n] / th->mw[n] * 1e-6;
                    wdot[n] = 0.0;
                }
                double dei = 0;
                if (stiff) {
                    std::vector<double> A(ns * ns, 0.0), A1(ns * ns);
                    double drho[FLAME_MAX_NS];
                    oracle_production_rate(wdot, sc, A.data(), T, th, M, ns);
                    for (int l = 0; l < ns; ++l)
                        for (int n = 0; n < ns; ++n)
                            A1[n + ns * l] = (n == l ? 1.0 : 0.0) -
                                             A[n + ns * l] * th->mw[n] / th->mw[l] * dt;
                    for (int n = 0; n < ns; ++n) drho[n] = wdot[n] * th->mw[n] * 1e6 * dt;
                    oracle_solve(dr, A1.data(), drho, ns);
                    for (int n = 0; n < ns; ++n) {
                        const double a6 = transposed ? th->coeffs_lo[n + 35] : th->coeffs_lo[5 + 7 * n];
                        dei += -a6 * dr[n] * th->Ru / th->mw[n];
                        r[n] += dr[n];
                    }
                } else {
                    oracle_production_rate(wdot, sc, nullptr, T, th, M, ns);
                    for (int n = 0; n < ns; ++n) {
                        const double d = wdot[n] * th->mw[n] * 1e6 * dt;
                        dei += -th->coeffs_lo[5 + 7 * n] * d * th->Ru / th->mw[n];
                        r[n] += d;
                    }
                }
                U[p + 4 * np] += dei;
                const double rho = jmax(Q[p], kEps);
                double sum = 0.0;
                for (int n = 0; n < ns; ++n) r[n] = jmax(r[n], 0.0), sum += r[n];
                for (int n = 0; n < ns; ++n) r[n] *= rho / sum;
                for (int n = 0; n < ns; ++n) rhoi[p + n * np] = r[n];
                double ein = Q[p + 6 * np];
                ein += dei;
                T = jmax(GetT(ein, r, th, ns), kEps);
                const double pr = jmax(Pmixture(T, r, th, ns), kEps);
                Q[p + 4 * np] = pr;
                Q[p + 5 * np] = T;
                Q[p + 6 * np] = ein;
            }
}

// One SSP-RK3 stage exactly as solver.jl:298-326 orders it (IBM off, periodic fill in place of
// the case-specific fillGhost/fillSpec).  All arrays are host arrays the caller owns.
struct OracleState {
    double *U, *Un, *Q, *rhoi, *rhon;
};

void oracle_rk_stage_seq(const FlameGrid *g, int stage, double dt, double *U, double *Un,
                         double *Q, double *rhoi, double *rhon, const FlameMetrics *m,
                         const FlameThermo *th, const FlameTransport *tr) {
    Dims D(g);
    const long np = D.np;
    const int ns = D.ns;
    const long nfx = (D.nx + 1L) * D.ny * D.nz, nfy = D.nx * (D.ny + 1L) * D.nz,
               nfz = D.nx * (long)D.ny * (D.nz + 1L);
    std::vector<double> Yi(np * ns), lam(np), mu(np), Dk(np * ns), phi(np, 0.0);
    std::vector<double> Fp(np * 5), Fm(np * 5), Fpi(np * ns), Fmi(np * ns);
    std::vector<double> Fx(nfx * 5), Fy(nfy * 5), Fz(nfz * 5);
    std::vector<double> Fvx(nfx * 4), Fvy(nfy * 4), Fvz(nfz * 4);
    std::vector<double> Fxi(nfx * ns), Fyi(nfy * ns), Fzi(nfz * ns);
    std::vector<double> Fdx(nfx * ns), Fdy(nfy * ns), Fdz(nfz * ns);
    std::vector<double> Fhx(nfx * 3), Fhy(nfy * 3), Fhz(nfz * 3);
    if (stage == 1) {
        std::memcpy(Un, U, sizeof(double) * np * 5);
        std::memcpy(rhon, rhoi, sizeof(double) * np * ns);
    }
    oracle_mixture(g, Q, rhoi, Yi.data(), lam.data(), mu.data(), Dk.data(), th, tr, nullptr);
    oracle_shockSensor(g, phi.data(), Q);
    // specAdvance, solver.jl:40-56
    const double *A[3][3] = {{m->dxidx, m->dxidy, m->dxidz},
                             {m->detadx, m->detady, m->detadz},
                             {m->dzetadx, m->dzetady, m->dzetadz}};
    double *Fi[3] = {Fxi.data(), Fyi.data(), Fzi.data()};
    for (int d = 0; d < 3; ++d) {
        oracle_split(g, rhoi, Q, Fpi.data(), Fmi.data(), A[d][0], A[d][1], A[d][2], nullptr);
        oracle_WENO(g, d, Fi[d], phi.data(), Fpi.data(), Fmi.data(), ns, nullptr);
    }
    double *Fd[3] = {Fdx.data(), Fdy.data(), Fdz.data()};
    double *Fh[3] = {Fhx.data(), Fhy.data(), Fhz.data()};
    for (int d = 0; d < 3; ++d)
        oracle_specViscousFlux(g, d, Fd[d], Q, Yi.data(), m, Dk.data(), Fh[d], th, nullptr);
    oracle_divSpecs(g, rhoi, Fxi.data(), Fyi.data(), Fzi.data(), Fdx.data(), Fdy.data(),
                    Fdz.data(), dt, m->J, nullptr);
    // flowAdvance, solver.jl:22-38
    double *Fc[3] = {Fx.data(), Fy.data(), Fz.data()};
    for (int d = 0; d < 3; ++d) {
        oracle_fluxSplit(g, Q, Fp.data(), Fm.data(), A[d][0], A[d][1], A[d][2], nullptr);
        oracle_WENO(g, d, Fc[d], phi.data(), Fp.data(), Fm.data(), 5, nullptr);
    }
    double *Fv[3] = {Fvx.data(), Fvy.data(), Fvz.data()};
    for (int d = 0; d < 3; ++d)
        oracle_viscousFlux(g, d, Fv[d], Q, m, lam.data(), mu.data(), Fh[d], nullptr);
    oracle_div(g, U, Fx.data(), Fy.data(), Fz.data(), Fvx.data(), Fvy.data(), Fvz.data(), dt,
               m->J, nullptr);
    if (stage == 2) {
        oracle_linComb(g, U, Un, 5, 0.25, 0.75, nullptr);
        oracle_linComb(g, rhoi, rhon, ns, 0.25, 0.75, nullptr);
    } else if (stage == 3) {
        oracle_linComb(g, U, Un, 5, 2.0 / 3.0, 1.0 / 3.0, nullptr);
        oracle_linComb(g, rhoi, rhon, ns, 2.0 / 3.0, 1.0 / 3.0, nullptr);
    }
    oracle_c2Prim(g, U, Q, rhoi, th, nullptr);
    oracle_fill_periodic(g, Q, 7);
    oracle_fill_periodic(g, rhoi, ns);
}

// Exposed thermo helpers for known-answer tests.
double oracle_GetT(double ein, const double *rhoi, const FlameThermo *th, int ns) {
    return GetT(ein, rhoi, th, ns);
}
double oracle_InternalEnergy(double T, const double *rhoi, const FlameThermo *th, int ns) {
    return InternalEnergy(T, rhoi, th, ns);
}
double oracle_CP(double T, const double *rhoi, const FlameThermo *th, int ns) {
    return CPv(T, rhoi, th, ns);
}
void oracle_h_specs(double *hi, double T, const FlameThermo *th, int ns) {
    h_specs(hi, T, th, ns);
}
void oracle_up7(double *c7) {
    for (int i = 0; i < 7; ++i) c7[i] = kUP7[i];
}
int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
