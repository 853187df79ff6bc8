// kernels_ref.cu — one sm_100a kernel per reference kernel, same index ranges and arithmetic.
//
// These are the drop-in replacements of the CUDA.jl kernels (same arguments, same layout) and
// the parity scaffold of the fused path.  This file is compiled with -fmad=false so its results
// are bit-identical to a strict IEEE CPU evaluation of the reference arithmetic.
//
// Launch shape: blocks of 32 x 4 x 2 threads with x fastest, so a warp reads 32 consecutive
// FP64 values (256 B) of one SoA row instead of the reference's 4-wide x blocks (run.jl:66).

#include "common.cuh"

namespace flame {
namespace {

constexpr int BX = 32, BY = 4, BZ = 2;

inline dim3 grid_for(long long nx, long long ny, long long nz) {
    return dim3((unsigned)((nx + BX - 1) / BX), (unsigned)((ny + BY - 1) / BY),
                (unsigned)((nz + BZ - 1) / BZ));
}
const dim3 kBlock(BX, BY, BZ);

// Face-array geometry of the swept direction d (0: xi, 1: eta, 2: zeta).
struct FaceGeom {
    long long fx, fy, fz, nf;
    long long sn;  // ghosted stride along the face normal
    long long s1, s2;  // ghosted strides of the tangential directions (d+1)%3, (d+2)%3
};
inline FaceGeom face_geom(const Dims &D, int d) {
    FaceGeom f;
    f.fx = D.nx + (d == 0), f.fy = D.ny + (d == 1), f.fz = D.nz + (d == 2);
    f.nf = f.fx * f.fy * f.fz;
    const long long s[3] = {1, D.tx, D.tx * D.ty};
    f.sn = s[d], f.s1 = s[(d + 1) % 3], f.s2 = s[(d + 2) % 3];
    return f;
}

// ------------------------------------------------------------------- schemes.jl:1-24
__global__ void k_shockSensor(Dims D, double *__restrict__ phi, const double *__restrict__ Q) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x + 1;
    long long j = blockIdx.y * (long long)BY + threadIdx.y + 1;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z + 1;
    if (i > D.tx - 2 || j > D.ty - 2 || k > D.tz - 2) return;
    const double *p = Q + 4 * D.np;
    long long c = D.P(i, j, k), sy = D.tx, sz = D.tx * D.ty;
    double Px1 = p[c - 1], Px2 = p[c], Px3 = p[c + 1];
    double Py1 = p[c - sy], Py2 = Px2, Py3 = p[c + sy];
    double Pz1 = p[c - sz], Pz2 = Px2, Pz3 = p[c + sz];
    double phx = fabs(-Px1 + 2 * Px2 - Px3) / (Px1 + 2 * Px2 + Px3);
    double phy = fabs(-Py1 + 2 * Py2 - Py3) / (Py1 + 2 * Py2 + Py3);
    double phz = fabs(-Pz1 + 2 * Pz2 - Pz3) / (Pz1 + 2 * Pz2 + Pz3);
    phi[c] = phx + phy + phz;
}

// ------------------------------------------------------------------- split.jl:17-89
// SWϵ2 = 0 (run.jl:51), so sqrt(E^2 + SWϵ2) = |E| exactly (sqrt of a correctly rounded square
// returns |E| in binary floating point barring under/overflow of E^2).
__global__ void k_fluxSplit(Dims D, const double *__restrict__ Q, double *__restrict__ Fp,
                            double *__restrict__ Fm, const double *__restrict__ Ax,
                            const double *__restrict__ Ay, const double *__restrict__ Az,
                            const int64_t *__restrict__ tag) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    const long long c = D.P(i, j, k), np = D.np;
    if (tag_at(tag, c) == 1) return;
    double rho = Q[c], u = Q[c + np], v = Q[c + 2 * np], w = Q[c + 3 * np], p = Q[c + 4 * np],
           ei = Q[c + 6 * np];
    double A1 = Ax[c], A2 = Ay[c], A3 = Az[c];
    double gam = p / ei + 1;
    double cs = sqrt(gam * p / rho);
    double ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
    double E1 = A1 * u + A2 * v + A3 * w;
    double E2 = E1 - cs * ss;
    double E3 = E1 + cs * ss;
    ss = 1 / ss;
    A1 *= ss, A2 *= ss, A3 *= ss;
    double E1P = (E1 + fabs(E1)) * 0.5, E2P = (E2 + fabs(E2)) * 0.5, E3P = (E3 + fabs(E3)) * 0.5;
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

// ------------------------------------------------------------------- split.jl:101-130
__global__ void k_split(Dims D, const double *__restrict__ rhoi, const double *__restrict__ Q,
                        double *__restrict__ Fp, double *__restrict__ Fm,
                        const double *__restrict__ Ax, const double *__restrict__ Ay,
                        const double *__restrict__ Az, const int64_t *__restrict__ tag) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    const long long c = D.P(i, j, k), np = D.np;
    if (tag_at(tag, c) == 1) return;
    double un = Ax[c] * Q[c + np] + Ay[c] * Q[c + 2 * np] + Az[c] * Q[c + 3 * np];
    double Ep = 0.5 * (un + fabs(un));
    double Em = 0.5 * (un - fabs(un));
    for (int n = 0; n < D.ns; ++n) {
        Fp[c + n * np] = Ep * rhoi[c + n * np];
        Fm[c + n * np] = Em * rhoi[c + n * np];
    }
}

// ------------------------------------------------------------------- schemes.jl:86-437
__global__ void k_WENO(Dims D, FaceGeom f, double *__restrict__ F, const double *__restrict__ phi,
                       const double *__restrict__ Fp, const double *__restrict__ Fm, int NV,
                       const int64_t *__restrict__ tag) {
    long long fi = blockIdx.x * (long long)BX + threadIdx.x;
    long long fj = blockIdx.y * (long long)BY + threadIdx.y;
    long long fk = blockIdx.z * (long long)BZ + threadIdx.z;
    if (fi >= f.fx || fj >= f.fy || fk >= f.fz) return;
    const long long c = D.P(fi + D.ng, fj + D.ng, fk + D.ng), s = f.sn;
    if (tag_at(tag, c) == 1) return;
    const double phif = jmax(phi[c - s], phi[c]);
    const long long fo = fi + f.fx * (fj + f.fy * fk);
    for (int n = 0; n < NV; ++n) {
        const double *p = Fp + n * D.np + c, *m = Fm + n * D.np + c;
        double pv[7], mv[7];
#pragma unroll
        for (int a = 0; a < 7; ++a) pv[a] = 0, mv[a] = 0;
        if (phif < kHybrid1) {
#pragma unroll
            for (int a = 0; a < 6; ++a) pv[a] = p[(a - 3) * s], mv[a] = m[(a - 3) * s];
        } else if (phif < kHybrid2) {
#pragma unroll
            for (int a = 0; a < 5; ++a) pv[a] = p[(a - 3) * s], mv[a + 1] = m[(a - 2) * s];
        } else {
#pragma unroll
            for (int a = 1; a < 4; ++a) pv[a] = p[(a - 3) * s];
#pragma unroll
            for (int a = 2; a < 5; ++a) mv[a] = m[(a - 3) * s];
        }
        F[fo + n * f.nf] = hybrid_face7<double>(pv, mv, phif);
    }
}

// ------------------------------------------------------------------- viscous.jl:1-428
// Derivative along the face normal (the 1.25 / -1/12 half-point stencil) and the averaged 4th
// order tangential central difference of the two cells that share the face.
__device__ __forceinline__ double dnorm4(const double *q, long long sn) {
    return 1.25 * (q[0] - q[-sn]) - (1.0 / 12.0) * (q[sn] - q[-2 * sn]);
}
__device__ __forceinline__ double dtan4(const double *q, long long sn, long long st) {
    return 0.5 * ((2.0 / 3.0) * (q[st] + q[-sn + st] - q[-st] - q[-sn - st]) -
                  (1.0 / 12.0) * (q[2 * st] + q[-sn + 2 * st] - q[-2 * st] - q[-sn - 2 * st]));
}

__global__ void k_viscousFlux(Dims D, FaceGeom f, int d, double *__restrict__ Fv,
                              const double *__restrict__ Q, FlameMetrics m,
                              const double *__restrict__ lambda, const double *__restrict__ mu,
                              const double *__restrict__ Fh, const int64_t *__restrict__ tag) {
    long long fi = blockIdx.x * (long long)BX + threadIdx.x;
    long long fj = blockIdx.y * (long long)BY + threadIdx.y;
    long long fk = blockIdx.z * (long long)BZ + threadIdx.z;
    if (fi >= f.fx || fj >= f.fy || fk >= f.fz) return;
    const long long c = D.P(fi + D.ng, fj + D.ng, fk + D.ng), sn = f.sn, np = D.np;
    if (tag_at(tag, c) == 1) return;
    const double c23 = 2.0 / 3.0;
    const double *M[9] = {m.dxidx,   m.dxidy,   m.dxidz,   m.detadx, m.detady,
                          m.detadz,  m.dzetadx, m.dzetady, m.dzetadz};
    double met[9];
#pragma unroll
    for (int a = 0; a < 9; ++a) met[a] = (M[a][c - sn] + M[a][c]) * 0.5;
    const double Jac = (m.J[c - sn] + m.J[c]) * 0.5;
    const double mui = (mu[c - sn] + mu[c]) * 0.5;
    const double lami = (lambda[c - sn] + lambda[c]) * 0.5;
    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
    double gr[4][3];
    const int qv[4] = {1, 2, 3, 5};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double *q = Q + qv[a] * np + c;
        double dq[3];
        dq[d] = dnorm4(q, sn);
        dq[d1] = dtan4(q, sn, f.s1);
        dq[d2] = dtan4(q, sn, f.s2);
#pragma unroll
        for (int x = 0; x < 3; ++x)
            gr[a][x] = (dq[0] * met[x] + dq[1] * met[3 + x] + dq[2] * met[6 + x]) * Jac;
    }
    const double u = (Q[c - sn + np] + Q[c + np]) * 0.5;
    const double v = (Q[c - sn + 2 * np] + Q[c + 2 * np]) * 0.5;
    const double w = (Q[c - sn + 3 * np] + Q[c + 3 * np]) * 0.5;
    const double div = gr[0][0] + gr[1][1] + gr[2][2];
    const double t11 = mui * (2 * gr[0][0] - c23 * div);
    const double t12 = mui * (gr[0][1] + gr[1][0]);
    const double t13 = mui * (gr[0][2] + gr[2][0]);
    const double t22 = mui * (2 * gr[1][1] - c23 * div);
    const double t23 = mui * (gr[2][1] + gr[1][2]);
    const double t33 = mui * (2 * gr[2][2] - c23 * div);
    const long long fo = fi + f.fx * (fj + f.fy * fk);
    const double E1 = u * t11 + v * t12 + w * t13 + lami * gr[3][0] + Fh[fo];
    const double E2 = u * t12 + v * t22 + w * t23 + lami * gr[3][1] + Fh[fo + f.nf];
    const double E3 = u * t13 + v * t23 + w * t33 + lami * gr[3][2] + Fh[fo + 2 * f.nf];
    const double *md = met + 3 * d;
    Fv[fo] = md[0] * t11 + md[1] * t12 + md[2] * t13;
    Fv[fo + f.nf] = md[0] * t12 + md[1] * t22 + md[2] * t23;
    Fv[fo + 2 * f.nf] = md[0] * t13 + md[1] * t23 + md[2] * t33;
    Fv[fo + 3 * f.nf] = md[0] * E1 + md[1] * E2 + md[2] * E3;
}

// ------------------------------------------------------------------- viscous.jl:430-665
__global__ void k_specViscousFlux(Dims D, FaceGeom f, int d, double *__restrict__ Fd,
                                  const double *__restrict__ Q, const double *__restrict__ Yi,
                                  FlameMetrics m, const double *__restrict__ Dk,
                                  double *__restrict__ Fh, const FlameThermo th,
                                  const int64_t *__restrict__ tag) {
    long long fi = blockIdx.x * (long long)BX + threadIdx.x;
    long long fj = blockIdx.y * (long long)BY + threadIdx.y;
    long long fk = blockIdx.z * (long long)BZ + threadIdx.z;
    if (fi >= f.fx || fj >= f.fy || fk >= f.fz) return;
    const long long c = D.P(fi + D.ng, fj + D.ng, fk + D.ng), sn = f.sn, np = D.np;
    if (tag_at(tag, c) == 1) return;
    const double *M[9] = {m.dxidx,   m.dxidy,   m.dxidz,   m.detadx, m.detady,
                          m.detadz,  m.dzetadx, m.dzetady, m.dzetadz};
    double met[9];
#pragma unroll
    for (int a = 0; a < 9; ++a) met[a] = (M[a][c - sn] + M[a][c]) * 0.5;
    const double Jac = (m.J[c - sn] + m.J[c]) * 0.5;
    const double rho = (Q[c - sn] + Q[c]) * 0.5;
    const double T = (Q[c - sn + 5 * np] + Q[c + 5 * np]) * 0.5;
    const double T2 = 0.5 * T * T, T3 = 2.0 / 3.0 * T2 * T, T4 = T2 * T2, T5 = 0.8 * T4 * T;
    const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
    double Vk1[FLAME_MAX_NS], Vk2[FLAME_MAX_NS], Vk3[FLAME_MAX_NS];
    double sum1 = 0, sum2 = 0, sum3 = 0;
    const int ns = D.ns;
    for (int n = 0; n < ns; ++n) {
        const double *y = Yi + n * np + c;
        const double rhoDi = (Dk[c - sn + n * np] + Dk[c + n * np]) * rho;
        double dY[3];
        dY[d] = dnorm4(y, sn);
        dY[d1] = 0.25 * (y[f.s1] + y[-sn + f.s1] - y[-f.s1] - y[-sn - f.s1]);
        dY[d2] = 0.25 * (y[f.s2] + y[-sn + f.s2] - y[-f.s2] - y[-sn - f.s2]);
        const double Vx = (dY[0] * met[0] + dY[1] * met[3] + dY[2] * met[6]) * Jac * rhoDi;
        const double Vy = (dY[0] * met[1] + dY[1] * met[4] + dY[2] * met[7]) * Jac * rhoDi;
        const double Vz = (dY[0] * met[2] + dY[1] * met[5] + dY[2] * met[8]) * Jac * rhoDi;
        Vk1[n] = Vx, Vk2[n] = Vy, Vk3[n] = Vz;
        sum1 += Vx, sum2 += Vy, sum3 += Vz;
    }
    const long long fo = fi + f.fx * (fj + f.fy * fk);
    const double *md = met + 3 * d;
    double fh1 = 0, fh2 = 0, fh3 = 0;
    for (int n = 0; n < ns; ++n) {
        const double Yn = 0.5 * (Yi[c - sn + n * np] + Yi[c + n * np]);
        const double hn = h_spec(th, n, T, T2, T3, T4, T5);
        const double V1 = Vk1[n] - sum1 * Yn, V2 = Vk2[n] - sum2 * Yn, V3 = Vk3[n] - sum3 * Yn;
        Fd[fo + n * f.nf] = V1 * md[0] + V2 * md[1] + V3 * md[2];
        fh1 += V1 * hn, fh2 += V2 * hn, fh3 += V3 * hn;
    }
    Fh[fo] = fh1, Fh[fo + f.nf] = fh2, Fh[fo + 2 * f.nf] = fh3;
}

// ------------------------------------------------------------------- div.jl:16-84
__global__ void k_div(Dims D, double *__restrict__ U, const double *__restrict__ Fx,
                      const double *__restrict__ Fy, const double *__restrict__ Fz,
                      const double *__restrict__ Fvx, const double *__restrict__ Fvy,
                      const double *__restrict__ Fvz, double dt, const double *__restrict__ J,
                      const int64_t *__restrict__ tag, int nv_inv, int species) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.nx || j >= D.ny || k >= D.nz) return;
    const long long c = D.P(i + D.ng, j + D.ng, k + D.ng), np = D.np;
    if (tag_at(tag, c) != 0) return;
    const long long nfx = (D.nx + 1LL) * D.ny * D.nz, nfy = D.nx * (D.ny + 1LL) * D.nz,
                    nfz = D.nx * (long long)D.ny * (D.nz + 1LL);
    const double Jact = J[c] * dt;
    const long long x0 = i + (D.nx + 1LL) * (j + D.ny * k), x1 = x0 + 1;
    const long long y0 = i + D.nx * (j + (D.ny + 1LL) * k), y1 = y0 + D.nx;
    const long long z0 = i + D.nx * (j + (long long)D.ny * k), z1 = z0 + (long long)D.nx * D.ny;
    if (species) {  // divSpecs: Fv_* hold the diffusion fluxes Fd_*
        for (int n = 0; n < nv_inv; ++n)
            U[c + n * np] += (Fx[x0 + n * nfx] - Fx[x1 + n * nfx] + Fy[y0 + n * nfy] -
                              Fy[y1 + n * nfy] + Fz[z0 + n * nfz] - Fz[z1 + n * nfz] +
                              Fvx[x1 + n * nfx] - Fvx[x0 + n * nfx] + Fvy[y1 + n * nfy] -
                              Fvy[y0 + n * nfy] + Fvz[z1 + n * nfz] - Fvz[z0 + n * nfz]) *
                             Jact;
        return;
    }
    double dV[4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
        dV[a] = (Fvx[x1 + a * nfx] - Fvx[x0 + a * nfx]) + (Fvy[y1 + a * nfy] - Fvy[y0 + a * nfy]) +
                (Fvz[z1 + a * nfz] - Fvz[z0 + a * nfz]);
#pragma unroll
    for (int n = 0; n < 5; ++n)
        U[c + n * np] += (Fx[x0 + n * nfx] - Fx[x1 + n * nfx] + Fy[y0 + n * nfy] -
                          Fy[y1 + n * nfy] + Fz[z0 + n * nfz] - Fz[z1 + n * nfz]) *
                         Jact;
#pragma unroll
    for (int a = 0; a < 4; ++a) U[c + (a + 1) * np] += dV[a] * Jact;
}

// ------------------------------------------------------------------- utils.jl:95-112
__global__ void k_linComb(Dims D, double *__restrict__ U, const double *__restrict__ Un, int NV,
                          double a, double b, const int64_t *__restrict__ tag) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.nx || j >= D.ny || k >= D.nz) return;
    const long long c = D.P(i + D.ng, j + D.ng, k + D.ng);
    if (tag_at(tag, c) != 0) return;
    for (int n = 0; n < NV; ++n) U[c + n * D.np] = U[c + n * D.np] * a + Un[c + n * D.np] * b;
}

// ------------------------------------------------------------------- utils.jl:2-48
__global__ void k_c2Prim(Dims D, const double *__restrict__ U, double *__restrict__ Q,
                         double *__restrict__ rhoi, const FlameThermo th,
                         const int64_t *__restrict__ tag) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.nx || j >= D.ny || k >= D.nz) return;
    const long long c = D.P(i + D.ng, j + D.ng, k + D.ng), np = D.np;
    if (tag_at(tag, c) != 0) return;
    const int ns = D.ns;
    const double rho = jmax(U[c], kEps);
    const double rhoinv = 1 / rho;
    double r[FLAME_MAX_NS];
    double sr = 0.0;
    for (int n = 0; n < ns; ++n) {
        r[n] = jmax(rhoi[c + n * np], 0.0);
        sr += r[n];
    }
    for (int n = 0; n < ns; ++n) r[n] *= rho / sr;
    const double u = U[c + np] * rhoinv, v = U[c + 2 * np] * rhoinv, w = U[c + 3 * np] * rhoinv;
    const double ei = jmax(U[c + 4 * np] - 0.5 * rho * (u * u + v * v + w * w), kEps);
    const double T = jmax(get_T<0>(th, ns, ei, r), kEps);
    const double p = jmax(p_mixture<0>(th, ns, T, r), kEps);
    for (int n = 0; n < ns; ++n) rhoi[c + n * np] = r[n];
    Q[c] = rho, Q[c + np] = u, Q[c + 2 * np] = v, Q[c + 3 * np] = w;
    Q[c + 4 * np] = p, Q[c + 5 * np] = T, Q[c + 6 * np] = ei;
}

// ------------------------------------------------------------------- utils.jl:71-92
__global__ void k_prim2c(Dims D, double *__restrict__ U, const double *__restrict__ Q) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= D.np) return;
    const long long np = D.np;
    const double rho = Q[c], u = Q[c + np], v = Q[c + 2 * np], w = Q[c + 3 * np],
                 ei = Q[c + 6 * np];
    U[c] = rho, U[c + np] = u * rho, U[c + 2 * np] = v * rho, U[c + 3 * np] = w * rho;
    U[c + 4 * np] = ei + 0.5 * rho * (u * u + v * v + w * w);
}

// ------------------------------------------------------------------- thermo.jl:371-403
__global__ void k_mixture(Dims D, const double *__restrict__ Q, const double *__restrict__ rhoi,
                          double *__restrict__ Yi, double *__restrict__ lambda,
                          double *__restrict__ mu, double *__restrict__ Dk, const FlameThermo th,
                          const FlameTransport tr, const int64_t *__restrict__ tag) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= D.np) return;
    if (tag_at(tag, c) == 1) return;
    const long long np = D.np;
    const int ns = D.ns;
    const double T = Q[c + 5 * np];
    const double rho = jmax(Q[c], kEps);
    const double rhoinv = 1 / rho;
    double Y[FLAME_MAX_NS];
    for (int n = 0; n < ns; ++n) {
        Y[n] = jmax(rhoi[c + n * np] * rhoinv, 0.0);
        Yi[c + n * np] = Y[n];
    }
    double mv, lv, dv;
    if (tr.law == 2) {  // Y2X (thermo.jl:38-52), then mixtureProperties
        double yow = 0;
        for (int n = 0; n < ns; ++n) yow += Y[n] / th.mw[n];
        const double yowinv = 1 / yow;
        double X[FLAME_MAX_NS], mui[FLAME_MAX_NS], W[FLAME_MAX_NS * FLAME_MAX_NS];
        for (int n = 0; n < ns; ++n) X[n] = Y[n] / th.mw[n] * yowinv;
        mixture_properties(T, Q[c + 4 * np], X, th, tr.poly, ns, W, mui, Dk + c, np, lv, mv);
        mu[c] = mv, lambda[c] = lv;
        return;
    }
    if (tr.law == 0) {
        mv = tr.mu_ref, lv = tr.lambda_ref, dv = tr.D_ref;
    } else {
        const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
        double cpm = 0;
        for (int n = 0; n < ns; ++n) cpm += cp_spec(th, n, T, T2, T3, T4) * Y[n] / th.mw[n];
        cpm *= th.Ru;
        mv = tr.mu_ref * pow(T / tr.T_ref, tr.exponent);
        lv = cpm * mv / tr.Pr;
        dv = lv / (rho * cpm);
    }
    mu[c] = mv, lambda[c] = lv;
    for (int n = 0; n < ns; ++n) Dk[c + n * np] = dv;
}

// ------------------------------------------------------------------- periodic ghost fill
__device__ __forceinline__ long long wrap_idx(long long i, int n, int ng, bool per) {
    if (!per || (i >= ng && i < n + ng)) return i;
    long long r = (i - ng) % n;
    if (r < 0) r += n;
    return ng + r;
}
__global__ void k_fill_periodic(Dims D, double *__restrict__ A, int nv, int periodic) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    const long long si = wrap_idx(i, D.nx, D.ng, periodic & 1);
    const long long sj = wrap_idx(j, D.ny, D.ng, periodic & 2);
    const long long sk = wrap_idx(k, D.nz, D.ng, periodic & 4);
    if (si == i && sj == j && sk == k) return;
    const long long dst = D.P(i, j, k), src = D.P(si, sj, sk);
    for (int n = 0; n < nv; ++n) A[dst + n * D.np] = A[src + n * D.np];
}

// ------------------------------------------------------------------ boundary.jl:1-176
// The inflow state of fill_x / fill_z (boundary.jl:10-43, 89-122): every Yi and ρi zeroed, the
// inflow's Y set, ρ = ρmixture(P, T, Y) (thermo.jl:29-35), ρi = Y ρ, e = InternalEnergy(T, ρi),
// then Q and U.
__device__ void set_inflow(const Dims &D, long long p, double *Q, double *U, double *rhoi,
                           double *Yi, const FlameThermo &th, const FlameInflow &in) {
    const int ns = D.ns;
    const long long np = D.np;
    for (int n = 0; n < ns; ++n) Yi[p + n * np] = 0.0, rhoi[p + n * np] = 0.0;
    for (int n = 0; n < ns; ++n) Yi[p + n * np] = in.Y[n];
    double yow = 0;
    for (int n = 0; n < ns; ++n) yow += Yi[p + n * np] / th.mw[n];
    const double rho = in.P / (th.Ru * in.T * yow);
    double r[FLAME_MAX_NS];
    for (int n = 0; n < ns; ++n) {
        rhoi[p + n * np] = Yi[p + n * np] * rho;
        r[n] = rhoi[p + n * np];
    }
    const double ei = internal_energy<0>(th, ns, in.T, r);
    const double u = in.u, v = in.v, w = in.w;
    const double q[7] = {rho, u, v, w, in.P, in.T, ei};
    for (int n = 0; n < 7; ++n) Q[p + n * np] = q[n];
    U[p] = rho;
    U[p + np] = u * rho;
    U[p + 2 * np] = v * rho;
    U[p + 3 * np] = w * rho;
    U[p + 4 * np] = ei + 0.5 * rho * (u * u + v * v + w * w);
}

__device__ void copy_point(const Dims &D, long long dst, long long src, double *Q, double *U,
                           double *rhoi) {
    for (int n = 0; n < 7 && Q; ++n) Q[dst + n * D.np] = Q[src + n * D.np];
    for (int n = 0; n < 5 && U; ++n) U[dst + n * D.np] = U[src + n * D.np];
    for (int n = 0; n < D.ns && rhoi; ++n) rhoi[dst + n * D.np] = rhoi[src + n * D.np];
}

// fill_x, boundary.jl:1-52 (0-based: inflow i <= NG, outlet i >= nx+NG-1 from nx+NG-2)
__global__ void k_fill_x(Dims D, double *Q, double *U, double *rhoi, double *Yi, FlameThermo th,
                         FlameInflow in, int rank, int nprocs) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    const long long p = D.P(i, j, k);
    if (rank == 0 && i <= D.ng) set_inflow(D, p, Q, U, rhoi, Yi, th, in);
    if (rank == nprocs - 1 && i >= D.nx + D.ng - 1)
        copy_point(D, p, D.P(D.nx + D.ng - 2, j, k), Q, U, rhoi);
}

// fill_y (boundary.jl:54-80) on Q, U and fill_y_s (139-158) on ρi: the same rule
__global__ void k_fill_y(Dims D, double *Q, double *U, double *rhoi) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    if (j <= D.ng)
        copy_point(D, D.P(i, j, k), D.P(i, D.ng + 1, k), Q, U, rhoi);
    else if (j >= D.ny + D.ng - 1)
        copy_point(D, D.P(i, j, k), D.P(i, D.ny + D.ng - 2, k), Q, U, rhoi);
}

// fill_z (boundary.jl:82-137): inflow k <= NG, outlet k >= nz+NG-1 copies Q, U only;
// fill_z_s (160-176) with Q = U = null: the outlet copy of ρi
__global__ void k_fill_z(Dims D, double *Q, double *U, double *rhoi, double *Yi, FlameThermo th,
                         FlameInflow in, int inflow) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    const long long p = D.P(i, j, k);
    if (inflow && k <= D.ng)
        set_inflow(D, p, Q, U, rhoi, Yi, th, in);
    else if (k >= D.nz + D.ng - 1)
        copy_point(D, p, D.P(i, j, D.nz + D.ng - 2), Q, U, inflow ? nullptr : rhoi);
}

// CFL rate of every interior cell, reduced to its maximum (see flame_cfl_max).  A non-negative
// double orders like its bit pattern read as an unsigned integer, so an integer atomicMax of
// the bits is the exact maximum in any order (a NaN rate sorts above every number and so
// propagates).
__global__ void k_cfl_max(Dims D, const double *__restrict__ Q, FlameMetrics m,
                          unsigned long long *out) {
    const long long c = blockIdx.x * 256LL + threadIdx.x;
    const long long ncell = (long long)D.nx * D.ny * D.nz;
    unsigned long long bits = 0;
    if (c < ncell) {
        const long long x = c % D.nx, y = (c / D.nx) % D.ny, z = c / ((long long)D.nx * D.ny);
        const long long p = D.P(x + D.ng, y + D.ng, z + D.ng), np = D.np;
        const double rho = Q[p], u = Q[p + np], v = Q[p + 2 * np], w = Q[p + 3 * np],
                     pr = Q[p + 4 * np], e = Q[p + 6 * np];
        const double gam = pr / e + 1;
        const double cs = sqrt(gam * pr / rho);
        const double J = m.J[p];
        const double *rows[3][3] = {{m.dxidx, m.dxidy, m.dxidz},
                                    {m.detadx, m.detady, m.detadz},
                                    {m.dzetadx, m.dzetady, m.dzetadz}};
        double tot = 0;
        for (int d = 0; d < 3; ++d) {
            const double mx = rows[d][0][p], my = rows[d][1][p], mz = rows[d][2][p];
            tot += J * (fabs(mx * u + my * v + mz * w) + cs * sqrt(mx * mx + my * my + mz * mz));
        }
        bits = (unsigned long long)__double_as_longlong(tot);
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long b = __shfl_down_sync(0xffffffffu, bits, o);
        bits = b > bits ? b : bits;
    }
    if ((threadIdx.x & 31) == 0 && bits) atomicMax(out, bits);
}

// fillIB, boundary.jl:193-279 (15-point stencils, 1-based Julia indices)
__global__ void k_fill_ib(Dims D, double *Q, double *U, double *rhoi, const int64_t *ni,
                          const int64_t *nj, const int64_t *nk, const double *cd,
                          const double *cn, const int64_t *tag, FlameThermo th, double Tw) {
    long long i = blockIdx.x * (long long)BX + threadIdx.x;
    long long j = blockIdx.y * (long long)BY + threadIdx.y;
    long long k = blockIdx.z * (long long)BZ + threadIdx.z;
    if (i >= D.tx || j >= D.ty || k >= D.tz) return;
    const long long p = D.P(i, j, k), np = D.np;
    if (tag[p] != 3) return;
    const int ns = D.ns;
    constexpr int NPT = 15;
    long long q[NPT];
    for (int m = 0; m < NPT; ++m)
        q[m] = D.P(ni[m + NPT * p] - 1, nj[m + NPT * p] - 1, nk[m + NPT * p] - 1);
    const double *cnp = cn + 16 * p, *cdp = cd + 16 * p;
    double Yg[FLAME_MAX_NS];
    for (int n = 0; n < ns; ++n) {  // Y: zero gradient
        double sum = 0.0;
        for (int m = 0; m < NPT; ++m) sum += cnp[m + 1] * (rhoi[q[m] + n * np] / Q[q[m]]);
        Yg[n] = -sum / cnp[0];
    }
    double sum = 0.0;  // p: zero gradient
    for (int m = 0; m < NPT; ++m) sum += cnp[m + 1] * Q[q[m] + 4 * np];
    const double pg = -sum / cnp[0];
    double vel[3];  // u, v, w: Dirichlet
    for (int c = 0; c < 3; ++c) {
        sum = 0.0;
        for (int m = 0; m < NPT; ++m) sum += cdp[m + 1] * Q[q[m] + (1 + c) * np];
        vel[c] = -sum / cdp[0];
    }
    double yow = 0;  // ρmixture, thermo.jl:29-35
    for (int n = 0; n < ns; ++n) yow += Yg[n] / th.mw[n];
    const double rho = pg / (th.Ru * Tw * yow);
    double r[FLAME_MAX_NS];
    for (int n = 0; n < ns; ++n) r[n] = Yg[n] * rho, rhoi[p + n * np] = r[n];
    const double ei = internal_energy<0>(th, ns, Tw, r);
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

// Non-finite values of an array (solver.jl:388-391 tests isnan over U).
__global__ void k_count_nonfinite(long long n, const double *__restrict__ A, unsigned int *count) {
    unsigned int c = 0;
    for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += (long long)gridDim.x * 256)
        c += isfinite(A[i]) ? 0u : 1u;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

}  // namespace
}  // namespace flame

using namespace flame;

// ========================================================================= C ABI
extern "C" {

int flame_shockSensor(const FlameGrid *g, flame_stream_t s, double *phi, const double *Q) {
    if (int e = flame_check_grid(g, "flame_shockSensor")) return e;
    if (!phi || !Q) return flame_fail(FLAME_EINVAL, "flame_shockSensor: NULL array");
    Dims D = make_dims(*g);
    k_shockSensor<<<grid_for(D.tx - 2, D.ty - 2, D.tz - 2), kBlock, 0, s>>>(D, phi, Q);
    return flame_check_launch("flame_shockSensor");
}

int flame_fluxSplit(const FlameGrid *g, flame_stream_t s, const double *Q, double *Fp, double *Fm,
                    const double *Ax, const double *Ay, const double *Az, const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_fluxSplit")) return e;
    if (!Q || !Fp || !Fm || !Ax || !Ay || !Az)
        return flame_fail(FLAME_EINVAL, "flame_fluxSplit: NULL array");
    Dims D = make_dims(*g);
    k_fluxSplit<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, Q, Fp, Fm, Ax, Ay, Az, tag);
    return flame_check_launch("flame_fluxSplit");
}

int flame_split(const FlameGrid *g, flame_stream_t s, const double *rhoi, const double *Q,
                double *Fp, double *Fm, const double *Ax, const double *Ay, const double *Az,
                const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_split")) return e;
    if (!rhoi || !Q || !Fp || !Fm || !Ax || !Ay || !Az)
        return flame_fail(FLAME_EINVAL, "flame_split: NULL array");
    Dims D = make_dims(*g);
    k_split<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, rhoi, Q, Fp, Fm, Ax, Ay, Az, tag);
    return flame_check_launch("flame_split");
}

static int weno_dir(const FlameGrid *g, flame_stream_t s, int d, double *F, const double *phi,
                    const double *Fp, const double *Fm, int NV, const int64_t *tag,
                    const char *name) {
    if (int e = flame_check_grid(g, name)) return e;
    if (!F || !phi || !Fp || !Fm) return flame_fail(FLAME_EINVAL, "%s: NULL array", name);
    if (NV < 1) return flame_fail(FLAME_EINVAL, "%s: NV=%d must be >= 1", name, NV);
    Dims D = make_dims(*g);
    FaceGeom f = face_geom(D, d);
    k_WENO<<<grid_for(f.fx, f.fy, f.fz), kBlock, 0, s>>>(D, f, F, phi, Fp, Fm, NV, tag);
    return flame_check_launch(name);
}
int flame_WENO_x(const FlameGrid *g, flame_stream_t s, double *F, const double *phi,
                 const double *Fp, const double *Fm, int NV, const int64_t *tag) {
    return weno_dir(g, s, 0, F, phi, Fp, Fm, NV, tag, "flame_WENO_x");
}
int flame_WENO_y(const FlameGrid *g, flame_stream_t s, double *F, const double *phi,
                 const double *Fp, const double *Fm, int NV, const int64_t *tag) {
    return weno_dir(g, s, 1, F, phi, Fp, Fm, NV, tag, "flame_WENO_y");
}
int flame_WENO_z(const FlameGrid *g, flame_stream_t s, double *F, const double *phi,
                 const double *Fp, const double *Fm, int NV, const int64_t *tag) {
    return weno_dir(g, s, 2, F, phi, Fp, Fm, NV, tag, "flame_WENO_z");
}

static bool metrics_ok(const FlameMetrics *m) {
    return m && m->dxidx && m->dxidy && m->dxidz && m->detadx && m->detady && m->detadz &&
           m->dzetadx && m->dzetady && m->dzetadz && m->J;
}

// The metric arguments of viscous.jl:1 and :430 (and of flowAdvance / specAdvance,
// solver.jl:21,40): the nine J^-1-scaled cofactors in xi, eta, zeta order, then J.
#define FLAME_METRIC_ARGS                                                                     \
    const double *dxidx, const double *dxidy, const double *dxidz, const double *detadx,     \
        const double *detady, const double *detadz, const double *dzetadx,                  \
        const double *dzetady, const double *dzetadz, const double *J
#define FLAME_METRIC_STRUCT \
    FlameMetrics { dxidx, dxidy, dxidz, detadx, detady, detadz, dzetadx, dzetady, dzetadz, J }

static int visc_dir(const FlameGrid *g, flame_stream_t s, int d, double *Fv, const double *Q,
                    const FlameMetrics &m, const double *lambda, const double *mu,
                    const double *Fh, const int64_t *tag, const char *name) {
    if (int e = flame_check_grid(g, name)) return e;
    if (!Fv || !Q || !lambda || !mu || !Fh || !metrics_ok(&m))
        return flame_fail(FLAME_EINVAL, "%s: NULL array", name);
    Dims D = make_dims(*g);
    FaceGeom f = face_geom(D, d);
    k_viscousFlux<<<grid_for(f.fx, f.fy, f.fz), kBlock, 0, s>>>(D, f, d, Fv, Q, m, lambda, mu,
                                                                 Fh, tag);
    return flame_check_launch(name);
}
int flame_viscousFlux_x(const FlameGrid *g, flame_stream_t s, double *Fv, const double *Q,
                        FLAME_METRIC_ARGS, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag) {
    return visc_dir(g, s, 0, Fv, Q, FLAME_METRIC_STRUCT, lambda, mu, Fh, tag,
                    "flame_viscousFlux_x");
}
int flame_viscousFlux_y(const FlameGrid *g, flame_stream_t s, double *Fv, const double *Q,
                        FLAME_METRIC_ARGS, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag) {
    return visc_dir(g, s, 1, Fv, Q, FLAME_METRIC_STRUCT, lambda, mu, Fh, tag,
                    "flame_viscousFlux_y");
}
int flame_viscousFlux_z(const FlameGrid *g, flame_stream_t s, double *Fv, const double *Q,
                        FLAME_METRIC_ARGS, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag) {
    return visc_dir(g, s, 2, Fv, Q, FLAME_METRIC_STRUCT, lambda, mu, Fh, tag,
                    "flame_viscousFlux_z");
}

static int spec_dir(const FlameGrid *g, flame_stream_t s, int d, double *Fd, const double *Q,
                    const double *Yi, const FlameMetrics &m, const double *Dk, double *Fh,
                    const FlameThermo *th, const int64_t *tag, const char *name) {
    if (int e = flame_check_grid(g, name)) return e;
    if (!Fd || !Q || !Yi || !Dk || !Fh || !th || !metrics_ok(&m))
        return flame_fail(FLAME_EINVAL, "%s: NULL argument", name);
    Dims D = make_dims(*g);
    FaceGeom f = face_geom(D, d);
    k_specViscousFlux<<<grid_for(f.fx, f.fy, f.fz), kBlock, 0, s>>>(D, f, d, Fd, Q, Yi, m, Dk,
                                                                     Fh, *th, tag);
    return flame_check_launch(name);
}
int flame_specViscousFlux_x(const FlameGrid *g, flame_stream_t s, double *Fd, const double *Q,
                            const double *Yi, FLAME_METRIC_ARGS, const double *Dk, double *Fh,
                            const FlameThermo *th, const int64_t *tag) {
    return spec_dir(g, s, 0, Fd, Q, Yi, FLAME_METRIC_STRUCT, Dk, Fh, th, tag,
                    "flame_specViscousFlux_x");
}
int flame_specViscousFlux_y(const FlameGrid *g, flame_stream_t s, double *Fd, const double *Q,
                            const double *Yi, FLAME_METRIC_ARGS, const double *Dk, double *Fh,
                            const FlameThermo *th, const int64_t *tag) {
    return spec_dir(g, s, 1, Fd, Q, Yi, FLAME_METRIC_STRUCT, Dk, Fh, th, tag,
                    "flame_specViscousFlux_y");
}
int flame_specViscousFlux_z(const FlameGrid *g, flame_stream_t s, double *Fd, const double *Q,
                            const double *Yi, FLAME_METRIC_ARGS, const double *Dk, double *Fh,
                            const FlameThermo *th, const int64_t *tag) {
    return spec_dir(g, s, 2, Fd, Q, Yi, FLAME_METRIC_STRUCT, Dk, Fh, th, tag,
                    "flame_specViscousFlux_z");
}

int flame_div(const FlameGrid *g, flame_stream_t s, double *U, const double *Fx, const double *Fy,
              const double *Fz, const double *Fvx, const double *Fvy, const double *Fvz, double dt,
              const double *J, const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_div")) return e;
    if (!U || !Fx || !Fy || !Fz || !Fvx || !Fvy || !Fvz || !J)
        return flame_fail(FLAME_EINVAL, "flame_div: NULL array");
    Dims D = make_dims(*g);
    k_div<<<grid_for(D.nx, D.ny, D.nz), kBlock, 0, s>>>(D, U, Fx, Fy, Fz, Fvx, Fvy, Fvz, dt, J,
                                                         tag, 5, 0);
    return flame_check_launch("flame_div");
}

int flame_divSpecs(const FlameGrid *g, flame_stream_t s, double *rhoi, const double *Fx,
                   const double *Fy, const double *Fz, const double *Fdx, const double *Fdy,
                   const double *Fdz, double dt, const double *J, const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_divSpecs")) return e;
    if (!rhoi || !Fx || !Fy || !Fz || !Fdx || !Fdy || !Fdz || !J)
        return flame_fail(FLAME_EINVAL, "flame_divSpecs: NULL array");
    Dims D = make_dims(*g);
    k_div<<<grid_for(D.nx, D.ny, D.nz), kBlock, 0, s>>>(D, rhoi, Fx, Fy, Fz, Fdx, Fdy, Fdz, dt, J,
                                                         tag, D.ns, 1);
    return flame_check_launch("flame_divSpecs");
}

int flame_linComb(const FlameGrid *g, flame_stream_t s, double *U, const double *Un, int NV,
                  double a, double b, const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_linComb")) return e;
    if (!U || !Un) return flame_fail(FLAME_EINVAL, "flame_linComb: NULL array");
    if (NV < 1) return flame_fail(FLAME_EINVAL, "flame_linComb: NV=%d must be >= 1", NV);
    Dims D = make_dims(*g);
    k_linComb<<<grid_for(D.nx, D.ny, D.nz), kBlock, 0, s>>>(D, U, Un, NV, a, b, tag);
    return flame_check_launch("flame_linComb");
}

int flame_c2Prim(const FlameGrid *g, flame_stream_t s, const double *U, double *Q, double *rhoi,
                 const FlameThermo *th, const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_c2Prim")) return e;
    if (!U || !Q || !rhoi || !th) return flame_fail(FLAME_EINVAL, "flame_c2Prim: NULL argument");
    Dims D = make_dims(*g);
    k_c2Prim<<<grid_for(D.nx, D.ny, D.nz), kBlock, 0, s>>>(D, U, Q, rhoi, *th, tag);
    return flame_check_launch("flame_c2Prim");
}

int flame_prim2c(const FlameGrid *g, flame_stream_t s, double *U, const double *Q) {
    if (int e = flame_check_grid(g, "flame_prim2c")) return e;
    if (!U || !Q) return flame_fail(FLAME_EINVAL, "flame_prim2c: NULL array");
    Dims D = make_dims(*g);
    k_prim2c<<<(unsigned)((D.np + 255) / 256), 256, 0, s>>>(D, U, Q);
    return flame_check_launch("flame_prim2c");
}

int flame_mixture(const FlameGrid *g, flame_stream_t s, const double *Q, const double *rhoi,
                  double *Yi, double *lambda, double *mu, double *Dk, const FlameThermo *th,
                  const FlameTransport *tr, const int64_t *tag) {
    if (int e = flame_check_grid(g, "flame_mixture")) return e;
    if (!Q || !rhoi || !Yi || !lambda || !mu || !Dk || !th || !tr)
        return flame_fail(FLAME_EINVAL, "flame_mixture: NULL argument");
    if (tr->law < 0 || tr->law > 2)
        return flame_fail(FLAME_EINVAL, "flame_mixture: transport law %d unknown", tr->law);
    if (tr->law == 2 && !tr->poly)
        return flame_fail(FLAME_EINVAL, "flame_mixture: law 2 needs the polynomial fits (poly)");
    Dims D = make_dims(*g);
    k_mixture<<<(unsigned)((D.np + 255) / 256), 256, 0, s>>>(D, Q, rhoi, Yi, lambda, mu, Dk, *th,
                                                              *tr, tag);
    return flame_check_launch("flame_mixture");
}

static int check_fill_grid(const FlameGrid *g, const char *what) {
    if (int e = flame_check_grid(g, what)) return e;
    if (g->nx < 3 || g->ny < 3 || g->nz < 3)
        return flame_fail(FLAME_EINVAL, "%s: the reference fills need at least 3 cells per axis",
                          what);
    return FLAME_OK;
}

int flame_fill_x(const FlameGrid *g, flame_stream_t s, double *Q, double *U, double *rhoi,
                 double *Yi, const FlameThermo *th, const FlameInflow *in, int rank, int nprocs) {
    if (int e = check_fill_grid(g, "flame_fill_x")) return e;
    if (!Q || !U || !rhoi || !Yi || !th || !in || nprocs < 1 || rank < 0 || rank >= nprocs)
        return flame_fail(FLAME_EINVAL, "flame_fill_x: NULL argument or bad rank/nprocs");
    const Dims D = make_dims(*g);
    k_fill_x<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, Q, U, rhoi, Yi, *th, *in, rank,
                                                           nprocs);
    return flame_check_launch("flame_fill_x");
}

int flame_fill_y(const FlameGrid *g, flame_stream_t s, double *Q, double *U) {
    if (int e = check_fill_grid(g, "flame_fill_y")) return e;
    if (!Q || !U) return flame_fail(FLAME_EINVAL, "flame_fill_y: NULL argument");
    const Dims D = make_dims(*g);
    k_fill_y<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, Q, U, nullptr);
    return flame_check_launch("flame_fill_y");
}

int flame_fill_z(const FlameGrid *g, flame_stream_t s, double *Q, double *U, double *rhoi,
                 double *Yi, const FlameThermo *th, const FlameInflow *in) {
    if (int e = check_fill_grid(g, "flame_fill_z")) return e;
    if (!Q || !U || !rhoi || !Yi || !th || !in)
        return flame_fail(FLAME_EINVAL, "flame_fill_z: NULL argument");
    const Dims D = make_dims(*g);
    k_fill_z<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, Q, U, rhoi, Yi, *th, *in, 1);
    return flame_check_launch("flame_fill_z");
}

int flame_fill_y_s(const FlameGrid *g, flame_stream_t s, double *rhoi) {
    if (int e = check_fill_grid(g, "flame_fill_y_s")) return e;
    if (!rhoi) return flame_fail(FLAME_EINVAL, "flame_fill_y_s: NULL argument");
    const Dims D = make_dims(*g);
    k_fill_y<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, nullptr, nullptr, rhoi);
    return flame_check_launch("flame_fill_y_s");
}

int flame_fill_z_s(const FlameGrid *g, flame_stream_t s, double *rhoi) {
    if (int e = check_fill_grid(g, "flame_fill_z_s")) return e;
    if (!rhoi) return flame_fail(FLAME_EINVAL, "flame_fill_z_s: NULL argument");
    const Dims D = make_dims(*g);
    const FlameThermo th{};
    const FlameInflow in{};
    k_fill_z<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, nullptr, nullptr, rhoi, nullptr,
                                                           th, in, 0);
    return flame_check_launch("flame_fill_z_s");
}

int flame_fillGhost(const FlameGrid *g, flame_stream_t s, double *Q, double *U, double *rhoi,
                    double *Yi, const FlameThermo *th, const FlameInflow *in, int rank,
                    int nprocs) {
    if (int e = flame_fill_x(g, s, Q, U, rhoi, Yi, th, in, rank, nprocs)) return e;
    if (int e = flame_fill_y(g, s, Q, U)) return e;
    return flame_fill_z(g, s, Q, U, rhoi, Yi, th, in);
}

int flame_fillSpec(const FlameGrid *g, flame_stream_t s, double *rhoi) {
    if (int e = flame_fill_y_s(g, s, rhoi)) return e;
    return flame_fill_z_s(g, s, rhoi);
}

int flame_fillIB(const FlameGrid *g, flame_stream_t s, double *Q, double *U, double *rhoi,
                 const int64_t *neari, const int64_t *nearj, const int64_t *neark,
                 const double *c_d, const double *c_n, const int64_t *tag, const FlameThermo *th,
                 double T_wall) {
    if (int e = flame_check_grid(g, "flame_fillIB")) return e;
    if (!Q || !U || !rhoi || !neari || !nearj || !neark || !c_d || !c_n || !tag || !th)
        return flame_fail(FLAME_EINVAL, "flame_fillIB: NULL argument");
    const Dims D = make_dims(*g);
    k_fill_ib<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, Q, U, rhoi, neari, nearj, neark,
                                                            c_d, c_n, tag, *th, T_wall);
    return flame_check_launch("flame_fillIB");
}

int flame_check_finite(const FlameGrid *g, flame_stream_t s, const double *A, int nv,
                       unsigned int *count) {
    if (int e = flame_check_grid(g, "flame_check_finite")) return e;
    if (!A || !count || nv < 1) return flame_fail(FLAME_EINVAL, "flame_check_finite: bad argument");
    const Dims D = make_dims(*g);
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "flame_check_finite: %s", cudaGetErrorString(e));
    const long long n = D.np * nv;
    const long long blocks = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
    k_count_nonfinite<<<(unsigned)blocks, 256, 0, s>>>(n, A, count);
    return flame_check_launch("flame_check_finite");
}

int flame_cfl_max(const FlameGrid *g, flame_stream_t s, const double *Q, const FlameMetrics *m,
                  double *out) {
    if (int e = flame_check_grid(g, "flame_cfl_max")) return e;
    if (!Q || !m || !out || !m->J || !m->dxidx || !m->dxidy || !m->dxidz || !m->detadx ||
        !m->detady || !m->detadz || !m->dzetadx || !m->dzetady || !m->dzetadz)
        return flame_fail(FLAME_EINVAL, "flame_cfl_max: NULL argument");
    const Dims D = make_dims(*g);
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
    if (e != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "flame_cfl_max: %s", cudaGetErrorString(e));
    const long long ncell = (long long)D.nx * D.ny * D.nz;
    k_cfl_max<<<(unsigned)((ncell + 255) / 256), 256, 0, s>>>(
        D, Q, *m, reinterpret_cast<unsigned long long *>(out));
    return flame_check_launch("flame_cfl_max");
}

int flame_fill_periodic(const FlameGrid *g, flame_stream_t s, double *A, int nv) {
    if (int e = flame_check_grid(g, "flame_fill_periodic")) return e;
    if (!A || nv < 1) return flame_fail(FLAME_EINVAL, "flame_fill_periodic: bad array/nv");
    Dims D = make_dims(*g);
    k_fill_periodic<<<grid_for(D.tx, D.ty, D.tz), kBlock, 0, s>>>(D, A, nv, g->periodic);
    return flame_check_launch("flame_fill_periodic");
}

// solver.jl:22-38
int flame_flowAdvance(const FlameGrid *g, flame_stream_t s, double *U, const double *Q, double *Fp,
                      double *Fm, double *Fx, double *Fy, double *Fz, double *Fvx, double *Fvy,
                      double *Fvz, FLAME_METRIC_ARGS, double dt, const double *phi,
                      const double *lambda, const double *mu, const double *Fhx,
                      const double *Fhy, const double *Fhz, const int64_t *tag) {
    const FlameMetrics m = FLAME_METRIC_STRUCT;
    if (!metrics_ok(&m)) return flame_fail(FLAME_EINVAL, "flame_flowAdvance: NULL metrics");
    int e;
    if ((e = flame_fluxSplit(g, s, Q, Fp, Fm, dxidx, dxidy, dxidz, tag))) return e;
    if ((e = flame_WENO_x(g, s, Fx, phi, Fp, Fm, 5, tag))) return e;
    if ((e = flame_fluxSplit(g, s, Q, Fp, Fm, detadx, detady, detadz, tag))) return e;
    if ((e = flame_WENO_y(g, s, Fy, phi, Fp, Fm, 5, tag))) return e;
    if ((e = flame_fluxSplit(g, s, Q, Fp, Fm, dzetadx, dzetady, dzetadz, tag))) return e;
    if ((e = flame_WENO_z(g, s, Fz, phi, Fp, Fm, 5, tag))) return e;
    if ((e = visc_dir(g, s, 0, Fvx, Q, m, lambda, mu, Fhx, tag, "flame_viscousFlux_x"))) return e;
    if ((e = visc_dir(g, s, 1, Fvy, Q, m, lambda, mu, Fhy, tag, "flame_viscousFlux_y"))) return e;
    if ((e = visc_dir(g, s, 2, Fvz, Q, m, lambda, mu, Fhz, tag, "flame_viscousFlux_z"))) return e;
    return flame_div(g, s, U, Fx, Fy, Fz, Fvx, Fvy, Fvz, dt, J, tag);
}

// solver.jl:40-56
int flame_specAdvance(const FlameGrid *g, flame_stream_t s, double *rhoi, const double *Q,
                      const double *Yi, double *Fpi, double *Fmi, double *Fxi, double *Fyi,
                      double *Fzi, double *Fdx, double *Fdy, double *Fdz, FLAME_METRIC_ARGS,
                      double dt, const double *phi, const double *Dk, double *Fhx, double *Fhy,
                      double *Fhz, const FlameThermo *th, const int64_t *tag) {
    const FlameMetrics m = FLAME_METRIC_STRUCT;
    if (!metrics_ok(&m)) return flame_fail(FLAME_EINVAL, "flame_specAdvance: NULL metrics");
    const int ns = g ? g->ns : 0;
    int e;
    if ((e = flame_split(g, s, rhoi, Q, Fpi, Fmi, dxidx, dxidy, dxidz, tag))) return e;
    if ((e = flame_WENO_x(g, s, Fxi, phi, Fpi, Fmi, ns, tag))) return e;
    if ((e = flame_split(g, s, rhoi, Q, Fpi, Fmi, detadx, detady, detadz, tag))) return e;
    if ((e = flame_WENO_y(g, s, Fyi, phi, Fpi, Fmi, ns, tag))) return e;
    if ((e = flame_split(g, s, rhoi, Q, Fpi, Fmi, dzetadx, dzetady, dzetadz, tag))) return e;
    if ((e = flame_WENO_z(g, s, Fzi, phi, Fpi, Fmi, ns, tag))) return e;
    if ((e = spec_dir(g, s, 0, Fdx, Q, Yi, m, Dk, Fhx, th, tag, "flame_specViscousFlux_x")))
        return e;
    if ((e = spec_dir(g, s, 1, Fdy, Q, Yi, m, Dk, Fhy, th, tag, "flame_specViscousFlux_y")))
        return e;
    if ((e = spec_dir(g, s, 2, Fdz, Q, Yi, m, Dk, Fhz, th, tag, "flame_specViscousFlux_z")))
        return e;
    return flame_divSpecs(g, s, rhoi, Fxi, Fyi, Fzi, Fdx, Fdy, Fdz, dt, J, tag);
}

}  // extern "C"
