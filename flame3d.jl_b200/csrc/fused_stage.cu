// fused_stage.cu — one launch per SSP-RK3 stage on periodic grids (sm_100a).
//
// A CTA owns a TX x TY x TZ tile of interior cells and performs, for that tile, everything
// solver.jl:298-326 does in ~30 launches:
//   point phase   shock sensor (schemes.jl:1-24) and 1/max(ρ, eps) (the mass-fraction factor of
//                 thermo.jl:391) on the tile and its halo, into shared memory;
//   sweeps        per direction, in chunks: Steger-Warming split of every pencil point into
//                 shared memory (split.jl:17-130), hybrid UP7 / WENO-Z / minmod face fluxes
//                 (schemes.jl:86-437), viscous and species-diffusion face fluxes
//                 (viscous.jl:1-665) and the face differences into per-cell accumulators;
//   epilogue      div (div.jl), RK3 combination (utils.jl:95-112), c2Prim with the Newton
//                 temperature solve (utils.jl:2-48, thermo.jl:231-282), the transport law of
//                 the new state (the stand-in for thermo.jl:371-403), and the writes of the
//                 result and of its periodic ghost images.
// Split fluxes are computed once per point and direction (plus the pencil halo); face fluxes
// once per face; μ, λ, D once per cell (by the epilogue of the stage before).  HBM traffic is
// the stage's inputs (halo re-reads are served by L2) and its outputs.
//
// Template parameters: a tile configuration, NS species (compile-time loops), QT the storage
// type of the primitive and transport arrays, CT the arithmetic type of split, reconstruction
// and viscous fluxes.  The plain path is <cfg, NS, double, double>; the mixed path is
// <cfg, NS, float, float> (reconstruction with its WENO-Z weights in FP32, wenoz_combine_fast
// <float>) with U, Un, rho_i, metrics, accumulators and the Newton solve kept in FP64.
//
// All indices are 32-bit: the host checks that every array holds fewer than 2^31 elements.

#include <atomic>

#include "common.cuh"

int flame_pencil_stage(const FlameGrid *g, cudaStream_t s, int stage, double dt,
                       const FlameStageBuffers *b, const FlameMetrics *m, const FlameThermo *th,
                       const FlameTransport *tr, int precision, void *scratch, int split_finish,
                       int split_species);

namespace flame {
namespace fused {

// Tile configurations the autotuner chooses from.  ZC / YC are the chunk depths of the x/y and
// z sweeps so that a chunk holds exactly NT cells: one owned cell per thread and chunk in the
// x/y sweeps; all owned cells of the threads with cy / YC == chunk in the z sweep.
template <int TX_, int TY_, int TZ_, int NT_, int MINB_>
struct TileCfg {
    static constexpr int TX = TX_, TY = TY_, TZ = TZ_, NT = NT_, MINB = MINB_;
    static constexpr int CELLS = TX * TY * TZ;
    static constexpr int CPT = CELLS / NT;
    static constexpr int ZC = NT / (TX * TY);
    static constexpr int YC = NT / (TX * TZ);
    static_assert(CELLS % NT == 0 && NT % (TX * TY) == 0 && NT % (TX * TZ) == 0, "tile");
    static_assert(TZ % ZC == 0 && TY % YC == 0 && CPT == TZ / ZC, "chunks");
    static constexpr int BX1 = TX + 2, BY1 = TY + 2, BZ1 = TZ + 2, NB1 = BX1 * BY1 * BZ1;
    static constexpr int BX2 = TX + 4, BY2 = TY + 4, BZ2 = TZ + 4, NB2 = BX2 * BY2 * BZ2;
};

using Cfg16x8x8 = TileCfg<16, 8, 8, 256, 1>;
using Cfg16x8x8b2 = TileCfg<16, 8, 8, 256, 2>;
using Cfg8x8x8 = TileCfg<8, 8, 8, 256, 2>;

template <class T, int NS>
struct Layout {
    static constexpr int VF = 10 + 2 * NS;  // split values per point
    static constexpr int VG = 5 + NS;       // face values
    static constexpr int NPX = (T::TX + 6) * T::TY * T::ZC, NPY = T::TX * (T::TY + 6) * T::ZC,
                         NPZ = T::TX * T::YC * (T::TZ + 6);
    static constexpr int NFX = (T::TX + 1) * T::TY * T::ZC, NFY = T::TX * (T::TY + 1) * T::ZC,
                         NFZ = T::TX * T::YC * (T::TZ + 1);
    static constexpr int NPMAX = NPX > NPY ? (NPX > NPZ ? NPX : NPZ) : (NPY > NPZ ? NPY : NPZ);
    static constexpr int NFMAX = NFX > NFY ? (NFX > NFZ ? NFX : NFZ) : (NFY > NFZ ? NFY : NFZ);
};

template <typename QT>
struct Args {
    int nx, ny, nz, ng, tx, ty, tz, np, sy, sz;
    int per;  // periodic axes (FlameGrid::periodic): ghost images are written on these only
    int stage;
    double dt, ca, cb;  // RK3 combination U = ca*U + cb*Un (stages 2, 3)
    double *U, *Un;
    const QT *Qi;
    QT *Qo;
    const QT *Ti;  // μ, λ, D of the stage input
    QT *To;        // μ, λ, D of the stage result
    const double *ri;
    double *ro, *rn;
    const double *met[10];  // ξx ξy ξz ηx ηy ηz ζx ζy ζz J
    FlameThermo th;
    FlameTransport tr;
};

template <class T, int NS, typename CT>
constexpr size_t smem_bytes() {
    using L = Layout<T, NS>;
    // working arrays, or the epilogue's accumulator hand-off if that is larger
    constexpr size_t work =
        sizeof(CT) * (T::NB1 + T::NB2 + L::VF * L::NPMAX + L::VG * L::NFMAX);
    constexpr size_t acc = sizeof(double) * T::CPT * L::VG * T::NT;
    return work > acc ? work : acc;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

template <typename CT, typename T>
__device__ __forceinline__ CT ldg(const T *p, int i) {
    return CT(__ldg(p + i));
}

// Steger-Warming splitting of the Euler flux along metric (A1, A2, A3), split.jl:17-89, with
// the reference's divisions folded into two reciprocals and one reciprocal square root (the
// results differ from the reference's rounding by a few ulp, far inside the 1e-12 bound).
template <typename CT>
__device__ __forceinline__ void sw_split(CT rho, CT u, CT v, CT w, CT p, CT ei, CT A1, CT A2,
                                         CT A3, CT *fp, CT *fm) {
    const CT h = CT(0.5);
    const CT gam = p * (CT(1) / ei) + 1;
    const CT gm1 = gam - 1;
    const CT inv = CT(1) / (rho * gam * gm1);  // 1/(ρ γ (γ-1))
    const CT cs = sqrt(gam * p * (gam * gm1 * inv));
    const CT r2 = A1 * A1 + A2 * A2 + A3 * A3;
    const CT rs = rsqrt(r2);
    const CT ss = r2 * rs;
    const CT E1 = A1 * u + A2 * v + A3 * w;
    const CT E2 = E1 - cs * ss;
    const CT E3 = E1 + cs * ss;
    A1 *= rs, A2 *= rs, A3 *= rs;
    const CT E1P = (E1 + fabs(E1)) * h, E2P = (E2 + fabs(E2)) * h, E3P = (E3 + fabs(E3)) * h;
    const CT E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    const CT uc1 = u - cs * A1, uc2 = u + cs * A1;
    const CT vc1 = v - cs * A2, vc2 = v + cs * A2;
    const CT wc1 = w - cs * A3, wc2 = w + cs * A3;
    const CT vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * h;
    const CT vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * h;
    const CT vv = gm1 * (u * u + v * v + w * w);
    const CT W2 = (3 - gam) * (h * rho * gam * inv) * (cs * cs);  // (3-γ)/(2(γ-1)) c²
    const CT tmp1 = h * rho * (rho * gm1 * inv);                  // ρ/(2γ)
    const CT tmp2 = 2 * gm1;
    fp[0] = tmp1 * (tmp2 * E1P + E2P + E3P);
    fp[1] = tmp1 * (tmp2 * E1P * u + E2P * uc1 + E3P * uc2);
    fp[2] = tmp1 * (tmp2 * E1P * v + E2P * vc1 + E3P * vc2);
    fp[3] = tmp1 * (tmp2 * E1P * w + E2P * wc1 + E3P * wc2);
    fp[4] = tmp1 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0] = tmp1 * (tmp2 * E1M + E2M + E3M);
    fm[1] = tmp1 * (tmp2 * E1M * u + E2M * uc1 + E3M * uc2);
    fm[2] = tmp1 * (tmp2 * E1M * v + E2M * vc1 + E3M * vc2);
    fm[3] = tmp1 * (tmp2 * E1M * w + E2M * wc1 + E3M * wc2);
    fm[4] = tmp1 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

// Transport law of one point (stand-in for mixtureProperties, thermo.jl:289-369); writes μ, λ, D.
template <int NS>
__device__ __forceinline__ void transport_point(const FlameThermo &th, const FlameTransport &tr,
                                                double T, double rho_raw, const double *r,
                                                double &mu, double &lam, double &D) {
    if (tr.law == 0) {
        mu = tr.mu_ref, lam = tr.lambda_ref, D = tr.D_ref;
        return;
    }
    const double rho = jmax(rho_raw, kEps);
    const double rinv = 1 / rho;
    const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
    double cpm = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n)
        cpm += cp_spec(th, n, T, T2, T3, T4) * jmax(r[n] * rinv, 0.0) / th.mw[n];
    cpm *= th.Ru;
    mu = tr.mu_ref * pow(T / tr.T_ref, tr.exponent);
    lam = cpm * mu / tr.Pr;
    D = lam / (rho * cpm);
}

template <class T, int NS, typename QT, typename CT>
struct Tile {
    using L = Layout<T, NS>;
    static constexpr int TX = T::TX, TY = T::TY, TZ = T::TZ, NT = T::NT, CPT = T::CPT;
    const Args<QT> &A;
    const int X0, Y0, Z0;  // interior index of the tile's first cell
    CT *sPhi, *sRinv, *sF, *sG;

    __device__ Tile(const Args<QT> &a, CT *smem)
        : A(a), X0(blockIdx.x * TX), Y0(blockIdx.y * TY), Z0(blockIdx.z * TZ) {
        sPhi = smem;
        sRinv = sPhi + T::NB1;
        sF = sRinv + T::NB2;
        sG = sF + L::VF * L::NPMAX;
    }

    // ghosted linear index of tile-relative cell (x, y, z), clamped into the array
    __device__ int gidx(int x, int y, int z) const {
        const int gx = clampi(X0 + A.ng + x, 0, A.tx - 1);
        const int gy = clampi(Y0 + A.ng + y, 0, A.ty - 1);
        const int gz = clampi(Z0 + A.ng + z, 0, A.tz - 1);
        return gx + A.sy * gy + A.sz * gz;
    }
    // ghosted index of the right cell of a DIR face, clamped so that the whole viscous stencil
    // (normal -2..+1, tangential ±2) stays inside the array even for tiles past the domain end
    template <int DIR>
    __device__ int gidx_face(int x, int y, int z) const {
        const int ng = A.ng;
        const int gx = clampi(X0 + ng + x, ng, A.nx + ng - (DIR != 0));
        const int gy = clampi(Y0 + ng + y, ng, A.ny + ng - (DIR != 1));
        const int gz = clampi(Z0 + ng + z, ng, A.nz + ng - (DIR != 2));
        return gx + A.sy * gy + A.sz * gz;
    }
    __device__ static int b1i(int x, int y, int z) {
        return (x + 1) + T::BX1 * ((y + 1) + T::BY1 * (z + 1));
    }
    __device__ static int b2i(int x, int y, int z) {
        return (x + 2) + T::BX2 * ((y + 2) + T::BY2 * (z + 2));
    }

    // ---------------------------------------------------------------- point phase
    __device__ void point_phase() {
        const QT *Q = A.Qi;
        for (int p = threadIdx.x; p < T::NB2; p += NT) {
            const int x = p % T::BX2 - 2, y = (p / T::BX2) % T::BY2 - 2, z = p / (T::BX2 * T::BY2) - 2;
            sRinv[p] = CT(1) / CT(jmax(double(Q[gidx(x, y, z)]), kEps));
        }
        const QT *P = Q + 4 * A.np;
        for (int p = threadIdx.x; p < T::NB1; p += NT) {
            const int x = p % T::BX1 - 1, y = (p / T::BX1) % T::BY1 - 1, z = p / (T::BX1 * T::BY1) - 1;
            // schemes.jl:10-22 with the exact divisions: the branch thresholds see the same ϕ
            const int gx = clampi(X0 + A.ng + x, 1, A.tx - 2);
            const int gy = clampi(Y0 + A.ng + y, 1, A.ty - 2);
            const int gz = clampi(Z0 + A.ng + z, 1, A.tz - 2);
            const int gc = gx + A.sy * gy + A.sz * gz;
            const CT P2 = CT(P[gc]);
            CT a1 = CT(P[gc - 1]), a3 = CT(P[gc + 1]);
            const CT phx = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
            a1 = CT(P[gc - A.sy]), a3 = CT(P[gc + A.sy]);
            const CT phy = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
            a1 = CT(P[gc - A.sz]), a3 = CT(P[gc + A.sz]);
            const CT phz = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
            sPhi[p] = phx + phy + phz;
        }
    }

    // ---------------------------------------------------------------- split of one point
    template <int DIR>
    __device__ void split_point(int g, CT *out, int stride) const {
        const double *Ax = A.met[3 * DIR], *Ay = A.met[3 * DIR + 1], *Az = A.met[3 * DIR + 2];
        const QT *Q = A.Qi;
        const int np = A.np;
        const CT rho = CT(Q[g]), u = CT(Q[g + np]), v = CT(Q[g + 2 * np]),
                 w = CT(Q[g + 3 * np]), p = CT(Q[g + 4 * np]), ei = CT(Q[g + 6 * np]);
        const CT A1 = ldg<CT>(Ax, g), A2 = ldg<CT>(Ay, g), A3 = ldg<CT>(Az, g);
        CT fp[5], fm[5];
        sw_split<CT>(rho, u, v, w, p, ei, A1, A2, A3, fp, fm);
#pragma unroll
        for (int n = 0; n < 5; ++n) out[n * stride] = fp[n], out[(5 + n) * stride] = fm[n];
        // species: split.jl:101-130
        const CT un = A1 * u + A2 * v + A3 * w;
        const CT Ep = CT(0.5) * (un + fabs(un));
        const CT Em = CT(0.5) * (un - fabs(un));
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            const CT r = CT(A.ri[g + n * np]);
            out[(10 + n) * stride] = Ep * r;
            out[(10 + NS + n) * stride] = Em * r;
        }
    }

    // ---------------------------------------------------------------- viscous face
    // Face between tile cells (x,y,z) - e_DIR and (x,y,z); ghosted index g of the right cell.
    // Subtracts Fv (viscous.jl:1-428) from G[1..4] and Fd_n (viscous.jl:430-665) from G[5+n],
    // so G holds F_inviscid - F_viscous with the sign convention of div.jl.
    template <int DIR>
    __device__ void viscous_face(int g, int x, int y, int z, CT *G) const {
        constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
        const int np = A.np;
        const int sn = DIR == 0 ? 1 : (DIR == 1 ? A.sy : A.sz);
        const int s1 = D1 == 0 ? 1 : (D1 == 1 ? A.sy : A.sz);
        const int s2 = D2 == 0 ? 1 : (D2 == 1 ? A.sy : A.sz);
        const QT *Q = A.Qi;
        const CT h = CT(0.5), c23 = CT(2.0 / 3.0), c12 = CT(1.0 / 12.0);
        CT met[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) met[a] = (ldg<CT>(A.met[a], g - sn) + ldg<CT>(A.met[a], g)) * h;
        const CT Jac = (ldg<CT>(A.met[9], g - sn) + ldg<CT>(A.met[9], g)) * h;
        const QT *Tr = A.Ti;
        const CT mui = (ldg<CT>(Tr, g - sn) + ldg<CT>(Tr, g)) * h;
        const CT lami = (ldg<CT>(Tr + np, g - sn) + ldg<CT>(Tr + np, g)) * h;
        const CT DL = ldg<CT>(Tr + 2 * np, g - sn), DR = ldg<CT>(Tr + 2 * np, g);

        // species diffusion first: it produces Fh for the energy flux (viscous.jl:446-505)
        const CT rho = (CT(Q[g - sn]) + CT(Q[g])) * h;
        const CT Tf = (CT(Q[g - sn + 5 * np]) + CT(Q[g + 5 * np])) * h;
        const int b2R = b2i(x, y, z);
        constexpr int o_n = DIR == 0 ? 1 : (DIR == 1 ? T::BX2 : T::BX2 * T::BY2);
        constexpr int o_1 = D1 == 0 ? 1 : (D1 == 1 ? T::BX2 : T::BX2 * T::BY2);
        constexpr int o_2 = D2 == 0 ? 1 : (D2 == 1 ? T::BX2 : T::BX2 * T::BY2);
        CT Vk1[NS], Vk2[NS], Vk3[NS], Yf[NS];
        CT sum1 = 0, sum2 = 0, sum3 = 0;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            const double *r = A.ri + n * np;
            // Y = max(ρi / max(ρ, eps), 0) at the stencil points (mixture, thermo.jl:391-394)
#define YAT(off, boff) (fmax(CT(r[g + (off)]) * sRinv[b2R + (boff)], CT(0)))
            const CT y0 = YAT(0, 0), ym = YAT(-sn, -o_n);
            const CT yp = YAT(sn, o_n), ymm = YAT(-2 * sn, -2 * o_n);
            const CT dYn = CT(1.25) * (y0 - ym) - c12 * (yp - ymm);
            const CT dY1 = CT(0.25) * (YAT(s1, o_1) + YAT(-sn + s1, -o_n + o_1) - YAT(-s1, -o_1) -
                                       YAT(-sn - s1, -o_n - o_1));
            const CT dY2 = CT(0.25) * (YAT(s2, o_2) + YAT(-sn + s2, -o_n + o_2) - YAT(-s2, -o_2) -
                                       YAT(-sn - s2, -o_n - o_2));
#undef YAT
            CT dY[3];
            dY[DIR] = dYn, dY[D1] = dY1, dY[D2] = dY2;
            const CT rhoDi = (DL + DR) * rho;  // viscous.jl:473 (no 1/2, as the reference)
            const CT Vx = (dY[0] * met[0] + dY[1] * met[3] + dY[2] * met[6]) * Jac * rhoDi;
            const CT Vy = (dY[0] * met[1] + dY[1] * met[4] + dY[2] * met[7]) * Jac * rhoDi;
            const CT Vz = (dY[0] * met[2] + dY[1] * met[5] + dY[2] * met[8]) * Jac * rhoDi;
            Vk1[n] = Vx, Vk2[n] = Vy, Vk3[n] = Vz;
            sum1 += Vx, sum2 += Vy, sum3 += Vz;
            Yf[n] = h * (ym + y0);
        }
        const CT *md = met + 3 * DIR;
        CT fh1 = 0, fh2 = 0, fh3 = 0;
        {
            const double Td = double(Tf);
            const double T2 = 0.5 * Td * Td, T3 = 2.0 / 3.0 * T2 * Td, T4 = T2 * T2,
                         T5 = 0.8 * T4 * Td;
#pragma unroll
            for (int n = 0; n < NS; ++n) {
                const CT hn = CT(h_spec(A.th, n, Td, T2, T3, T4, T5));
                const CT V1 = Vk1[n] - sum1 * Yf[n], V2 = Vk2[n] - sum2 * Yf[n],
                         V3 = Vk3[n] - sum3 * Yf[n];
                G[5 + n] -= V1 * md[0] + V2 * md[1] + V3 * md[2];
                fh1 += V1 * hn, fh2 += V2 * hn, fh3 += V3 * hn;
            }
        }

        // momentum and energy (viscous.jl:14-141)
        CT gr[4][3];
        const int qv[4] = {1, 2, 3, 5};
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const QT *q = Q + qv[a] * np + g;
            CT dq[3];
            dq[DIR] = CT(1.25) * (CT(q[0]) - CT(q[-sn])) - c12 * (CT(q[sn]) - CT(q[-2 * sn]));
            dq[D1] = h * (c23 * (CT(q[s1]) + CT(q[-sn + s1]) - CT(q[-s1]) - CT(q[-sn - s1])) -
                          c12 * (CT(q[2 * s1]) + CT(q[-sn + 2 * s1]) - CT(q[-2 * s1]) -
                                 CT(q[-sn - 2 * s1])));
            dq[D2] = h * (c23 * (CT(q[s2]) + CT(q[-sn + s2]) - CT(q[-s2]) - CT(q[-sn - s2])) -
                          c12 * (CT(q[2 * s2]) + CT(q[-sn + 2 * s2]) - CT(q[-2 * s2]) -
                                 CT(q[-sn - 2 * s2])));
#pragma unroll
            for (int xx = 0; xx < 3; ++xx)
                gr[a][xx] = (dq[0] * met[xx] + dq[1] * met[3 + xx] + dq[2] * met[6 + xx]) * Jac;
        }
        const CT u = (CT(Q[g - sn + np]) + CT(Q[g + np])) * h;
        const CT v = (CT(Q[g - sn + 2 * np]) + CT(Q[g + 2 * np])) * h;
        const CT w = (CT(Q[g - sn + 3 * np]) + CT(Q[g + 3 * np])) * h;
        const CT div = gr[0][0] + gr[1][1] + gr[2][2];
        const CT t11 = mui * (2 * gr[0][0] - c23 * div);
        const CT t12 = mui * (gr[0][1] + gr[1][0]);
        const CT t13 = mui * (gr[0][2] + gr[2][0]);
        const CT t22 = mui * (2 * gr[1][1] - c23 * div);
        const CT t23 = mui * (gr[2][1] + gr[1][2]);
        const CT t33 = mui * (2 * gr[2][2] - c23 * div);
        const CT E1 = u * t11 + v * t12 + w * t13 + lami * gr[3][0] + fh1;
        const CT E2 = u * t12 + v * t22 + w * t23 + lami * gr[3][1] + fh2;
        const CT E3 = u * t13 + v * t23 + w * t33 + lami * gr[3][2] + fh3;
        G[1] -= md[0] * t11 + md[1] * t12 + md[2] * t13;
        G[2] -= md[0] * t12 + md[1] * t22 + md[2] * t23;
        G[3] -= md[0] * t13 + md[1] * t23 + md[2] * t33;
        G[4] -= md[0] * E1 + md[1] * E2 + md[2] * E3;
    }

    // tile-relative cell of (along a, cross b1, chunk-local b2) in chunk ch of sweep DIR
    template <int DIR>
    __device__ static void sweep_cell(int a, int b, int ch, int &x, int &y, int &z) {
        if (DIR == 0) x = a, y = b % TY, z = ch * T::ZC + b / TY;
        else if (DIR == 1) y = a, x = b % TX, z = ch * T::ZC + b / TX;
        else z = a, x = b % TX, y = ch * T::YC + b / TX;
    }

    // ---------------------------------------------------------------- one sweep direction
    template <int DIR>
    __device__ void sweep(double (&acc)[CPT][L::VG]) {
        constexpr int LEN = DIR == 0 ? TX : (DIR == 1 ? TY : TZ);
        constexpr int NP = DIR == 0 ? L::NPX : (DIR == 1 ? L::NPY : L::NPZ);
        constexpr int NF = DIR == 0 ? L::NFX : (DIR == 1 ? L::NFY : L::NFZ);
        constexpr int NCH = DIR == 2 ? TY / T::YC : TZ / T::ZC;
        const int tid = threadIdx.x;
        const int cx = tid % TX, cy = (tid / TX) % TY, cz0 = tid / (TX * TY);
#pragma unroll 1
        for (int ch = 0; ch < NCH; ++ch) {
            // split fluxes of every pencil point of the chunk
            for (int p = tid; p < NP; p += NT) {
                int x, y, z;
                sweep_cell<DIR>(p % (LEN + 6) - 3, p / (LEN + 6), ch, x, y, z);
                split_point<DIR>(gidx(x, y, z), sF + p, L::NPMAX);
            }
            __syncthreads();
            // face fluxes
            for (int f = tid; f < NF; f += NT) {
                const int a = f % (LEN + 1), b = f / (LEN + 1);
                int x, y, z;
                sweep_cell<DIR>(a, b, ch, x, y, z);
                const int xl = x - (DIR == 0), yl = y - (DIR == 1), zl = z - (DIR == 2);
                const CT phif = CT(jmax(double(sPhi[b1i(xl, yl, zl)]), double(sPhi[b1i(x, y, z)])));
                const int p0 = a + (LEN + 6) * b;  // point index of along-coordinate a-3
                CT G[L::VG];
#pragma unroll
                for (int n = 0; n < L::VG; ++n) {
                    const int vp = n < 5 ? n : 5 + n;  // F+ row (species rows start at 10)
                    const int vm = n < 5 ? 5 + n : 5 + NS + n;
                    // the hybrid face reads F±[c-3..c+2] only (UP7[1] = 0 drops F+[c-4], and
                    // F-[c+3] carries the weight UP7[1] too), i.e. six points of the pencil
                    CT pv[7], mv[7];
#pragma unroll
                    for (int i = 0; i < 6; ++i) {
                        pv[i] = sF[vp * L::NPMAX + p0 + i];
                        mv[i] = sF[vm * L::NPMAX + p0 + i];
                    }
                    pv[6] = mv[6] = CT(0);
                    G[n] = hybrid_face_fast<CT>(pv, mv, phif);
                }
                viscous_face<DIR>(gidx_face<DIR>(x, y, z), x, y, z, G);
#pragma unroll
                for (int n = 0; n < L::VG; ++n) sG[n * L::NFMAX + f] = G[n];
            }
            __syncthreads();
            // face differences into the owned cells of this chunk
#pragma unroll
            for (int m = 0; m < CPT; ++m) {
                const int z = cz0 + T::ZC * m;
                bool in;
                int a, b;
                if (DIR == 2) {
                    in = (cy / T::YC) == ch;
                    a = z, b = cx + TX * (cy - ch * T::YC);
                } else {
                    in = m == ch;
                    a = DIR == 0 ? cx : cy;
                    b = (DIR == 0 ? cy + TY * cz0 : cx + TX * cz0);
                }
                if (in) {
                    const int f0 = a + (LEN + 1) * b;
#pragma unroll
                    for (int n = 0; n < L::VG; ++n)
                        acc[m][n] += double(sG[n * L::NFMAX + f0]) - double(sG[n * L::NFMAX + f0 + 1]);
                }
            }
            __syncthreads();
        }
    }

    // ---------------------------------------------------------------- epilogue
    // The accumulators leave registers through shared memory so the (not unrolled) cell loop
    // below does not force them into local memory for the whole kernel.
    __device__ void epilogue(const double (&acc)[CPT][L::VG]) {
        const int tid = threadIdx.x;
        double *sAcc = reinterpret_cast<double *>(sPhi);
#pragma unroll
        for (int m = 0; m < CPT; ++m)
#pragma unroll
            for (int n = 0; n < L::VG; ++n) sAcc[(m * L::VG + n) * NT + tid] = acc[m][n];
        const int cx = tid % TX, cy = (tid / TX) % TY, cz0 = tid / (TX * TY);
        const int np = A.np, ng = A.ng;
#pragma unroll 1
        for (int m = 0; m < CPT; ++m) {
            const int ix = X0 + cx, iy = Y0 + cy, iz = Z0 + cz0 + T::ZC * m;
            if (ix >= A.nx || iy >= A.ny || iz >= A.nz) continue;
            const int g = (ix + ng) + A.sy * (iy + ng) + A.sz * (iz + ng);
            const double Jact = A.met[9][g] * A.dt;
            double Uc[5], r[NS];
#pragma unroll
            for (int n = 0; n < 5; ++n) {
                const double u0 = A.U[g + n * np];
                if (A.stage == 1) A.Un[g + n * np] = u0;
                double un = u0 + sAcc[(m * L::VG + n) * NT + tid] * Jact;
                if (A.stage > 1) un = un * A.ca + A.Un[g + n * np] * A.cb;
                Uc[n] = un;
                A.U[g + n * np] = un;
            }
#pragma unroll
            for (int n = 0; n < NS; ++n) {
                const double r0 = A.ri[g + n * np];
                if (A.stage == 1) A.rn[g + n * np] = r0;
                double rv = r0 + sAcc[(m * L::VG + 5 + n) * NT + tid] * Jact;
                if (A.stage > 1) rv = rv * A.ca + A.rn[g + n * np] * A.cb;
                r[n] = rv;
            }
            // c2Prim, utils.jl:2-48
            const double rho = jmax(Uc[0], kEps);
            const double rinv = 1 / rho;
            double sr = 0.0;
#pragma unroll
            for (int n = 0; n < NS; ++n) r[n] = jmax(r[n], 0.0), sr += r[n];
            const double sc = rho / sr;
#pragma unroll
            for (int n = 0; n < NS; ++n) r[n] *= sc;
            const double u = Uc[1] * rinv, v = Uc[2] * rinv, w = Uc[3] * rinv;
            const double ei = jmax(Uc[4] - 0.5 * rho * (u * u + v * v + w * w), kEps);
            const double Tn = jmax(NS < 4 ? get_T<NS>(A.th, NS, ei, r)
                                           : get_T_mix<NS>(MixPoly<NS>(A.th, r), A.th, ei, r),
                                   kEps);
            const double p = jmax(p_mixture<NS>(A.th, NS, Tn, r), kEps);
            double mu, lam, D;
            transport_point<NS>(A.th, A.tr, Tn, rho, r, mu, lam, D);
            const double qv[7] = {rho, u, v, w, p, Tn, ei};
            const double tv[3] = {mu, lam, D};
            // the cell and its ghost images along the periodic axes (new: the reference fills
            // ghosts with case-specific kernels, boundary.jl:1-191, which the caller runs after
            // the stage for the other axes)
            const int gx = ix + ng, gy = iy + ng, gz = iz + ng;
            // up to two images per axis: an axis shorter than 2 NG has cells near both ends
            int ox[3] = {0, 0, 0}, oy[3] = {0, 0, 0}, oz[3] = {0, 0, 0};
            int nxo = 1, nyo = 1, nzo = 1;
            if (A.per & 1) {
                if (gx < 2 * ng) ox[nxo++] = A.nx;
                if (gx >= A.nx) ox[nxo++] = -A.nx;
            }
            if (A.per & 2) {
                if (gy < 2 * ng) oy[nyo++] = A.ny;
                if (gy >= A.ny) oy[nyo++] = -A.ny;
            }
            if (A.per & 4) {
                if (gz < 2 * ng) oz[nzo++] = A.nz;
                if (gz >= A.nz) oz[nzo++] = -A.nz;
            }
            for (int c = 0; c < nzo; ++c)
                for (int b = 0; b < nyo; ++b)
                    for (int a = 0; a < nxo; ++a) {
                        const int t = (gx + ox[a]) + A.sy * (gy + oy[b]) + A.sz * (gz + oz[c]);
#pragma unroll
                        for (int n = 0; n < 7; ++n) A.Qo[t + n * np] = QT(qv[n]);
#pragma unroll
                        for (int n = 0; n < 3; ++n) A.To[t + n * np] = QT(tv[n]);
#pragma unroll
                        for (int n = 0; n < NS; ++n) A.ro[t + n * np] = r[n];
                    }
        }
    }
};

template <class T, int NS, typename QT, typename CT>
__global__ void __launch_bounds__(T::NT, T::MINB) k_stage(const __grid_constant__ Args<QT> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Tile<T, NS, QT, CT> t(A, reinterpret_cast<CT *>(smem_raw));
    double acc[T::CPT][Layout<T, NS>::VG];
#pragma unroll
    for (int m = 0; m < T::CPT; ++m)
#pragma unroll
        for (int n = 0; n < Layout<T, NS>::VG; ++n) acc[m][n] = 0.0;
    t.point_phase();
    __syncthreads();
    t.template sweep<0>(acc);
    t.template sweep<1>(acc);
    t.template sweep<2>(acc);
    __syncthreads();  // every thread is done with the working arrays before the hand-off
    t.epilogue(acc);
}

// The points whose transport a ghost fill can invalidate: with `on` set, a ghosted point is
// taken when, on an axis that is not periodic, it is a ghost or the first or last interior
// plane (the planes the reference's fills overwrite, boundary.jl:1-176); otherwise every point.
struct Shell {
    int on, tx, ty, nx, ny, nz, ng, per;
    __device__ __forceinline__ bool take(int c) const {
        if (!on) return true;
        const int gx = c % tx, gy = (c / tx) % ty, gz = c / (tx * ty);
        const auto edge = [this](int g, int n) { return g <= ng || g >= n + ng - 1; };
        return (!(per & 1) && edge(gx, nx)) || (!(per & 2) && edge(gy, ny)) ||
               (!(per & 4) && edge(gz, nz));
    }
};

// Transport of the ghosted points of a state (every point once, to start the fused stage loop;
// the boundary shell after a ghost fill).
template <int NS, typename QT>
__global__ void k_transport(int np, const QT *__restrict__ Q, const double *__restrict__ ri,
                            QT *__restrict__ To, const FlameThermo th, const FlameTransport tr,
                            const Shell sh) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= np || !sh.take(c)) return;
    double r[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) r[n] = ri[c + n * np];
    double mu, lam, D;
    transport_point<NS>(th, tr, double(Q[c + 5 * np]), double(Q[c]), r, mu, lam, D);
    To[c] = QT(mu), To[c + np] = QT(lam), To[c + 2 * np] = QT(D);
}

// The same with the mixture-averaged law (law 2): μ, λ and the per-species D_k (fields 2 + n).
template <int NS, typename QT>
__global__ void k_transport_mix(int np, const QT *__restrict__ Q, const double *__restrict__ ri,
                                QT *__restrict__ To, const FlameThermo th,
                                const FlameTransport tr, const Shell sh) {
    __shared__ MixTables<NS, QT> mt;
    mix_tables_fill<NS, QT>(th, tr, mt);
    __syncthreads();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= np || !sh.take(c)) return;
    double r[NS], Dk[NS], mu, lam;
#pragma unroll
    for (int n = 0; n < NS; ++n) r[n] = ri[c + n * np];
    mixture_point<NS, QT>(th, tr, mt, double(Q[c + 5 * np]), double(Q[c + 4 * np]), double(Q[c]), r,
                      mu, lam, Dk);
    To[c] = QT(mu), To[c + np] = QT(lam);
#pragma unroll
    for (int n = 0; n < NS; ++n) To[c + (2 + n) * np] = QT(Dk[n]);
}

template <typename QT>
Args<QT> make_args(const FlameGrid &g, int stage, double dt, const FlameStageBuffers &b,
                   const FlameMetrics &m, const FlameThermo &th, const FlameTransport &tr) {
    Args<QT> A;
    A.nx = g.nx, A.ny = g.ny, A.nz = g.nz, A.ng = g.ng;
    A.tx = g.nx + 2 * g.ng, A.ty = g.ny + 2 * g.ng, A.tz = g.nz + 2 * g.ng;
    A.np = A.tx * A.ty * A.tz;
    A.sy = A.tx, A.sz = A.tx * A.ty;
    A.per = g.periodic & 7;
    A.stage = stage;
    A.dt = dt;
    A.ca = stage == 2 ? 0.25 : 2.0 / 3.0;
    A.cb = stage == 2 ? 0.75 : 1.0 / 3.0;
    A.U = b.U, A.Un = b.Un;
    A.Qi = static_cast<const QT *>(b.Q_in);
    A.Qo = static_cast<QT *>(b.Q_out);
    A.Ti = static_cast<const QT *>(b.trans_in);
    A.To = static_cast<QT *>(b.trans_out);
    A.ri = b.rhoi_in, A.ro = b.rhoi_out, A.rn = b.rhon;
    const double *mm[10] = {m.dxidx,   m.dxidy,   m.dxidz,   m.detadx, m.detady,
                            m.detadz,  m.dzetadx, m.dzetady, m.dzetadz, m.J};
    for (int i = 0; i < 10; ++i) A.met[i] = mm[i];
    A.th = th, A.tr = tr;
    return A;
}

template <class T, int NS, typename QT, typename CT>
int launch(const FlameGrid &g, cudaStream_t s, int stage, double dt, const FlameStageBuffers &b,
           const FlameMetrics &m, const FlameThermo &th, const FlameTransport &tr) {
    const Args<QT> A = make_args<QT>(g, stage, dt, b, m, th, tr);
    constexpr size_t sm = smem_bytes<T, NS, CT>();
    // the attribute is per function and device; atomic, as host threads on other streams may
    // launch the same kernel at the same time (both then set it, to the same value)
    static std::atomic<bool> attr_set[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev].load(std::memory_order_acquire)) {
        cudaError_t e = cudaFuncSetAttribute(k_stage<T, NS, QT, CT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess)
            return flame_fail(FLAME_ELAUNCH, "flame_rk_stage: %zu B shared memory: %s", sm,
                              cudaGetErrorString(e));
        if (dev >= 0 && dev < 64) attr_set[dev].store(true, std::memory_order_release);
    }
    dim3 grid((g.nx + T::TX - 1) / T::TX, (g.ny + T::TY - 1) / T::TY, (g.nz + T::TZ - 1) / T::TZ);
    k_stage<T, NS, QT, CT><<<grid, T::NT, sm, s>>>(A);
    return flame_check_launch("flame_rk_stage");
}

template <class T, typename QT, typename CT>
int dispatch_ns(int ns, const FlameGrid &g, cudaStream_t s, int stage, double dt,
                const FlameStageBuffers &b, const FlameMetrics &m, const FlameThermo &th,
                const FlameTransport &tr) {
    switch (ns) {
#define CASE(N) \
    case N: return launch<T, N, QT, CT>(g, s, stage, dt, b, m, th, tr);
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9)
#undef CASE
        default:
            return flame_fail(FLAME_EUNSUPPORTED, "flame_rk_stage: ns=%d (fused path has 1..9)",
                              ns);
    }
}

template <typename QT, typename CT>
int dispatch_tile(int tile, int ns, const FlameGrid &g, cudaStream_t s, int stage, double dt,
                  const FlameStageBuffers &b, const FlameMetrics &m, const FlameThermo &th,
                  const FlameTransport &tr) {
    switch (tile) {
        case 0: return dispatch_ns<Cfg16x8x8, QT, CT>(ns, g, s, stage, dt, b, m, th, tr);
        case 1: return dispatch_ns<Cfg16x8x8b2, QT, CT>(ns, g, s, stage, dt, b, m, th, tr);
        case 2: return dispatch_ns<Cfg8x8x8, QT, CT>(ns, g, s, stage, dt, b, m, th, tr);
        case 3:
        case 4:
        case 5:
        case 6:
            return flame_pencil_stage(&g, s, stage, dt, &b, &m, &th, &tr,
                                      sizeof(QT) == 8 ? 0 : 1, b.scratch, tile == 4 || tile == 6,
                                      tile >= 5);
        default: return flame_fail(FLAME_EINVAL, "flame_rk_stage: tile config %d unknown", tile);
    }
}

template <typename QT>
int transport_ns(int ns, int np, cudaStream_t s, const void *Q, const double *ri, void *To,
                 const FlameThermo &th, const FlameTransport &tr, const Shell &sh) {
    const unsigned blocks = (unsigned)((np + 255) / 256);
    const QT *q = static_cast<const QT *>(Q);
    QT *t = static_cast<QT *>(To);
    switch (ns) {
#define CASE(N)                                                                              \
    case N:                                                                                  \
        if (tr.law == 2) k_transport_mix<N, QT><<<blocks, 256, 0, s>>>(np, q, ri, t, th, tr, sh); \
        else k_transport<N, QT><<<blocks, 256, 0, s>>>(np, q, ri, t, th, tr, sh);           \
        break;
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9)
#undef CASE
        default: return flame_fail(FLAME_EUNSUPPORTED, "flame_transport: ns=%d", ns);
    }
    return flame_check_launch("flame_transport");
}

}  // namespace fused
}  // namespace flame

namespace {
// Every array of the stage must hold fewer than 2^31 elements (32-bit indices).  Extents are
// widened to 64 bits and multiplied one at a time, so absurd extents cannot wrap into a small
// product: before each multiplication the partial product is below 2^28 and the factor below
// 2^32.
int check_sizes(const FlameGrid *g, const char *what) {
    const long long nv = g->ns > 10 ? g->ns : 10;
    const long long ext[3] = {(long long)g->nx + 2LL * g->ng, (long long)g->ny + 2LL * g->ng,
                              (long long)g->nz + 2LL * g->ng};
    long long np = 1;
    for (long long e : ext) {
        np *= e;
        if (np * nv >= (1LL << 31))
            return flame_fail(FLAME_EINVAL,
                              "%s: %dx%dx%d cells with %lld fields exceed 2^31 elements per array",
                              what, g->nx, g->ny, g->nz, nv);
    }
    return FLAME_OK;
}
}  // namespace

static int transport_call(const FlameGrid *g, flame_stream_t s, const void *Q,
                          const double *rhoi, void *trans, const FlameThermo *th,
                          const FlameTransport *tr, int precision, bool shell,
                          const char *what) {
    if (int e = flame_check_grid(g, what)) return e;
    if (int e = check_sizes(g, what)) return e;
    if (!Q || !rhoi || !trans || !th || !tr) return flame_fail(FLAME_EINVAL, "%s: NULL argument", what);
    if (tr->law < 0 || tr->law > 2)
        return flame_fail(FLAME_EINVAL, "%s: transport law %d unknown", what, tr->law);
    if (tr->law == 2 && !tr->poly)
        return flame_fail(FLAME_EINVAL, "%s: law 2 needs the polynomial fits (poly)", what);
    const int np = (g->nx + 2 * g->ng) * (g->ny + 2 * g->ng) * (g->nz + 2 * g->ng);
    const flame::fused::Shell sh{shell ? 1 : 0, g->nx + 2 * g->ng, g->ny + 2 * g->ng, g->nx,
                                 g->ny, g->nz, g->ng, g->periodic & 7};
    if (shell && sh.per == 7) return FLAME_OK;  // no axis is filled by the caller
    if (precision == 0)
        return flame::fused::transport_ns<double>(g->ns, np, s, Q, rhoi, trans, *th, *tr, sh);
    if (precision == 1)
        return flame::fused::transport_ns<float>(g->ns, np, s, Q, rhoi, trans, *th, *tr, sh);
    return flame_fail(FLAME_EINVAL, "%s: precision=%d must be 0 or 1", what, precision);
}

extern "C" int flame_transport(const FlameGrid *g, flame_stream_t s, const void *Q,
                               const double *rhoi, void *trans, const FlameThermo *th,
                               const FlameTransport *tr, int precision) {
    return transport_call(g, s, Q, rhoi, trans, th, tr, precision, false, "flame_transport");
}

extern "C" int flame_transport_boundary(const FlameGrid *g, flame_stream_t s, const void *Q,
                                        const double *rhoi, void *trans, const FlameThermo *th,
                                        const FlameTransport *tr, int precision) {
    return transport_call(g, s, Q, rhoi, trans, th, tr, precision, true,
                          "flame_transport_boundary");
}

extern "C" int flame_rk_stage_tiled(const FlameGrid *g, flame_stream_t s, int stage, double dt,
                                    const FlameStageBuffers *b, const FlameMetrics *m,
                                    const FlameThermo *th, const FlameTransport *tr,
                                    int precision, int tile) {
    static const char *kNames[3] = {"flame_rk_stage 1", "flame_rk_stage 2", "flame_rk_stage 3"};
    flame::NvtxRange range(kNames[(stage >= 1 && stage <= 3) ? stage - 1 : 0]);
    if (int e = flame_check_grid(g, "flame_rk_stage")) return e;
    if (int e = check_sizes(g, "flame_rk_stage")) return e;
    if (!b || !m || !th || !tr || !b->U || !b->Un || !b->Q_in || !b->Q_out || !b->rhoi_in ||
        !b->rhoi_out || !b->rhon || !b->trans_in || !b->trans_out || !m->J || !m->dxidx ||
        !m->dxidy || !m->dxidz || !m->detadx || !m->detady || !m->detadz || !m->dzetadx ||
        !m->dzetady || !m->dzetadz)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: NULL argument");
    if (stage < 1 || stage > 3)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: stage=%d must be 1, 2 or 3", stage);
    if (tr->law < 0 || tr->law > 2)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: transport law %d unknown", tr->law);
    if (tr->law == 2 && !tr->poly)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: law 2 needs the polynomial fits (poly)");
    if (tr->law == 2 && tile >= 0 && tile <= 2)
        return flame_fail(FLAME_EUNSUPPORTED,
                          "flame_rk_stage: transport law 2 (per-species D_k) runs on the pencil "
                          "configurations 3-6, not on tile configuration %d", tile);
    if (g->nx < FLAME_NG || g->ny < FLAME_NG || g->nz < FLAME_NG)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: extents must be >= %d", FLAME_NG);
    if (b->Q_in == b->Q_out || (const void *)b->rhoi_in == (const void *)b->rhoi_out ||
        b->trans_in == b->trans_out)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: in and out buffers must differ");
    if (precision == 0)
        return flame::fused::dispatch_tile<double, double>(tile, g->ns, *g, s, stage, dt, *b, *m,
                                                           *th, *tr);
    if (precision == 1)
        return flame::fused::dispatch_tile<float, float>(tile, g->ns, *g, s, stage, dt, *b, *m,
                                                         *th, *tr);
    return flame_fail(FLAME_EINVAL, "flame_rk_stage: precision=%d must be 0 or 1", precision);
}

extern "C" int flame_rk_stage(const FlameGrid *g, flame_stream_t s, int stage, double dt,
                              const FlameStageBuffers *b, const FlameMetrics *m,
                              const FlameThermo *th, const FlameTransport *tr, int precision) {
    return flame_rk_stage_tiled(g, s, stage, dt, b, m, th, tr, precision, 0);
}
