// pencil_stage.cu — the RK3 stage as four barrier-free sweeps (sm_100a).
//
// One stage of solver.jl:298-326 on a periodic grid, organised for latency hiding instead of
// shared-memory tiling:
//   k_prep      every ghosted point: shock sensor ϕ (schemes.jl:1-24) and the mass fractions
//               Y = max(ρi / max(ρ, eps), 0) (thermo.jl:391-394) into a scratch array;
//   k_pencil<2> z sweep, k_pencil<1> y sweep, k_pencil<0> x sweep: a warp owns a pencil of 32
//               points along the sweep axis (26 owned cells plus the 3 + 3 stencil halo).  Each
//               lane splits its point once (split.jl:17-130), computes the cell-centred
//               tangential derivatives the viscous fluxes average across a face, and publishes
//               everything in the warp's slice of shared memory; the face between lanes l-1 and
//               l then forms the hybrid UP7 / WENO-Z / minmod flux (schemes.jl:86-437) minus the
//               viscous and species-diffusion flux (viscous.jl:1-665); the difference of two
//               faces is the cell's contribution.  Only __syncwarp orders the phases.
//   The z and y sweeps accumulate into a scratch right-hand side; the x sweep (lanes along x,
//   so its stores coalesce) finishes the stage: div (div.jl), RK3 combination (utils.jl:95-112),
//   c2Prim with the Newton temperature (utils.jl:2-48, thermo.jl:231-282), the transport law of
//   the new state, and the periodic ghost images.
// Configurations (flame_rk_stage_tiled): 3 as above; 4 moves the finish into k_finish, one
// thread per cell; 5 and 6 are 3 and 4 with each z / y sweep split into a flow sweep (the NS = 0
// instance of the same kernel) and a species sweep (PART 2: species fluxes and the
// enthalpy-diffusion term of the energy flux, with fewer slots and registers).  The flame_batch_*
// persistent kernels at the end of the file run configuration 3 over many cases.
//
// Template parameters as in fused_stage.cu: NS species, QT storage of Q / transport, CT
// arithmetic type of split, reconstruction and viscous fluxes.  All indices are 32-bit.

#include <atomic>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "common.cuh"

namespace flame {
namespace pencil {

constexpr int OWN = 26;  // cells owned by a 32-lane pencil (3 halo lanes below, 3 above)

// Warps per block.  The x sweep reads whole rows per warp; the y and z sweeps read one value per
// lane from 32 different rows, so their blocks take 16 consecutive x columns and together use
// every byte of each 128-byte line they touch.
template <int DIR>
struct Wpb {
    static constexpr int value = DIR == 0 ? 4 : 16;
};

template <typename QT>
struct Args {
    int nx, ny, nz, ng, tx, ty, tz, np, sy, sz;
    int per;  // periodic axes (FlameGrid::periodic): ghost images are written on these only
    int stage;
    double dt, ca, cb;
    double *U, *Un;
    const QT *Qi;
    QT *Qo;
    const QT *Ti;
    QT *To;
    const double *ri;
    double *ro, *rn;
    const double *met[10];
    const QT *metq;  // the metrics rounded to QT once (mixed precision), or null
    QT *aux;     // ϕ (1) and Y (NS), ghosted
    double *R;   // right-hand side accumulator (5 + NS), ghosted indexing: z sweep, then all
    double *R2;  // the y sweep's contribution (5 + NS), written, never read-modify-written
    FlameThermo th;
    FlameTransport tr;
};

// Shared-memory slots of one lane's point (CT each).  REUSE (the FP64 y and z sweeps): the
// metrics are staged after the reconstruction has read the split fluxes, into their slots, so a
// point needs ten slots fewer and three 8-column blocks fit on an SM.
template <int NS, bool REUSE = false>
struct Slots {
    static constexpr int FP = 0;                // F+ flow (5), F- flow (5), F+ sp (NS), F- sp (NS)
    static constexpr int VF = 10 + 2 * NS;
    static constexpr int Q4 = VF;               // u v w T
    static constexpr int MET = REUSE ? FP : Q4 + 4;    // 9 metrics + J
    static constexpr int TR = REUSE ? Q4 + 4 : MET + 10;  // μ λ D
    static constexpr int RHO = TR + 3;
    static constexpr int Y = RHO + 1;           // NS
    static constexpr int DQ1 = Y + NS;          // tangential derivatives of u v w T along d+1
    static constexpr int DQ2 = DQ1 + 4;         // ... along d+2
    static constexpr int DY1 = DQ2 + 4;         // Y[+] - Y[-] along d+1 (NS)
    static constexpr int DY2 = DY1 + NS;        // ... along d+2 (NS)
    static constexpr int PHI = DY2 + NS;
    static constexpr int N = PHI + 1;
    static constexpr int G = FP;                // face flux, reuses the split slots (5 + NS)
    static constexpr int SPP = 10, SPM = 10 + NS;  // F+ / F- of species 0
    static constexpr int D = TR + 2, T = Q4 + 3;
};

// Slots of the species sweep (PART 2): only what the species fluxes and the enthalpy
// diffusion term of the energy flux read.  MIXD (law 2): D holds D_0 and DK the other species'
// D_1 .. D_{NS-1}.
template <int NS, bool MIXD = false>
struct SpSlots {
    static constexpr int FP = 0;                // F+ sp (NS), F- sp (NS)
    static constexpr int SPP = 0, SPM = NS;
    static constexpr int MET = 2 * NS;          // 9 metrics + J
    static constexpr int D = MET + 10;
    static constexpr int RHO = D + 1;
    static constexpr int T = RHO + 1;
    static constexpr int PHI = T + 1;
    static constexpr int Y = PHI + 1;           // NS
    static constexpr int DY1 = Y + NS;          // NS
    static constexpr int DY2 = DY1 + NS;        // NS
    static constexpr int DK = DY2 + NS;         // NS - 1 (MIXD only)
    static constexpr int N = DK + (MIXD ? NS - 1 : 0);  // 5 NS + 14 (+ NS - 1)
    static constexpr int G = FP;                // NS species fluxes + the energy term
};

// PART 0: the whole face flux; PART 2: the species fluxes and the enthalpy-diffusion term of the
// energy flux only (the flow part then runs as the NS = 0 instance of the same sweep).
template <int NS, int PART, bool MIXD = false, bool REUSE = false>
using SlotsOf = std::conditional_t<PART == 2, SpSlots<NS, MIXD>, Slots<NS, REUSE>>;

template <int NS, typename CT, int WPB>
constexpr size_t smem_bytes() {
    return sizeof(CT) * Slots<NS>::N * 32 * WPB;
}

// Asks L2 for the line holding p ahead of its use (no register is held meanwhile).
__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

template <typename CT, typename T>
__device__ __forceinline__ CT ldg(const T *p, int i) {
    return CT(__ldg(p + i));
}

// ----------------------------------------------------------------------------------- prep
template <int NS, typename QT, int PTS = 256>
__device__ __forceinline__ void prep_block(const Args<QT> &A, int bid) {
    const int c = bid * PTS + threadIdx.x;
    if (c >= A.np) return;
    const int gx = c % A.tx, gy = (c / A.tx) % A.ty, gz = c / A.sz;
    const QT *P = A.Qi + 4 * A.np;
    // the inputs of Y before any store (a later load could not pass a store it may alias)
    const double rinv = 1 / jmax(double(A.Qi[c]), kEps);
    double ri[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) ri[n] = A.ri[c + n * A.np];
    double phi = 0;
    if (gx > 0 && gx < A.tx - 1 && gy > 0 && gy < A.ty - 1 && gz > 0 && gz < A.tz - 1) {
        // schemes.jl:10-22 in the arithmetic type of Q with exact divisions, so the branch
        // thresholds see the same ϕ as the reference
        using CT = QT;
        const CT P2 = P[c];
        CT a1 = P[c - 1], a3 = P[c + 1];
        const CT phx = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
        a1 = P[c - A.sy], a3 = P[c + A.sy];
        const CT phy = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
        a1 = P[c - A.sz], a3 = P[c + A.sz];
        const CT phz = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
        phi = phx + phy + phz;
    }
    A.aux[c] = QT(phi);
#pragma unroll
    for (int n = 0; n < NS; ++n) A.aux[c + (1 + n) * A.np] = QT(jmax(ri[n] * rinv, 0.0));
}

template <int NS, typename QT>
__global__ void __launch_bounds__(256) k_prep(const __grid_constant__ Args<QT> A) {
    prep_block<NS, QT>(A, blockIdx.x);
}

// ----------------------------------------------------------------------------------- sweep
template <int DIR>
struct Dir {
    static constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
};

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

// ---- phase A: everything the faces of a pencil need from one point, into the point's
// column of shared memory (slot stride 32).  l is the point's position along the pencil.
template <int DIR, int NS, typename QT, typename CT, bool REUSE = false>
__device__ __forceinline__ void point_phase(const Args<QT> &A, CT *S, int l, int g) {
    using SL = Slots<NS, REUSE>;
    constexpr int D1 = Dir<DIR>::D1, D2 = Dir<DIR>::D2;
    const int np = A.np;
    const int s1 = D1 == 0 ? 1 : (D1 == 1 ? A.sy : A.sz);
    const int s2 = D2 == 0 ? 1 : (D2 == 1 ? A.sy : A.sz);
    const QT *Q = A.Qi;
    const CT h = CT(0.5), c23 = CT(2.0 / 3.0), c12 = CT(1.0 / 12.0);
#define SV(slot) S[(slot) * 32 + l]
    const CT rho = CT(Q[g]), u = CT(Q[g + np]), v = CT(Q[g + 2 * np]), w = CT(Q[g + 3 * np]),
             p = CT(Q[g + 4 * np]), T = CT(Q[g + 5 * np]), ei = CT(Q[g + 6 * np]);
    CT mv[10];
    if (A.metq) {  // once-rounded copy: the same values without a conversion per load
#pragma unroll
        for (int m = 0; m < 10; ++m) mv[m] = CT(__ldg(A.metq + m * np + g));
    } else {
#pragma unroll
        for (int m = 0; m < 10; ++m) mv[m] = ldg<CT>(A.met[m], g);
    }
    const CT A1 = mv[3 * DIR], A2 = mv[3 * DIR + 1], A3 = mv[3 * DIR + 2];
    // Steger-Warming split, split.jl:17-89 (divisions folded into reciprocals)
    {
        const CT gam = p * (CT(1) / ei) + 1;
        const CT gm1 = gam - 1;
        const CT inv = CT(1) / (rho * gam * gm1);
        const CT cs = sqrt(gam * p * (gam * gm1 * inv));
        const CT r2 = A1 * A1 + A2 * A2 + A3 * A3;
        const CT rs = rsqrt(r2);
        const CT ss = r2 * rs;
        const CT E1 = A1 * u + A2 * v + A3 * w;
        const CT E2 = E1 - cs * ss, E3 = E1 + cs * ss;
        const CT B1 = A1 * rs, B2 = A2 * rs, B3 = A3 * rs;
        const CT E1P = (E1 + fabs(E1)) * h, E2P = (E2 + fabs(E2)) * h, E3P = (E3 + fabs(E3)) * h;
        const CT E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
        const CT uc1 = u - cs * B1, uc2 = u + cs * B1;
        const CT vc1 = v - cs * B2, vc2 = v + cs * B2;
        const CT wc1 = w - cs * B3, wc2 = w + cs * B3;
        const CT vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * h;
        const CT vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * h;
        const CT vv = gm1 * (u * u + v * v + w * w);
        const CT W2 = (3 - gam) * (h * rho * gam * inv) * (cs * cs);
        const CT tmp1 = h * rho * (rho * gm1 * inv);
        const CT tmp2 = 2 * gm1;
        SV(0) = tmp1 * (tmp2 * E1P + E2P + E3P);
        SV(1) = tmp1 * (tmp2 * E1P * u + E2P * uc1 + E3P * uc2);
        SV(2) = tmp1 * (tmp2 * E1P * v + E2P * vc1 + E3P * vc2);
        SV(3) = tmp1 * (tmp2 * E1P * w + E2P * wc1 + E3P * wc2);
        SV(4) = tmp1 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
        SV(5) = tmp1 * (tmp2 * E1M + E2M + E3M);
        SV(6) = tmp1 * (tmp2 * E1M * u + E2M * uc1 + E3M * uc2);
        SV(7) = tmp1 * (tmp2 * E1M * v + E2M * vc1 + E3M * vc2);
        SV(8) = tmp1 * (tmp2 * E1M * w + E2M * wc1 + E3M * wc2);
        SV(9) = tmp1 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
        // species, split.jl:101-130
        const CT Ep = h * (E1 + fabs(E1)), Em = h * (E1 - fabs(E1));
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            const CT r = CT(A.ri[g + n * np]);
            SV(10 + n) = Ep * r;
            SV(10 + NS + n) = Em * r;
        }
    }
    SV(SL::Q4 + 0) = u, SV(SL::Q4 + 1) = v, SV(SL::Q4 + 2) = w, SV(SL::Q4 + 3) = T;
    if constexpr (!REUSE) {  // REUSE: staged later, into the split slots (stage_metrics)
#pragma unroll
        for (int m = 0; m < 10; ++m) SV(SL::MET + m) = mv[m];
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) SV(SL::TR + m) = CT(A.Ti[g + m * np]);
    SV(SL::RHO) = rho;
    SV(SL::PHI) = CT(A.aux[g]);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        const QT *Y = A.aux + (1 + n) * np;
        SV(SL::Y + n) = CT(Y[g]);
        SV(SL::DY1 + n) = CT(Y[g + s1]) - CT(Y[g - s1]);
        SV(SL::DY2 + n) = CT(Y[g + s2]) - CT(Y[g - s2]);
    }
    // cell-centred 4th-order tangential derivatives of u, v, w, T; the face value the reference
    // forms (viscous.jl:36-53) is the mean of the two cells' values
    const int qv[4] = {1, 2, 3, 5};
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const QT *q = Q + qv[m] * np + g;
        SV(SL::DQ1 + m) = c23 * (CT(q[s1]) - CT(q[-s1])) - c12 * (CT(q[2 * s1]) - CT(q[-2 * s1]));
        SV(SL::DQ2 + m) = c23 * (CT(q[s2]) - CT(q[-s2])) - c12 * (CT(q[2 * s2]) - CT(q[-2 * s2]));
    }
#undef SV
}

// ---- phase B: the face between pencil positions l-1 and l; G = F_inviscid − F_viscous.
// The species part runs one species at a time in two passes (the sums of the diffusion
// velocities first, then each species' reconstruction, corrected diffusion flux and enthalpy
// flux), recomputing the few gradient terms instead of holding per-species arrays in registers.
// MIXD (the mixture-averaged law, law 2): each species has its own D_k; Dk points at D_0 of
// point l in the transport fields (field 2 + n holds D_n) and dstep is the pencil's stride, so
// point l - 1 is Dk - dstep.  The other laws use the one D of the shared-memory slots and
// compile without the per-species loads.
// MODE 0: the whole face.  With the REUSE slots the face runs in two calls, between which the
// metrics overwrite the split fluxes: MODE 1 reconstructs every flux into G, MODE 2 subtracts
// the viscous and diffusion fluxes from it (the same operations in the same order as MODE 0).
template <int DIR, int NS, typename QT, typename CT, int PART = 0, bool MIXD = false,
          int MODE = 0, bool REUSE = false>
__device__ __forceinline__ void face_phase(const Args<QT> &A, const CT *S, int l, CT *G,
                                           const QT *Dk, int dstep) {
    using SL = SlotsOf<NS, PART, MIXD, REUSE>;
    constexpr int GS = PART == 2 ? 0 : 5;  // G index of species 0
    constexpr int D1 = Dir<DIR>::D1, D2 = Dir<DIR>::D2;
    const CT h = CT(0.5), c23 = CT(2.0 / 3.0), c12 = CT(1.0 / 12.0);
#define SV(slot, ll) S[(slot) * 32 + (ll)]
    const int lm = l - 1;
    const CT phif = CT(jmax(double(SV(SL::PHI, lm)), double(SV(SL::PHI, l))));
    auto recon = [&](int vp, int vm) {
        CT pv[7], mv[7];
#pragma unroll
        for (int i = 0; i < 6; ++i) pv[i] = SV(vp, l - 3 + i), mv[i] = SV(vm, l - 3 + i);
        pv[6] = mv[6] = CT(0);
        return hybrid_face_fast<CT>(pv, mv, phif);
    };
    if constexpr (PART != 2 && MODE != 2) {
#pragma unroll
        for (int n = 0; n < 5; ++n) G[n] = recon(n, 5 + n);
    }
    if constexpr (MODE == 1) {
#pragma unroll
        for (int n = 0; n < NS; ++n) G[GS + n] = recon(SL::SPP + n, SL::SPM + n);
        return;
    }
    CT met[9];
#pragma unroll
    for (int m = 0; m < 9; ++m) met[m] = (SV(SL::MET + m, lm) + SV(SL::MET + m, l)) * h;
    const CT Jac = (SV(SL::MET + 9, lm) + SV(SL::MET + 9, l)) * h;
    const CT DL = SV(SL::D, lm), DR = SV(SL::D, l);
    const CT rho = (SV(SL::RHO, lm) + SV(SL::RHO, l)) * h;
    const CT Tf = (SV(SL::T, lm) + SV(SL::T, l)) * h;
    const CT *md = met + 3 * DIR;
    // species diffusion (viscous.jl:430-507): the diffusion velocity of species n at the face
    const CT rhoD1 = (DL + DR) * rho;  // viscous.jl:473 (no 1/2, as the reference)
    auto diffusion = [&](int n, CT &Vx, CT &Vy, CT &Vz) {
        CT rhoDi = rhoD1;
        if constexpr (MIXD && PART == 2) {  // staged with the species slots
            constexpr int dk = SpSlots<NS, true>::DK;
            if (n > 0) rhoDi = (SV(dk + n - 1, lm) + SV(dk + n - 1, l)) * rho;
        } else if constexpr (MIXD) {  // the x sweep: coalesced loads
            const QT *dn = Dk + (size_t)n * A.np;
            rhoDi = (CT(dn[-dstep]) + CT(dn[0])) * rho;
        }
        const CT y0 = SV(SL::Y + n, l), ym = SV(SL::Y + n, lm);
        const CT yp = SV(SL::Y + n, l + 1), ymm = SV(SL::Y + n, l - 2);
        CT dY[3];
        dY[DIR] = CT(1.25) * (y0 - ym) - c12 * (yp - ymm);
        dY[D1] = CT(0.25) * (SV(SL::DY1 + n, l) + SV(SL::DY1 + n, lm));
        dY[D2] = CT(0.25) * (SV(SL::DY2 + n, l) + SV(SL::DY2 + n, lm));
        Vx = (dY[0] * met[0] + dY[1] * met[3] + dY[2] * met[6]) * Jac * rhoDi;
        Vy = (dY[0] * met[1] + dY[1] * met[4] + dY[2] * met[7]) * Jac * rhoDi;
        Vz = (dY[0] * met[2] + dY[1] * met[5] + dY[2] * met[8]) * Jac * rhoDi;
        return h * (ym + y0);
    };
    CT sum1 = 0, sum2 = 0, sum3 = 0;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        CT Vx, Vy, Vz;
        diffusion(n, Vx, Vy, Vz);
        sum1 += Vx, sum2 += Vy, sum3 += Vz;
    }
    CT fh1 = 0, fh2 = 0, fh3 = 0;
    {
        const double Td = double(Tf);
        const double T2 = 0.5 * Td * Td, T3 = 2.0 / 3.0 * T2 * Td, T4 = T2 * T2, T5 = 0.8 * T4 * Td;
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            CT Vx, Vy, Vz;
            const CT Yf = diffusion(n, Vx, Vy, Vz);
            const CT hn = CT(h_spec(A.th, n, Td, T2, T3, T4, T5));
            const CT V1 = Vx - sum1 * Yf, V2 = Vy - sum2 * Yf, V3 = Vz - sum3 * Yf;
            const CT gi = MODE == 2 ? G[GS + n] : recon(SL::SPP + n, SL::SPM + n);
            G[GS + n] = gi - (V1 * md[0] + V2 * md[1] + V3 * md[2]);
            fh1 += V1 * hn, fh2 += V2 * hn, fh3 += V3 * hn;
        }
    }
    if constexpr (PART == 2) {  // the energy flux's enthalpy-diffusion term, viscous.jl:120-141
        G[NS] = -(md[0] * fh1 + md[1] * fh2 + md[2] * fh3);
    } else {
    const CT mui = (SV(SL::TR, lm) + SV(SL::TR, l)) * h;
    const CT lami = (SV(SL::TR + 1, lm) + SV(SL::TR + 1, l)) * h;
    // momentum and energy, viscous.jl:14-141
    CT gr[4][3];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        CT dq[3];
        dq[DIR] = CT(1.25) * (SV(SL::Q4 + m, l) - SV(SL::Q4 + m, lm)) -
                  c12 * (SV(SL::Q4 + m, l + 1) - SV(SL::Q4 + m, l - 2));
        dq[D1] = h * (SV(SL::DQ1 + m, l) + SV(SL::DQ1 + m, lm));
        dq[D2] = h * (SV(SL::DQ2 + m, l) + SV(SL::DQ2 + m, lm));
#pragma unroll
        for (int x = 0; x < 3; ++x)
            gr[m][x] = (dq[0] * met[x] + dq[1] * met[3 + x] + dq[2] * met[6 + x]) * Jac;
    }
    const CT u = (SV(SL::Q4 + 0, lm) + SV(SL::Q4 + 0, l)) * h;
    const CT v = (SV(SL::Q4 + 1, lm) + SV(SL::Q4 + 1, l)) * h;
    const CT w = (SV(SL::Q4 + 2, lm) + SV(SL::Q4 + 2, l)) * h;
#undef SV
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
}

// ---- phase A of the species sweep: the species slots of one point.
template <int DIR, int NS, typename QT, typename CT, bool MIXD = false>
__device__ __forceinline__ void species_point_phase(const Args<QT> &A, CT *S, int l, int g) {
    using SL = SpSlots<NS, MIXD>;
    constexpr int D1 = Dir<DIR>::D1, D2 = Dir<DIR>::D2;
    const int np = A.np;
    const int s1 = D1 == 0 ? 1 : (D1 == 1 ? A.sy : A.sz);
    const int s2 = D2 == 0 ? 1 : (D2 == 1 ? A.sy : A.sz);
    const QT *Q = A.Qi;
    const CT h = CT(0.5);
#define SV(slot) S[(slot) * 32 + l]
    const CT rho = CT(Q[g]), u = CT(Q[g + np]), v = CT(Q[g + 2 * np]), w = CT(Q[g + 3 * np]);
    CT mv[10];
    if (A.metq) {
#pragma unroll
        for (int m = 0; m < 10; ++m) mv[m] = CT(__ldg(A.metq + m * np + g));
    } else {
#pragma unroll
        for (int m = 0; m < 10; ++m) mv[m] = ldg<CT>(A.met[m], g);
    }
    // species split, split.jl:101-130 (the contravariant velocity as in point_phase)
    const CT E1 = mv[3 * DIR] * u + mv[3 * DIR + 1] * v + mv[3 * DIR + 2] * w;
    const CT Ep = h * (E1 + fabs(E1)), Em = h * (E1 - fabs(E1));
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        const CT r = CT(A.ri[g + n * np]);
        SV(SL::SPP + n) = Ep * r;
        SV(SL::SPM + n) = Em * r;
    }
#pragma unroll
    for (int m = 0; m < 10; ++m) SV(SL::MET + m) = mv[m];
    SV(SL::D) = CT(A.Ti[g + 2 * np]);
    if constexpr (MIXD) {
#pragma unroll
        for (int n = 1; n < NS; ++n) SV(SL::DK + n - 1) = CT(A.Ti[g + (2 + n) * np]);
    }
    SV(SL::RHO) = rho;
    SV(SL::T) = CT(Q[g + 5 * np]);
    SV(SL::PHI) = CT(A.aux[g]);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        const QT *Y = A.aux + (1 + n) * np;
        SV(SL::Y + n) = CT(Y[g]);
        SV(SL::DY1 + n) = CT(Y[g + s1]) - CT(Y[g - s1]);
        SV(SL::DY2 + n) = CT(Y[g + s2]) - CT(Y[g - s2]);
    }
#undef SV
}

// ---- last sweep: div, RK3 combination, c2Prim, transport, ghost images of one cell.
// LAW2: the mixture-averaged transport, written as μ, λ, D_0 .. D_{NS-1}.
// mt: the block's MixTables (LAW2 only).
template <int NS, typename QT, bool LAW2 = false>
__device__ __forceinline__ void finish_cell(const Args<QT> &A, int g, int gx, int gy, int gz,
                                            const double *rhs,
                                            const MixTables<NS, QT> *mt = nullptr) {
    const int np = A.np;
    const double Jact = A.met[9][g] * A.dt;
    // every input first: the stores below could alias them as far as the compiler knows, so
    // loads placed after a store would each wait for the one before
    double u0[5], r0[NS], un0[5], rn0[NS];
#pragma unroll
    for (int n = 0; n < 5; ++n) u0[n] = A.U[g + n * np];
#pragma unroll
    for (int n = 0; n < NS; ++n) r0[n] = A.ri[g + n * np];
    if (A.stage > 1) {
#pragma unroll
        for (int n = 0; n < 5; ++n) un0[n] = A.Un[g + n * np];
#pragma unroll
        for (int n = 0; n < NS; ++n) rn0[n] = A.rn[g + n * np];
    }
    // the RK3 update, utils.jl:95-112 (the multiply-adds spelled out, so that every kernel
    // that inlines this rounds them alike)
    double Uc[5], r[NS];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
        if (A.stage == 1) A.Un[g + n * np] = u0[n];
        double un = fma(rhs[n], Jact, u0[n]);
        if (A.stage > 1) un = fma(un, A.ca, un0[n] * A.cb);
        Uc[n] = un;
        A.U[g + n * np] = un;
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        if (A.stage == 1) A.rn[g + n * np] = r0[n];
        double rv = fma(rhs[5 + n], Jact, r0[n]);
        if (A.stage > 1) rv = fma(rv, A.ca, rn0[n] * A.cb);
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
    double mu, lam, D, Tn, p;
    double Dk[LAW2 ? NS : 1];
    if constexpr (NS < 4) {  // few species: the per-species sums are as cheap
        Tn = jmax(get_T<NS>(A.th, NS, ei, r), kEps);
        p = jmax(p_mixture<NS>(A.th, NS, Tn, r), kEps);
        if constexpr (!LAW2) transport_point<NS>(A.th, A.tr, Tn, rho, r, mu, lam, D);
    } else {  // the mixture's own polynomials (MixPoly): one evaluation per Newton iteration
        const MixPoly<NS> M(A.th, r);
        Tn = jmax(get_T_mix<NS>(M, A.th, ei, r), kEps);
        p = jmax(p_mixture<NS>(A.th, NS, Tn, r), kEps);
        if constexpr (!LAW2) {
            if (A.tr.law == 0) {
                mu = A.tr.mu_ref, lam = A.tr.lambda_ref, D = A.tr.D_ref;
            } else {  // transport_point with cp_mix = Σ_n w_n cp_n / ρ from the same polynomials
                const double rh = jmax(rho, kEps);
                const double cpm = (M.cv(Tn) + A.th.Ru * M.wsum) / rh;
                mu = A.tr.mu_ref * pow(Tn / A.tr.T_ref, A.tr.exponent);
                lam = cpm * mu / A.tr.Pr;
                D = lam / (rh * cpm);
            }
        }
    }
    if constexpr (LAW2) {  // the next stage's mixture kernel (thermo.jl:371-403), per cell
        mixture_point<NS, QT>(A.th, A.tr, *mt, Tn, p, rho, r, mu, lam, Dk);
        D = Dk[0];
    }
    const double qv[7] = {rho, u, v, w, p, Tn, ei};
    const double tv[3] = {mu, lam, D};
    // the cell and its ghost images along the periodic axes (new: the reference fills ghosts
    // with case-specific kernels, boundary.jl:1-191, which the caller runs after the stage for
    // the other axes)
    const int ng = A.ng;
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
            for (int aa = 0; aa < nxo; ++aa) {
                const int t = (gx + ox[aa]) + A.sy * (gy + oy[b]) + A.sz * (gz + oz[c]);
#pragma unroll
                for (int n = 0; n < 7; ++n) A.Qo[t + n * np] = QT(qv[n]);
#pragma unroll
                for (int n = 0; n < 3; ++n) A.To[t + n * np] = QT(tv[n]);
                if constexpr (LAW2) {
#pragma unroll
                    for (int n = 1; n < NS; ++n) A.To[t + (2 + n) * np] = QT(Dk[n]);
                }
#pragma unroll
                for (int n = 0; n < NS; ++n) A.ro[t + n * np] = r[n];
            }
}

// x sweep (lanes along x, every access coalesced); it is the last sweep.  FIN: it finishes the
// stage itself (configuration 3); otherwise it adds its differences to R and k_finish follows
// (configuration 4: the FP64 finish then runs at full occupancy, apart from the sweep's
// registers and shared memory).  Both form (R + R2) + rhs the same way, so they agree bit for
// bit.
template <int NS, typename QT, typename CT, bool FIN = true, bool MIXD = false,
          int WPB = Wpb<0>::value>
__device__ __forceinline__ void x_block(const Args<QT> &A, int bid, unsigned char *smem_raw) {
    using SL = Slots<NS>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    CT *S = reinterpret_cast<CT *>(smem_raw) + warp * SL::N * 32;
    const int nseg = (A.nx + OWN - 1) / OWN;
    const int gw = bid * WPB + warp;
    const int seg = gw % nseg;
    const int y = (gw / nseg) % A.ny, z = (gw / nseg) / A.ny;
    if (z >= A.nz) return;
    const int a = seg * OWN - 3 + lane;
    const int gx = clampi(a + A.ng, 0, A.nx + 2 * A.ng - 1), gy = y + A.ng, gz = z + A.ng;
    const int g = gx + A.sy * gy + A.sz * gz;
    if (lane >= 3 && lane < 3 + OWN && a < A.nx) {  // what the end of this sweep reads
#pragma unroll
        for (int n = 0; n < 5 + NS; ++n) {
            prefetch_l2(A.R + g + n * A.np);
            prefetch_l2(A.R2 + g + n * A.np);
        }
        if constexpr (FIN) {
#pragma unroll
            for (int n = 0; n < 5; ++n) {
                prefetch_l2(A.U + g + n * A.np);
                if (A.stage > 1) prefetch_l2(A.Un + g + n * A.np);
            }
#pragma unroll
            for (int n = 0; n < NS; ++n) {
                prefetch_l2(A.ri + g + n * A.np);
                if (A.stage > 1) prefetch_l2(A.rn + g + n * A.np);
            }
        }
    }
    point_phase<0, NS, QT, CT>(A, S, lane, g);
    __syncwarp();
    CT G[5 + NS];
    const bool face = lane >= 3 && lane <= 3 + OWN && a <= A.nx;
    if (face) face_phase<0, NS, QT, CT, 0, MIXD>(A, S, lane, G, A.Ti + 2 * A.np + g, 1);
    __syncwarp();
    if (face) {
#pragma unroll
        for (int n = 0; n < 5 + NS; ++n) S[(SL::G + n) * 32 + lane] = G[n];
    }
    __syncwarp();
    if (lane < 3 || lane >= 3 + OWN || a >= A.nx) return;
    double rhs[5 + NS];  // the complete right-hand side: (z + y) + x, one rounding per sum
#pragma unroll
    for (int n = 0; n < 5 + NS; ++n)
        rhs[n] = (A.R[g + n * A.np] + A.R2[g + n * A.np]) +
                 (double(S[(SL::G + n) * 32 + lane]) - double(S[(SL::G + n) * 32 + lane + 1]));
    if constexpr (FIN) {
        finish_cell<NS, QT>(A, g, gx, gy, gz, rhs);
    } else {
#pragma unroll
        for (int n = 0; n < 5 + NS; ++n) A.R[g + n * A.np] = rhs[n];
    }
}

template <int NS, typename QT, typename CT, bool FIN, bool MIXD = false>
__global__ void __launch_bounds__(Wpb<0>::value * 32) k_pencil_x(const __grid_constant__ Args<QT> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    x_block<NS, QT, CT, FIN, MIXD>(A, blockIdx.x, smem_raw);
}

// The stage's finish for configuration 4: one thread per interior cell, x fastest, with the
// complete right-hand side already in R (the x sweep summed it).
template <int NS, typename QT, bool LAW2>
__device__ __forceinline__ void finish_thread(const Args<QT> &A, const MixTables<NS, QT> *mt,
                                              int block) {
    const int c = block * 128 + threadIdx.x;
    if (c >= A.nx * A.ny * A.nz) return;
    const int x = c % A.nx, y = (c / A.nx) % A.ny, z = c / (A.nx * A.ny);
    const int gx = x + A.ng, gy = y + A.ng, gz = z + A.ng;
    const int g = gx + A.sy * gy + A.sz * gz;
    double rhs[5 + NS];
#pragma unroll
    for (int n = 0; n < 5 + NS; ++n) rhs[n] = A.R[g + n * A.np];
    finish_cell<NS, QT, LAW2>(A, g, gx, gy, gz, rhs, mt);
}

template <int NS, typename QT>
__global__ void __launch_bounds__(128) k_finish(const __grid_constant__ Args<QT> A) {
    finish_thread<NS, QT, false>(A, nullptr, blockIdx.x);
}

// The finish with the mixture-averaged law (law 2).  Its mixture rule needs up to 166 registers
// at nine species (three blocks per SM); capped at 128 (four blocks, at most 72 bytes of spill)
// it runs faster.  A separate kernel, so that the bound does not touch the other laws' finish.
template <int NS, typename QT>
__global__ void __launch_bounds__(128, 4) k_finish_mix(const __grid_constant__ Args<QT> A) {
    __shared__ MixTables<NS, QT> mt;
    mix_tables_fill<NS, QT>(A.th, A.tr, mt);
    __syncthreads();
    finish_thread<NS, QT, true>(A, &mt, blockIdx.x);
}

// Columns per block of the staged y / z sweeps.  Single precision: 16 consecutive x columns, so
// the block's loads use whole 128-byte lines; 8 when the column slots would not fit in shared
// memory.  (Sizing for two blocks per SM instead, 16/8/4 columns under 112 KB, measured 0-2 %
// faster with few species and 6 % slower with nine.)  FP64 sweeps that carry species: always 8
// columns.  With one or two species a 16-column FP64 block holds 172-199 KB, one block per SM,
// and its warps wait at the phase barriers with nothing else to run; two 8-column blocks keep
// the same warp count and one block's loads overlap the other's arithmetic (2-3 % faster on the
// 256x128x128 jet, neutral with two species); from three species on 16 columns would not fit
// anyway.  The flow-only sweep of configurations 5 and 6 (ns = 0) keeps 16 columns: 8 measured
// 8 % slower there.  Host and device use this rule: the batch planner sizes its work list with
// it.
constexpr int slots_of(int ns) { return 37 + 5 * ns; }
constexpr int staged_cols(int ns, size_t csz) {
    return (csz == 8 && ns > 0) ? 8 : (csz * slots_of(ns) * 33 * 16 <= 200 * 1024 ? 16 : 8);
}

template <int NS, typename CT, int PART = 0, bool MIXD = false>
struct Staged {
    static_assert(Slots<NS>::N == slots_of(NS), "slots_of must follow Slots");
    // FP64 sweeps with one or two species stage the metrics into the split slots once the
    // reconstruction is done: ten slots fewer per point let three blocks share an SM (more
    // species would not fit three blocks anyway)
    static constexpr bool REUSE = sizeof(CT) == 8 && PART == 0 && NS >= 1 && NS <= 2;
    static constexpr int NSLOT = SlotsOf<NS, PART, MIXD, REUSE>::N;
    static constexpr int STRIDE = NSLOT * 32 + 1;  // padded column region (bank spread)
    // (the species sweep in 8-column blocks capped at three per SM measured 7-12 % slower in
    // mixed precision: the register cap spills)
    static constexpr int COLS =
        PART == 2 ? (sizeof(CT) * NSLOT * 33 * 16 <= 200 * 1024 ? 16 : 8)
                  : staged_cols(NS, sizeof(CT));
    static constexpr size_t SMEM = sizeof(CT) * STRIDE * COLS;
    // three 8-column FP64 blocks per SM when their shared memory fits (228 KB per SM, 1 KB
    // reserved per block): at most 80 registers; otherwise no bound
    static constexpr int MINB =
        (sizeof(CT) == 8 && COLS == 8 && 3 * (SMEM + 1024) <= 228 * 1024) ? 3 : 1;
};

// y or z sweep (DIR 1, 2).  The block stages the points of COLS neighbouring pencils with
// x-fastest threads (coalesced loads), then each warp works its own pencil from shared memory
// exactly like the x sweep, and the right-hand side goes back with x-fastest threads.
// PASS 0 writes R, PASS 1 adds to it.
template <int DIR, int PASS, int NS, typename QT, typename CT, int PART = 0, bool MIXD = false>
__device__ __forceinline__ void staged_block(const Args<QT> &A, int block, unsigned char *smem_raw) {
    constexpr int COLS = Staged<NS, CT, PART, MIXD>::COLS;
    constexpr int STRIDE = Staged<NS, CT, PART, MIXD>::STRIDE;
    constexpr bool REUSE = Staged<NS, CT, PART, MIXD>::REUSE;
    using SL = SlotsOf<NS, PART, MIXD, REUSE>;
    constexpr int NG_OUT = PART == 2 ? NS + 1 : 5 + NS;  // face values a lane produces
    CT *base = reinterpret_cast<CT *>(smem_raw);
    const int n_along = DIR == 1 ? A.ny : A.nz;
    const int n_c2 = DIR == 1 ? A.nz : A.ny;
    const int nseg = (n_along + OWN - 1) / OWN;
    const int nxb = (A.nx + COLS - 1) / COLS;
    int bid = block;
    const int xb = bid % nxb;
    bid /= nxb;
    const int seg = bid % nseg, c2 = bid / nseg;
    if (c2 >= n_c2) return;
    const int tid = threadIdx.x;
    if constexpr (PASS == 1 && PART == 2) {  // the energy field this thread adds to in phase C
        const int cx = tid % COLS, l = tid / COLS;
        const int x = xb * COLS + cx, ac = seg * OWN - 3 + l;
        if (l >= 3 && l < 3 + OWN && ac < n_along && x < A.nx) {
            const int gy = DIR == 1 ? ac + A.ng : c2 + A.ng;
            const int gz = DIR == 1 ? c2 + A.ng : ac + A.ng;
            prefetch_l2(A.R2 + (x + A.ng) + A.sy * gy + A.sz * gz + 4 * A.np);
        }
    }
    // ---- phase A, x-fastest: thread -> (column cx, pencil position l)
    int gA;  // the thread's phase-A point
    {
        const int cx = tid % COLS, l = tid / COLS;
        const int x = clampi(xb * COLS + cx, 0, A.nx - 1);
        const int a = seg * OWN - 3 + l;
        const int ga = clampi(a + A.ng, 0, n_along + 2 * A.ng - 1);
        const int gx = x + A.ng;
        const int gy = DIR == 1 ? ga : c2 + A.ng;
        const int gz = DIR == 1 ? c2 + A.ng : ga;
        gA = gx + A.sy * gy + A.sz * gz;
        if constexpr (PART == 2)
            species_point_phase<DIR, NS, QT, CT, MIXD>(A, base + cx * STRIDE, l, gA);
        else
            point_phase<DIR, NS, QT, CT, REUSE>(A, base + cx * STRIDE, l, gA);
    }
    __syncthreads();
    // ---- phase B, one warp per pencil (column)
    const int warp = tid >> 5, lane = tid & 31;
    CT *S = base + warp * STRIDE;
    const int a = seg * OWN - 3 + lane;
    CT G[NG_OUT];
    const bool face = lane >= 3 && lane <= 3 + OWN && a <= n_along;
    // the lane's point in the transport fields (per-species D_k of law 2)
    const int gxw = clampi(xb * COLS + warp, 0, A.nx - 1) + A.ng, gaw = a + A.ng;
    const int gl = gxw + (DIR == 1 ? A.sy * gaw + A.sz * (c2 + A.ng)
                                   : A.sy * (c2 + A.ng) + A.sz * gaw);
    if constexpr (REUSE) {
        // the reconstruction, then every warp is done with the split fluxes: the x-fastest
        // threads stage their point's metrics into those slots (coalesced loads), and the faces
        // take their viscous fluxes
        if (face)
            face_phase<DIR, NS, QT, CT, PART, MIXD, 1, true>(A, S, lane, G, A.Ti + 2 * A.np + gl,
                                                             DIR == 1 ? A.sy : A.sz);
        __syncthreads();
        {
            const int cx = tid % COLS, l = tid / COLS;
            CT *Sc = base + cx * STRIDE;
#pragma unroll
            for (int m = 0; m < 10; ++m)
                Sc[(SL::MET + m) * 32 + l] =
                    A.metq ? CT(__ldg(A.metq + m * A.np + gA)) : ldg<CT>(A.met[m], gA);
        }
        __syncthreads();
        if (face)
            face_phase<DIR, NS, QT, CT, PART, MIXD, 2, true>(A, S, lane, G, A.Ti + 2 * A.np + gl,
                                                             DIR == 1 ? A.sy : A.sz);
    } else if (face) {
        face_phase<DIR, NS, QT, CT, PART, MIXD>(A, S, lane, G, A.Ti + 2 * A.np + gl,
                                                DIR == 1 ? A.sy : A.sz);
    }
    __syncwarp();
    if (face) {
#pragma unroll
        for (int n = 0; n < NG_OUT; ++n) S[(SL::G + n) * 32 + lane] = G[n];
    }
    __syncthreads();
    // ---- phase C, x-fastest again: cell differences into R
    const int cx = tid % COLS, l = tid / COLS;
    const int x = xb * COLS + cx;
    const int ac = seg * OWN - 3 + l;
    if (l < 3 || l >= 3 + OWN || ac >= n_along || x >= A.nx) return;
    const int gy = DIR == 1 ? ac + A.ng : c2 + A.ng;
    const int gz = DIR == 1 ? c2 + A.ng : ac + A.ng;
    const int g = (x + A.ng) + A.sy * gy + A.sz * gz;
    const CT *Sc = base + cx * STRIDE;
#pragma unroll
    for (int n = 0; n < NG_OUT; ++n) {
        const double d = double(Sc[(SL::G + n) * 32 + l]) - double(Sc[(SL::G + n) * 32 + l + 1]);
        // the z sweep (PASS 0) writes R, the y sweep (PASS 1) R2; PART 2: G[n] is species n
        // (field 5 + n) and G[NS] the energy term, added to field 4, which the flow sweep of
        // the same direction wrote just before
        double *Rt = PASS == 0 ? A.R : A.R2;
        const int f = PART == 2 ? (n < NS ? 5 + n : 4) : n;
        if (PART == 2 && n == NS) Rt[g + f * A.np] += d;
        else Rt[g + f * A.np] = d;
    }
}

template <int DIR, int PASS, int NS, typename QT, typename CT, int PART = 0, bool MIXD = false>
__global__ void __launch_bounds__(Staged<NS, CT, PART, MIXD>::COLS * 32)
    k_pencil_staged(const __grid_constant__ Args<QT> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    staged_block<DIR, PASS, NS, QT, CT, PART, MIXD>(A, blockIdx.x, smem_raw);
}

// The same sweep held to the registers of three blocks per SM (Staged::MINB == 3).  A separate
// kernel: naming a minimum of one block per SM changes the compiler's register choices against
// leaving it out, so the other instances keep the plain bound above.
template <int DIR, int PASS, int NS, typename QT, typename CT, int PART = 0, bool MIXD = false>
__global__ void __launch_bounds__(Staged<NS, CT, PART, MIXD>::COLS * 32, 3)
    k_pencil_staged3(const __grid_constant__ Args<QT> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    staged_block<DIR, PASS, NS, QT, CT, PART, MIXD>(A, blockIdx.x, smem_raw);
}

// ---------------------------------------------------------------------- batched, persistent
// Persistent launches per chunk of cases (one species count and transport family) and stage,
// over a work list of (case, block) items in phase order.  Laws 0 and 1 (configuration 3's
// shape), two launches: k_batch_sweeps<V = 0> takes the prep, z-sweep and y-sweep blocks of all
// the chunk's cases, k_batch_x<false> the x-sweep blocks, which finish the stage.  Law 2
// (configuration 6's shape, per-species D_k), four: k_batch_sweeps<V = 1> the prep blocks and
// the flow-only (ns = 0) z and y sweeps, k_batch_sweeps<V = 2> the species z and y sweeps
// (which add the enthalpy-diffusion term to the flow sweeps' energy field), k_batch_x<true> the
// x sweeps without the finish, k_batch_finish the finishing blocks with the mixture rule.
// Each launch takes its items in list order from its own atomic counter, so an item only ever
// waits for items taken before it: a case's sweep item waits until the case's prep items are
// done (a counter in device memory; every wait bounded: on timeout the batch's error word is
// set, the item is skipped and every later wait gives up at once; flame_batch_status reports
// FLAME_ETIMEOUT).  Every other order is the stream's: each launch follows the one before, so
// each kernel keeps the registers of its own phases.  Cases never read each other's data, so a
// case's result does not depend on which other cases share the batch.
struct BatchItem {
    int c, b;  // case (index within the chunk), block within the case's phase
};

struct BatchLaunch {
    const BatchItem *items;  // work list
    const int4 *need;        // per case: prep items (x)
    int *next;               // this launch's item counter (zeroed before the chunk's launches)
    int *done;               // per case: completed prep items (zeroed before the launches)
    int *err;                // the batch's error word (FLAME_ETIMEOUT)
    int lo, hi;              // this launch's items: list positions [lo, hi)
    int p1, p2;              // sweep launches: first item of the second and of the third phase
    int stall;               // test hook: case 0 waits for one prep item more than exists
};

constexpr int kWaitSpins = 1 << 22;  // x 128 ns: about half a second per wait

// Spins (thread 0) until *count >= target; false if the batch already failed or the bound ran
// out (then the error word is set).
__device__ __forceinline__ bool wait_count(const int *count, int target, int *err) {
    for (int i = 0; i < kWaitSpins; ++i) {
        if (*(volatile const int *)err) return false;
        if (*(volatile const int *)count >= target) {
            __threadfence();  // acquire: the counted items' writes are visible from here on
            return true;
        }
        __nanosleep(128);
    }
    atomicExch(err, FLAME_ETIMEOUT);
    return false;
}

// The staged sweep of a sweeps launch: V 0 the whole sweep, V 1 the flow-only sweep (the ns = 0
// instance), V 2 the species sweep with per-species D_k.
template <int NS, typename CT, int V>
using SweepOf = Staged<V == 1 ? 0 : NS, CT, V == 2 ? 2 : 0, V == 2>;

template <int NS, typename QT, typename CT, int V = 0>
struct BatchShape {
    using ST = SweepOf<NS, CT, V>;
    static constexpr int COLS = ST::COLS;
    static constexpr int NT = ST::COLS * 32;  // threads of a sweep block (prep, z, y items)
    static constexpr int XW = Wpb<0>::value;  // pencils of an x item (its warps)
    static constexpr size_t SMEM = sizeof(CT) * ST::STRIDE * ST::COLS;
    static constexpr size_t SMEM_X = smem_bytes<NS, CT, XW>();
    // x blocks per SM, as the register bound: what the shared memory allows (228 KB, 1 KB
    // reserved per block), but at most what the stand-alone x sweep's own register count gives
    // at this species count and precision (its item loop and indexed descriptors cost the
    // persistent kernel registers: unbounded it takes more and fits fewer blocks, bounded
    // tighter it spills; measured on single cases and the 64-case ensemble)
    static constexpr int FIT_X = int((228 * 1024) / (SMEM_X + 1024));
    static constexpr int CAP_X = sizeof(CT) == 8 ? (NS <= 1 ? 5 : NS == 2 ? 4 : NS <= 5 ? 3 : 2)
                                                 : (NS <= 1 ? 7 : NS <= 3 ? 5 : NS <= 7 ? 4 : 3);
    static constexpr int MINB_X = FIT_X < 1 ? 1 : (FIT_X > CAP_X ? CAP_X : FIT_X);
};

constexpr int kPrepPerThread = 4;  // points each thread of a prep item handles

// The descriptors of the cases a launch advances, in constant memory: copied (device to device)
// before each launch, so the kernels read them through the constant cache as the stand-alone
// kernels read their parameters (a descriptor read from shared or global memory costs a load
// for every field, and from global memory the compiler must also assume that stores alias it).
// One table per device context: persistent batches on one device run one after the other.
constexpr int kConstCases = 20;
__constant__ __align__(16) unsigned char c_batch_args[kConstCases * sizeof(Args<double>)];
static_assert(sizeof(Args<double>) == sizeof(Args<float>), "one table for both precisions");

template <typename QT>
__device__ __forceinline__ const Args<QT> &batch_args(int c) {
    return reinterpret_cast<const Args<QT> *>(c_batch_args)[c];
}

// Sweep items (list positions [L.lo, L.hi)): prep items up to L.p1, then z-sweep items up to
// L.p2, then y-sweep items.  A sweep item first waits until its case's prep items are done (in
// the species launch, V 2, which has no prep items, the prep launch before it has done them
// all and the wait ends at its first look).  Thread 0 takes the next item from the counter
// while the block works on the current one.
template <int NS, typename QT, typename CT, int V>
__global__ void __launch_bounds__(BatchShape<NS, QT, CT, V>::NT)
    k_batch_sweeps(const __grid_constant__ BatchLaunch L) {
    using BS = BatchShape<NS, QT, CT, V>;
    constexpr int SN = V == 1 ? 0 : NS;               // the species the sweeps carry
    constexpr int PART = V == 2 ? 2 : 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item, s_next, s_ok;
    if (threadIdx.x == 0) s_next = L.lo + atomicAdd(L.next, 1);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = s_next;
        __syncthreads();
        const int item = s_item;
        if (item >= L.hi) return;
        const BatchItem it = L.items[item];
        const int ph = item < L.p1 ? 0 : item < L.p2 ? 1 : 2;
        if (threadIdx.x == 0) {
            s_next = L.lo + atomicAdd(L.next, 1);  // in flight while the item runs
            s_ok = ph == 0 || wait_count(L.done + 4 * it.c,
                                         L.need[it.c].x + (L.stall && it.c == 0), L.err);
        }
        __syncthreads();
        const Args<QT> &A = batch_args<QT>(it.c);
        if (s_ok) {
            if (ph == 0) {
                if constexpr (V != 2) {
#pragma unroll
                    for (int k = 0; k < kPrepPerThread; ++k)
                        prep_block<NS, QT, BS::NT>(A, it.b * kPrepPerThread + k);
                }
            } else if (ph == 1) {
                staged_block<2, 0, SN, QT, CT, PART, V == 2>(A, it.b, smem_raw);
            } else {
                staged_block<1, 1, SN, QT, CT, PART, V == 2>(A, it.b, smem_raw);
            }
        }
        __syncthreads();  // the item's writes are done and its shared memory is free
        if (threadIdx.x == 0 && ph == 0) {
            __threadfence();  // release: publish the prep block's writes before counting it
            atomicAdd(L.done + 4 * it.c, 1);
        }
    }
}

// x-sweep items (list positions [L.lo, L.hi)), launched after the sweeps on the same stream, so
// all of every case's z and y items are done.  MIX (law 2): the x sweep with per-species D_k,
// which leaves the finish to k_batch_finish; otherwise the x sweep finishes the stage.
template <int NS, typename QT, typename CT, bool MIX>
__global__ void __launch_bounds__(BatchShape<NS, QT, CT>::XW * 32, BatchShape<NS, QT, CT>::MINB_X)
    k_batch_x(const __grid_constant__ BatchLaunch L) {
    using BS = BatchShape<NS, QT, CT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item, s_next;
    if (threadIdx.x == 0) s_next = L.lo + atomicAdd(L.next, 1);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = s_next;
        __syncthreads();
        const int item = s_item;
        if (item >= L.hi) return;
        const BatchItem it = L.items[item];
        if (threadIdx.x == 0) s_next = L.lo + atomicAdd(L.next, 1);
        if (!*(volatile const int *)L.err)
            x_block<NS, QT, CT, !MIX, MIX, BS::XW>(batch_args<QT>(it.c), it.b, smem_raw);
    }
}

// Finishing items of law 2 (list positions [L.lo, L.hi)), after the x items: 128 cells each,
// with the mixture rule's tables of the item's case in shared memory (filled again when the
// block moves on to another case; items come in case order, so that is rare).
template <int NS, typename QT>
__global__ void __launch_bounds__(128, 4) k_batch_finish(const __grid_constant__ BatchLaunch L) {
    __shared__ MixTables<NS, QT> mt;
    __shared__ int s_item, s_next;
    int filled = -1;  // the case whose tables mt holds
    if (threadIdx.x == 0) s_next = L.lo + atomicAdd(L.next, 1);
    for (;;) {
        __syncthreads();  // also: every thread is done with mt before it is filled again
        if (threadIdx.x == 0) s_item = s_next;
        __syncthreads();
        const int item = s_item;
        if (item >= L.hi) return;
        const BatchItem it = L.items[item];
        if (threadIdx.x == 0) s_next = L.lo + atomicAdd(L.next, 1);
        const Args<QT> &A = batch_args<QT>(it.c);
        if (it.c != filled) {  // block-uniform
            mix_tables_fill<NS, QT>(A.th, A.tr, mt);
            __syncthreads();
            filled = it.c;
        }
        if (!*(volatile const int *)L.err) finish_thread<NS, QT, true>(A, &mt, it.b);
    }
}

template <typename QT>
Args<QT> make_args(const FlameGrid &g, int stage, double dt, const FlameStageBuffers &b,
                   const FlameMetrics &m, const FlameThermo &th, const FlameTransport &tr,
                   void *scratch) {
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
    A.metq = sizeof(QT) == 4 ? static_cast<const QT *>(b.metrics_lo) : nullptr;
    // scratch: R and R2 (5 + NS doubles per point each) first, then ϕ and Y (1 + NS of QT)
    A.R = static_cast<double *>(scratch);
    A.R2 = A.R + (size_t)(5 + g.ns) * A.np;
    A.aux = reinterpret_cast<QT *>(A.R2 + (size_t)(5 + g.ns) * A.np);
    A.th = th, A.tr = tr;
    return A;
}

template <typename K>
int set_smem(K kernel, size_t sm, std::atomic<bool> *done) {
    int dev = 0;
    cudaGetDevice(&dev);
    // atomic flags: host threads on other streams may launch the same kernel at the same time
    // (two that both find the flag unset both set the attribute, to the same value)
    if (dev >= 0 && dev < 64 && done[dev].load(std::memory_order_acquire)) return FLAME_OK;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "pencil sweep: %zu B shared memory: %s", sm,
                          cudaGetErrorString(e));
    if (dev >= 0 && dev < 64) done[dev].store(true, std::memory_order_release);
    return FLAME_OK;
}

template <int DIR, int PASS, int NS, typename QT, typename CT, int PART = 0, bool MIXD = false>
int launch_staged(const Args<QT> &A, cudaStream_t s) {
    using ST = Staged<NS, CT, PART, MIXD>;
    constexpr size_t sm = sizeof(CT) * ST::STRIDE * ST::COLS;
    static std::atomic<bool> done[64];
    const int n_along = DIR == 1 ? A.ny : A.nz;
    const int n_c2 = DIR == 1 ? A.nz : A.ny;
    const long long blocks = (long long)((A.nx + ST::COLS - 1) / ST::COLS) *
                             ((n_along + OWN - 1) / OWN) * n_c2;
    if constexpr (ST::MINB == 3) {
        if (int e = set_smem(k_pencil_staged3<DIR, PASS, NS, QT, CT, PART, MIXD>, sm, done)) return e;
        k_pencil_staged3<DIR, PASS, NS, QT, CT, PART, MIXD><<<(unsigned)blocks, ST::COLS * 32, sm, s>>>(A);
    } else {
        if (int e = set_smem(k_pencil_staged<DIR, PASS, NS, QT, CT, PART, MIXD>, sm, done)) return e;
        k_pencil_staged<DIR, PASS, NS, QT, CT, PART, MIXD><<<(unsigned)blocks, ST::COLS * 32, sm, s>>>(A);
    }
    return flame_check_launch("flame_rk_stage (pencil)");
}

template <int NS, typename QT, typename CT, bool FIN, bool MIXD = false>
int launch_x(const Args<QT> &A, cudaStream_t s) {
    constexpr int WPB = Wpb<0>::value;
    constexpr size_t sm = smem_bytes<NS, CT, WPB>();
    static std::atomic<bool> done[64];
    if (int e = set_smem(k_pencil_x<NS, QT, CT, FIN, MIXD>, sm, done)) return e;
    const long long warps = (long long)A.ny * A.nz * ((A.nx + OWN - 1) / OWN);
    k_pencil_x<NS, QT, CT, FIN, MIXD><<<(unsigned)((warps + WPB - 1) / WPB), WPB * 32, sm, s>>>(A);
    return flame_check_launch("flame_rk_stage (pencil)");
}

template <int NS, typename QT, typename CT>
int launch(const FlameGrid &g, cudaStream_t s, int stage, double dt, const FlameStageBuffers &b,
           const FlameMetrics &m, const FlameThermo &th, const FlameTransport &tr,
           void *scratch, bool split_finish, bool split_species) {
    const Args<QT> A = make_args<QT>(g, stage, dt, b, m, th, tr, scratch);
    k_prep<NS, QT><<<(unsigned)((A.np + 255) / 256), 256, 0, s>>>(A);
    if (int e = flame_check_launch("flame_rk_stage (prep)")) return e;
    if (tr.law == 2) {  // per-species D_k: configuration 6's launches with the MIXD sweeps
        if (int e = launch_staged<2, 0, 0, QT, CT>(A, s)) return e;
        if (int e = launch_staged<2, 0, NS, QT, CT, 2, true>(A, s)) return e;
        if (int e = launch_staged<1, 1, 0, QT, CT>(A, s)) return e;
        if (int e = launch_staged<1, 1, NS, QT, CT, 2, true>(A, s)) return e;
        if (int e = launch_x<NS, QT, CT, false, true>(A, s)) return e;
        k_finish_mix<NS, QT><<<(unsigned)(((long long)A.nx * A.ny * A.nz + 127) / 128), 128, 0,
                               s>>>(A);
        return flame_check_launch("flame_rk_stage (finish)");
    }
    if (split_species) {  // configurations 5, 6: flow sweep (the NS = 0 instance) + species sweep
        if (int e = launch_staged<2, 0, 0, QT, CT>(A, s)) return e;
        if (int e = launch_staged<2, 0, NS, QT, CT, 2>(A, s)) return e;
        if (int e = launch_staged<1, 1, 0, QT, CT>(A, s)) return e;
        if (int e = launch_staged<1, 1, NS, QT, CT, 2>(A, s)) return e;
    } else {
        if (int e = launch_staged<2, 0, NS, QT, CT>(A, s)) return e;
        if (int e = launch_staged<1, 1, NS, QT, CT>(A, s)) return e;
    }
    if (!split_finish) return launch_x<NS, QT, CT, true>(A, s);
    if (int e = launch_x<NS, QT, CT, false>(A, s)) return e;
    const long long cells = (long long)A.nx * A.ny * A.nz;
    k_finish<NS, QT><<<(unsigned)((cells + 127) / 128), 128, 0, s>>>(A);
    return flame_check_launch("flame_rk_stage (finish)");
}

template <typename QT, typename CT>
int dispatch(int ns, const FlameGrid &g, cudaStream_t s, int stage, double dt,
             const FlameStageBuffers &b, const FlameMetrics &m, const FlameThermo &th,
             const FlameTransport &tr, void *scratch, bool split_finish, bool split_species) {
    switch (ns) {
#define CASE(N) \
    case N: return launch<N, QT, CT>(g, s, stage, dt, b, m, th, tr, scratch, split_finish, split_species);
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9)
#undef CASE
        default:
            return flame_fail(FLAME_EUNSUPPORTED, "flame_rk_stage: ns=%d (pencil path has 1..9)",
                              ns);
    }
}

}  // namespace pencil
}  // namespace flame

// Entry used by fused_stage.cu's dispatcher for tile configuration 3.
int flame_pencil_stage(const FlameGrid *g, cudaStream_t s, int stage, double dt,
                       const FlameStageBuffers *b, const FlameMetrics *m, const FlameThermo *th,
                       const FlameTransport *tr, int precision, void *scratch, int split_finish,
                       int split_species) {
    if (!scratch)
        return flame_fail(FLAME_EINVAL,
                          "flame_rk_stage: the pencil configuration needs scratch (see "
                          "flame_stage_scratch_bytes)");
    if (precision == 0)
        return flame::pencil::dispatch<double, double>(g->ns, *g, s, stage, dt, *b, *m, *th, *tr,
                                                       scratch, split_finish != 0,
                                                       split_species != 0);
    return flame::pencil::dispatch<float, float>(g->ns, *g, s, stage, dt, *b, *m, *th, *tr,
                                                 scratch, split_finish != 0, split_species != 0);
}

// SIZE_MAX when the product does not fit in size_t (then no buffer can be large enough).
extern "C" size_t flame_stage_scratch_bytes(const FlameGrid *g, int precision) {
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1 || g->ng < 0 || g->ns < 0) return 0;
    const size_t q = precision == 0 ? sizeof(double) : sizeof(float);
    size_t bytes = 2 * (5 + (size_t)g->ns) * sizeof(double) + (1 + (size_t)g->ns) * q;
    const size_t ext[3] = {(size_t)g->nx + 2 * (size_t)g->ng, (size_t)g->ny + 2 * (size_t)g->ng,
                           (size_t)g->nz + 2 * (size_t)g->ng};
    for (size_t e : ext)
        if (__builtin_mul_overflow(bytes, e, &bytes)) return SIZE_MAX;
    return bytes;
}

// ============================================================================= batches
// A batch advances many independent cases per stage: the cases are grouped by species count and
// transport family (laws 0 and 1, or law 2) and the groups cut into chunks of at most
// kConstCases cases; per chunk and stage a copy of the chunk's descriptors into the constant
// table, a memset of its counters and its persistent launches (two, or four for law 2).
// Descriptors for the three stages and both in/out parities, the work lists and the per-case
// item counts are uploaded once, into device workspace the caller owns, so flame_batch_stage
// issues copies, memsets and launches only (capturable as a CUDA graph).
#include <algorithm>
#include <array>

namespace flame {
namespace pencil {

constexpr int kMaxPhases = 7;

// The work-list shape of a chunk: its phases and the block sizes their item counts follow.
struct BatchDims {
    int phases = 4;  // 4 (prep, z, y, x) or, law 2, 7 (prep, flow z, flow y, species z,
                     // species y, x, finish)
    int nt = 0;      // threads of a prep item (those of the first sweeps launch's blocks)
    int cols = 0;    // staged columns of the first sweeps launch's blocks
    int cols_s = 0;  // law 2: staged columns of the species sweeps' blocks
};

struct BatchChunk {
    int ns = 0, n = 0;
    bool mix = false;            // law 2
    const void *args[6] = {};    // device Args arrays of the chunk, index (stage - 1) * 2 + parity
    const BatchItem *items = nullptr;
    const int4 *need = nullptr;  // per case: prep items (x)
    int *counters = nullptr;     // item counters (ints 0-3, one per launch), per case done[4]
                                 // from int 4 on
    int bound[kMaxPhases + 1] = {};  // first item of each phase; bound[phases] = item count
    int grid[4] = {1, 1, 1, 1};      // persistent blocks of the launches
};

}  // namespace pencil
}  // namespace flame

struct FlameBatch {
    int precision = 0;
    int *err = nullptr;  // device error word (FLAME_ETIMEOUT)
    int stall = 0;       // test hook (flame_batch_test_stall)
    std::vector<flame::pencil::BatchChunk> chunks;
};

namespace flame {
namespace pencil {

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <typename QT>
size_t args_size() { return sizeof(Args<QT>); }

// Items of one case in each phase of a chunk of shape d.
inline void case_items(const FlameGrid &g, const BatchDims &d, int items[kMaxPhases]) {
    const long long tx = g.nx + 2LL * g.ng, ty = g.ny + 2LL * g.ng, tz = g.nz + 2LL * g.ng;
    const long long np = tx * ty * tz;
    auto zsweep = [&](int cols) { return ((g.nx + cols - 1) / cols) * ((g.nz + OWN - 1) / OWN) * g.ny; };
    auto ysweep = [&](int cols) { return ((g.nx + cols - 1) / cols) * ((g.ny + OWN - 1) / OWN) * g.nz; };
    const long long per = (long long)d.nt * kPrepPerThread;
    items[0] = (int)((np + per - 1) / per);
    items[1] = zsweep(d.cols);
    items[2] = ysweep(d.cols);
    int k = 3;
    if (d.phases == 7) items[3] = zsweep(d.cols_s), items[4] = ysweep(d.cols_s), k = 5;
    const long long warps = (long long)g.ny * g.nz * ((g.nx + OWN - 1) / OWN);
    items[k] = (int)((warps + Wpb<0>::value - 1) / Wpb<0>::value);
    if (d.phases == 7) items[6] = (int)(((long long)g.nx * g.ny * g.nz + 127) / 128);
}

template <int NS, typename QT, typename CT>
BatchDims batch_dims(bool mix) {
    BatchDims d;
    if (mix) {
        d.phases = 7;
        d.nt = BatchShape<NS, QT, CT, 1>::NT;
        d.cols = BatchShape<NS, QT, CT, 1>::COLS;
        d.cols_s = BatchShape<NS, QT, CT, 2>::COLS;
    } else {
        d.nt = BatchShape<NS, QT, CT>::NT;
        d.cols = BatchShape<NS, QT, CT>::COLS;
    }
    return d;
}

// Blocks of a persistent launch: as many as fit on the device at once, at most one per item.
template <typename K>
int persistent_grid(K kernel, int threads, size_t smem, std::atomic<bool> *done, int items,
                    int &grid) {
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (smem)
        if (int e = set_smem(kernel, smem, done)) return e;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem);
    grid = std::max(1, std::min(items, sms * std::max(occ, 1)));
    return FLAME_OK;
}

template <int NS, typename QT, typename CT>
int batch_grid(BatchChunk &bc) {
    using B0 = BatchShape<NS, QT, CT>;
    using B1 = BatchShape<NS, QT, CT, 1>;
    using B2 = BatchShape<NS, QT, CT, 2>;
    static std::atomic<bool> d[5][64];
    const int *b = bc.bound;
    int e = FLAME_OK;
    if (!bc.mix) {
        if (!e) e = persistent_grid(k_batch_sweeps<NS, QT, CT, 0>, B0::NT, B0::SMEM, d[0], b[3] - b[0], bc.grid[0]);
        if (!e) e = persistent_grid(k_batch_x<NS, QT, CT, false>, B0::XW * 32, B0::SMEM_X, d[1], b[4] - b[3], bc.grid[1]);
    } else {
        if (!e) e = persistent_grid(k_batch_sweeps<NS, QT, CT, 1>, B1::NT, B1::SMEM, d[2], b[3] - b[0], bc.grid[0]);
        if (!e) e = persistent_grid(k_batch_sweeps<NS, QT, CT, 2>, B2::NT, B2::SMEM, d[3], b[5] - b[3], bc.grid[1]);
        if (!e) e = persistent_grid(k_batch_x<NS, QT, CT, true>, B0::XW * 32, B0::SMEM_X, d[4], b[6] - b[5], bc.grid[2]);
        if (!e) e = persistent_grid(k_batch_finish<NS, QT>, 128, 0, nullptr, b[7] - b[6], bc.grid[3]);
    }
    if (e) return e;
    return flame_check_launch("flame_batch_create");
}

template <int NS, typename QT, typename CT>
int batch_launch(const BatchChunk &bc, cudaStream_t s, int stage, int parity, int *err,
                 int stall) {
    using B0 = BatchShape<NS, QT, CT>;
    using B1 = BatchShape<NS, QT, CT, 1>;
    using B2 = BatchShape<NS, QT, CT, 2>;
    cudaError_t ce = cudaMemcpyToSymbolAsync(c_batch_args, bc.args[(stage - 1) * 2 + parity],
                                             sizeof(Args<QT>) * (size_t)bc.n, 0,
                                             cudaMemcpyDeviceToDevice, s);
    if (ce == cudaSuccess)
        ce = cudaMemsetAsync(bc.counters, 0, sizeof(int) * (4 + 4 * (size_t)bc.n), s);
    if (ce != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "flame_batch_stage: %s", cudaGetErrorString(ce));
    BatchLaunch L;
    L.items = bc.items;
    L.need = bc.need;
    L.done = bc.counters + 4;
    L.err = err;
    L.stall = stall;
    // launch k: its counter, items [lo, hi) and, for the sweeps, the starts of phases 1 and 2
    auto set = [&](int k, int lo, int hi, int p1, int p2) {
        L.next = bc.counters + k;
        L.lo = lo, L.hi = hi, L.p1 = p1, L.p2 = p2;
    };
    const int *b = bc.bound;
    if (!bc.mix) {
        set(0, b[0], b[3], b[1], b[2]);
        k_batch_sweeps<NS, QT, CT, 0><<<bc.grid[0], B0::NT, B0::SMEM, s>>>(L);
        if (int e = flame_check_launch("flame_batch_stage")) return e;
        set(1, b[3], b[4], b[4], b[4]);
        k_batch_x<NS, QT, CT, false><<<bc.grid[1], B0::XW * 32, B0::SMEM_X, s>>>(L);
        return flame_check_launch("flame_batch_stage");
    }
    set(0, b[0], b[3], b[1], b[2]);
    k_batch_sweeps<NS, QT, CT, 1><<<bc.grid[0], B1::NT, B1::SMEM, s>>>(L);
    if (int e = flame_check_launch("flame_batch_stage")) return e;
    set(1, b[3], b[5], b[3], b[4]);  // no prep phase: p1 = lo
    k_batch_sweeps<NS, QT, CT, 2><<<bc.grid[1], B2::NT, B2::SMEM, s>>>(L);
    if (int e = flame_check_launch("flame_batch_stage")) return e;
    set(2, b[5], b[6], b[6], b[6]);
    k_batch_x<NS, QT, CT, true><<<bc.grid[2], B0::XW * 32, B0::SMEM_X, s>>>(L);
    if (int e = flame_check_launch("flame_batch_stage")) return e;
    set(3, b[6], b[7], b[7], b[7]);
    k_batch_finish<NS, QT><<<bc.grid[3], 128, 0, s>>>(L);
    return flame_check_launch("flame_batch_stage");
}

// what: 0 the chunk's work-list shape (*dims), 1 its persistent grids, 2 a stage launch
template <typename QT, typename CT>
int batch_dispatch(int what, BatchChunk &bc, cudaStream_t s, int stage, int parity, int *err,
                   int stall, BatchDims *dims) {
    switch (bc.ns) {
#define CASE(N)                                                                   \
    case N:                                                                       \
        if (what == 0) return *dims = batch_dims<N, QT, CT>(bc.mix), FLAME_OK;    \
        if (what == 1) return batch_grid<N, QT, CT>(bc);                          \
        return batch_launch<N, QT, CT>(bc, s, stage, parity, err, stall);
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9)
#undef CASE
        default:
            return flame_fail(FLAME_EUNSUPPORTED, "flame_batch: ns=%d (1..9)", bc.ns);
    }
}

inline int batch_dispatch_p(int precision, int what, BatchChunk &bc, cudaStream_t s, int stage,
                            int parity, int *err, int stall, BatchDims *dims = nullptr) {
    return precision == 0
               ? batch_dispatch<double, double>(what, bc, s, stage, parity, err, stall, dims)
               : batch_dispatch<float, float>(what, bc, s, stage, parity, err, stall, dims);
}

template <typename QT>
void fill_args(std::vector<unsigned char> &host, size_t at, const FlameCaseDesc &c, int stage,
               int parity) {
    FlameStageBuffers b = c.buf;
    if (parity) {  // the stage reads what the buffers call "out" and writes "in"
        const void *q = b.Q_in, *t = b.trans_in;
        const double *r = b.rhoi_in;
        b.Q_in = b.Q_out, b.Q_out = const_cast<void *>(q);
        b.rhoi_in = b.rhoi_out, b.rhoi_out = const_cast<double *>(r);
        b.trans_in = b.trans_out, b.trans_out = const_cast<void *>(t);
    }
    const Args<QT> A =
        make_args<QT>(c.grid, stage, c.dt, b, c.metrics, c.thermo, c.transport, c.buf.scratch);
    memcpy(host.data() + at, &A, sizeof(A));
}

}  // namespace pencil
}  // namespace flame

namespace {

// Chunks (cases of one species count, at most kConstCases each) and the byte layout of the
// workspace: the batch's error word, then per chunk six descriptor arrays, the work list, the
// per-case counts and the counters, each aligned to 256 bytes.
struct ChunkPlan {
    int ns = 0;
    bool mix = false;  // law 2
    flame::pencil::BatchDims dims;
    std::vector<int> members;  // case indices
    long long total = 0;
    size_t args_at[6] = {}, items_at = 0, need_at = 0, counters_at = 0;
};

struct Layout {
    std::vector<ChunkPlan> chunks;
    size_t bytes = 0;
};

// A case's group: its species count, and whether it has per-species D_k (law 2).
int group_of(const FlameCaseDesc &c) { return 2 * c.grid.ns + (c.transport.law == 2); }

int plan_layout(const FlameCaseDesc *cases, int n, int precision, Layout &L) {
    std::vector<int> groups;
    for (int i = 0; i < n; ++i)
        if (std::find(groups.begin(), groups.end(), group_of(cases[i])) == groups.end())
            groups.push_back(group_of(cases[i]));
    for (int grp : groups) {
        flame::pencil::BatchChunk probe;
        probe.ns = grp / 2, probe.mix = grp % 2;
        flame::pencil::BatchDims dims;
        if (int e = flame::pencil::batch_dispatch_p(precision, 0, probe, nullptr, 1, 0, nullptr,
                                                    0, &dims))
            return e;
        bool fresh = true;
        for (int i = 0; i < n; ++i) {
            if (group_of(cases[i]) != grp) continue;
            if (fresh || (int)L.chunks.back().members.size() == flame::pencil::kConstCases) {
                L.chunks.emplace_back();
                L.chunks.back().ns = probe.ns, L.chunks.back().mix = probe.mix;
                L.chunks.back().dims = dims;
                fresh = false;
            }
            ChunkPlan &c = L.chunks.back();
            c.members.push_back(i);
            int it[flame::pencil::kMaxPhases] = {};
            flame::pencil::case_items(cases[i].grid, dims, it);
            for (int ph = 0; ph < dims.phases; ++ph) c.total += it[ph];
        }
    }
    const size_t asz = precision == 0 ? flame::pencil::args_size<double>()
                                      : flame::pencil::args_size<float>();
    using flame::pencil::align256;
    size_t at = 256;  // the error word
    for (ChunkPlan &c : L.chunks) {
        if (c.total >= (1LL << 31))
            return flame_fail(FLAME_EINVAL, "flame_batch: %lld work items in one chunk", c.total);
        const size_t m = c.members.size();
        for (int v = 0; v < 6; ++v) c.args_at[v] = at, at = align256(at + asz * m);
        c.items_at = at, at = align256(at + sizeof(flame::pencil::BatchItem) * c.total);
        c.need_at = at, at = align256(at + sizeof(int4) * m);
        c.counters_at = at, at = align256(at + sizeof(int) * (4 + 4 * m));
    }
    L.bytes = at;
    return FLAME_OK;
}

int check_case(const FlameCaseDesc &c, int i) {
    if (int e = flame_check_grid(&c.grid, "flame_batch")) return e;
    if ((c.grid.periodic & 7) != 7)
        return flame_fail(FLAME_EUNSUPPORTED, "flame_batch: case %d is not periodic", i);
    if (c.grid.ns > 9) return flame_fail(FLAME_EUNSUPPORTED, "flame_batch: case %d ns > 9", i);
    if (c.grid.nx < FLAME_NG || c.grid.ny < FLAME_NG || c.grid.nz < FLAME_NG)
        return flame_fail(FLAME_EINVAL, "flame_batch: case %d extents must be >= %d", i, FLAME_NG);
    const long long np =
        ((long long)c.grid.nx + 8) * ((long long)c.grid.ny + 8) * ((long long)c.grid.nz + 8);
    if (c.grid.nx > (1 << 20) || c.grid.ny > (1 << 20) || c.grid.nz > (1 << 20) ||
        np * 10 >= (1LL << 31))
        return flame_fail(FLAME_EINVAL, "flame_batch: case %d too large", i);
    const FlameStageBuffers &b = c.buf;
    if (!b.U || !b.Un || !b.Q_in || !b.Q_out || !b.rhoi_in || !b.rhoi_out || !b.rhon ||
        !b.trans_in || !b.trans_out || !b.scratch || !c.metrics.J || !c.metrics.dxidx)
        return flame_fail(FLAME_EINVAL, "flame_batch: case %d has a NULL buffer", i);
    if (c.transport.law < 0 || c.transport.law > 2)
        return flame_fail(FLAME_EINVAL, "flame_batch: case %d: transport law %d", i,
                          c.transport.law);
    return FLAME_OK;
}

}  // namespace

extern "C" size_t flame_batch_workspace_bytes(const FlameCaseDesc *cases, int n, int precision) {
    if (!cases || n < 1 || (precision != 0 && precision != 1)) return 0;
    for (int i = 0; i < n; ++i)
        if (check_case(cases[i], i)) return 0;
    Layout L;
    if (plan_layout(cases, n, precision, L)) return 0;
    return L.bytes;
}

extern "C" int flame_batch_create(FlameBatch **out, const FlameCaseDesc *cases, int n,
                                  int precision, void *workspace, size_t bytes,
                                  flame_stream_t s) {
    if (!out || !cases || n < 1) return flame_fail(FLAME_EINVAL, "flame_batch_create: no cases");
    if (precision != 0 && precision != 1)
        return flame_fail(FLAME_EINVAL, "flame_batch_create: precision=%d", precision);
    for (int i = 0; i < n; ++i)
        if (int e = check_case(cases[i], i)) return e;
    Layout L;
    if (int e = plan_layout(cases, n, precision, L)) return e;
    if (!workspace || bytes < L.bytes)
        return flame_fail(FLAME_EINVAL, "flame_batch_create: workspace of %zu bytes, need %zu",
                          bytes, L.bytes);
    std::vector<unsigned char> host(L.bytes, 0);
    FlameBatch *B = new FlameBatch();
    B->precision = precision;
    unsigned char *dev = static_cast<unsigned char *>(workspace);
    B->err = reinterpret_cast<int *>(dev);
    const size_t asz = precision == 0 ? flame::pencil::args_size<double>()
                                      : flame::pencil::args_size<float>();
    using flame::pencil::BatchItem;
    for (const ChunkPlan &cp : L.chunks) {
        flame::pencil::BatchChunk bc;
        bc.ns = cp.ns;
        bc.mix = cp.mix;
        bc.n = (int)cp.members.size();
        const int phases = cp.dims.phases;
        std::vector<int4> need(bc.n);
        std::vector<std::array<int, flame::pencil::kMaxPhases>> counts(bc.n);
        for (int j = 0; j < bc.n; ++j) {
            const FlameCaseDesc &c = cases[cp.members[j]];
            counts[j].fill(0);
            flame::pencil::case_items(c.grid, cp.dims, counts[j].data());
            need[j] = make_int4(counts[j][0], 0, 0, 0);
            for (int st = 1; st <= 3; ++st)
                for (int par = 0; par < 2; ++par) {
                    const size_t at = cp.args_at[(st - 1) * 2 + par] + asz * j;
                    if (precision == 0) flame::pencil::fill_args<double>(host, at, c, st, par);
                    else flame::pencil::fill_args<float>(host, at, c, st, par);
                }
        }
        // work list: phase by phase (prep, z, y, ... as BatchDims lists them), each phase's
        // items case by case
        BatchItem *items = reinterpret_cast<BatchItem *>(host.data() + cp.items_at);
        long long w = 0;
        for (int ph = 0; ph < phases; ++ph) {
            bc.bound[ph] = (int)w;
            for (int j = 0; j < bc.n; ++j)
                for (int b = 0; b < counts[j][ph]; ++b) items[w++] = BatchItem{j, b};
        }
        bc.bound[phases] = (int)w;
        memcpy(host.data() + cp.need_at, need.data(), sizeof(int4) * bc.n);
        for (int v = 0; v < 6; ++v) bc.args[v] = dev + cp.args_at[v];
        bc.items = reinterpret_cast<const BatchItem *>(dev + cp.items_at);
        bc.need = reinterpret_cast<const int4 *>(dev + cp.need_at);
        bc.counters = reinterpret_cast<int *>(dev + cp.counters_at);
        if (int e = flame::pencil::batch_dispatch_p(precision, 1, bc, s, 1, 0, B->err, 0)) {
            delete B;
            return e;
        }
        B->chunks.push_back(bc);
    }
    cudaError_t ce = cudaMemcpyAsync(workspace, host.data(), L.bytes, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) {
        delete B;
        return flame_fail(FLAME_ELAUNCH, "flame_batch_create: upload: %s", cudaGetErrorString(ce));
    }
    *out = B;
    return FLAME_OK;
}

extern "C" int flame_batch_stage(FlameBatch *B, flame_stream_t s, int stage, int parity) {
    flame::NvtxRange range("flame_batch_stage");
    if (!B) return flame_fail(FLAME_EINVAL, "flame_batch_stage: NULL batch");
    if (stage < 1 || stage > 3 || (parity != 0 && parity != 1))
        return flame_fail(FLAME_EINVAL, "flame_batch_stage: stage=%d parity=%d", stage, parity);
    for (flame::pencil::BatchChunk &bc : B->chunks)
        if (int e = flame::pencil::batch_dispatch_p(B->precision, 2, bc, s, stage, parity, B->err,
                                                    B->stall))
            return e;
    return FLAME_OK;
}

extern "C" int flame_batch_status(FlameBatch *B, flame_stream_t s) {
    if (!B) return flame_fail(FLAME_EINVAL, "flame_batch_status: NULL batch");
    int h = 0;
    cudaError_t ce = cudaMemcpyAsync(&h, B->err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce == cudaSuccess && h) ce = cudaMemsetAsync(B->err, 0, sizeof(int), s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "flame_batch_status: %s", cudaGetErrorString(ce));
    if (h)
        return flame_fail(FLAME_ETIMEOUT,
                          "flame_batch_stage: a wait for another work item's completion ran out; "
                          "the items after it were skipped and the cases' states are invalid");
    return FLAME_OK;
}

extern "C" int flame_batch_test_stall(FlameBatch *B, int on) {
    if (!B) return flame_fail(FLAME_EINVAL, "flame_batch_test_stall: NULL batch");
    B->stall = on != 0;
    return FLAME_OK;
}

extern "C" int flame_batch_destroy(FlameBatch *B) {
    delete B;
    return FLAME_OK;
}
