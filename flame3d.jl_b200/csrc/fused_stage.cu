// fused_stage.cu — one launch per SSP-RK3 stage on periodic grids (sm_100a).
//
// A CTA owns a 16 x 8 x 8 tile of interior cells and performs, for that tile, everything
// solver.jl:298-326 does in ~30 launches:
//   point phase   shock sensor (schemes.jl:1-24), transport law (stand-in for thermo.jl:371),
//                 1/max(ρ, eps) for the mass fractions, into shared memory;
//   sweeps        per direction, in chunks: Steger-Warming split of every pencil point into
//                 shared memory (split.jl:17-130), hybrid UP7 / WENO-Z / minmod face fluxes
//                 (schemes.jl:86-437), viscous and species-diffusion face fluxes
//                 (viscous.jl:1-665) and the face differences into per-cell accumulators;
//   epilogue      div (div.jl), RK3 combination (utils.jl:95-112), c2Prim with the Newton
//                 temperature solve (utils.jl:2-48, thermo.jl:231-282), and the writes of the
//                 result and of its periodic ghost images.
// Split fluxes are computed once per point and direction (plus the pencil halo); face
// fluxes are computed once per face.  The only HBM traffic is the stage's inputs (with halo
// re-reads served by L2) and its outputs.
//
// Template parameters: NS species (compile-time loops), QT storage type of the primitive
// array Q, CT arithmetic type of split / reconstruction / viscous fluxes.  The plain path is
// <NS, double, double>; the mixed path is <NS, float, float> with U, Un, rhoi, metrics, the
// accumulators and the Newton solve kept in FP64.

#include "common.cuh"

namespace flame {
namespace fused {

constexpr int TX = 16, TY = 8, TZ = 8, NT = 256;
constexpr int CPT = TX * TY * TZ / NT;  // cells per thread (4): z = cz0 + 2*m
constexpr int BX1 = TX + 2, BY1 = TY + 2, BZ1 = TZ + 2, NB1 = BX1 * BY1 * BZ1;  // box [-1,T]
constexpr int BX2 = TX + 4, BY2 = TY + 4, BZ2 = TZ + 4, NB2 = BX2 * BY2 * BZ2;  // box [-2,T+1]

template <int NS>
struct Cfg {
    static constexpr int ZC = NS <= 4 ? 2 : 1;  // planes per chunk (x, y sweeps)
    static constexpr int YC = ZC;               // rows per chunk (z sweep)
    static constexpr int VF = 10 + 2 * NS;      // split values per point
    static constexpr int VG = 5 + NS;           // face values
    static constexpr int NPX = (TX + 6) * TY * ZC, NPY = TX * (TY + 6) * ZC,
                         NPZ = TX * YC * (TZ + 6);
    static constexpr int NFX = (TX + 1) * TY * ZC, NFY = TX * (TY + 1) * ZC,
                         NFZ = TX * YC * (TZ + 1);
    static constexpr int NPMAX = NPX > NPY ? (NPX > NPZ ? NPX : NPZ) : (NPY > NPZ ? NPY : NPZ);
    static constexpr int NFMAX = NFX > NFY ? (NFX > NFZ ? NFX : NFZ) : (NFY > NFZ ? NFY : NFZ);
};

template <typename QT>
struct Args {
    Dims D;
    int stage;
    double dt, ca, cb;  // RK3 combination U = ca*U + cb*Un (stage 2, 3)
    double *U, *Un;
    const QT *Qi;
    QT *Qo;
    const double *ri;
    double *ro, *rn;
    FlameMetrics m;
    FlameThermo th;
    FlameTransport tr;
};

template <int NS, typename CT>
constexpr size_t smem_bytes() {
    // working arrays, or the epilogue's accumulator hand-off if that is larger
    constexpr size_t work = sizeof(CT) * (4 * NB1 + NB2 + Cfg<NS>::VF * Cfg<NS>::NPMAX +
                                          Cfg<NS>::VG * Cfg<NS>::NFMAX);
    constexpr size_t acc = sizeof(double) * CPT * Cfg<NS>::VG * NT;
    return work > acc ? work : acc;
}

__device__ __forceinline__ long long clampll(long long v, long long lo, long long hi) {
    return v < lo ? lo : (v > hi ? hi : v);
}

template <typename CT>
__device__ __forceinline__ CT ld(const double *p, long long i) {
    return CT(__ldg(p + i));
}
template <typename CT>
__device__ __forceinline__ CT ld(const float *p, long long i) {
    return CT(__ldg(p + i));
}

// Steger-Warming splitting of the Euler flux along metric (A1, A2, A3), split.jl:17-89.
template <typename CT>
__device__ __forceinline__ void sw_split(CT rho, CT u, CT v, CT w, CT p, CT ei, CT A1, CT A2,
                                         CT A3, CT *fp, CT *fm) {
    const CT gam = p / ei + 1;
    const CT cs = sqrt(gam * p / rho);
    CT ss = sqrt(A1 * A1 + A2 * A2 + A3 * A3);
    const CT E1 = A1 * u + A2 * v + A3 * w;
    const CT E2 = E1 - cs * ss;
    const CT E3 = E1 + cs * ss;
    ss = 1 / ss;
    A1 *= ss, A2 *= ss, A3 *= ss;
    const CT h = CT(0.5);
    const CT E1P = (E1 + fabs(E1)) * h, E2P = (E2 + fabs(E2)) * h, E3P = (E3 + fabs(E3)) * h;
    const CT E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    const CT uc1 = u - cs * A1, uc2 = u + cs * A1;
    const CT vc1 = v - cs * A2, vc2 = v + cs * A2;
    const CT wc1 = w - cs * A3, wc2 = w + cs * A3;
    const CT vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * h;
    const CT vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * h;
    const CT vv = (gam - 1) * (u * u + v * v + w * w);
    const CT W2 = (3 - gam) / (2 * (gam - 1)) * (cs * cs);
    const CT tmp1 = rho / (2 * gam);
    const CT tmp2 = 2 * (gam - 1);
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

// Geometry of a sweep chunk along direction DIR.  "a" runs along the sweep, (b1, b2) across.
template <int NS, int DIR>
struct Sweep {
    using C = Cfg<NS>;
    static constexpr int L = DIR == 0 ? TX : (DIR == 1 ? TY : TZ);        // cells along
    static constexpr int C1 = DIR == 0 ? TY : TX;                         // first cross extent
    static constexpr int C2 = DIR == 2 ? C::YC : C::ZC;                   // chunk depth
    static constexpr int NCH = DIR == 2 ? TY / C::YC : TZ / C::ZC;        // chunks
    static constexpr int NP = (L + 6) * C1 * C2;
    static constexpr int NF = (L + 1) * C1 * C2;
    // tile-relative cell of (along a, cross b1, chunk-local b2) in chunk ch
    __device__ static void cell(int a, int b1, int b2, int ch, int &x, int &y, int &z) {
        if (DIR == 0) x = a, y = b1, z = ch * C2 + b2;
        else if (DIR == 1) x = b1, y = a, z = ch * C2 + b2;
        else x = b1, y = ch * C2 + b2, z = a;
    }
};

template <int NS, typename QT, typename CT>
struct Tile {
    using C = Cfg<NS>;
    const Args<QT> &A;
    const long long X0, Y0, Z0;  // interior index of the tile's first cell
    const long long sy, sz, np;
    CT *sPhi, *sMu, *sLam, *sD, *sRinv, *sF, *sG;

    __device__ Tile(const Args<QT> &a, CT *smem)
        : A(a),
          X0((long long)blockIdx.x * TX),
          Y0((long long)blockIdx.y * TY),
          Z0((long long)blockIdx.z * TZ),
          sy(a.D.tx),
          sz(a.D.tx * a.D.ty),
          np(a.D.np) {
        sPhi = smem;
        sMu = sPhi + NB1;
        sLam = sMu + NB1;
        sD = sLam + NB1;
        sRinv = sD + NB1;
        sF = sRinv + NB2;
        sG = sF + C::VF * C::NPMAX;
    }

    // ghosted linear index of tile-relative cell (x, y, z), clamped into the array
    __device__ long long gidx(int x, int y, int z) const {
        const long long gx = clampll(X0 + A.D.ng + x, 0, A.D.tx - 1);
        const long long gy = clampll(Y0 + A.D.ng + y, 0, A.D.ty - 1);
        const long long gz = clampll(Z0 + A.D.ng + z, 0, A.D.tz - 1);
        return gx + sy * (gy + A.D.ty * gz);
    }
    // ghosted index of the right cell of a DIR face, clamped so that the whole viscous stencil
    // (normal -2..+1, tangential ±2) stays inside the array even for tiles past the domain end
    template <int DIR>
    __device__ long long gidx_face(int x, int y, int z) const {
        const int ng = A.D.ng;
        const long long gx = clampll(X0 + ng + x, ng, A.D.nx + ng - (DIR != 0));
        const long long gy = clampll(Y0 + ng + y, ng, A.D.ny + ng - (DIR != 1));
        const long long gz = clampll(Z0 + ng + z, ng, A.D.nz + ng - (DIR != 2));
        return gx + sy * (gy + A.D.ty * gz);
    }
    __device__ static int b1i(int x, int y, int z) {
        return (x + 1) + BX1 * ((y + 1) + BY1 * (z + 1));
    }
    __device__ static int b2i(int x, int y, int z) {
        return (x + 2) + BX2 * ((y + 2) + BY2 * (z + 2));
    }

    // ---------------------------------------------------------------- point phase
    __device__ void point_phase() {
        const QT *Q = A.Qi;
        // 1/max(ρ, eps) on the box [-2, T+1]^3 (mixture: thermo.jl:391)
        for (int p = threadIdx.x; p < NB2; p += NT) {
            const int x = p % BX2 - 2, y = (p / BX2) % BY2 - 2, z = p / (BX2 * BY2) - 2;
            const long long g = gidx(x, y, z);
            sRinv[p] = CT(1) / CT(jmax(double(Q[g]), kEps));
        }
        // sensor, μ, λ, D on the box [-1, T]^3
        for (int p = threadIdx.x; p < NB1; p += NT) {
            const int x = p % BX1 - 1, y = (p / BX1) % BY1 - 1, z = p / (BX1 * BY1) - 1;
            long long g = gidx(x, y, z);
            // schemes.jl:10-22; the neighbours of a clamped point stay inside the array
            {
                const long long gx = g % sy, gy = (g / sy) % A.D.ty, gz = g / sz;
                const long long gc = clampll(gx, 1, A.D.tx - 2) +
                                     sy * (clampll(gy, 1, A.D.ty - 2) +
                                           A.D.ty * clampll(gz, 1, A.D.tz - 2));
                const QT *P = Q + 4 * np;
                const CT P2 = CT(P[gc]);
                CT a1 = CT(P[gc - 1]), a3 = CT(P[gc + 1]);
                const CT phx = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
                a1 = CT(P[gc - sy]), a3 = CT(P[gc + sy]);
                const CT phy = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
                a1 = CT(P[gc - sz]), a3 = CT(P[gc + sz]);
                const CT phz = fabs(-a1 + 2 * P2 - a3) / (a1 + 2 * P2 + a3);
                sPhi[p] = phx + phy + phz;
            }
            // transport law in place of mixtureProperties (thermo.jl:289-369)
            CT mu, lam, dd;
            if (A.tr.law == 0) {
                mu = CT(A.tr.mu_ref), lam = CT(A.tr.lambda_ref), dd = CT(A.tr.D_ref);
            } else {
                const double T = double(Q[g + 5 * np]);
                const double rho = jmax(double(Q[g]), kEps);
                const double rinv = 1 / rho;
                const double T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
                double cpm = 0;
#pragma unroll
                for (int n = 0; n < NS; ++n) {
                    const double Y = jmax(A.ri[g + n * np] * rinv, 0.0);
                    cpm += cp_spec(A.th, n, T, T2, T3, T4) * Y / A.th.mw[n];
                }
                cpm *= A.th.Ru;
                const double m = A.tr.mu_ref * pow(T / A.tr.T_ref, A.tr.exponent);
                const double l = cpm * m / A.tr.Pr;
                mu = CT(m), lam = CT(l), dd = CT(l / (rho * cpm));
            }
            sMu[p] = mu, sLam[p] = lam, sD[p] = dd;
        }
    }

    // ---------------------------------------------------------------- split of one point
    template <int DIR>
    __device__ void split_point(long long g, CT *out, int stride) const {
        const double *Ax = DIR == 0 ? A.m.dxidx : (DIR == 1 ? A.m.detadx : A.m.dzetadx);
        const double *Ay = DIR == 0 ? A.m.dxidy : (DIR == 1 ? A.m.detady : A.m.dzetady);
        const double *Az = DIR == 0 ? A.m.dxidz : (DIR == 1 ? A.m.detadz : A.m.dzetadz);
        const QT *Q = A.Qi;
        const CT rho = CT(Q[g]), u = CT(Q[g + np]), v = CT(Q[g + 2 * np]), w = CT(Q[g + 3 * np]),
                 p = CT(Q[g + 4 * np]), ei = CT(Q[g + 6 * np]);
        const CT A1 = ld<CT>(Ax, g), A2 = ld<CT>(Ay, g), A3 = ld<CT>(Az, g);
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
    // Writes G[1..4] -= Fv (viscous.jl:1-428) and G[5+n] -= Fd_n (viscous.jl:430-665), so that
    // G holds F_inviscid - F_viscous with the sign convention of div.jl.
    template <int DIR>
    __device__ void viscous_face(long long g, int x, int y, int z, CT *G) const {
        constexpr int D1 = (DIR + 1) % 3, D2 = (DIR + 2) % 3;
        const long long sn = DIR == 0 ? 1 : (DIR == 1 ? sy : sz);
        const long long s1 = D1 == 0 ? 1 : (D1 == 1 ? sy : sz);
        const long long s2 = D2 == 0 ? 1 : (D2 == 1 ? sy : sz);
        const int xl = x - (DIR == 0), yl = y - (DIR == 1), zl = z - (DIR == 2);
        const int bR = b1i(x, y, z), bL = b1i(xl, yl, zl);
        const QT *Q = A.Qi;
        const double *M[9] = {A.m.dxidx,   A.m.dxidy,   A.m.dxidz,   A.m.detadx, A.m.detady,
                              A.m.detadz,  A.m.dzetadx, A.m.dzetady, A.m.dzetadz};
        const CT h = CT(0.5), c23 = CT(2.0 / 3.0), c12 = CT(1.0 / 12.0);
        CT met[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) met[a] = (ld<CT>(M[a], g - sn) + ld<CT>(M[a], g)) * h;
        const CT Jac = (ld<CT>(A.m.J, g - sn) + ld<CT>(A.m.J, g)) * h;
        const CT mui = (sMu[bL] + sMu[bR]) * h;
        const CT lami = (sLam[bL] + sLam[bR]) * h;

        // species diffusion first: it produces Fh for the energy flux (viscous.jl:446-505)
        const CT rho = (CT(Q[g - sn]) + CT(Q[g])) * h;
        const CT T = (CT(Q[g - sn + 5 * np]) + CT(Q[g + 5 * np])) * h;
        const int b2R = b2i(x, y, z);
        const int o_n = DIR == 0 ? 1 : (DIR == 1 ? BX2 : BX2 * BY2);
        const int o_1 = D1 == 0 ? 1 : (D1 == 1 ? BX2 : BX2 * BY2);
        const int o_2 = D2 == 0 ? 1 : (D2 == 1 ? BX2 : BX2 * BY2);
        CT Vk1[NS], Vk2[NS], Vk3[NS], Yf[NS];
        CT sum1 = 0, sum2 = 0, sum3 = 0;
        const CT DL = sD[bL], DR = sD[bR];
#pragma unroll
        for (int n = 0; n < NS; ++n) {
            const double *r = A.ri + n * np;
            // Y = max(ρi / max(ρ, eps), 0) at the stencil points
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
            const double Td = double(T);
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

    // ---------------------------------------------------------------- one sweep direction
    template <int DIR>
    __device__ void sweep(double (&acc)[CPT][C::VG]) {
        using SW = Sweep<NS, DIR>;
        const int tid = threadIdx.x;
        const int cx = tid % TX, cy = (tid / TX) % TY, cz0 = tid / (TX * TY);
#pragma unroll 1
        for (int ch = 0; ch < SW::NCH; ++ch) {
            // split fluxes of every pencil point of the chunk
            for (int p = tid; p < SW::NP; p += NT) {
                const int a = p % (SW::L + 6) - 3, b = p / (SW::L + 6);
                int x, y, z;
                SW::cell(a, b % SW::C1, b / SW::C1, ch, x, y, z);
                split_point<DIR>(gidx(x, y, z), sF + p, C::NPMAX);
            }
            __syncthreads();
            // face fluxes
            for (int f = tid; f < SW::NF; f += NT) {
                const int a = f % (SW::L + 1), b = f / (SW::L + 1);
                int x, y, z;
                SW::cell(a, b % SW::C1, b / SW::C1, ch, x, y, z);
                const int xl = x - (DIR == 0), yl = y - (DIR == 1), zl = z - (DIR == 2);
                const CT phif = CT(jmax(double(sPhi[b1i(xl, yl, zl)]), double(sPhi[b1i(x, y, z)])));
                const int p0 = a + (SW::L + 6) * b;  // point index of along-coordinate a-3
                CT G[C::VG];
#pragma unroll
                for (int n = 0; n < C::VG; ++n) {
                    const int vp = n < 5 ? n : 5 + n;  // F+ row (species rows start at 10)
                    const int vm = n < 5 ? 5 + n : 5 + NS + n;
                    // the hybrid face reads F±[c-3..c+2] only (UP7[1] = 0 drops F+[c-4], and
                    // F-[c+3] carries the weight UP7[1] too), i.e. six points of the pencil
                    CT pv[7], mv[7];
#pragma unroll
                    for (int i = 0; i < 6; ++i) {
                        pv[i] = sF[vp * C::NPMAX + p0 + i];
                        mv[i] = sF[vm * C::NPMAX + p0 + i];
                    }
                    pv[6] = mv[6] = CT(0);
                    G[n] = hybrid_face7<CT>(pv, mv, phif);
                }
                viscous_face<DIR>(gidx_face<DIR>(x, y, z), x, y, z, G);
#pragma unroll
                for (int n = 0; n < C::VG; ++n) sG[n * C::NFMAX + f] = G[n];
            }
            __syncthreads();
            // face differences into the owned cells of this chunk
#pragma unroll
            for (int m = 0; m < CPT; ++m) {
                const int z = cz0 + 2 * m;
                bool in;
                int a, b;
                if (DIR == 2) {
                    in = (cy / C::YC) == ch;
                    a = z, b = cx + TX * (cy - ch * C::YC);
                } else {
                    in = (z / C::ZC) == ch;
                    a = DIR == 0 ? cx : cy;
                    b = (DIR == 0 ? cy : cx) + SW::C1 * (z - ch * C::ZC);
                }
                if (in) {
                    const int f0 = a + (SW::L + 1) * b;
#pragma unroll
                    for (int n = 0; n < C::VG; ++n)
                        acc[m][n] += double(sG[n * C::NFMAX + f0]) - double(sG[n * C::NFMAX + f0 + 1]);
                }
            }
            __syncthreads();
        }
    }

    // ---------------------------------------------------------------- epilogue
    // The accumulators leave registers through shared memory so the (not unrolled) cell loop
    // below does not force them into local memory for the whole kernel.
    __device__ void epilogue(const double (&acc)[CPT][C::VG]) {
        const int tid = threadIdx.x;
        __syncthreads();  // every thread is done reading the working arrays
        double *sAcc = reinterpret_cast<double *>(sPhi);
#pragma unroll
        for (int m = 0; m < CPT; ++m)
#pragma unroll
            for (int n = 0; n < C::VG; ++n) sAcc[(m * C::VG + n) * NT + tid] = acc[m][n];
        const int cx = tid % TX, cy = (tid / TX) % TY, cz0 = tid / (TX * TY);
        const Dims &D = A.D;
#pragma unroll 1
        for (int m = 0; m < CPT; ++m) {
            const int cz = cz0 + 2 * m;
            const long long ix = X0 + cx, iy = Y0 + cy, iz = Z0 + cz;
            if (ix >= D.nx || iy >= D.ny || iz >= D.nz) continue;
            const long long g = (ix + D.ng) + sy * ((iy + D.ng) + D.ty * (iz + D.ng));
            const double Jact = A.m.J[g] * A.dt;
            double Uc[5], r[NS];
#pragma unroll
            for (int n = 0; n < 5; ++n) {
                const double u0 = A.U[g + n * np];
                if (A.stage == 1) A.Un[g + n * np] = u0;
                double un = u0 + sAcc[(m * C::VG + n) * NT + tid] * Jact;
                if (A.stage > 1) un = un * A.ca + A.Un[g + n * np] * A.cb;
                Uc[n] = un;
                A.U[g + n * np] = un;
            }
#pragma unroll
            for (int n = 0; n < NS; ++n) {
                const double r0 = A.ri[g + n * np];
                if (A.stage == 1) A.rn[g + n * np] = r0;
                double rv = r0 + sAcc[(m * C::VG + 5 + n) * NT + tid] * Jact;
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
            const double T = jmax(get_T<NS>(A.th, NS, ei, r), kEps);
            const double p = jmax(p_mixture<NS>(A.th, NS, T, r), kEps);
            const double qv[7] = {rho, u, v, w, p, T, ei};
            // the cell and its periodic ghost images (new: the reference fills ghosts with
            // case-specific kernels, boundary.jl:1-191)
            const long long gx = ix + D.ng, gy = iy + D.ng, gz = iz + D.ng;
            long long ox[2] = {0, 0}, oy[2] = {0, 0}, oz[2] = {0, 0};
            int nxo = 1, nyo = 1, nzo = 1;
            if (gx < 2 * D.ng) ox[nxo++] = D.nx; else if (gx >= D.nx) ox[nxo++] = -D.nx;
            if (gy < 2 * D.ng) oy[nyo++] = D.ny; else if (gy >= D.ny) oy[nyo++] = -D.ny;
            if (gz < 2 * D.ng) oz[nzo++] = D.nz; else if (gz >= D.nz) oz[nzo++] = -D.nz;
            for (int c = 0; c < nzo; ++c)
                for (int b = 0; b < nyo; ++b)
                    for (int a = 0; a < nxo; ++a) {
                        const long long t = (gx + ox[a]) + sy * ((gy + oy[b]) + D.ty * (gz + oz[c]));
#pragma unroll
                        for (int n = 0; n < 7; ++n) A.Qo[t + n * np] = QT(qv[n]);
#pragma unroll
                        for (int n = 0; n < NS; ++n) A.ro[t + n * np] = r[n];
                    }
        }
    }
};

template <int NS, typename QT, typename CT>
__global__ void __launch_bounds__(NT, 1) k_stage(const __grid_constant__ Args<QT> A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Tile<NS, QT, CT> t(A, reinterpret_cast<CT *>(smem_raw));
    double acc[CPT][Cfg<NS>::VG];
#pragma unroll
    for (int m = 0; m < CPT; ++m)
#pragma unroll
        for (int n = 0; n < Cfg<NS>::VG; ++n) acc[m][n] = 0.0;
    t.point_phase();
    __syncthreads();
    t.template sweep<0>(acc);
    t.template sweep<1>(acc);
    t.template sweep<2>(acc);
    t.epilogue(acc);
}

template <int NS, typename QT, typename CT>
int launch(const FlameGrid &g, cudaStream_t s, int stage, double dt, const FlameStageBuffers &b,
           const FlameMetrics &m, const FlameThermo &th, const FlameTransport &tr) {
    Args<QT> A;
    A.D = make_dims(g);
    A.stage = stage;
    A.dt = dt;
    A.ca = stage == 2 ? 0.25 : 2.0 / 3.0;
    A.cb = stage == 2 ? 0.75 : 1.0 / 3.0;
    A.U = b.U, A.Un = b.Un;
    A.Qi = reinterpret_cast<const QT *>(b.Q_in);
    A.Qo = reinterpret_cast<QT *>(b.Q_out);
    A.ri = b.rhoi_in, A.ro = b.rhoi_out, A.rn = b.rhon;
    A.m = m, A.th = th, A.tr = tr;
    constexpr size_t sm = smem_bytes<NS, CT>();
    static bool attr_set[64] = {};  // the attribute is per function and device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(
            k_stage<NS, QT, CT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess)
            return flame_fail(FLAME_ELAUNCH, "flame_rk_stage: %zu B shared memory: %s", sm,
                              cudaGetErrorString(e));
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
    }
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, (g.nz + TZ - 1) / TZ);
    k_stage<NS, QT, CT><<<grid, NT, sm, s>>>(A);
    return flame_check_launch("flame_rk_stage");
}

template <typename QT, typename CT>
int dispatch(int ns, const FlameGrid &g, cudaStream_t s, int stage, double dt,
             const FlameStageBuffers &b, const FlameMetrics &m, const FlameThermo &th,
             const FlameTransport &tr) {
    switch (ns) {
#define CASE(N) \
    case N: return launch<N, QT, CT>(g, s, stage, dt, b, m, th, tr);
        CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8) CASE(9)
#undef CASE
        default:
            return flame_fail(FLAME_EUNSUPPORTED, "flame_rk_stage: ns=%d (fused path has 1..9)",
                              ns);
    }
}

}  // namespace fused
}  // namespace flame

extern "C" int flame_rk_stage(const FlameGrid *g, flame_stream_t s, int stage, double dt,
                              const FlameStageBuffers *b, const FlameMetrics *m,
                              const FlameThermo *th, const FlameTransport *tr, int precision) {
    if (int e = flame_check_grid(g, "flame_rk_stage")) return e;
    if (!b || !m || !th || !tr || !b->U || !b->Un || !b->Q_in || !b->Q_out || !b->rhoi_in ||
        !b->rhoi_out || !b->rhon || !m->J || !m->dxidx || !m->dzetadz)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: NULL argument");
    if (stage < 1 || stage > 3)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: stage=%d must be 1, 2 or 3", stage);
    if ((g->periodic & 7) != 7)
        return flame_fail(FLAME_EUNSUPPORTED,
                          "flame_rk_stage: the fused stage needs a grid periodic in x, y and z; "
                          "use the per-kernel entry points with the case's own ghost fill");
    if (g->nx < FLAME_NG || g->ny < FLAME_NG || g->nz < FLAME_NG)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: extents must be >= %d", FLAME_NG);
    if ((const void *)b->Q_in == (const void *)b->Q_out ||
        (const void *)b->rhoi_in == (const void *)b->rhoi_out)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: in and out buffers must differ");
    if (tr->law != 0 && tr->law != 1)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage: transport law %d unknown", tr->law);
    if (precision == 0)
        return flame::fused::dispatch<double, double>(g->ns, *g, s, stage, dt, *b, *m, *th, *tr);
    if (precision == 1)
        return flame::fused::dispatch<float, float>(g->ns, *g, s, stage, dt, *b, *m, *th, *tr);
    return flame_fail(FLAME_EINVAL, "flame_rk_stage: precision=%d must be 0 or 1", precision);
}
