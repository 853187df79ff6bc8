// chemistry.cu — the finite-rate chemistry step of the reference (reactions.jl), 1:1.
//
// eval_gpu (explicit) and eval_gpu_stiff (point-implicit) advance the partial densities of every
// interior cell hotter than T_criteria by the mass production rates of the mechanism, add the
// formation-enthalpy release to the total energy, clip and rescale ρi to ρ and recover T, p, e.
// Rates follow vproductionRate / vproductionRate_Jac: Arrhenius forward rates, equilibrium
// constants from the Gibbs energy (thermo.jl:163-191), third-body and Troe falloff reactions.
//
// Built with -fmad=false, like kernels_ref.cu: apart from exp / log / pow (the device math
// library against the host's) the arithmetic is the oracle's, operation by operation.  One
// thread per cell; the per-cell work arrays (ns, nreacs and ns x ns doubles) live in local
// memory, as MVector / MMatrix do in the reference.

#include "common.cuh"

namespace flame {
namespace chem {

constexpr int kMaxReacs = 64;

struct Mech {
    int nr;
    double atm;
    const int64_t *type, *sgm, *vf, *vr;
    const double *Arr, *ef, *loP, *Troe;
};

// x^k for the small integer stoichiometric powers (repeated multiplication, both signs)
__device__ __forceinline__ double ipow(double x, long long k) {
    double r = 1.0;
    const long long m = k < 0 ? -k : k;
    for (long long i = 0; i < m; ++i) r *= x;
    return k < 0 ? 1.0 / r : r;
}

// gibbs, thermo.jl:163-191 (dimensionless g/RT per species)
__device__ void gibbs(double *gi, double T, double lgT, double invT, const FlameThermo &th,
                      int ns) {
    const double mlogT = 1 - lgT;
    const double T1 = 0.5 * T;
    const double T2 = 1.0 / 6.0 * T * T;
    const double T3 = T1 * T2;
    const double T4 = 1.8 * T2 * T2;
    for (int n = 0; n < ns; ++n) {
        const double *c = T < th.coeffs_sep[n] ? th.coeffs_lo + 7 * n : th.coeffs_hi + 7 * n;
        gi[n] = c[0] * mlogT - c[1] * T1 - c[2] * T2 - c[3] * T3 - c[4] * T4 + c[5] * invT - c[6];
    }
}

// vproductionRate (reactions.jl:311-380) and, with JAC, vproductionRate_Jac (:383-462):
// wdot [mol/(cm^3 s)] from the concentrations sc [mol/cm^3]; A (ns x ns, column-major) gets
// the Jacobian of wdot with respect to sc.
template <bool JAC>
__device__ void production(double *wdot, const double *sc, double *A, double T,
                           const FlameThermo &th, const Mech &M, int ns) {
    double gi[FLAME_MAX_NS], kf[kMaxReacs], Kc[kMaxReacs];
    const double lgT = log(T);
    const double invT = 1.0 / T;
    for (int n = 0; n < M.nr; ++n)
        kf[n] = M.Arr[3 * n] * exp(M.Arr[3 * n + 1] * lgT - M.Arr[3 * n + 2] * invT);
    gibbs(gi, T, lgT, invT, th, ns);
    const double RsT = th.Ru / M.atm * 1e6 * T;
    for (int n = 0; n < M.nr; ++n) {
        double dg = 0;
        for (int m = 0; m < ns; ++m) dg += gi[m] * double(M.vf[m + ns * n] - M.vr[m + ns * n]);
        Kc[n] = ipow(RsT, M.sgm[n]) * exp(dg);
    }
    for (int n = 0; n < M.nr; ++n) {
        double qf = kf[n];
        double qr = qf / Kc[n];
        for (int m = 0; m < ns; ++m) {
            const long long vf = M.vf[m + ns * n], vr = M.vr[m + ns * n];
            if (vf != 0) qf *= ipow(sc[m], vf);
            if (vr != 0) qr *= ipow(sc[m], vr);
        }
        double mix = 0.0;
        if (M.type[n] == 2) {  // three-body
            for (int m = 0; m < ns; ++m) mix += M.ef[m + ns * n] * sc[m];
            qf *= mix;
            qr *= mix;
        } else if (M.type[n] == 3) {  // falloff, Troe form
            for (int m = 0; m < ns; ++m) mix += M.ef[m + ns * n] * sc[m];
            const double *lo = M.loP + 3 * n, *tr = M.Troe + 4 * n;
            const double redP = mix / kf[n] * lo[0] * exp(lo[1] * lgT - lo[2] * invT);
            const double logPred = log10(redP);
            const double a = tr[0];
            const double logFcent =
                log10((1 - a) * exp(-T / tr[1]) + a * exp(-T / tr[2]) + exp(-tr[3] * invT));
            const double troe_c = -0.4 - 0.67 * logFcent;
            const double troe_n = 0.75 - 1.27 * logFcent;
            const double troe = (troe_c + logPred) / (troe_n - 0.14 * (troe_c + logPred));
            const double F = pow(10.0, logFcent / (1.0 + troe * troe));
            const double k1 = (redP / (1.0 + redP)) * F;
            qf *= k1;
            qr *= k1;
        }
        for (int m = 0; m < ns; ++m) {
            const double nu = double(M.vr[m + ns * n] - M.vf[m + ns * n]);
            wdot[m] += (qf - qr) * nu;
            if constexpr (JAC) {
                const double invsc = 1 / (sc[m] + kEps);
                const double Awf = double(M.vf[m + ns * n]) * qf * invsc;
                const double Awr = double(M.vr[m + ns * n]) * qr * invsc;
                for (int l = 0; l < ns; ++l)
                    A[l + ns * m] += (Awf - Awr) * double(M.vr[l + ns * n] - M.vf[l + ns * n]);
            }
        }
    }
}

// solve, reactions.jl:465-504: Gaussian elimination with partial pivoting; a (ns x ns,
// column-major) and b are overwritten.
__device__ void solve(double *x, double *a, double *b, int ns) {
#define AT(i, j) a[(i) + ns * (j)]
    for (int k = 0; k < ns - 1; ++k) {
        double fmax = fabs(AT(k, k));
        int kk = k;
        for (int i = k + 1; i < ns; ++i) {
            const double absa = fabs(AT(i, k));
            if (absa > fmax) fmax = absa, kk = i;
        }
        for (int j = k; j < ns; ++j) {
            const double t = AT(k, j);
            AT(k, j) = AT(kk, j);
            AT(kk, j) = t;
        }
        const double t = b[k];
        b[k] = b[kk];
        b[kk] = t;
        for (int i = k + 1; i < ns; ++i) {
            const double f = -AT(i, k) / AT(k, k);
            for (int j = 0; j < ns; ++j) AT(i, j) += f * AT(k, j);
            b[i] += f * b[k];
        }
    }
    x[ns - 1] = b[ns - 1] / AT(ns - 1, ns - 1);
    for (int i = ns - 2; i >= 0; --i) {
        x[i] = b[i];
        for (int j = i + 1; j < ns; ++j) x[i] -= AT(i, j) * x[j];
        x[i] /= AT(i, i);
    }
#undef AT
}

// eval_gpu (STIFF false, reactions.jl:187-232) and eval_gpu_stiff (STIFF true, :235-309)
template <bool STIFF>
__global__ void k_eval(Dims D, double *U, double *Q, double *rhoi, double dt, FlameThermo th,
                       Mech M, const int64_t *tag, double Tcrit, int transposed) {
    const long long c = blockIdx.x * 128LL + threadIdx.x;
    const long long ncell = (long long)D.nx * D.ny * D.nz;
    if (c >= ncell) return;
    const long long x = c % D.nx, y = (c / D.nx) % D.ny, z = c / ((long long)D.nx * D.ny);
    const long long p = D.P(x + D.ng, y + D.ng, z + D.ng), np = D.np;
    if (tag && tag[p] != 0) return;
    double T = Q[p + 5 * np];
    if (!(T > Tcrit)) return;
    const int ns = D.ns;
    double sc[FLAME_MAX_NS], wdot[FLAME_MAX_NS], r[FLAME_MAX_NS], dr[FLAME_MAX_NS];
    for (int n = 0; n < ns; ++n) {
        r[n] = rhoi[p + n * np];
        sc[n] = r[n] / th.mw[n] * 1e-6;
        wdot[n] = 0.0;
    }
    double dei = 0;
    if constexpr (STIFF) {
        double A[FLAME_MAX_NS * FLAME_MAX_NS], A1[FLAME_MAX_NS * FLAME_MAX_NS];
        double drho[FLAME_MAX_NS];
        for (int i = 0; i < ns * ns; ++i) A[i] = 0.0;
        production<true>(wdot, sc, A, T, th, M, ns);
        for (int l = 0; l < ns; ++l)  // I - A dt, with the mass weights
            for (int n = 0; n < ns; ++n)
                A1[n + ns * l] = (n == l ? 1.0 : 0.0) - A[n + ns * l] * th.mw[n] / th.mw[l] * dt;
        for (int n = 0; n < ns; ++n) drho[n] = wdot[n] * th.mw[n] * 1e6 * dt;
        solve(dr, A1, drho, ns);
        for (int n = 0; n < ns; ++n) {
            const double a6 = transposed ? th.coeffs_lo[n + 35] : th.coeffs_lo[5 + 7 * n];
            dei += -a6 * dr[n] * th.Ru / th.mw[n];
            r[n] += dr[n];
        }
    } else {
        production<false>(wdot, sc, nullptr, T, th, M, ns);
        for (int n = 0; n < ns; ++n) {
            const double d = wdot[n] * th.mw[n] * 1e6 * dt;
            dei += -th.coeffs_lo[5 + 7 * n] * d * th.Ru / th.mw[n];
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
    T = jmax(get_T<0>(th, ns, ein, r), kEps);
    const double pr = jmax(p_mixture<0>(th, ns, T, r), kEps);
    Q[p + 4 * np] = pr;
    Q[p + 5 * np] = T;
    Q[p + 6 * np] = ein;
}

int launch(bool stiff, const FlameGrid *g, cudaStream_t s, double *U, double *Q, double *rhoi,
           double dt, const FlameThermo *th, const FlameReactions *re, const int64_t *tag,
           double Tcrit, int transposed, const char *what) {
    if (int e = flame_check_grid(g, what)) return e;
    if (!U || !Q || !rhoi || !th || !re || !re->reaction_type || !re->sgm || !re->vf ||
        !re->vr || !re->Arr || !re->ef || !re->loP || !re->Troe)
        return flame_fail(FLAME_EINVAL, "%s: NULL argument", what);
    if (re->nreacs < 1 || re->nreacs > kMaxReacs)
        return flame_fail(FLAME_EUNSUPPORTED, "%s: %d reactions (1..%d supported)", what,
                          re->nreacs, kMaxReacs);
    if (stiff && transposed && g->ns + 35 > 7 * FLAME_MAX_NS)
        return flame_fail(FLAME_EINVAL, "%s: transposed read outside coeffs_lo", what);
    const Dims D = make_dims(*g);
    const Mech M{re->nreacs, re->atm, re->reaction_type, re->sgm, re->vf, re->vr,
                 re->Arr, re->ef, re->loP, re->Troe};
    const long long ncell = (long long)D.nx * D.ny * D.nz;
    const unsigned blocks = (unsigned)((ncell + 127) / 128);
    if (stiff)
        k_eval<true><<<blocks, 128, 0, s>>>(D, U, Q, rhoi, dt, *th, M, tag, Tcrit, transposed);
    else
        k_eval<false><<<blocks, 128, 0, s>>>(D, U, Q, rhoi, dt, *th, M, tag, Tcrit, 0);
    return flame_check_launch(what);
}

}  // namespace chem
}  // namespace flame

extern "C" int flame_eval_gpu(const FlameGrid *g, flame_stream_t s, double *U, double *Q,
                              double *rhoi, double dt, const FlameThermo *thermo,
                              const FlameReactions *react, const int64_t *tag, double T_criteria) {
    return flame::chem::launch(false, g, s, U, Q, rhoi, dt, thermo, react, tag, T_criteria, 0,
                               "flame_eval_gpu");
}

extern "C" int flame_eval_gpu_stiff(const FlameGrid *g, flame_stream_t s, double *U, double *Q,
                                    double *rhoi, double dt, const FlameThermo *thermo,
                                    const FlameReactions *react, const int64_t *tag,
                                    double T_criteria, int transposed) {
    return flame::chem::launch(true, g, s, U, Q, rhoi, dt, thermo, react, tag, T_criteria,
                               transposed, "flame_eval_gpu_stiff");
}
