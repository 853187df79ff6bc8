/*
 * flame3d_b200.h — C ABI of libflame3d_b200.so, the sm_100a (B200) implementation of
 * Flame3D.jl's per-stage right-hand side on curvilinear grids and its SSP-RK3 stage update.
 *
 * Conventions (shared by every entry point):
 *   - Arrays are the reference's Julia arrays, column-major with i fastest, SoA by variable:
 *     ghosted point (i, j, k, n), 0-based, lives at  i + Tx*(j + Ty*(k + Tz*n))  with
 *     Tx = nx + 2*ng, Ty = ny + 2*ng, Tz = nz + 2*ng.  Face arrays are unghosted with one extra
 *     face along the swept axis: an x-face array is (nx+1, ny, nz, NV), face f lies between
 *     ghosted cells ng+f-1 and ng+f.  Same shapes as solver.jl:141-167.
 *   - All floating point arrays are FP64 device pointers owned by the caller (Julia CuArray or
 *     torch tensor); the library only borrows them for the duration of the (asynchronous) call.
 *   - `tag` is the IBM tag field (Int64, solver.jl:123).  NULL means "all fluid" (tag == 0),
 *     which is the only value the fused entry points accept.
 *   - Every call is asynchronous on `stream` (NULL = legacy default stream) and returns
 *     FLAME_OK or an error code; flame_last_error() gives the message of the calling thread.
 *   - Global state of the library: a per-thread error string; per device, atomic flags
 *     recording that a kernel's dynamic shared-memory limit has been raised (set once, never
 *     cleared; host threads on different streams may call concurrently); the
 *     persistent batch's constant-memory descriptor table (one per device, see flame_batch_*);
 *     and, used only by flame_rk_stage_noalloc, a library-held scratch array with its
 *     per-device address cache (described at that entry point).  No call allocates device
 *     memory.
 *
 * The argument order after (grid, stream) is the argument order of the reference kernel each
 * entry point replaces, so a Julia `ccall` is a mechanical rewrite of the `@cuda` launch.
 */
#ifndef FLAME3D_B200_H
#define FLAME3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *flame_stream_t; /* identical to cudaStream_t */

#define FLAME_NG 4      /* ghost layers; parse_mesh.jl:5 */
/* Largest species count: every 1:1 entry point and the fills take 1..FLAME_MAX_NS species; the
 * fused stage (flame_rk_stage*, flame_transport, flame_rk_stage_noalloc) and the batches are
 * compiled for 1..FLAME_FUSED_MAX_NS and return FLAME_EUNSUPPORTED above (the reference's CH4
 * mechanism, 21 species, runs on the 1:1 path only once FLAME_MAX_NS is raised). */
#define FLAME_MAX_NS 16
#define FLAME_FUSED_MAX_NS 9

enum {
    FLAME_OK = 0,
    FLAME_EINVAL = 1,      /* bad argument (NULL pointer, size, ng != 4, ns out of range) */
    FLAME_ELAUNCH = 2,     /* CUDA reported an error at launch */
    FLAME_ETIMEOUT = 3,    /* a bounded device wait gave up */
    FLAME_ENONFINITE = 4,  /* a non-finite conserved value was detected */
    FLAME_EUNSUPPORTED = 5 /* valid request this build does not implement */
};

/* Grid extents; the reference keeps these as compile-time constants (run.jl:59-63). */
typedef struct FlameGrid {
    int32_t nx, ny, nz; /* interior cells (Nxp, Ny, Nz) */
    int32_t ng;         /* ghost layers, must be FLAME_NG */
    int32_t ns;         /* species count (Nspecs), 1..FLAME_MAX_NS */
    int32_t periodic;   /* bit 0/1/2: x/y/z periodic (ghost fill and fused stage) */
} FlameGrid;

/* NASA-7 thermodynamics; the by-value counterpart of thermoProperty (run.jl:71-82).
 * coeffs_lo / coeffs_hi are the Julia (7, ns) matrices, column-major: [a + 7*n]. */
typedef struct FlameThermo {
    double Ru;       /* J/(mol K) */
    double min_temp; /* K */
    double max_temp; /* K */
    int32_t ns;
    int32_t pad;
    double mw[FLAME_MAX_NS];         /* kg/mol */
    double coeffs_sep[FLAME_MAX_NS]; /* K, switch between the low and high range */
    double coeffs_lo[7 * FLAME_MAX_NS];
    double coeffs_hi[7 * FLAME_MAX_NS];
} FlameThermo;

/* Transport law (thermo.jl:289-403).
 *   law 0: mu = mu_ref, lambda = lambda_ref, D_k = D_ref (constants)
 *   law 1: mu = mu_ref * (T / T_ref)^exponent, lambda = cp * mu / Pr with cp the mass-specific
 *          mixture heat capacity, D_k = lambda / (rho * cp) for every species (unity Lewis).
 *   law 2: the reference's mixture-averaged properties, mixtureProperties thermo.jl:289-369:
 *          Mathur lambda, Wilke mu and mixture-averaged D_k from the log(T) polynomial fits
 *          that initThermo takes from Cantera (thermo.jl:405-436), here supplied by the
 *          caller in `poly`: visc_poly (5, ns), conduct_poly (5, ns), binarydiff_poly
 *          (5, ns, ns), each column-major as in thermoProperty, back to back (10 ns + 5 ns^2
 *          doubles, device memory for the GPU entry points).  Laws 0 and 1 run everywhere;
 *          law 2 runs on the per-kernel path (flame_mixture) and on the fused stage's pencil
 *          configurations 3-6, whose transport fields then hold one D_k per species. */
typedef struct FlameTransport {
    int32_t law;
    int32_t pad;
    double mu_ref, T_ref, exponent, Pr, lambda_ref, D_ref;
    const double *poly; /* law 2 only */
} FlameTransport;

/* Curvilinear metrics (J^-1-scaled cofactors, parse_mesh.jl:210-221) and J, all ghosted. */
typedef struct FlameMetrics {
    const double *dxidx, *dxidy, *dxidz;
    const double *detadx, *detady, *detadz;
    const double *dzetadx, *dzetady, *dzetadz;
    const double *J;
} FlameMetrics;

/* ---------------------------------------------------------------------------------------
 * 1:1 replacements of the reference kernels (same index ranges, same arithmetic).
 * ------------------------------------------------------------------------------------- */

/* schemes.jl:1-24  shockSensor(ϕ, Q) */
int flame_shockSensor(const FlameGrid *g, flame_stream_t stream, double *phi, const double *Q);

/* split.jl:17-89  fluxSplit(Q, Fp, Fm, Ax, Ay, Az, tag); Fp/Fm are ghosted (…, 5) */
int flame_fluxSplit(const FlameGrid *g, flame_stream_t stream, const double *Q, double *Fp,
                    double *Fm, const double *Ax, const double *Ay, const double *Az,
                    const int64_t *tag);

/* split.jl:101-130  split(ρi, Q, Fp, Fm, Ax, Ay, Az, tag); Fp/Fm are ghosted (…, ns) */
int flame_split(const FlameGrid *g, flame_stream_t stream, const double *rhoi, const double *Q,
                double *Fp, double *Fm, const double *Ax, const double *Ay, const double *Az,
                const int64_t *tag);

/* schemes.jl:86-437  WENO_x/y/z(F, ϕ, Fp, Fm, NV, tag): hybrid UP7 / WENO-Z5 / minmod */
int flame_WENO_x(const FlameGrid *g, flame_stream_t stream, double *F, const double *phi,
                 const double *Fp, const double *Fm, int NV, const int64_t *tag);
int flame_WENO_y(const FlameGrid *g, flame_stream_t stream, double *F, const double *phi,
                 const double *Fp, const double *Fm, int NV, const int64_t *tag);
int flame_WENO_z(const FlameGrid *g, flame_stream_t stream, double *F, const double *phi,
                 const double *Fp, const double *Fm, int NV, const int64_t *tag);

/* viscous.jl:1-428  viscousFlux_x/y/z(Fv, Q, dξdx, dξdy, dξdz, dηdx, dηdy, dηdz, dζdx, dζdy,
 * dζdz, J, λ, μ, Fh, tag): the reference's argument list (viscous.jl:1, 144, 287), the nine
 * J^-1-scaled metric cofactors and J as separate ghosted arrays.  Fv is (faces, 4). */
int flame_viscousFlux_x(const FlameGrid *g, flame_stream_t stream, double *Fv, const double *Q,
                        const double *dxidx, const double *dxidy, const double *dxidz,
                        const double *detadx, const double *detady, const double *detadz,
                        const double *dzetadx, const double *dzetady, const double *dzetadz,
                        const double *J, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag);
int flame_viscousFlux_y(const FlameGrid *g, flame_stream_t stream, double *Fv, const double *Q,
                        const double *dxidx, const double *dxidy, const double *dxidz,
                        const double *detadx, const double *detady, const double *detadz,
                        const double *dzetadx, const double *dzetady, const double *dzetadz,
                        const double *J, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag);
int flame_viscousFlux_z(const FlameGrid *g, flame_stream_t stream, double *Fv, const double *Q,
                        const double *dxidx, const double *dxidy, const double *dxidz,
                        const double *detadx, const double *detady, const double *detadz,
                        const double *dzetadx, const double *dzetady, const double *dzetadz,
                        const double *J, const double *lambda, const double *mu,
                        const double *Fh, const int64_t *tag);

/* viscous.jl:430-665  specViscousFlux_x/y/z(Fd, Q, Yi, dξdx, dξdy, dξdz, dηdx, dηdy, dηdz,
 * dζdx, dζdy, dζdz, J, D, Fh, thermo, tag): the reference's argument list (viscous.jl:430, 509,
 * 588).  Fd is (faces, ns), Fh (faces, 3) is written. */
int flame_specViscousFlux_x(const FlameGrid *g, flame_stream_t stream, double *Fd,
                            const double *Q, const double *Yi, const double *dxidx,
                            const double *dxidy, const double *dxidz, const double *detadx,
                            const double *detady, const double *detadz, const double *dzetadx,
                            const double *dzetady, const double *dzetadz, const double *J,
                            const double *D, double *Fh, const FlameThermo *thermo,
                            const int64_t *tag);
int flame_specViscousFlux_y(const FlameGrid *g, flame_stream_t stream, double *Fd,
                            const double *Q, const double *Yi, const double *dxidx,
                            const double *dxidy, const double *dxidz, const double *detadx,
                            const double *detady, const double *detadz, const double *dzetadx,
                            const double *dzetady, const double *dzetadz, const double *J,
                            const double *D, double *Fh, const FlameThermo *thermo,
                            const int64_t *tag);
int flame_specViscousFlux_z(const FlameGrid *g, flame_stream_t stream, double *Fd,
                            const double *Q, const double *Yi, const double *dxidx,
                            const double *dxidy, const double *dxidz, const double *detadx,
                            const double *detady, const double *detadz, const double *dzetadx,
                            const double *dzetady, const double *dzetadz, const double *J,
                            const double *D, double *Fh, const FlameThermo *thermo,
                            const int64_t *tag);

/* div.jl:16-54  div(U, Fx, Fy, Fz, Fv_x, Fv_y, Fv_z, dt, J, tag): U += J dt (−ΔF + ΔFv) */
int flame_div(const FlameGrid *g, flame_stream_t stream, double *U, const double *Fx,
              const double *Fy, const double *Fz, const double *Fv_x, const double *Fv_y,
              const double *Fv_z, double dt, const double *J, const int64_t *tag);

/* div.jl:61-84  divSpecs(ρi, Fx, Fy, Fz, Fd_x, Fd_y, Fd_z, dt, J, tag) */
int flame_divSpecs(const FlameGrid *g, flame_stream_t stream, double *rhoi, const double *Fx,
                   const double *Fy, const double *Fz, const double *Fd_x, const double *Fd_y,
                   const double *Fd_z, double dt, const double *J, const int64_t *tag);

/* utils.jl:95-112  linComb(U, Un, NV, a, b, tag): U = a U + b Un on interior points */
int flame_linComb(const FlameGrid *g, flame_stream_t stream, double *U, const double *Un,
                  int NV, double a, double b, const int64_t *tag);

/* utils.jl:2-48 (+ thermo.jl:231-282 GetT)  c2Prim(U, Q, ρi, thermo, tag) */
int flame_c2Prim(const FlameGrid *g, flame_stream_t stream, const double *U, double *Q,
                 double *rhoi, const FlameThermo *thermo, const int64_t *tag);

/* utils.jl:71-92  prim2c(U, Q) over all ghosted points */
int flame_prim2c(const FlameGrid *g, flame_stream_t stream, double *U, const double *Q);

/* thermo.jl:371-403  mixture(Q, ρi, Yi, λ, μ, D, thermo, tag) with the FlameTransport law in
 * place of Cantera's fits; Yi = max(ρi / max(ρ, eps), 0) exactly as the reference. */
int flame_mixture(const FlameGrid *g, flame_stream_t stream, const double *Q, const double *rhoi,
                  double *Yi, double *lambda, double *mu, double *D, const FlameThermo *thermo,
                  const FlameTransport *transport, const int64_t *tag);

/* Periodic ghost fill of `nv` ghosted fields (new: the reference's fills, boundary.jl:1-191,
 * are case-specific inflow / zero-gradient; all benchmark cases are periodic). */
int flame_fill_periodic(const FlameGrid *g, flame_stream_t stream, double *A, int nv);

/* boundary.jl:193-279  fillIB(Q, U, ρi, neari, nearj, neark, c_d, c_n, tag, thermo): at every
 * immersed-boundary ghost point (tag == 3) Y and p take the zero-gradient value -Σ c_n[m+1] f_m
 * / c_n[1] and u, v, w the Dirichlet value with c_d over the 15 stencil points (neari / nearj /
 * neark: (15, Tx, Ty, Tz) Int64, 1-based as in Julia; c_d, c_n: (16, Tx, Ty, Tz)); T is the wall
 * temperature (300 K in the reference, here T_wall); ρ from ρmixture, then ρi, e, Q and U.  The
 * stencil points are read while ghost points are written, so, as in the reference, a stencil
 * must not contain another ghost point for the result to be defined. */
int flame_fillIB(const FlameGrid *g, flame_stream_t stream, double *Q, double *U, double *rhoi,
                 const int64_t *neari, const int64_t *nearj, const int64_t *neark,
                 const double *c_d, const double *c_n, const int64_t *tag,
                 const FlameThermo *thermo, double T_wall);

/* The inflow state of the reference's fills.  fill_x / fill_z hard-code it (boundary.jl:17-25,
 * 96-104): P = 79.8 Pa, T = 270.65 K, u = 1000 m/s, v = w = 0, Y(2) = 0.233, Y(5) = 0.767
 * (1-based species), every other Y zero; here the caller passes it. */
typedef struct FlameInflow {
    double P, T, u, v, w;
    double Y[FLAME_MAX_NS];
} FlameInflow;

/* boundary.jl:1-52  fill_x(Q, U, ρi, Yi, thermo, rank): on the first x-slab rank the planes
 * i <= NG+1 (1-based; the first interior plane included) take the inflow state (ρ from
 * ρmixture, thermo.jl:29-35; e from InternalEnergy), on the last rank the planes i >= Nxp+NG
 * copy Q, U, ρi from i = Nxp+NG-1.  One GPU: rank 0 of nprocs 1. */
int flame_fill_x(const FlameGrid *g, flame_stream_t stream, double *Q, double *U, double *rhoi,
                 double *Yi, const FlameThermo *thermo, const FlameInflow *inflow, int rank,
                 int nprocs);

/* boundary.jl:54-80  fill_y(Q, U): j <= NG+1 copy j = NG+2, j >= Ny+NG copy j = Ny+NG-1. */
int flame_fill_y(const FlameGrid *g, flame_stream_t stream, double *Q, double *U);

/* boundary.jl:82-137  fill_z(Q, U, ρi, Yi, thermo): k <= NG+1 inflow (as fill_x), k >= Nz+NG
 * copy Q, U from k = Nz+NG-1. */
int flame_fill_z(const FlameGrid *g, flame_stream_t stream, double *Q, double *U, double *rhoi,
                 double *Yi, const FlameThermo *thermo, const FlameInflow *inflow);

/* boundary.jl:139-158  fill_y_s(ρi): the fill_y rule on ρi. */
int flame_fill_y_s(const FlameGrid *g, flame_stream_t stream, double *rhoi);

/* boundary.jl:160-176  fill_z_s(ρi): k >= Nz+NG copy k = Nz+NG-1. */
int flame_fill_z_s(const FlameGrid *g, flame_stream_t stream, double *rhoi);

/* boundary.jl:180-184  fillGhost: fill_x, fill_y, fill_z in that order on the stream. */
int flame_fillGhost(const FlameGrid *g, flame_stream_t stream, double *Q, double *U,
                    double *rhoi, double *Yi, const FlameThermo *thermo,
                    const FlameInflow *inflow, int rank, int nprocs);

/* boundary.jl:188-191  fillSpec: fill_y_s, fill_z_s. */
int flame_fillSpec(const FlameGrid *g, flame_stream_t stream, double *rhoi);

/* reactionProperty (run.jl:84-94), the mechanism initReact builds (reactions.jl:506-575), for the
 * grid's ns species and nreacs reactions.  Every array is device memory in Julia's column-major
 * layout: reaction_type (nreacs: 1 Arrhenius, 2 three-body, 3 falloff-Troe), sgm (nreacs:
 * reactant minus product stoichiometric sum), vf / vr (ns, nreacs: stoichiometric coefficients),
 * Arr (3, nreacs: A in m, mol, s units, b, E/R in K), ef (ns, nreacs: third-body efficiencies),
 * loP (3, nreacs: the low-pressure Arrhenius of falloff reactions), Troe (4, nreacs). */
typedef struct FlameReactions {
    int32_t nreacs;
    int32_t pad;
    double atm; /* Pa */
    const int64_t *reaction_type, *sgm, *vf, *vr;
    const double *Arr, *ef, *loP, *Troe;
} FlameReactions;

/* reactions.jl:187-232  eval_gpu(U, Q, ρi, dt, thermo, react, tag): explicit finite-rate
 * chemistry on the interior cells hotter than T_criteria (a constant in run.jl:12): ρi += ẇ W
 * dt, U[5] gains the formation-enthalpy release, ρi is clipped and rescaled to ρ, then T (GetT),
 * p and e of Q are updated.  thermo needs the full NASA-7 set (a7 enters the Gibbs energy). */
int flame_eval_gpu(const FlameGrid *g, flame_stream_t stream, double *U, double *Q,
                   double *rhoi, double dt, const FlameThermo *thermo,
                   const FlameReactions *react, const int64_t *tag, double T_criteria);

/* reactions.jl:235-309  eval_gpu_stiff(…): the point-implicit form, (I − A dt) Δρ = ẇ W dt with
 * the production-rate Jacobian A (vproductionRate_Jac, :383-462) solved by Gaussian elimination
 * with partial pivoting (:465-504).  The reference reads the formation coefficient as
 * coeffs_lo[n, 6] here but coeffs_lo[6, n] in eval_gpu; transposed = 1 reproduces the former
 * (the linear element n + 35 of the 7 x ns matrix), 0 uses coeffs_lo[6, n] as eval_gpu does. */
int flame_eval_gpu_stiff(const FlameGrid *g, flame_stream_t stream, double *U, double *Q,
                         double *rhoi, double dt, const FlameThermo *thermo,
                         const FlameReactions *react, const int64_t *tag, double T_criteria,
                         int transposed);

/* solver.jl:388-391  `any(isnan, U)` every 10 steps, as a count: writes to the device unsigned
 * *count how many of the nv ghosted FP64 fields' values are NaN or infinite (the reference
 * tests NaN only; an infinity is as fatal).  The caller reads it and stops the case, the
 * reference's "Oops, NaN detected" (FLAME_ENONFINITE on the host side). */
int flame_check_finite(const FlameGrid *g, flame_stream_t stream, const double *A, int nv,
                       unsigned int *count);

/* Largest per-cell CFL rate max over interior cells of Σ_d J (|m_d·u| + c |m_d|), with m_d the
 * stored metric rows (dξ/dx … scaled by 1/J), c = sqrt(γ p / ρ) and γ = p/e + 1 (split.jl:40-41),
 * written to the device double *out (a stable time step is dt = CFL / *out).  New: the reference
 * runs a fixed dt (run.jl:30).  Deterministic: the maximum does not depend on reduction order. */
int flame_cfl_max(const FlameGrid *g, flame_stream_t stream, const double *Q,
                  const FlameMetrics *m, double *out);

/* solver.jl:22-38  flowAdvance(U, Q, Fp, Fm, Fx, Fy, Fz, Fv_x, Fv_y, Fv_z, dξdx, dξdy, dξdz,
 * dηdx, dηdy, dηdz, dζdx, dζdy, dζdz, J, dt, ϕ, λ, μ, Fhx, Fhy, Fhz, tag): fluxSplit+WENO per
 * direction, viscousFlux ×3, div.  Fp/Fm are ghosted (…,5) scratch; Fx/Fy/Fz face (…,5);
 * Fv_* face (…,4); Fh* face (…,3). */
int flame_flowAdvance(const FlameGrid *g, flame_stream_t stream, double *U, const double *Q,
                      double *Fp, double *Fm, double *Fx, double *Fy, double *Fz, double *Fv_x,
                      double *Fv_y, double *Fv_z, const double *dxidx, const double *dxidy,
                      const double *dxidz, const double *detadx, const double *detady,
                      const double *detadz, const double *dzetadx, const double *dzetady,
                      const double *dzetadz, const double *J, double dt, const double *phi,
                      const double *lambda, const double *mu, const double *Fhx,
                      const double *Fhy, const double *Fhz, const int64_t *tag);

/* solver.jl:40-56  specAdvance(ρi, Q, Yi, Fp_i, Fm_i, Fx_i, Fy_i, Fz_i, Fd_x, Fd_y, Fd_z, dξdx,
 * dξdy, dξdz, dηdx, dηdy, dηdz, dζdx, dζdy, dζdz, J, dt, ϕ, D, Fhx, Fhy, Fhz, thermo, tag):
 * split+WENO per direction, specViscousFlux ×3, divSpecs. */
int flame_specAdvance(const FlameGrid *g, flame_stream_t stream, double *rhoi, const double *Q,
                      const double *Yi, double *Fp_i, double *Fm_i, double *Fx_i, double *Fy_i,
                      double *Fz_i, double *Fd_x, double *Fd_y, double *Fd_z,
                      const double *dxidx, const double *dxidy, const double *dxidz,
                      const double *detadx, const double *detady, const double *detadz,
                      const double *dzetadx, const double *dzetady, const double *dzetadz,
                      const double *J, double dt, const double *phi, const double *D,
                      double *Fhx, double *Fhy, double *Fhz, const FlameThermo *thermo,
                      const int64_t *tag);

/* ---------------------------------------------------------------------------------------
 * Fused path: one RK3 stage in one to seven launches (solver.jl:297-326, IBM off).
 * Reads Q_in / rhoi_in / trans_in (ghosts filled), writes U in place and Q_out / rhoi_out /
 * trans_out on the interior cells and, along every periodic axis (FlameGrid::periodic), their
 * ghost images, so the caller swaps every in/out pair after each stage.  On an axis that is not
 * periodic the stage writes interior cells only, and the caller fills the ghosts of the result
 * as the reference does after c2Prim (solver.jl:321-325): flame_fillGhost on (Q_out, U,
 * rhoi_out), flame_fillSpec on rhoi_out, then flame_transport_boundary on (Q_out, rhoi_out,
 * trans_out) for the points the fills changed (FP64 storage, precision 0: the fills are FP64).
 * Stage 1 also writes Un = U and rhon = rhoi (solver.jl:299-302).
 * trans_* hold the transport of the state, (…, 3) = μ, λ, D, as computed by flame_transport;
 * with law 2 (mixture-averaged, per-species D_k) they are (…, 2 + ns) = μ, λ, D_0 .. D_{ns-1}.
 * The stage computes the next one in its epilogue, so the law is evaluated once per cell.
 * Q_* and trans_* are double arrays for precision 0 and float arrays for precision 1.
 * ------------------------------------------------------------------------------------- */
typedef struct FlameStageBuffers {
    double *U;             /* (…,5) conserved, interior updated in place */
    double *Un;            /* (…,5) RK3 stage-0 copy */
    const void *Q_in;      /* (…,7) primitives of the stage input, ghosts filled */
    void *Q_out;           /* (…,7) primitives of the stage result, ghosts filled */
    const double *rhoi_in; /* (…,ns) partial densities of the stage input, ghosts filled */
    double *rhoi_out;      /* (…,ns) partial densities of the stage result, ghosts filled */
    double *rhon;          /* (…,ns) RK3 stage-0 copy */
    const void *trans_in;  /* (…,3) μ, λ, D of the stage input; law 2: (…,2+ns) */
    void *trans_out;       /* (…,3) μ, λ, D of the stage result; law 2: (…,2+ns) */
    void *scratch;         /* flame_stage_scratch_bytes() bytes for configurations 3 to 6,
                              else unused (may be NULL); contents need not survive calls */
    const void *metrics_lo; /* optional, precision 1 and configurations 3-4: the ten metric
                               fields rounded once to float, back to back in FlameMetrics
                               order (10 x ghosted points); NULL rounds them at every load.
                               The FP64 metrics are still read for J in the RK3 update. */
} FlameStageBuffers;

/* stage in {1,2,3}; precision 0 = plain FP64, 1 = mixed (FP32 storage of Q and transport, FP32
 * split / reconstruction with its WENO-Z weights / viscous fluxes and, with law 2, the mixture
 * rule; FP64 conserved accumulation, metrics and Newton temperature).  No reference counterpart: it replaces the launch sequence
 * of solver.jl:298-326. */
int flame_rk_stage(const FlameGrid *g, flame_stream_t stream, int stage, double dt,
                   const FlameStageBuffers *b, const FlameMetrics *m, const FlameThermo *thermo,
                   const FlameTransport *transport, int precision);

/* flame_rk_stage with an explicit configuration: 0, 1, 2 = one tile kernel per stage (16x8x8
 * with one CTA per SM, 16x8x8 with two, 8x8x8 with two); 3 = four barrier-free launches
 * (a prep pass and z, y, x warp-per-pencil sweeps, the x sweep finishing the stage) that need
 * b->scratch; 4 = configuration 3 with the finish (RK3 update, c2Prim, transport, ghosts) in a
 * fifth, per-cell launch, bit-identical to 3; 5, 6 = configurations 3, 4 with each y / z sweep
 * split into a flow sweep and a species sweep (fewer registers and shared-memory slots per
 * sweep when there are many species).  The autotuner picks the configuration per grid,
 * species count and precision.  Transport law 2 runs on configurations 3-6, always with
 * configuration 6's launches (its species sweeps and x sweep read each species' D_k, and the
 * finish evaluates the mixture rule per cell); configurations 0-2 refuse it with
 * FLAME_EUNSUPPORTED. */
int flame_rk_stage_tiled(const FlameGrid *g, flame_stream_t stream, int stage, double dt,
                         const FlameStageBuffers *b, const FlameMetrics *m,
                         const FlameThermo *thermo, const FlameTransport *transport,
                         int precision, int tile);

/* Bytes of scratch the pencil configurations need: 2 (5 + ns) doubles (the right-hand side of
 * the z sweep and of the y sweep) and (1 + ns) values of the storage type per ghosted point. */
size_t flame_stage_scratch_bytes(const FlameGrid *g, int precision);

/* No counterpart in the reference.  The pencil-sweep stage (configuration 3) for callers that
 * cannot allocate device memory for it: a Julia program whose device memory all belongs to
 * CUDA.jl's pool, or a serving process that has committed its whole HBM budget, must not have
 * the library cudaMalloc for them, and an allocation can synchronize the device.  The scratch
 * lives in one array of FLAME_NOALLOC_SCRATCH_BYTES (64 MiB) that the library's GPU code holds
 * on every device it is loaded on until the process exits; b->scratch is ignored.  Grids whose
 * flame_stage_scratch_bytes() exceeds it are rejected with FLAME_EINVAL (FP64, ns = 1: up to
 * about 600 thousand ghosted points).  The first call on a device looks up the array's address
 * with that device current, so make it before any stream capture; the address is then cached
 * for the life of the process, so cudaDeviceReset between calls is not supported (the array
 * may come back at another address).  All calls on a device share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  Nothing in the array has to
 * start at zero; allocates nothing. */
#define FLAME_NOALLOC_SCRATCH_BYTES (64u << 20)
int flame_rk_stage_noalloc(const FlameGrid *g, flame_stream_t stream, int stage, double dt,
                           const FlameStageBuffers *b, const FlameMetrics *m,
                           const FlameThermo *thermo, const FlameTransport *transport,
                           int precision);

/* μ, λ, D of every ghosted point of a state (Q, rhoi) into trans (…, 3), or (…, 2 + ns) with
 * law 2: the transport law of flame_mixture without the mass-fraction output; starts the fused
 * stage loop. */
int flame_transport(const FlameGrid *g, flame_stream_t stream, const void *Q, const double *rhoi,
                    void *trans, const FlameThermo *thermo, const FlameTransport *transport,
                    int precision);

/* flame_transport restricted to the points a ghost fill can change on a grid that is not
 * periodic on every axis: on each non-periodic axis the ghost layers and the first and last
 * interior planes (the planes the reference's fill_x / fill_y / fill_z and fill_y_s / fill_z_s
 * overwrite, boundary.jl:1-176).  Nothing to do on a fully periodic grid.  New: the reference
 * recomputes the whole mixture every stage (solver.jl:304). */
int flame_transport_boundary(const FlameGrid *g, flame_stream_t stream, const void *Q,
                             const double *rhoi, void *trans, const FlameThermo *thermo,
                             const FlameTransport *transport, int precision);

/* ---------------------------------------------------------------------------------------
 * Batches (no reference counterpart): many independent periodic cases, each with its own
 * grid, species count, thermodynamics, transport (laws 0, 1 and 2), dt and buffers, advanced
 * together by persistent kernels.  Cases are grouped by species count and transport family
 * (laws 0 and 1, or law 2) and cut into chunks of at most 20; per chunk and stage the chunk's
 * descriptors go into a constant-memory table and the persistent kernels run one after the
 * other on the stream, each over its part of a (case, block) work list.  Laws 0 and 1 take
 * configuration 3's shape, two kernels: the prep, z-sweep and y-sweep blocks of every case of
 * the chunk in list order, a case's sweep blocks waiting on a device counter for that case's
 * prep blocks; then the x-sweep blocks, which finish the stage.  Law 2 takes configuration 6's
 * shape, four: prep and flow-only sweeps (with the same waits), the species sweeps, the x
 * sweeps, and the finish with the mixture rule.  Every wait is bounded: when one runs out
 * (about half a second) the batch's error word is set and the remaining items are skipped;
 * flame_batch_status reports it.  The constant table is one per device: persistent batches on
 * one device must not run concurrently.  Descriptors and work lists for all stages and both
 * in/out parities go once into caller-owned device workspace, so a captured CUDA graph of
 * flame_batch_stage calls replays without host work.  parity 0 advances buf.*_in -> buf.*_out,
 * parity 1 the other way.  Every case needs buf.scratch (flame_stage_scratch_bytes).  A
 * case's result is the same as when it runs alone: cases share no data and no reduction.
 * ------------------------------------------------------------------------------------- */
typedef struct FlameCaseDesc {
    FlameGrid grid;
    double dt;
    FlameStageBuffers buf;
    FlameMetrics metrics;
    FlameThermo thermo;
    FlameTransport transport;
} FlameCaseDesc;

typedef struct FlameBatch FlameBatch; /* opaque host-side plan */

size_t flame_batch_workspace_bytes(const FlameCaseDesc *cases, int n, int precision);
int flame_batch_create(FlameBatch **out, const FlameCaseDesc *cases, int n, int precision,
                       void *workspace, size_t bytes, flame_stream_t stream);
int flame_batch_stage(FlameBatch *batch, flame_stream_t stream, int stage, int parity);
/* Synchronizes `stream` and returns FLAME_ETIMEOUT (and clears it) if a wait of an earlier
 * flame_batch_stage ran out, else FLAME_OK. */
int flame_batch_status(FlameBatch *batch, flame_stream_t stream);
/* Test hook: with on != 0, the next stages make the first case of every chunk wait for one
 * more prep block than exists, a completion that never comes, so its waits run out and
 * flame_batch_status reports FLAME_ETIMEOUT (a host-side injection; nothing faults). */
int flame_batch_test_stall(FlameBatch *batch, int on);
int flame_batch_destroy(FlameBatch *batch);

/* Message of the last error on the calling thread; returns its length. */
int flame_last_error(char *buf, size_t n);

/* ABI version (major*10000 + minor*100 + patch). */
int flame_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FLAME3D_B200_H */
