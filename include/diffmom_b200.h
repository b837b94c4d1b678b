/*
 * diffmom_b200.h -- C ABI of the B200 library for DiffMoM.jl's dense
 * surface-EFIE hot path (libdiffmom_b200.so).
 *
 * Plain C types only: pointers, sizes, doubles.  Complex arrays are
 * interleaved (re, im) doubles in Julia's ComplexF64 layout; matrices are
 * column-major.  Index arrays are Julia's 1-based Int64.  Every entry point
 * returns a dmb_status; dmb_last_error() holds the message of the last
 * failure on that context.
 *
 * Status codes map onto the Julia exceptions the reference raises:
 *   DMB_ERR_ARGUMENT   -> ArgumentError      (invalid input, e.g. EFIE.jl:297-330)
 *   DMB_ERR_OVERFLOW   -> OverflowError      (non-finite results)
 *   DMB_ERR_DIMENSION  -> DimensionMismatch
 *   DMB_ERR_BUDGET     -> ArgumentError      (resource limit, Types.jl:85)
 *   DMB_ERR_NOT_CONVERGED -> ErrorException  (IterativeSolve.jl:50-61)
 *   DMB_ERR_BREAKDOWN  -> SingularException  (factorisation pivot failure)
 *   DMB_ERR_CUDA / DMB_ERR_STATE / DMB_ERR_TIMEOUT -> ErrorException
 *
 * Thread safety: calls on one context are serialised by a context mutex;
 * contexts are independent.  All entry points block until their device work
 * has finished unless stated otherwise.
 */
#ifndef DIFFMOM_B200_H
#define DIFFMOM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dmb_ctx dmb_ctx;
typedef int dmb_status;

#define DMB_OK 0
#define DMB_ERR_ARGUMENT 1
#define DMB_ERR_OVERFLOW 2
#define DMB_ERR_DIMENSION 3
#define DMB_ERR_BUDGET 4
#define DMB_ERR_NOT_CONVERGED 5
#define DMB_ERR_CUDA 6
#define DMB_ERR_STATE 7
#define DMB_ERR_BREAKDOWN 8
#define DMB_ERR_TIMEOUT 9

/* precision of the impedance matrix */
#define DMB_PREC_FP64 0  /* FP64 everywhere, complex128 Z */
#define DMB_PREC_MIXED 1 /* FP32 far pairs, FP64 singular terms, complex64 Z */

/* preconditioner kinds */
#define DMB_PRECOND_NONE 0
#define DMB_PRECOND_NF_LU 1      /* near-field matrix, exact factorisation */
#define DMB_PRECOND_NF_DIAG 2    /* Jacobi on the diagonal, 1e-10*max floor */
#define DMB_PRECOND_LOCAL_INV 3  /* per-RWG near-block local inverses */
#define DMB_PRECOND_LEARNED 4    /* learned correction of the local inverses */
#define DMB_PRECOND_RING 5       /* plain ring-step correction of the local inverses */

#define DMB_SIDE_LEFT 0
#define DMB_SIDE_RIGHT 1

typedef struct {
  int32_t niter;        /* Arnoldi steps taken (max over right-hand sides) */
  int32_t solved;       /* 1 when every right-hand side met the tolerance */
  double residual;      /* last residual estimate (max over RHS), relative */
  double true_residual; /* ||b - Z x|| / ||b|| in FP64 (max over RHS) */
  int32_t restarts;     /* restart / refinement cycles */
  int32_t reserved;     /* times the true-residual check continued a left-
                           preconditioned cycle (DMB_OPT_TRUE_RESIDUAL) */
} dmb_gmres_stats;

typedef struct {
  double geometry_ms;   /* cache precompute (areas, quadrature, RWG values) */
  double assembly_ms;   /* impedance matrix assembly */
  double precond_ms;    /* preconditioner build */
  double rhs_ms;        /* excitation assembly */
  double solve_ms;      /* GMRES / direct solve */
  double nnz_ratio;     /* near-field fill of the last preconditioner */
  int64_t kernels;      /* kernels launched by this context so far */
  double gmres_ms;      /* the GMRES part alone (resident solves put their total in solve_ms) */
} dmb_timings;

/* ---- context ----------------------------------------------------------- */
/* No reference counterpart: owns device buffers, stream and error text. */
dmb_status dmb_ctx_create(int device, dmb_ctx **out);
dmb_status dmb_ctx_destroy(dmb_ctx *ctx);
/* ctx == NULL: the message of the calling thread's last failed call that
 * takes no context (dmb_aca_plan, dmb_aca_admissible). */
const char *dmb_last_error(const dmb_ctx *ctx);
dmb_status dmb_get_timings(dmb_ctx *ctx, dmb_timings *out);
/* Library version string, e.g. "diffmom_b200 0.1 sm_100a". */
const char *dmb_version(void);

/* Implementation options (no reference counterpart).
 * DMB_OPT_TENSOR_CORES: 1 (default) runs the complex64 factorisation update on
 * the tcgen05 tensor cores (3xTF32), 0 on FP32 SIMT units.
 * DMB_OPT_TC_MIN_RHS: from this many right-hand sides (default 64) a complex64
 * Z X (dmb_matvec and the GMRES operator) and the panel updates of the batched
 * near-field solves run on the tensor cores (3xTF32, FP32 accumulation); GMRES
 * then confirms convergence on the FP64 residual and refines where needed. */
#define DMB_OPT_TENSOR_CORES 1
#define DMB_OPT_TC_MIN_RHS 2
/* DMB_OPT_FAR_TILE: width T of the RWG tiles of the assembly's far-pair
 * kernel (one CTA per T x T block of Z): 16 or 32 for FP64, 32 or 64 for
 * mixed precision; 0 (default) lets the autotuner pick it per mesh-size
 * bucket (each width timed once per process).  Every width writes the same
 * bits. */
#define DMB_OPT_FAR_TILE 3
/* DMB_OPT_EXACT_KRYLOV: 1 (default) runs the many-RHS GMRES operator on the
 * FP64-accurate INT8-slice product (no refinement cycle needed); 0 runs it in
 * 3xTF32 with FP64-residual refinement. */
#define DMB_OPT_EXACT_KRYLOV 4
/* DMB_OPT_PRECOND_TF32_TERMS: products per complex MAC in the tensor-core
 * updates of the complex64 factorisation and in the batched triangular sweeps
 * that apply it: 3 (default, hi*hi + hi*lo + lo*hi) or 1 (hi*hi only, a third
 * of the tensor-core work); the pieces are TF32 or BF16 (DMB_OPT_PRECOND_BF16).  Only the
 * preconditioner changes; right-preconditioned GMRES keeps the preconditioned
 * vectors (flexible form), so the solution accuracy is unaffected. */
#define DMB_OPT_PRECOND_TF32_TERMS 5
/* DMB_OPT_GMRES_GRAPHS: 1 (default) replays the GMRES iterations between two
 * host convergence checks of solves with fewer than 32 right-hand sides as
 * captured CUDA graphs (captured the second time an iteration range is met
 * with the same problem shape and device buffers, replayed afterwards); 0
 * launches every kernel directly.  Results are identical either way.  The
 * lanes of dmb_batch_* contexts launch directly. */
#define DMB_OPT_GMRES_GRAPHS 6
/* DMB_OPT_OPERATOR: the operator of dmb_matvec / dmb_gmres / dmb_gmres_adjoint:
 * 0 the assembled dense Z, 1 the H-matrix of dmb_aca_build (each build or
 * assembly selects its own; switching drops the preconditioner). */
#define DMB_OPT_OPERATOR 7
/* DMB_OPT_TRUE_RESIDUAL: 1 (default) makes the unpreconditioned FP64 residual
 * ||b - Z x|| / ||b|| the convergence test of dmb_gmres / dmb_gmres_adjoint and the
 * resident solves.  For left preconditioning (Krylov.gmres stops on the
 * preconditioned residual, IterativeSolve.jl:364-384) the trial solution is
 * checked when a system's estimate meets the tolerance, and a system whose
 * true residual does not continues the same Arnoldi process with a lower
 * threshold; a system that still misses it after its cycle (basis capacity,
 * inexact operator) is refined by further cycles from its current iterate.
 * All within maxiter; a system counts as solved only once its true residual
 * meets the tolerance.  0 stops exactly where Krylov.gmres stops (iteration
 * counts of the reference). */
#define DMB_OPT_TRUE_RESIDUAL 8
/* DMB_OPT_SPIN_LIMIT: polls a waiting CTA of the chained triangular sweeps
 * (complex128 factors, and 2-7 right-hand sides of complex64 ones) makes
 * before it gives up; the call then fails with DMB_ERR_TIMEOUT and the context
 * stays usable.  A negative value restores the default (2e7 polls, seconds);
 * small values exercise the timeout path without any GPU fault. */
#define DMB_OPT_SPIN_LIMIT 9
/* DMB_OPT_TUNE_TC_GEMM / DMB_OPT_TUNE_TC_SYRK: pin a candidate of the online
 * autotuner (0, the default, lets it choose): the tile width of the
 * tensor-core sweep GEMMs (1: 256, 2: 128 complex columns per tile; 3:
 * persistent grid of 256-column tiles, double-buffered accumulators) and the schedule of
 * the complex64 factor updates (1: 4 stages, one CTA per SM; 2: 2 stages, two
 * CTAs per SM; 3: persistent grid over the lower tiles only, double-buffered
 * accumulators).  Unpinned, each launch shape bucket runs every candidate on
 * its first real calls, timed with events, and keeps the fastest for the
 * process; the candidates give the same bits. */
#define DMB_OPT_TUNE_TC_GEMM 10
#define DMB_OPT_TUNE_TC_SYRK 11
/* DMB_OPT_PRECOND_BF16: the operands of the complex64 factor updates and of
 * the packed many-RHS sweeps as BF16 pieces (hi + lo, ~16 bits, the three
 * products on the kind::f16 tensor-core path at twice the TF32 rate, FP32
 * accumulation) instead of TF32 pieces (~21 bits).  1: always; 0: never; -1
 * (default): inside the resident solves only (dmb_solve_resident,
 * dmb_solve_resident_many, dmb_batch_solve), whose GMRES is checked on the FP64
 * residual, so the preconditioner's precision changes the iteration count,
 * not the result; dmb_nf_build / dmb_nf_apply / dmb_gmres keep TF32 pieces. */
#define DMB_OPT_PRECOND_BF16 12
/* DMB_OPT_INT8_SCHEME: how the FP64-accurate complex64 Z X (refinement and
 * true residuals, the exact Krylov operator) is made of exact int8
 * tensor-core products.  0 (default): residues modulo 13 pairwise coprime
 * moduli <= 256 of Z and X scaled to 44-bit integers, one int8 product per
 * modulus, recombined by the Chinese remainder theorem as a 96-bit fixed-point
 * fraction of the moduli's product (13 products, 12 for the Krylov operator).
 * 1: seven-bit fixed-point slices, products of slice pairs up to a level
 * (26 products, 21 for the Krylov operator).  Both are deterministic and
 * agree with the FP64 product to ~1e-12 normwise. */
#define DMB_OPT_INT8_SCHEME 13
/* DMB_OPT_TUNE_INT8_TILE: pin the tile shape of the residue-scheme int8
 * product (0, the default, lets the online autotuner choose per shape
 * bucket): 1: one SM per 64 x 256 complex output tile (M 128 int8 MMA);
 * 2: a CTA pair (two SMs of a cluster, tcgen05 cta_group::2, M 256 MMA) per
 * 128 x 256 complex tile, each SM loading half of the right-hand operand.
 * Both give the same bits. */
#define DMB_OPT_TUNE_INT8_TILE 14
dmb_status dmb_set_option(dmb_ctx *ctx, int option, int value);
/* The far-pair RWG tile width used by the last assembly on this context. */
dmb_status dmb_get_far_tile(dmb_ctx *ctx, int *width_out);
/* The autotuner's measurements and choices so far (all contexts of the
 * process), one line per (device, kernel family, shape bucket); writes at
 * most cap - 1 characters and a terminating zero, *len_out = full length.
 * No reference counterpart. */
dmb_status dmb_tune_report(char *buf, size_t cap, size_t *len_out);

/* ---- mesh and basis ---------------------------------------------------- */
/* TriMesh (src/Types.jl:123-126): xyz 3 x Nv column-major, tri 3 x Nt
 * 1-based.  Replaces the host-side cache geometry of _build_efie_cache
 * (src/assembly/EFIE.jl:332-398). */
dmb_status dmb_mesh_upload(dmb_ctx *ctx, const double *xyz, const int64_t *tri, int64_t nv,
                           int64_t nt);
/* RWGData (src/Types.jl:138-152, built by src/basis/RWG.jl:102-143).
 * evert is 2 x N column-major 1-based. */
dmb_status dmb_rwg_upload(dmb_ctx *ctx, int64_t n, const int64_t *tplus, const int64_t *tminus,
                          const int64_t *evert, const int64_t *vplus_opp,
                          const int64_t *vminus_opp, const double *len,
                          const double *area_plus, const double *area_minus);

/* ---- impedance matrix -------------------------------------------------- */
/* assemble_Z_efie (src/assembly/EFIE.jl:699-753).  Z stays resident on the
 * device; when Z_out is non-NULL the N x N ComplexF64 matrix is also copied
 * out (column-major).  precision: DMB_PREC_FP64 or DMB_PREC_MIXED. */
dmb_status dmb_assemble_z(dmb_ctx *ctx, double k, double eta0, int quad_order, int precision,
                          double *Z_out);
/* Copy selected entries of the resident Z (1-based m, n); for efie_entry
 * (src/assembly/EFIE.jl:1002-1007). */
dmb_status dmb_z_entries(dmb_ctx *ctx, const int64_t *m, const int64_t *n, int64_t count,
                         double *out);
/* Impedance loading Z -= sum_t zs[t] M_t (src/assembly/Impedance.jl:304-408,
 * src/solver/Solve.jl:1412-1449 with one patch per triangle). zs: Nt complex. */
dmb_status dmb_apply_impedance(dmb_ctx *ctx, const double *zs);

/* ---- operators --------------------------------------------------------- */
/* Dense Z*x (the zgemv inside Krylov.gmres) for nrhs column-major
 * right-hand sides: y = Z x.  FP64 accumulation; for a complex64 Z with many
 * right-hand sides on the tensor cores: the FP64-accurate INT8-slice product
 * (nrhs >= 32, DMB_OPT_EXACT_KRYLOV on) or 3xTF32 (nrhs >= DMB_OPT_TC_MIN_RHS,
 * ~2e-5 relative). */
dmb_status dmb_matvec(dmb_ctx *ctx, const double *x, double *y, int64_t nrhs);
/* (After dmb_aca_build, dmb_matvec applies the context's H-matrix instead.) */
/* Matrix-free Z*x (MatrixFreeEFIEOperator mul!, src/assembly/EFIE.jl:867-909):
 * entries are recomputed from the geometry on every call, nothing of size
 * N^2 is stored.  Requires a prior dmb_assemble_z or dmb_prepare_operator. */
dmb_status dmb_prepare_operator(dmb_ctx *ctx, double k, double eta0, int quad_order);
/* The near-field entries are added with atomics, so repeated products agree
 * to rounding (about 1e-15 relative), not bit for bit. */
dmb_status dmb_matvec_free(dmb_ctx *ctx, const double *x, double *y);
/* No counterpart in the reference.  The same matrix-free product for callers
 * that cannot allocate device memory mid-run (device memory owned by an
 * external pool, or a fixed budget that forbids allocation after set-up):
 * x_dev and y_dev are DEVICE pointers to N complex128 values, and the call
 * allocates nothing -- its slot-space scratch is a static device array of
 * 3 MiB held by every GPU that loads the library until exit.  Meshes with more
 * than 32,768 triangles are rejected with DMB_ERR_BUDGET.  Every call looks up
 * that array's device address (cudaGetSymbolAddress, which allocates nothing)
 * with the context's device current; the first lookup on a device may load
 * the module, so make the first call before any stream capture.  Not for use
 * across a reset of the device (cudaDeviceReset) by another part of the
 * process while a call is running.  All calls share the array and
 * it keeps the last call's contents, so calls that overlap on the GPU (other
 * contexts or threads on the same device at the same time) race.  Requires a
 * prior dmb_prepare_operator (or dmb_assemble_z) on the context. */
dmb_status dmb_matvec_free_noalloc(dmb_ctx *ctx, const double *x_dev, double *y_dev);

/* ---- near-field preconditioner ---------------------------------------- */
/* build_nearfield_preconditioner(Z, mesh, rwg, cutoff; factorization)
 * (src/solver/NearFieldPreconditioner.jl:670-758).  kind: DMB_PRECOND_NF_LU
 * or DMB_PRECOND_NF_DIAG.  nnz_ratio_out may be NULL. */
dmb_status dmb_nf_build(dmb_ctx *ctx, double cutoff, int kind, double *nnz_ratio_out);
/* NearFieldOperator apply y = Z_nf^-1 x (NearFieldPreconditioner.jl:1034-1054). */
dmb_status dmb_nf_apply(dmb_ctx *ctx, const double *x, double *y, int64_t nrhs);

/* ---- local-inverse and learned preconditioners ------------------------- */
/* No reference counterpart (the near-field preconditioner above is their
 * fallback).  dmb_local_build: per-RWG near blocks (the <= 64 nearest RWG
 * centres within `radius`) are solved exactly; their rows form a sparse right
 * preconditioner (DMB_PRECOND_LOCAL_INV).  The "ring" of m is the rest of its
 * 2x-radius neighbourhood E_m (<= 128); the ring residual of a row z is
 * r = Z[E_m, S_m] z - e_m.
 *   mode 0: local inverse rows.
 *   mode 1: local inverse + one exactly line-searched ring-residual step along
 *           g (1 + o), g = Z[E,S]^H r, o the trained network's per-entry
 *           modulation (DMB_PRECOND_LEARNED).
 *   mode 2: least-squares rows min || Z[E_m, S_m] z - e_m || (the exact rows
 *           the network is trained toward).
 *   mode 3: local inverse + one plain line-searched ring step (o = 0)
 *           (DMB_PRECOND_RING): the learned method without its network. */
dmb_status dmb_local_build(dmb_ctx *ctx, double radius, int mode);
/* Train the network on the current body (resident Z): features of the
 * local-inverse rows and their ring gradients as input; targets from the
 * least-squares rows (exact local block solves the method generates); Adam
 * over minibatches; mean loss of the last epoch in loss_out.  Weights persist
 * in the context across bodies. */
dmb_status dmb_net_train(dmb_ctx *ctx, double radius, int epochs, int batch, double lr, uint64_t seed,
                         double *loss_out);
/* Flat FP32 weight vector (save/load/check): count, get, set. */
int dmb_net_param_count(void);
dmb_status dmb_net_get(dmb_ctx *ctx, float *w);
dmb_status dmb_net_set(dmb_ctx *ctx, const float *w);
/* Loss and gradient of the network for caller-supplied rows (gradient check):
 * feat nrows x 64 x 13, tgt nrows x 64 x 2, per-entry weights nrows x 64,
 * cnt nrows (1..64).  loss = mean over rows of sum_j w_j |out_j - tgt_j|^2. */
dmb_status dmb_net_loss_grad(dmb_ctx *ctx, const float *feat, const float *tgt, const float *wgt,
                             const int *cnt, int64_t nrows, float *grad, float *loss);

/* ---- excitation -------------------------------------------------------- */
/* assemble_plane_wave / assemble_multiple_excitations for R plane waves
 * (src/assembly/Excitation.jl:2738-2797, 2866-2896).  kvecs, pols: 3 x R
 * column-major, E0s: R.  V_out: N x R complex column-major. */
dmb_status dmb_rhs_plane_waves(dmb_ctx *ctx, const double *kvecs, const double *E0s,
                               const double *pols, int64_t R, int quad_order, double *V_out);
/* assemble_dipole / assemble_loop (src/assembly/Excitation.jl:2924-2985) for R
 * sources: positions R x 3, complex moments R x 3 (re, im interleaved: R x 6
 * doubles), magnetic[r] 0 = electric (C m), 1 = magnetic (A m^2; a loop of
 * radius a, current I and normal n is the magnetic dipole I pi a^2 n),
 * frequencies R (Hz; k = 2 pi f sqrt(eps0 mu0) as the reference).  V_out
 * N x R column-major. */
dmb_status dmb_rhs_dipoles(dmb_ctx *ctx, int64_t R, const double *positions, const double *moments,
                           const int *magnetic, const double *frequencies, int quad_order, double *V_out);
/* assemble_pattern_feed (src/assembly/Excitation.jl:3044-3071) with the field
 * of _pattern_feed_field_unchecked (:1417-1460): E = exp(-ikR)/R (F_theta
 * e_theta + F_phi e_phi) about phase_center[3], k = 2 pi frequency /
 * 299792458, F bilinear on the (theta, phi) grid (radians; theta clamped,
 * phi periodic).  Ftheta, Fphi: ntheta x nphi column-major complex (re, im
 * interleaved).  conj_convention = 1 for exp(-i omega t) coefficients
 * (:exp_minus_iwt).  Grid rules of _validate_pattern_grid (:999-1025).
 * V_out: N complex values. */
dmb_status dmb_rhs_pattern_feed(dmb_ctx *ctx, int ntheta, const double *theta, int nphi, const double *phi,
                                const double *Ftheta, const double *Fphi, double frequency,
                                const double *phase_center, int conj_convention, int quad_order, double *V_out);

/* ---- impedance gradients ----------------------------------------------- */
/* gradient_impedance(Mp, I, lambda; reactive) (src/optimization/Adjoint.jl:
 * 1081-1119) with Mp = precompute_patch_mass(mesh, rwg, partition;
 * quad_order) (src/assembly/Impedance.jl:304-377), for R (I, lambda) pairs:
 * g[p + r P] = 2 Re(lambda_r^H M_p I_r), or -2 Im(...) with reactive = 1.
 * tri_patch: nt 0-based patch ids (PatchPartition.tri_patch - 1); I, lambda:
 * N x R column-major complex (re, im interleaved); g_out: P x R doubles.
 * The patch mass entries are evaluated on the fly per triangle. */
dmb_status dmb_gradient_impedance(dmb_ctx *ctx, int64_t R, const double *I, const double *lambda,
                                  const int *tri_patch, int64_t P, int reactive, int quad_order, double *g_out);

/* ---- solvers ----------------------------------------------------------- */
/* solve_gmres (src/solver/IterativeSolve.jl:341-392): GMRES without
 * restart (Krylov.gmres, memory grows), rtol=tol, atol=0, left or right
 * preconditioner, nrhs independent right-hand sides solved as a block.
 * rhs, x: N x nrhs column-major.  Returns DMB_ERR_NOT_CONVERGED (x still
 * written) when check_convergence != 0 and a system did not converge. */
dmb_status dmb_gmres(dmb_ctx *ctx, const double *rhs, double *x, int64_t nrhs, double tol,
                     int maxiter, int precond_kind, int precond_side, int check_convergence,
                     dmb_gmres_stats *stats);
/* solve_gmres_adjoint (IterativeSolve.jl:409-470) with NearFieldAdjointOperator
 * (NearFieldPreconditioner.jl:1237): GMRES on Z^H x = rhs.  Z (and its
 * near-field matrix) is complex symmetric, so this is the conjugate of the
 * forward solve with conj(rhs); the near-field preconditioners only (none,
 * NF_LU, NF_DIAG). */
dmb_status dmb_gmres_adjoint(dmb_ctx *ctx, const double *rhs, double *x, int64_t nrhs, double tol, int maxiter,
                             int precond_kind, int precond_side, int check_convergence, dmb_gmres_stats *stats);
/* solve_forward(Z, v; solver=:direct) (src/solver/Solve.jl:1342-1382):
 * factorisation of the resident Z plus FP64 iterative refinement. */
dmb_status dmb_solve_direct(dmb_ctx *ctx, const double *rhs, double *x, int64_t nrhs,
                            double *backward_error_out);

/* ---- whole solve, device resident ------------------------------------- */
/* solve_scattering(mesh, freq, plane wave; method=:dense_gmres) body
 * (src/Workflow.jl:160-317) on the uploaded mesh/RWG: assemble Z at
 * `precision`, build the preconditioner (kind; near-field cutoff in metres),
 * assemble the plane-wave RHS, run GMRES to `tol`.  The current vector stays
 * on the device (dmb_copy_solution fetches it). */
typedef struct {
  double k, eta0, cutoff, tol;
  int32_t quad_order, precision, precond_kind, precond_side, maxiter, reserved;
  double kvec[3], pol[3], E0;
} dmb_solve_params;
dmb_status dmb_solve_resident(dmb_ctx *ctx, const dmb_solve_params *p, dmb_gmres_stats *stats);
/* Many incidences at once: the per-column loop over
 * assemble_multiple_excitations (src/assembly/Excitation.jl:2738-2797) with
 * solve_scattering's dense GMRES, and backscatter_rcs
 * (src/postprocessing/Diagnostics.jl:460-517) of each solution.  Z and the
 * preconditioner are built once, the R right-hand sides (kvecs, pols R x 3
 * row-major, E0s R; p->kvec/pol/E0 are ignored) are solved by block GMRES,
 * and, when sigma_out is non-NULL, sigma_out[r] = 4 pi |E_inf(-k_hat_r)|^2 /
 * |E0_r|^2 is computed on the device (only these R values are copied back).
 * The N x R currents stay on the device. */
dmb_status dmb_solve_resident_many(dmb_ctx *ctx, const dmb_solve_params *p, int64_t R, const double *kvecs,
                                   const double *E0s, const double *pols, double *sigma_out,
                                   dmb_gmres_stats *stats);
/* Copy the resident currents (N x 1, or N x R after dmb_solve_resident_many,
 * column-major complex128). */
dmb_status dmb_copy_solution(dmb_ctx *ctx, double *I_out);

/* ---- many independent surfaces ------------------------------------------ */
/* No single reference call: the loop of solve_scattering (src/Workflow.jl:
 * 67-317) over independent bodies, each with its own mesh and RWG basis, an
 * optional per-triangle surface impedance (assemble_full_Z with
 * precompute_patch_mass, Impedance.jl:304-408) and its own plane wave, plus
 * backscatter_rcs (Diagnostics.jl:460-517).  A batch keeps one device context
 * per surface of a call (reused, buffers grow only).  dmb_batch_solve
 * uploads the surfaces on `lanes` host threads, then assembles EVERY
 * surface's impedance matrix with one far-pair tile launch (a task list of
 * all surfaces' RWG tile pairs, largest surface first) and one launch each
 * for the near values and near sums, and then runs the per-surface stages
 * (impedance loading, preconditioner, right-hand side, GMRES, sigma) on the
 * `lanes` host threads, largest surface first, each surface on its own
 * stream.  The solve of each surface follows dmb_solve_resident with `p`
 * (kvec/pol/E0 of p are ignored).  The batch holds the device memory of its
 * largest call until dmb_batch_destroy. */
typedef struct dmb_batch dmb_batch;
typedef struct {
  /* inputs: host arrays in the layouts of dmb_mesh_upload / dmb_rwg_upload */
  const double *xyz;
  const int64_t *tri;
  int64_t nv, nt;
  int64_t n;
  const int64_t *tplus, *tminus, *evert, *vplus_opp, *vminus_opp;
  const double *len, *area_plus, *area_minus;
  const double *zs;       /* nt complex surface impedances (re, im interleaved), or NULL for PEC */
  double kvec[3], pol[3], E0;
  /* outputs */
  double *I_out;          /* n complex currents, or NULL */
  double sigma;           /* monostatic RCS at -k_hat */
  dmb_gmres_stats stats;
  double latency_ms;      /* device time from the batch start to the end of this surface */
  double solve_ms;        /* device time of this surface's stages after the batch-wide assembly */
} dmb_batch_item;
dmb_status dmb_batch_create(int device, int lanes, dmb_batch **out);
dmb_status dmb_batch_destroy(dmb_batch *b);
const char *dmb_batch_last_error(const dmb_batch *b);
/* Device time of the last dmb_batch_solve's batch-wide assembly (the far
 * tiles, near values and near sums of all its surfaces). */
dmb_status dmb_batch_assembly_ms(const dmb_batch *b, double *ms_out);
/* device_ms_out (may be NULL): device time of the whole batch. */
dmb_status dmb_batch_solve(dmb_batch *b, const dmb_solve_params *p, dmb_batch_item *items, int64_t count,
                           double *device_ms_out);

/* ---- measurement hooks -------------------------------------------------- */
/* No reference counterpart.  The CUDA stream the context launches on (a
 * cudaStream_t), for events recorded by the caller. */
dmb_status dmb_get_stream(dmb_ctx *ctx, void **stream_out);
/* When enabled, the context brackets every launch of its dominant kernel
 * (the factorisation trailing update) with CUDA events and accumulates the
 * device time, launch count and algorithmic FLOPs. */
dmb_status dmb_set_kernel_timing(dmb_ctx *ctx, int enable);
dmb_status dmb_kernel_timing(dmb_ctx *ctx, double *ms, int64_t *launches, double *flops);
/* Same per kernel family: 0 = tensor-core 3xTF32 Krylov and triangular-sweep
 * GEMMs (work in complex flops, 8 per complex MAC), 1 = INT8-slice
 * FP64-accurate GEMMs (work in int8 multiply-adds x 2), 2 = factorisation
 * trailing updates (3xTF32 tensor cores for complex64 factors; complex flops),
 * 3 = H-matrix products of dmb_aca_build's operator (one bracket per
 * right-hand side: gather, low-rank inner products, leaf sums; work in bytes:
 * the stored blocks plus x and y once), 4 = FP64-pipe complex128 GEMMs (Z X
 * of a complex128 Z with >= 16 right-hand sides and the many-column sweep
 * updates of a complex128 factor; complex flops), 5 = far-pair tiles of the
 * assembly (work in bytes of Z written: N^2 x 16 for complex128, x 8 for
 * complex64).  dmb_kernel_timing reports family 0. */
dmb_status dmb_kernel_timing_family(dmb_ctx *ctx, int family, double *ms, int64_t *launches, double *work);

/* ---- H-matrix operator (adaptive cross approximation) ------------------ */
/* Block plan of build_aca_operator without a GPU: the cluster tree of
 * build_cluster_tree (src/fast/ClusterTree.jl:82-166; median bisection along
 * the longest bounding-box axis, stable sort) and the block tasks of
 * _enum_block_tasks! (src/fast/ACA.jl:696-738) with is_admissible
 * (src/fast/ClusterTree.jl:223-246, exact decision near the boundary).
 * centers: n x 3 row-major points.  perm_out (n, may be NULL): tree order ->
 * original index, 1-based.  nodes_out (5 per node: first, last (1-based tree
 * order), left, right (1-based node ids, 0 = leaf), level) and boxes_out
 * (6 per node: bbox_min, bbox_max) may be NULL; *n_nodes_out gets the count.
 * tasks_out (5 per task: row node, col node (1-based ids), kind 0 = dense,
 * 1 = low-rank, 0, 0) is written when tasks_cap >= the count, which
 * *n_tasks_out always receives.  Errors: dmb_last_error(NULL). */
dmb_status dmb_aca_plan(const double *centers, int64_t n, int leaf_size, double eta, int64_t max_block_tasks,
                        int64_t *perm_out, int64_t *n_nodes_out, int64_t *nodes_out, double *boxes_out,
                        int64_t *n_tasks_out, int64_t *tasks_out, int64_t tasks_cap);
/* is_admissible(tree, i, j; eta) (src/fast/ClusterTree.jl:223-246) for two
 * boxes given as (bbox_min, bbox_max) 6-vectors; *out = 0 or 1. */
dmb_status dmb_aca_admissible(const double *box_i, const double *box_j, double eta, int *out);

typedef struct {
  int64_t n_dense;          /* dense (inadmissible) blocks, fallbacks included */
  int64_t n_lowrank;        /* low-rank blocks */
  int64_t n_fallback;       /* admissible blocks stored dense after a non-finite ACA update */
  int64_t max_rank_used;    /* largest rank of a low-rank block */
  int64_t entries_stored;   /* complex entries held (dense data + U + V at their ranks) */
  int64_t n_unconverged;    /* low-rank blocks that reached max_rank without meeting tol */
  double build_ms;          /* host + device time of the build */
  double plan_ms;           /* of which: cache, tree and block tasks on the host */
  double dense_ms;          /*           dense block fill */
  double lowrank_ms;        /*           ACA of the admissible blocks */
} dmb_aca_info;
/* build_aca_operator(mesh, rwg, k; leaf_size, eta, aca_tol, max_rank,
 * quad_order, eta0, max_block_tasks, max_storage_bytes)
 * (src/fast/ACA.jl:802-1103) on the device: dense blocks filled with the
 * FP64 EFIE entries, admissible blocks compressed by partially pivoted ACA
 * (aca_lowrank, src/fast/ACA.jl:351-554) with the reference's relative
 * Frobenius stopping rule.  The context's operator becomes this H-matrix:
 * dmb_gmres / dmb_gmres_adjoint use it until the next dmb_assemble_z. */
dmb_status dmb_aca_build(dmb_ctx *ctx, double k, double eta0, int quad_order, int leaf_size, double eta,
                         double aca_tol, int max_rank, int64_t max_block_tasks, int64_t max_storage_bytes,
                         dmb_aca_info *info_out);
/* mode 0: y = A x (mul!, src/fast/ACA.jl:1130-1221); 1: y = A^H x
 * (ACAAdjointOperator, :1231-1323); 2: y = A^T x.  nrhs column-major
 * right-hand sides, host buffers. */
dmb_status dmb_aca_matvec(dmb_ctx *ctx, const double *x, double *y, int64_t nrhs, int mode);
/* Blocks in task order, 7 per block: kind (0 dense, 1 low-rank), first row,
 * last row, first column, last column (1-based tree order), rank (low-rank)
 * or 0, 1 when the block is a dense fallback of an admissible task. */
dmb_status dmb_aca_blocks(dmb_ctx *ctx, int64_t *out);
/* Data of block b (0-based, task order): dense: a_out = m x n column-major;
 * low-rank: a_out = U (m x rank), b_out = V (n x rank), block = U V^H. */
dmb_status dmb_aca_block_data(dmb_ctx *ctx, int64_t b, double *a_out, double *b_out);
/* getindex(A::ACAOperator, i, j) (src/fast/ACA.jl:220-222): EFIE entries
 * evaluated on the device (1-based m, n). */
dmb_status dmb_aca_entries(dmb_ctx *ctx, const int64_t *m, const int64_t *n, int64_t count, double *out);
/* The operator's tree permutation (tree order -> original index, 1-based;
 * may be NULL) and the RWG centres it was built on (n x 3 row-major; may be
 * NULL). */
dmb_status dmb_aca_tree(dmb_ctx *ctx, int64_t *perm_out, double *centers_out);
/* aca_lowrank(cache, row_indices, col_indices; tol, max_rank,
 * max_output_bytes) (src/fast/ACA.jl:351-554) on one block of RWG index lists
 * (1-based) with the EFIE entries of (k, eta0, quad_order).  U_out (m x r) and
 * V_out (n x r) must hold min(max_rank, m, n) columns; *rank_out = r.  A
 * non-finite update fails with DMB_ERR_OVERFLOW. */
dmb_status dmb_aca_lowrank(dmb_ctx *ctx, double k, double eta0, int quad_order, const int64_t *rows, int64_t m,
                           const int64_t *cols, int64_t n, double tol, int max_rank, int64_t max_output_bytes,
                           double *U_out, double *V_out, int64_t *rank_out);
/* build_nearfield_preconditioner(A_aca; factorization)
 * (src/solver/NearFieldPreconditioner.jl:952-1000): the near-field matrix is
 * the union of the operator's dense blocks.  kind: DMB_PRECOND_NF_LU or
 * DMB_PRECOND_NF_DIAG; precision: DMB_PREC_FP64 (complex128 factor) or
 * DMB_PREC_MIXED (complex64 factor on the tensor cores). */
dmb_status dmb_aca_nf_build(dmb_ctx *ctx, int kind, int precision, double *nnz_ratio_out);

/* ---- far field --------------------------------------------------------- */
/* radiation_vectors + compute_farfield (src/postprocessing/FarField.jl:
 * 425-611): E_out is 3 x NO x nrhs complex for directions rhat (3 x NO). */
dmb_status dmb_farfield(dmb_ctx *ctx, const double *rhat, int64_t NO, double k, double eta0,
                        int quad_order, const double *I, int64_t nrhs, double *E_out);

#ifdef __cplusplus
}
#endif
#endif /* DIFFMOM_B200_H */
