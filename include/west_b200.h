/*
 * west_b200 — B200-native Wstat dielectric-response operator, C ABI.
 *
 * Drop-in boundary: WEST's
 *     SUBROUTINE apply_operator(m, dvg, dng, tr2, iq)      Wstat/apply_operator.f90:14
 * which applies dng = sqvc * chi0(sqvc * dvg) to m perturbations by solving
 * Gamma-point Sternheimer equations (DFPT_kernel/dfpt_module.f90:22).
 *
 * All entry points are extern "C", take plain pointers and sizes, never abort
 * and report errors as negative status codes with a message available from
 * wb_last_error().  Complex arrays are interleaved (re, im) doubles, i.e.
 * Fortran COMPLEX(DP) / C double _Complex, column-major with an explicit
 * leading dimension.  A Fortran caller binds them with iso_c_binding.
 */
#ifndef WEST_B200_H
#define WEST_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define WB_OK 0
#define WB_ERR_ARG (-1)         /* invalid argument or inconsistent system data */
#define WB_ERR_CUDA (-2)        /* a CUDA call failed */
#define WB_ERR_UNSUPPORTED (-3) /* valid in WEST but not provided here (k-points, non-cubic box...) */
#define WB_ERR_NOMEM (-4)       /* device allocation failed */

#define WB_PRECISION_FP64 0
#define WB_PRECISION_MIXED 1

typedef struct wb_ctx wb_ctx;

/*
 * Ground-state data that dfpt reads from QE/WEST modules.  Every pointer is a
 * host pointer and is only read during wb_ctx_create (the context keeps
 * device copies).  Field-by-field origin in WEST/QE:
 */
typedef struct wb_system {
  int npw;             /* pwcom npw = ngk(1) = westcom npwq at Gamma              */
  int npwx;            /* leading dimension of evc and vkb (pwcom npwx)           */
  int nr1, nr2, nr3;   /* dffts%nr1..nr3 (a cubic box: all three equal)           */
  int nbnd_occ;        /* westcom nbnd_occ(1)                                     */
  int nkb;             /* uspp nkb                                                */
  int n_dfpt_maxiter;  /* westcom n_dfpt_maxiter                                  */
  int l_kinetic_only;  /* westcom l_kinetic_only (k_psi instead of h_psi)         */
  int gstart;          /* gvect gstart: must be 2 (this process holds G=0)        */
  const int* nl;       /* [npw] dffts%nl, 1-based box index of +G                 */
  const int* nlm;      /* [npw] dffts%nlm, 1-based box index of -G                */
  const double* g2kin; /* [npw] wvfct g2kin (Ry)                                  */
  const double* vrs;   /* [nr1*nr2*nr3] scf vrs(:,1) on the smooth grid (Ry)      */
  const double* evc;   /* [npwx, nbnd_occ] complex: wavefunctions evc             */
  const double* et;    /* [nbnd_occ] wvfct et(:,1) (Ry)                           */
  const double* occupation; /* [nbnd_occ] westcom occupation(:,1); bands below
                               1 - 1e-3 are fractionally occupied (l_frac_occ,
                               dfpt_module.f90:328-401, set_nbndocc.f90:58-69) */
  const double* vkb;   /* [npwx, nkb] complex: uspp vkb after init_us_2           */
  const double* deeq;  /* [nkb, nkb] KB coupling D, dense (block-diagonal per atom) */
  const double* sqvc;  /* [npw] pot3D%sqvc (Coulomb_kernel/class_coulomb.f90:173) */
  double alpha_pv;     /* westcom alphapv_dfpt (Tools/get_alpha_pv.f90)           */
  double omega;        /* cell_base omega (bohr^3)                                */
  double wk;           /* k_grid%weight(1) (QE wk; 2 for a spin-unpolarised Gamma) */
} wb_system;

/* Pipeline stages timed by wb_set_profiling (CUDA events on the library's stream). */
#define WB_STAGE_VLOC_ZINV 0   /* local potential: sphere -> sticks, inverse z FFT   */
#define WB_STAGE_VLOC_PLANE 1  /* local potential: x-y FFTs, V(r) product, back      */
#define WB_STAGE_VLOC_ZFWD 2   /* local potential: forward z FFT, unpack, kinetic    */
#define WB_STAGE_GEMM_TN 3     /* <W|X> bra-ket GEMM (calbec, Pv, Pc)                */
#define WB_STAGE_GEMM_REDUCE 4 /* split-K reduction, Gamma G=0 term, D / alpha       */
#define WB_STAGE_GEMM_NN 5     /* W C accumulation (add_vuspsi, Pv, Pc)              */
#define WB_STAGE_CG 6          /* PCG vector steps and compaction                    */
#define WB_STAGE_RHS 7         /* dv(r), psi_v dv products, forward FFTs             */
#define WB_STAGE_DRHO 8        /* density response and its forward FFT               */
#define WB_STAGE_OTHER 9       /* permutation, Pc, preconditioner, copies            */
#define WB_NSTAGES 10

/* Counters of the last wb_apply_operator call. */
typedef struct wb_stats {
  int m;                   /* perturbations processed                         */
  int cg_iterations;       /* PCG iterations of the longest chunk             */
  long long cg_active_sum; /* sum over iterations of active (pert, band) systems */
  long long fft_boxes;     /* complex 3D box transforms performed             */
  long long launches;      /* kernel launches issued by the library           */
  double ms_total;         /* device time of the call (ms, CUDA events)       */
  double stage_ms[WB_NSTAGES];          /* per-stage device time (profiling on) */
  long long stage_launches[WB_NSTAGES]; /* per-stage kernel launches            */
  long long stage_items[WB_NSTAGES];    /* per-stage work items (FFT boxes, columns) */
  int refinements;         /* FP64 refinement steps (mixed form), 0 in FP64 */
} wb_stats;

/*
 * Create a context on CUDA device `device` and upload the ground state.
 * Replaces the setup part of dfpt (dfpt_module.f90:93-225: allocations,
 * set_eprec, et/eprec gathering) and QE's FFT/projector setup.
 */
int wb_ctx_create(wb_ctx** ctx, const wb_system* sys, int device);

/* Release all device memory of the context. */
int wb_ctx_destroy(wb_ctx* ctx);

/*
 * The drop-in for apply_operator (Wstat/apply_operator.f90:14-69).
 *   m            number of perturbations (columns)
 *   dvg          [ld_dvg, m] complex, host memory, IN
 *   dng          [ld_dng, m] complex, host memory, OUT (rows >= npw set to 0)
 *   tr2          PCG threshold on <r|M^-1 r>; tr2 < 0 = lite solver (no PCG),
 *                dfpt_module.f90:130,350
 *   iq           q-point index; only 1 (Gamma) is provided
 *   unconverged  [m] OUT (may be NULL): bands left unconverged per
 *                perturbation (dfpt's ierr, dfpt_module.f90:356-359)
 * Synchronous: returns when dng is written.
 */
int wb_apply_operator(wb_ctx* ctx, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng, double tr2,
                      int iq, int* unconverged);

/* Same contract with dvg and dng in device memory of the context's device. */
int wb_apply_operator_device(wb_ctx* ctx, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng,
                             double tr2, int iq, int* unconverged);

/*
 * WB_PRECISION_FP64 (default): every step in FP64, the reference's arithmetic.
 * WB_PRECISION_MIXED: the Sternheimer PCG runs in FP32 (FFTs, projector GEMMs,
 * vector updates) as correction solves inside an FP64 iterative refinement:
 * the residual b - A x and its preconditioned norm <r|M^-1 r> are formed in
 * FP64 and each system stops on the same tr2 test as the FP64 form.
 */
int wb_set_precision(wb_ctx* ctx, int mode);

/* Upper bound on perturbations processed per device batch (0 = automatic). */
int wb_set_batch(wb_ctx* ctx, int max_perturbations);

int wb_get_stats(const wb_ctx* ctx, wb_stats* out);

/* Bit mask of the WB_STAGE_* stages to time with CUDA events (bit s = stage s);
 * 0 = off (default), WB_PROFILE_ALL = every stage. */
#define WB_PROFILE_ALL ((1 << WB_NSTAGES) - 1)
int wb_set_profiling(wb_ctx* ctx, int stage_mask);

/*
 * Several ground states in one call (uneven cells, bands and batch sizes):
 * context i maps dvg[i] [ld_dvg[i], m[i]] to dng[i] exactly as
 * wb_apply_operator (on_device = 0: host arrays) or wb_apply_operator_device
 * (on_device = 1) would.  No counterpart in the reference, whose images each
 * hold one system.  The contexts run concurrently, one host thread and one
 * CUDA stream each, their PCG loops as graph launches, so the GPU interleaves
 * the systems' kernels and the SMs a system leaves when it converges go to
 * the others.  unconverged[i] may be NULL.  Returns the first failure.
 */
int wb_apply_operator_multi(int nctx, wb_ctx* const* ctx, const int* m, const double* const* dvg, const int* ld_dvg,
                            double* const* dng, const int* ld_dng, double tr2, int iq, int* const* unconverged,
                            int on_device);

/* Launch shapes chosen by the library's autotuner, which times the candidates
 * on the first batch of each form (FP64, mixed) on the batch's own buffers
 * before its PCG loop starts, then keeps them for the context. */
typedef struct wb_tuning {
  int autotune;              /* 1: tune on first use (default); 0: built-in shapes   */
  int tuned_fp64;            /* 1 once the FP64 form was tuned                        */
  int tuned_mixed;           /* 1 once the mixed form was tuned                       */
  int dmma_ctas_per_sm;      /* FP64 bra-ket split-K target, CTAs per SM (1, 2, 4)    */
  int tc_braket_ctas_per_sm; /* tcgen05 bra-ket split-K target, CTAs per SM (1..3)    */
  int tc_update_systems;     /* systems per CTA of the tcgen05 update (64, 128; 0 default) */
  int plane_fused_fp64;      /* 1: one-pass fused plane kernel in the FP64 operator   */
  int plane_fused_mixed;     /* 1: the same in the FP32 inner operator                */
  int dmma_prefetch;         /* FP64 bra-ket: k steps between operand load and MMA (1, 2) */
  float tuning_ms;           /* host time spent tuning                                */
} wb_tuning;
int wb_get_tuning(const wb_ctx* ctx, wb_tuning* out);
int wb_set_autotune(wb_ctx* ctx, int enable);

/* CUDA graphs: 1 (default) runs each batch's masked PCG loop from one graph
 * launch whose conditional WHILE node tests convergence on the device, and each
 * wb_davidson iteration's dense steps as two cached graph launches around the
 * operator call; 0 runs both eagerly, reading the PCG's active count back to the
 * host every iteration.  Stage profiling always runs the PCG loop eagerly.  The
 * same results either way, to rounding (the eager PCG may split its GEMMs
 * differently). */
int wb_set_graphs(wb_ctx* ctx, int enable);

/*
 * Allocation-free form of wb_apply_operator_device.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory while
 * they run (a host code whose GPU memory is owned by its own pool, a
 * latency-bound loop that cannot take cudaMalloc's implicit synchronisation,
 * an allocation policy that forbids allocations after set-up).  Same
 * arguments and results as wb_apply_operator_device in the FP64 form; dvg and
 * dng are device buffers supplied by the caller.  Limits:
 *   - FP64 only: on a context set to WB_PRECISION_MIXED it returns
 *     WB_ERR_UNSUPPORTED;
 *   - every per-call buffer comes from one file-scope device array of
 *     WB_NOALLOC_SCRATCH_BYTES that each GPU loading the library holds until
 *     the process exits; a call whose buffers do not fit returns WB_ERR_ARG
 *     with the size it would need;
 *   - the PCG loop runs eagerly (a host read of the active count per
 *     iteration, no CUDA graph) with the built-in launch shapes (no
 *     autotuning), and wb_get_stats reports only m, cg_iterations and
 *     cg_active_sum for it;
 *   - the first call on each context looks up the array's device address
 *     (cudaGetSymbolAddress) with the context's device current, so make that
 *     first call before any stream capture;
 *   - all calls, from every context on the device, share the one array and
 *     its leftover contents: calls that overlap on the GPU (other threads or
 *     streams) race and corrupt each other.
 * Nothing is allocated by this call; the context (wb_ctx_create) must exist.
 */
#define WB_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
int wb_apply_operator_device_noalloc(wb_ctx* ctx, int m, const double* dvg, int ld_dvg, double* dng, int ld_dng,
                                     double tr2, int iq, int* unconverged);

/* PDEP Davidson input keys (westcom wstat_control; Pytools/west_fetch_input.py:31-46). */
typedef struct wb_davidson_params {
  int n_pdep_eigen;    /* nvec: PDEP eigenpairs wanted                          */
  int n_pdep_basis;    /* nvecx = n_pdep_eigen * n_pdep_times                   */
  int n_pdep_maxiter;  /* Davidson iterations                                   */
  double tr2_dfpt;     /* PCG threshold of the iterations                        */
  double trev_pdep;    /* absolute eigenvalue convergence                        */
  double trev_pdep_rel;/* relative eigenvalue convergence                        */
  int n_steps_write_restart; /* 0: no restart files; k: write them every k iterations
                                (k = 1: also after the two starting steps)         */
  int restart;         /* 1: resume from restart_dir (wstat_calculation 'R')      */
  const char* restart_dir;   /* wstat_restart_dir (Wstat/davidson_restart.f90 layout) */
} wb_davidson_params;

/* What davidson_diago_gamma reports (exec.davitr of wstat.json). */
typedef struct wb_davidson_info {
  int dav_iter;             /* iterations run                                   */
  int notcnv;               /* roots still unconverged at exit                  */
  int converged;            /* 1 when every root converged                      */
  int apply_calls;          /* apply_operator calls                             */
  long long perturbations;  /* columns pushed through apply_operator            */
  double seconds;           /* wall time of the solve                           */
  double seconds_apply;     /* of which inside apply_operator                   */
} wb_davidson_info;

/*
 * The PDEP Davidson eigensolver, davidson_diago_gamma (Wstat/davidson_diago.f90:31-437)
 * with do_mgs (:909), build_hr_real (Wstat/wstat_tools.f90:345), diagox_dsy (:48),
 * redistribute_vr_distr_real (:591), update_with_vr_distr_real (:945) and
 * refresh_with_vr_distr_real (:1245), on one GPU.  dvg0 [ld_dvg0, n_pdep_eigen] is
 * the randomised starting basis (do_randomize, davidson_diago.f90:1121, host
 * memory).  Returns the n_pdep_eigen lowest eigenvalues of sqvc chi0 sqvc in
 * ev, their convergence flags in conv and, when pdep != NULL, the eigenvectors
 * [ld_pdep, n_pdep_eigen] (host memory).  The subspace eigensolver is
 * wb_diagox's Jacobi method on the GPU (diagox uses LAPACK DSYEV / cuSOLVER in
 * WEST); n_pdep_basis up to 4096.  The basis, hr, vr, the eigenvalues and the
 * convergence flags stay on the GPU: each iteration runs its dense steps as two
 * CUDA graph launches around the operator call (cached per basis size; eager
 * with wb_set_graphs(ctx, 0)) and the host reads back only the state it needs
 * to choose the next batch.
 */
/*
 * Operator hook of the Davidson: when set, wb_davidson calls fn instead of its
 * own apply_operator for every batch of new basis vectors.  dvg/dng are device
 * pointers to the batch (columns col0 .. col0+m-1 of the basis, WEST's G order,
 * leading dimension ld); fn writes dng = sqvc chi0 sqvc dvg with PCG threshold
 * tr2 (< 0: lite solver) and returns 0 or a wb error code.  The hook is how the
 * perturbation-sharded multi-GPU Davidson runs: each rank applies the operator
 * to its cyclic share of the columns (WEST's pert%l2g, davidson_diago.f90:
 * 185-196,313-324) and one all-gather of dng (NCCL over NVLink) gives every rank
 * the whole batch; the small dense steps then run redundantly on every rank.
 * fn = NULL restores the library's own apply_operator.
 */
typedef int (*wb_apply_fn)(void* user, int col0, int m, const double* dvg, double* dng, int ld, double tr2);
int wb_davidson_set_apply(wb_ctx* ctx, wb_apply_fn fn, void* user);

/*
 * Restart hand-off (Wstat/davidson_restart.f90:33-411, same files as WEST):
 * restart_dir/summary.json (dav_iter, notcnv, nbase, conv, ev, ew), hr_vr.dat
 * (Fortran unformatted sequential: hr then vr, n_pdep_basis^2 doubles each) and
 * V<j>.dat / N<j>.dat (j = 000001..nbase, the pdep file format) are written at
 * the reference's checkpoints and removed on convergence; with restart = 1 the
 * solve resumes from them (dvg0 may then be NULL).
 */
int wb_davidson(wb_ctx* ctx, const wb_davidson_params* params, const double* dvg0, int ld_dvg0, double* ev,
                int* conv, double* pdep, int ld_pdep, wb_davidson_info* info);

/*
 * Subspace eigensolver of the Davidson, diagox_dsy (Wstat/wstat_tools.f90:48,
 * serial_diagox_dsy :208, matdiago_dsy Tools/linear_algebra_kernel.f90:84):
 * the nvec lowest eigenvalues of the real symmetric hr(1:nbase, 1:nbase)
 * (upper triangle read, as DSYEV 'U') in ascending order into ew (host), and
 * their orthonormal eigenvectors into vr(:, 1:nvec).  hr [ldh, nbase] and vr
 * [ldv, nvec] are column-major device arrays of the context's device.  Cyclic
 * Jacobi in one CTA up to nbase = 112, a parallel two-sided block Jacobi over
 * many CTAs above (up to 4096); WEST uses LAPACK DSYEV / cuSOLVER here.
 */
int wb_diagox(wb_ctx* ctx, int nbase, int nvec, const double* hr, int ldh, double* ew, double* vr, int ldv);

/*
 * PDEP database in WEST's format: pdep_db_write (IO_kernel/pdep_db.f90:56) with
 * pdep_merge_and_write_G (IO_kernel/pdep_io.f90:35) and pdep_db_read (pdep_db.f90:212)
 * with pdep_read_G_and_distribute (pdep_io.f90:158).  One stream file per
 * eigenvector, Q<iq>E<j>.dat: 32 int32 header (210405, little-endian flag,
 * npw) then npw complex128 coefficients; summary.json with the cell
 * (cell = a1, a2, a3 in bohr then b1, b2, b3 in bohr^-1: 18 doubles), iq, q,
 * eigenval and eigenvec.  pdep [ld, n] complex, host memory.  Gamma only (iq = 1).
 * Host-only: no GPU work.
 */
int wb_pdep_db_write(const char* dir, int iq, const double* q_cryst, const double* cell, int n_pdep_eigen,
                     const double* ev, const double* pdep, int ld, int npw);
int wb_pdep_db_read(const char* dir, int iq, int nglob, double* ev, double* pdep, int ld, int npw);

/* Message of the last failed call in this thread ("" if none). */
const char* wb_last_error(void);

/* Library version: major * 10000 + minor * 100 + patch. */
int wb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* WEST_B200_H */
