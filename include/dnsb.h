/*
 * dnsb.h -- C ABI of libdnsb.so, the B200 (sm_100a) time-step kernels for
 * dnsjax (gokhanyalniz/dnsjax).
 *
 * Conventions
 *   - Every function returns 0 on success and a nonzero dnsb_status code
 *     otherwise; dnsb_last_error() gives a message for the calling thread.
 *   - Arrays are plain device pointers (complex128 = interleaved double
 *     pairs) in the reference's layouts; the caller owns them.  Contexts own
 *     only their coefficient copies and workspace (allocated once, at
 *     creation, with cudaMalloc) and are not thread-safe.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls only
 *     enqueue work: no host synchronisation happens inside, except where a
 *     function's comment says it returns a host value.
 *   - Scalars such as the corrector error are written to device memory
 *     (`double* out_dev`) so a whole step can be enqueued without a sync.
 *
 * Reference interfaces replaced (paths within the reference project):
 *   triply-periodic   src/dnsjax/flows/monochromatic.py:366-410 (_get_rhs,
 *                     _predict, _correct, _norm handed to make_stepper at
 *                     :413-415), :516-565 (correct_velocity), :433-510 (stats)
 *   plane Couette     src/dnsjax/flows/plane_couette.py:274-289 (_get_rhs),
 *                     :376-549 (_imm_iteration, _predict, _correct, _norm),
 *                     :591-613 (stats)
 *   banded solve      src/dnsjax/geometries/cartesian.py:360-488
 *                     (_banded_solve_device, PerModeBandedOperator.solve)
 *   transforms        src/dnsjax/operators.py:59-146 (spec_to_phys,
 *                     spec_to_phys_2d, phys_to_spec[_2d]) over
 *                     src/dnsjax/fft.py:193-408
 */
#ifndef DNSB_H_
#define DNSB_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum dnsb_status {
  DNSB_OK = 0,
  DNSB_ERR_ARG = 1,      /* invalid argument / unsupported size */
  DNSB_ERR_CUDA = 2,     /* a CUDA runtime call failed */
  DNSB_ERR_PIVOT = 3     /* a pivot index outside [j, j+kl] was met */
};

int dnsb_version(void);
const char* dnsb_last_error(void);
/* Number of kernel launches this library has enqueued in this process. */
long long dnsb_launch_count(void);

/* ------------------------------------------------------------------ */
/* Triply periodic flows (Kolmogorov, Waleffe, decaying box).          */
/* Spectral layout (3, ny-1, nz-1, nx/2) complex128, [ky][kz][kx].     */
/* Physical layout (3, ny_p, nz_p, nx_p) float64, [y][z][x].           */
/* ------------------------------------------------------------------ */
typedef struct dnsb_periodic dnsb_periodic;

typedef struct {
  int nx, ny, nz;         /* Fourier modes before the 3/2 rule (even) */
  int nx_p, ny_p, nz_p;   /* padded physical sizes, each 2^a 3^b */
  double dt, implicitness;
  /* host arrays, copied at creation */
  const double* kx;       /* nx/2, 2 pi/lx * [0 .. nx/2-1] */
  const double* ky;       /* ny-1, FFT order, Nyquist omitted */
  const double* kz;       /* nz-1 */
  const double* base_flow;        /* [3][ny_p] U(y) */
  const double* curl_base_flow;   /* [3][ny_p] curl U */
  const double* nonlin_base_flow; /* [3][ny_p] U x curl U */
  const double* ldt_1;    /* (ny-1)(nz-1)(nx/2), mean mode 0 */
  const double* ildt_2;   /* (ny-1)(nz-1)(nx/2), mean mode 0 */
} dnsb_periodic_desc;

int dnsb_periodic_create(const dnsb_periodic_desc* desc, dnsb_periodic** out);
int dnsb_periodic_destroy(dnsb_periodic* ctx);
/* Bytes of device workspace the context holds. */
size_t dnsb_periodic_workspace_bytes(const dnsb_periodic* ctx);

/* rhs = NL(u) - grad lapl^-1 div NL(u)   (monochromatic.py:366-386) */
int dnsb_periodic_rhs(dnsb_periodic* ctx, const void* state, void* rhs,
                      void* stream);
/* res.double_precision = False for the periodic flows (parameters.py:63):
 * with fp32 != 0 the RHS transforms (y, z, x passes) and the rotational
 * product run in FP32 on FP32 pass buffers; the state is read, the curl
 * formed and the projection applied in FP64, and the RHS is written in
 * complex128.  Only for padded sizes in {48, 72, 96, 192} with
 * nx_p = 3 nx / 2 (else DNSB_ERR_ARG).  fp32 = 2: the same FP32 passes with
 * compensated (two-sum) accumulation in their register DFT butterflies
 * (each value carried as h + l, the rounding errors of the butterflies'
 * sums and constant products kept in l and folded back at the DFT's
 * outputs); the twiddle products between stages and the pass buffers stay
 * FP32. */
int dnsb_periodic_set_rhs_precision(dnsb_periodic* ctx, int fp32);
/* out = (state ldt_1 + rhs) ildt_2       (monochromatic.py:320-333) */
int dnsb_periodic_predict(dnsb_periodic* ctx, const void* state,
                          const void* rhs, void* out, void* stream);
/* corr = c (rhs_next - rhs_prev) ildt_2; pred_out = pred + corr;
 * err_dev[0] = sqrt(sum conj(corr) k_metric corr)  (monochromatic.py:336-355,
 * 408-410).  pred_out may alias pred; corr_out and err_dev may be NULL. */
int dnsb_periodic_correct(dnsb_periodic* ctx, const void* pred,
                          const void* rhs_prev, const void* rhs_next,
                          void* pred_out, void* corr_out, double* err_dev,
                          void* stream);
/* out_dev[0] = sqrt(sum conj(v) k_metric v)  (triply_periodic.py:81-101) */
int dnsb_periodic_norm(dnsb_periodic* ctx, const void* v, double* out_dev,
                       void* stream);
/* out = v - grad lapl^-1 div v (if divergence), mean mode zeroed
 * (monochromatic.py:516-565).  out may alias v. */
int dnsb_periodic_correct_velocity(dnsb_periodic* ctx, const void* v,
                                   void* out, int divergence, void* stream);
/* One full time step as a CUDA graph, for callers that step without host
 * synchronisation (the reference driver's step, __main__.py:125-203, with its
 * corrector loop -- iterate while error > tol and iterations < max_iter,
 * :166-180 -- as a device-controlled conditional node): predictor and first
 * correction from `state`, corrector iterations, correct_velocity (with
 * `divergence`) back into `state`.  The graph is bound to `state` (updated in
 * place by every launch) and owns its prediction, RHS and control buffers;
 * creation captures the context's launches and allocates, launching does
 * neither. */
typedef struct dnsb_step_graph dnsb_step_graph;
int dnsb_periodic_step_graph_create(dnsb_periodic* ctx, void* state, double tol,
                                    int max_iter, int divergence,
                                    dnsb_step_graph** out);
int dnsb_step_graph_launch(dnsb_step_graph* g, void* stream);
/* Corrector iterations and final corrector error of the last launched step
 * (host values; synchronises `stream`). */
int dnsb_step_graph_status(dnsb_step_graph* g, int* iters, double* err,
                           void* stream);
int dnsb_step_graph_destroy(dnsb_step_graph* g);
/* Corrector iterations that periodic step graphs captured afterwards on this
 * context hold as straight-line kernels ahead of the WHILE node (no
 * counterpart in the reference; see dnsb_couette_set_graph_unroll).  n in
 * [0, 64] (capped at the graph's max_iter); it applies when the context runs
 * the two-stage passes at the compiled sizes (every pass variant 0), else
 * graphs are captured without unrolling. */
int dnsb_periodic_set_graph_unroll(dnsb_periodic* ctx, int n);

/* Ensembles of independent periodic trajectories (the driver's time step,
 * __main__.py:125-203, for every member; no counterpart for several
 * trajectories in the reference): one ensemble step is one CUDA graph in
 * which every stage -- each of the five RHS passes, the projection, the
 * predictor, the correction with its norm, correct_velocity -- is ONE
 * launch over all members (a work list of the members' blocks walked by a
 * persistent grid), and the corrector loop is a device-controlled WHILE
 * node that runs while any member iterates; a member that has converged or
 * reached max_iter[m] is skipped.  Every member computes exactly what its
 * own step graph computes (the same blocks, the same reduction order).
 * Members: FP64 contexts with the default pass variants and padded lengths
 * 48, 72, 96 or 192 with nx_p = 3 nx / 2; at most 1024.  states[m] is bound
 * (advanced in place by every step).  Creation allocates the members'
 * prediction and RHS buffers and the work lists; stepping allocates
 * nothing. */
typedef struct dnsb_ensemble dnsb_ensemble;
int dnsb_ensemble_create(dnsb_periodic* const* ctxs, void* const* states, int n,
                         const double* tol, const int* max_iter, int divergence,
                         dnsb_ensemble** out);
int dnsb_ensemble_step(dnsb_ensemble* e, void* stream);
/* Per member: corrector iterations and final corrector error of the last
 * step (host arrays of n; synchronises `stream`). */
int dnsb_ensemble_status(dnsb_ensemble* e, int* iters, double* errs, void* stream);
int dnsb_ensemble_destroy(dnsb_ensemble* e);

/* out_dev[0] = sum k_metric |v|^2, out_dev[1] = sum -lapl |v|^2 (the two
 * reductions of monochromatic.py:433-466). */
int dnsb_periodic_energy_sums(dnsb_periodic* ctx, const void* v,
                              double* out_dev, void* stream);
/* Inverse / forward dealiased 3D transforms of 3 components
 * (operators.py:59-101). */
int dnsb_periodic_spec_to_phys(dnsb_periodic* ctx, const void* spec,
                               double* phys, void* stream);
int dnsb_periodic_phys_to_spec(dnsb_periodic* ctx, const double* phys,
                               void* spec, void* stream);

/* ------------------------------------------------------------------ */
/* Plane Couette.                                                      */
/* Spectral layout (3, nz-1, nx/2, ny) complex128, [kz][kx][y].        */
/* Physical layout (3, ny, nz_p, nx_p) float64, [y][z][x].             */
/* ------------------------------------------------------------------ */
typedef struct dnsb_couette dnsb_couette;

typedef struct {
  int nx, ny, nz;         /* Fourier modes in x, z; CGL points in y (odd) */
  int nx_p, nz_p;         /* padded sizes, 2^a 3^b */
  int fd_order;           /* p: D1 on p+1 points, D2 on p+2, kl = ku = p */
  double dt, implicitness, nu, ly;
  /* host arrays, copied at creation */
  const double* kx;       /* nx/2 */
  const double* kz;       /* nz-1 */
  const double* ys;       /* ny CGL points */
  const int* d1_j0;       /* [ny] first column of the D1 stencil of row i */
  const double* d1_w;     /* [ny][p+1] */
  const int* d2_j0;       /* [ny] */
  const double* d2_w;     /* [ny][p+2] */
  const double* base_flow;        /* [3][ny] */
  const double* curl_base_flow;   /* [3][ny] */
  const double* nonlin_base_flow; /* [3][ny] */
} dnsb_couette_desc;

/* IMM operators in the reference's layouts (cartesian.py:575-801): device
 * pointers owned by the caller, kept alive while bound. */
typedef struct {
  const double* Lk_ab;  /* (nz-1, nx/2, 3p+1, ny), LAPACK gbtrf factors */
  const int* Lk_piv;    /* (nz-1, nx/2, ny), 0-based */
  const double* Hk_ab;
  const int* Hk_piv;
  const double* v1;     /* (nz-1, nx/2, ny) */
  const double* v2;
  const double* q1;
  const double* q2;
  const double* M_inv;  /* (nz-1, nx/2, 2, 2) */
} dnsb_imm_ops;

int dnsb_couette_create(const dnsb_couette_desc* desc, dnsb_couette** out);
int dnsb_couette_destroy(dnsb_couette* ctx);
size_t dnsb_couette_workspace_bytes(const dnsb_couette* ctx);
int dnsb_couette_bind_imm(dnsb_couette* ctx, const dnsb_imm_ops* ops);

/* rhs = NL(u) on the padded grid (plane_couette.py:274-289) */
int dnsb_couette_rhs(dnsb_couette* ctx, const void* state, void* rhs,
                     void* stream);
/* Arithmetic of dnsb_couette_rhs (the reference's res.double_precision,
 * parameters.py:63, __main__.py:287): fp32 = 1 runs the transforms and the
 * rotational product in FP32 -- the state is read and the RHS written in
 * complex128, the IMM, its banded substitutions and every norm stay FP64;
 * fp32 = 0 (the default) is FP64 throughout; fp32 = 2 is fp32 = 1 with
 * compensated (two-sum) accumulation in the register DFT butterflies, as
 * for dnsb_periodic_set_rhs_precision.  FP32 needs padded sizes in
 * {48, 72, 96, 192} with nx_p = 3 nx / 2 (DNSB_ERR_ARG otherwise). */
int dnsb_couette_set_rhs_precision(dnsb_couette* ctx, int fp32);
/* One influence-matrix iteration (plane_couette.py:376-504):
 * vel_new = IMM(vel_n, vel_j, nl_n, nl_j); corr_out = vel_new - vel_j
 * (nullable); err_dev[0] = Simpson norm of the correction (nullable).
 * vel_new may alias vel_j when vel_j != vel_n; it must not alias vel_n. */
int dnsb_couette_imm(dnsb_couette* ctx, const void* vel_n, const void* vel_j,
                     const void* nl_n, const void* nl_j, void* vel_new,
                     void* corr_out, double* err_dev, void* stream);
/* out_dev[0] = sqrt(Simpson_y(sum conj(v) k_metric v) / ly)
 * (cartesian.py:72-103). */
int dnsb_couette_norm(dnsb_couette* ctx, const void* v, double* out_dev,
                      void* stream);
/* out_dev[0] = Simpson_y(sum conj(v) k_metric v) / ly (no square root). */
int dnsb_couette_norm2(dnsb_couette* ctx, const void* v, double* out_dev,
                       void* stream);
int dnsb_couette_spec_to_phys(dnsb_couette* ctx, const void* spec,
                              double* phys, void* stream);
int dnsb_couette_phys_to_spec(dnsb_couette* ctx, const double* phys,
                              void* spec, void* stream);
/* Reads the context's device status word (synchronising `stream`):
 * DNSB_ERR_PIVOT when a bound operator holds a pivot index outside
 * [j, j+kl] (found when the operators are bound; such a pivot is not
 * followed), DNSB_ERR_CUDA when a bounded wait inside the IMM substitution
 * kernel gave up (its results are then invalid), else 0. */
int dnsb_couette_check(dnsb_couette* ctx, void* stream);
/* Failure detection (no counterpart in the reference): the status word stays
 * set until cleared; the ring waits of the IMM substitution kernel give up
 * after `polls` polls of a slot's mbarrier (default 2^20; 0 makes every
 * wait give up at once, which sets the status and invalidates the call's
 * results but leaves no copy in flight and the context usable).  Step
 * graphs keep the limit they were captured with. */
int dnsb_couette_clear_status(dnsb_couette* ctx, void* stream);
int dnsb_couette_set_wait_limit(dnsb_couette* ctx, int polls);

/* One full plane-Couette time step as a CUDA graph, like
 * dnsb_periodic_step_graph_create: predictor (the IMM iteration with
 * (u^n, u^n, N^n, N^n), plane_couette.py:507-519), first correction, and
 * corrector iterations (plane_couette.py:522-540) in a device-controlled
 * loop while error > tol and iterations < max_iter (__main__.py:166-180);
 * correct_velocity is the identity for this flow (plane_couette.py:575-582),
 * so the converged iterate is copied back into `state`.  Needs bound IMM
 * operators; launch/status/destroy through dnsb_step_graph_*. */
int dnsb_couette_step_graph_create(dnsb_couette* ctx, void* state, double tol,
                                   int max_iter, dnsb_step_graph** out);

/* Corrector iterations that step graphs captured afterwards on this context
 * (dnsb_couette_step_graph_create, dnsb_couette_mixed_graph_create) hold as
 * straight-line kernels before the WHILE node (no counterpart in the
 * reference).  Every entry into a conditional node's body leaves the GPU idle
 * for tens of microseconds; the unrolled iterations enter none, and once the
 * loop has ended their kernels return at once.  n in [0, 64] (capped at the
 * graph's max_iter); it applies when the context runs the two-stage passes at
 * the compiled sizes and the batched IMM (the defaults there), else graphs
 * are captured without unrolling.  The states and iteration counts are those
 * of the graphs without unrolling, bit for bit. */
int dnsb_couette_set_graph_unroll(dnsb_couette* ctx, int n);

/* The restarted, mixed-precision corrector step as two CUDA graphs (no
 * counterpart in the reference: the device form of the learned corrector
 * step, dnsjax_b200.learned.LearnedGuess.step, whose corrector is
 * iterate_correction, plane_couette.py:522-540, from a guessed start).
 * Bound to three distinct complex128 (3, nz-1, nx/2, ny) buffers:
 *   dnsb_mixed_graph_predict: RHS of `state` (u^n), the predictor
 *     (plane_couette.py:507-519) into `up`, copied into `cur`; the caller
 *     may then overwrite `cur` with a guessed start;
 *   dnsb_mixed_graph_correct: the first correction from `cur` (restart != 0:
 *     the start's RHS in both RHS slots, else N^n as the previous RHS), the
 *     corrector loop on the device while error > tol and iterations <
 *     max_iter (__main__.py:166-180), and `cur` copied into `state`.
 * mixed = 0: every RHS in FP64.  mixed = 1 (FP32) or 2 (FP32, compensated
 * butterflies): the RHS runs at that precision until the error after a
 * correction is <= switch_tol or > stall x the error two corrections back
 * (the corrector's errors fall in pairs), then in FP64
 * for the rest of the step (needs the FP32 pass sizes of
 * dnsb_couette_set_rhs_precision).  status: corrector iterations after the
 * first correction, the last and the first error, and the RHS evaluations at
 * reduced precision / FP64 of the last step (synchronises `stream`). */
typedef struct dnsb_mixed_graph dnsb_mixed_graph;
int dnsb_couette_mixed_graph_create(dnsb_couette* ctx, void* state, void* up, void* cur,
                                    double tol, int max_iter, int mixed, double switch_tol,
                                    double stall, int restart, dnsb_mixed_graph** out);
int dnsb_mixed_graph_predict(dnsb_mixed_graph* g, void* stream);
int dnsb_mixed_graph_correct(dnsb_mixed_graph* g, void* stream);
int dnsb_mixed_graph_status(dnsb_mixed_graph* g, int* iters, double* err, double* first_err,
                            int* n32, int* n64, void* stream);
int dnsb_mixed_graph_destroy(dnsb_mixed_graph* g);

/* Allocation-free Couette norm (no counterpart in the reference; it exists
 * for callers that cannot allocate device memory, such as an XLA FFI handler
 * working inside memory its framework owns).  Computes what dnsb_couette_norm computes, from the field alone
 * (the CGL grid and its Simpson weights are generated in the kernel), with
 * the per-mode partial sums kept in a file-scope device array instead of
 * context workspace:
 *   out_dev[0] = sqrt(Simpson_y(sum conj(v) k_metric v) / ly)
 *   v: (3, nz-1, nx/2, ny) complex128.  At most 32768 (kz, kx) modes;
 *   larger fields return DNSB_ERR_ARG.  The array (256 KiB) stays on every
 *   device that loads the library until exit; every call shares it, so calls
 *   that may overlap on the GPU race and must be ordered by the caller.  The
 *   first call on a device looks up the array's device address (with that
 *   device current) and caches it with the ID of the current CUDA context;
 *   the cache assumes that the address stays valid while that context
 *   lives, and a call from another context (after cudaDeviceReset, or with
 *   a different driver-API context current) looks it up again.  Make the
 *   first call on a device, and the first after a reset, before any stream
 *   capture.  Device ordinals of 64 and above return DNSB_ERR_ARG. */
int dnsb_couette_norm_noalloc(const void* v, int nx, int ny, int nz, double ly,
                              double* out_dev, void* stream);

/* ------------------------------------------------------------------ */
/* Autotuning (no counterpart in the reference).  Times every kernel    */
/* variant of each pass on the context's own sizes and buffers, from    */
/* `state` (spectral, complex128), `reps` calls each after one warm-up  */
/* call, and keeps the fastest (the default unless another is 5%       */
/* faster) for the context's later calls and later step graphs.        */
/* Variants: 0 the two-stage register                                   */
/* pass where it is compiled for the length (the default), 1 Stockham   */
/* stages with the compile-time plan, 2 Stockham stages with the        */
/* runtime plan; the FP32 forms have variant 0 only.                   */
/*   periodic: chosen[5] for the y inverse (0: two-stage pass with the  */
/*     curl formed at the load), z inverse, x, z forward and y forward  */
/*     (0: two-stage pass, then the projection as a separate pointwise  */
/*     kernel) passes; ms[5][3] mean times (-1 where not tried).        */
/*   Couette: chosen[4] for the z inverse, x and z forward passes and   */
/*     the IMM (0 five-kernel batched form, 1 one-kernel register-window */
/*     form, 2 one-kernel form); ms[4][3].                              */
/* Results of different variants agree to rounding, not bit for bit.   */
/* ------------------------------------------------------------------ */
int dnsb_periodic_autotune(dnsb_periodic* ctx, const void* state, int reps, int* chosen,
                           float* ms, void* stream);
/* Sets the variants directly (same meaning and order as `chosen`). */
int dnsb_periodic_set_variants(dnsb_periodic* ctx, const int* variants);
int dnsb_couette_set_variants(dnsb_couette* ctx, const int* variants);
int dnsb_couette_autotune(dnsb_couette* ctx, const void* state, int reps, int* chosen,
                          float* ms, void* stream);

/* ------------------------------------------------------------------ */
/* Learned corrector guess for plane Couette (no counterpart in the     */
/* reference): kernels of a per-(kz, kx)-mode MLP, BF16 weights and     */
/* activations, FP32 accumulation, trained online on the pairs          */
/* (predictor -> converged correction) the solver generates.  The       */
/* guess replaces the predictor's output before the first correction;   */
/* the corrector still iterates to the tolerance from it.  Every array  */
/* is device memory.                                                    */
/* ------------------------------------------------------------------ */
/* C[m][n] = sum_k A(m, k) B(n, k) on the tensor cores (BF16 operands,
 * FP32 accumulation); A(m, k) = ta ? A[k lda + m] : A[m lda + k],
 * B(n, k) = tb ? B[k ldb + n] : B[n ldb + k].  Epilogue: + bias[n] (FP32,
 * optional), max(., 0) when relu, times (mask[m ldm + n] > 0) when mask
 * (BF16) is given; written to Cf (FP32) and / or Cb (BF16) at [m ldc + n].
 * With ta = tb = 0, lda and ldb multiples of 8 and 16-byte aligned A, B it
 * runs on tcgen05 (TMA tiles, TMEM accumulator); other layouts run on
 * mma.sync.  work (optional, work_elems floats) lets the tcgen05 path split
 * K when the output tiles cannot fill the GPU: the partial tiles are summed
 * in a fixed order, so results are the same run to run.  status (optional,
 * device int): bit 0 is set if a pipeline wait of the tcgen05 kernel gave
 * up (bounded waits; the call then returns normally with that bit set). */
int dnsb_mlp_gemm(int ta, int tb, int M, int N, int K, const void* A, int lda, const void* B,
                  int ldb, const float* bias, int relu, const void* mask, int ldm, float* Cf,
                  void* Cb, int ldc, float* work, long long work_elems, int* status,
                  void* stream);
/* out[c][r] = A[r][c] for an R x C BF16 matrix (row strides lda, ldo). */
int dnsb_mlp_transpose(const void* A, int R, int C, int lda, void* out, int ldo, void* stream);
/* Features of every mode m (spectral layout (3, nz-1, nx/2, ny) complex128):
 * X[m][((F*3 + c)*ny + y)*2 + part] (BF16) with F = 0: (up - un) / s_m,
 * F = 1: dprev / s_m (zero when dprev is NULL), then kx / kx_max,
 * kz / kz_max at 12 ny, 12 ny + 1; scale[m] = s_m = rms of up - un over
 * the mode, at least s_floor; T[m][(c*ny + y)*2 + part] = target / s_m (FP32) when target is
 * given.  ldx >= 12 ny + 2, ldt >= 6 ny. */
int dnsb_learned_features(dnsb_couette* ctx, const void* un, const void* up, const void* dprev,
                          const void* target, double kx_max, double kz_max, double s_floor,
                          void* X, int ldx, float* T, int ldt, float* scale, void* stream);
/* out = up + scale[m] * Y[m][(c*ny + y)*2 + part] (complex128 out). */
int dnsb_learned_guess(dnsb_couette* ctx, const void* up, const float* Y, int ldy,
                       const float* scale, void* out, void* stream);
/* Mean-squared-error gradient dY = 2 (Y - T) / M (FP32 dYf and BF16 dYb),
 * err[m] = sum_n (Y - T)^2, ref[m] = sum_n T^2. */
int dnsb_mlp_loss_grad(const float* Y, const float* T, int M, int N, int ld, float* dYf,
                       void* dYb, float* err, float* ref, void* stream);
/* out[n] = sum_m A[m lda + n]; A is BF16 when bf16 != 0, else FP32.  Sums
 * in a fixed order through work (at least min(M, 128) x N floats). */
int dnsb_mlp_colsum(const void* A, int bf16, int M, int N, int lda, float* out, float* work,
                    long long work_elems, void* stream);
/* One Adam update (step >= 1, bias-corrected) of FP32 weights w with
 * moments m, v from grad; wb (BF16, optional) gets the rounded weights. */
int dnsb_mlp_adam(float* w, float* m, float* v, const float* grad, void* wb, long long n,
                  float lr, float b1, float b2, float eps, int step, void* stream);

/* ------------------------------------------------------------------ */
/* Influence-matrix precompute on the GPU (precompute_imm, banded      */
/* backend, geometries/cartesian.py:575-801).  For every (kz, kx) mode  */
/* (k2 = kx^2 + kz^2): L_k = D2 - k2 I with Neumann wall rows (row 0    */
/* pinned to e_0 when k2 = 0; build_Lk_neumann, :491-526) and           */
/* H_k = I/dt - c nu (D2 - k2 I) with identity wall rows               */
/* (build_Hk_dirichlet, :529-572), packed as LAPACK ab (:291-320) and  */
/* factored by banded LU with partial pivoting (LAPACK dgbtf2, what    */
/* SciPy's gbtrf runs for these bandwidths; :323-357); p1, p2 = L_k^-1 */
/* e_0, e_{ny-1}; v1, v2 = H_k^-1 (-D1 p1), H_k^-1 (-D1 p2) and q1,    */
/* q2 = H_k^-1 p1, H_k^-1 p2 (wall rows of the right-hand sides zero); */
/* M_inv = inverse of [D1[0].v1 D1[0].v2; D1[ny-1].v1 D1[ny-1].v2]      */
/* ([[0, 0], [0, 1/M11]] when k2 = 0).  The p, v, q solves use the     */
/* banded factors (the reference uses dense LU), so they agree with    */
/* the reference to rounding.  kl = ku = p.                            */
/*   D1, D2 : (ny, ny) float64 row-major; kx (nkx), kz (nkz) float64   */
/*   p1..q2 : (nkz, nkx, ny) float64; M_inv (nkz, nkx, 2, 2) float64   */
/*   Lk_ab, Hk_ab : (nkz, nkx, 3p+1, ny) float64; Lk_piv, Hk_piv       */
/*          (nkz, nkx, ny) int32, 0-based                              */
/*   info_dev : device int, zeroed by the caller; OR'ed with 2 when    */
/*          some L_k, 4 when some H_k has a zero pivot (the reference  */
/*          raises ValueError for LAPACK info > 0)                     */
/* Every array is device memory; the call allocates stream-ordered    */
/* workspace (6 nkz nkx ny doubles) and frees it before returning.     */
/* ------------------------------------------------------------------ */
int dnsb_imm_precompute(const double* D1, const double* D2, const double* kx, int nkx,
                        const double* kz, int nkz, int ny, int p, double dt, double c,
                        double nu, double* p1, double* p2, double* v1, double* v2,
                        double* q1, double* q2, double* M_inv, double* Lk_ab, int* Lk_piv,
                        double* Hk_ab, int* Hk_piv, int* info_dev, void* stream);

/* ------------------------------------------------------------------ */
/* Per-mode banded LU substitution (PerModeBandedOperator.solve,       */
/* cartesian.py:444-488; dgbtrs 'N').                                  */
/*   ab   : (nmodes, 2kl+ku+1, ny) float64, LAPACK ab packing          */
/*   ipiv : (nmodes, ny) int32, 0-based (SciPy gbtrf convention)       */
/*   b    : (nmodes, ny, ncols) float64, solved in place; a complex    */
/*          right-hand side is ncols = 2 (real, imaginary interleaved) */
/*   status_dev: optional device int, OR'ed with 1 on a bad pivot      */
/* ------------------------------------------------------------------ */
int dnsb_banded_solve(const double* ab, const int* ipiv, double* b,
                      int nmodes, int ny, int kl, int ku, int ncols,
                      int* status_dev, void* stream);

/* ------------------------------------------------------------------ */
/* Slab decomposition over several GPUs: the reference's multi-device  */
/* scheme (fft.py:193-392, sharding.py:107-129; jax shard_map with a   */
/* reshard between the column passes and the x pass).                  */
/*   A slab context of rank r of nranks holds the kx modes             */
/*   [r nx/2/nranks, (r+1) nx/2/nranks) of every spectral array (its   */
/*   tensors are the reference's shards: (3, ny-1, nz-1, nx/2/nranks)   */
/*   periodic, (3, nz-1, nx/2/nranks, ny) Couette).  desc is the whole  */
/*   problem's; the context keeps its share of kx, ldt_1, ildt_2.      */
/*   Between the column passes and the x pass the padded grid is       */
/*   sharded on z (nz_p / nranks rows per rank).  The z inverse and    */
/*   the x pass store every output straight into the receive buffer    */
/*   of the rank that owns it (the exchange is fused into those        */
/*   kernels): dnsb_*_slab_buffers gives this rank's two receive       */
/*   buffers, dnsb_*_slab_connect takes every rank's, as this process  */
/*   addresses them (dnsb_ipc_open of another process's handles, or    */
/*   the buffers of other contexts on the same GPU).                   */
/*   dnsb_*_rhs_phase(phase = 0, 1, 2) is the RHS: the caller makes     */
/*   every rank's phase k complete before any rank starts phase k+1    */
/*   (a collective on the stream, or the order of one stream).         */
/*   The corrector's err_dev and dnsb_*_norm return this rank's share  */
/*   of the squared norm: the caller sums the shares over the ranks    */
/*   and takes the square root.  The mean mode (kx = 0) lives on rank  */
/*   0.  Slab contexts run the FP64 two-stage passes (padded sizes in  */
/*   {48, 72, 96, 192}, nx_p = 3 nx / 2, nx/2 and nz_p multiples of    */
/*   nranks, nranks <= 8), step through the host loop (no step graph,  */
/*   no autotune) and refuse dnsb_*_rhs.                               */
/* ------------------------------------------------------------------ */
int dnsb_periodic_create_slab(const dnsb_periodic_desc* desc, int nranks, int rank,
                              dnsb_periodic** out);
int dnsb_periodic_slab_buffers(dnsb_periodic* ctx, void** bx, void** bk);
int dnsb_periodic_slab_connect(dnsb_periodic* ctx, void* const* bx, void* const* bk);
int dnsb_periodic_rhs_phase(dnsb_periodic* ctx, const void* state, void* rhs, int phase,
                            void* stream);
int dnsb_couette_create_slab(const dnsb_couette_desc* desc, int nranks, int rank,
                             dnsb_couette** out);
int dnsb_couette_slab_buffers(dnsb_couette* ctx, void** bx, void** bk);
int dnsb_couette_slab_connect(dnsb_couette* ctx, void* const* bx, void* const* bk);
int dnsb_couette_rhs_phase(dnsb_couette* ctx, const void* state, void* rhs, int phase,
                           void* stream);
/* CUDA IPC of a device allocation made by this library (the slab      */
/* receive buffers): a 64-byte handle; dnsb_ipc_open maps it with peer */
/* access in another process, dnsb_ipc_close unmaps it.                */
int dnsb_ipc_handle(const void* dev_ptr, void* handle);
int dnsb_ipc_open(const void* handle, void** dev_ptr);
int dnsb_ipc_close(void* dev_ptr);

#ifdef __cplusplus
}
#endif

#endif /* DNSB_H_ */
