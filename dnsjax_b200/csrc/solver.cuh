// Per-mode solves and pointwise kernels of the time step.
#pragma once

#include <string>

#include "common.cuh"

namespace dnsb {

// ---- deterministic reductions --------------------------------------------
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 592;  // 4 x 148 SMs; fixed so sums are reproducible

// out[0] = scale * sum(partials[0..n)), sqrt'ed if do_sqrt.
cudaError_t launch_finalize(const double* partials, int n, double* out,
                            double scale, int do_sqrt, cudaStream_t st,
                            const int* skip = nullptr);

// ---- periodic pointwise ----------------------------------------------------
struct PeriodicPointArgs {
  int S;  // scalar spectral size (ny-1)(nz-1)(nx/2)
  int NY1, NZ1, NKX;
  const double* ldt_1;
  const double* ildt_2;
  const double* kx;
  const double* ky;
  const double* kz;
  const double* inv_lapl;
  const double* lapl;
  double c;
  int kx0;  // 1: local kx index 0 is the kx = 0 mode (weight 1 in the norms; else 2)
  // Unrolled step-graph iterations: when non-null and *skip != 0, the
  // correct and projection kernels return at once (the work-list forms
  // ignore it).
  const int* skip = nullptr;
};

// One member's pointwise call in an ensemble work list: predict (op 0:
// out = (in0 ldt_1 + in1) ildt_2), correct (op 1: out = in0 + c (in2 - in1)
// ildt_2, the norm partials into `partials`), correct_velocity / projection
// (op 2: in0 -> out).
struct EnsPointItem {
  PeriodicPointArgs a;
  const double2* in0;
  const double2* in1;
  const double2* in2;
  double2* out;
  double* partials;
  int member;
};
cudaError_t launch_ens_point(const EnsPointItem* items, int n, const int* active, int op,
                             int divergence, int zero_mean, int grid, cudaStream_t st);
// err[member] = sqrt(sum of the member's kRedBlocks partials), one block each.
cudaError_t launch_ens_finalize(const EnsPointItem* items, int n, const int* active,
                                double* err, cudaStream_t st);

cudaError_t launch_periodic_predict(const PeriodicPointArgs& a,
                                    const double2* state, const double2* rhs,
                                    double2* out, cudaStream_t st);
// pred_out = pred + c (next - prev) ildt_2; partials of k_metric |corr|^2.
cudaError_t launch_periodic_correct(const PeriodicPointArgs& a,
                                    const double2* pred,
                                    const double2* rhs_prev,
                                    const double2* rhs_next, double2* pred_out,
                                    double2* corr_out, double* partials,
                                    cudaStream_t st);
cudaError_t launch_periodic_norm2(const PeriodicPointArgs& a,
                                  const double2* v, double* partials,
                                  cudaStream_t st);
cudaError_t launch_periodic_correct_velocity(const PeriodicPointArgs& a,
                                             const double2* in, double2* out,
                                             int divergence, cudaStream_t st);
cudaError_t launch_periodic_project(const PeriodicPointArgs& a, double2* rhs,
                                   cudaStream_t st);
// partials[0..kRedBlocks) of k_metric|u|^2, partials[kRedBlocks..2 kRedBlocks)
// of -lapl |u|^2.
cudaError_t launch_periodic_stats(const PeriodicPointArgs& a,
                                  const double2* v, double* partials,
                                  cudaStream_t st);

// ---- plane Couette ---------------------------------------------------------
struct ImmArgs {
  int NZ1, NKX, Ny, kl, ku;
  int s1, s2;             // D1 / D2 stencil widths (p+1, p+2)
  const int* d1_j0;       // [Ny]
  const double* d1_w;     // [Ny][s1]
  const int* d2_j0;       // [Ny]
  const double* d2_w;     // [Ny][s2]
  const double* d1_wT;    // [s1][Ny] (the same weights, tap-major)
  const double* d2_wT;    // [s2][Ny]
  const double* kx;       // [NKX]
  const double* kz;       // [NZ1]
  const double* simpson;  // [Ny] Simpson weights (norm)
  double dt, c, nu;
  // IMM operators, reference layouts (cartesian.py:575-801)
  const double* Lk_ab;    // [NZ1][NKX][2kl+ku+1][Ny]
  const int* Lk_piv;      // [NZ1][NKX][Ny]
  const double* Hk_ab;
  const int* Hk_piv;
  const double* v1;       // [NZ1][NKX][Ny]
  const double* v2;
  const double* q1;
  const double* q2;
  const double* M_inv;    // [NZ1][NKX][2][2]
  int* status;            // set nonzero on a pivot index out of range
  int ab_row0;            // first ab row with a nonzero entry in any mode
  int pair_modes;         // 1: (s, kx) and (nz-1-s, kx) share LU factors
  int kx0;                // 1: local kx index 0 is the kx = 0 mode (norm weight 1)
  // Unrolled step-graph iterations (the batched pipeline): when non-null and
  // *skip != 0, every kernel of the call returns at once.
  const int* skip = nullptr;
};

constexpr int kImmWarps = 4;  // modes per CTA (one warp each)

// vel_new = IMM(vel_n, vel_j, nl_n, nl_j); partials[mode] gets the
// Simpson-weighted k_metric |vel_new - vel_j|^2 of the mode when partials
// is non-null; corr_out (nullable) receives vel_new - vel_j.
cudaError_t launch_imm(const ImmArgs& a, const double2* vel_n,
                       const double2* vel_j, const double2* nl_n,
                       const double2* nl_j, double2* vel_new,
                       double2* corr_out, double* partials, cudaStream_t st);
size_t imm_smem(int Ny);
cudaError_t set_solver_attributes(int max_smem);

// Register-window IMM kernel (kl in {2, 4, 6, 8}), one warp per mode.
bool imm_v2_supported(int kl, int ny);
size_t imm_v2_smem(int Ny, int kl, int row0);
cudaError_t launch_imm_v2(const ImmArgs& a, const double2* vel_n,
                          const double2* vel_j, const double2* nl_n,
                          const double2* nl_j, double2* vel_new,
                          double2* corr_out, double* partials, cudaStream_t st);
cudaError_t set_imm_v2_attributes(int max_smem);
cudaError_t launch_ab_first_row(const double* ab, long long nmodes, int rows,
                                int ny, int kuu, int* out, cudaStream_t st);
cudaError_t launch_ab_pair_check(const double* ab, const int* piv, int nz1,
                                 int nkx, int rows, int ny, int* out,
                                 cudaStream_t st);

// Five-kernel IMM iteration (csrc/imm_batch.cu) over factors repacked at
// bind time (record-major, item index fastest; 1/U_jj and U/U_jj pre-scaled;
// pivots as validated offsets) and workspace F [NM][Ny], R [3][NM][Ny].
struct ImmBatch {
  // per operator (0 = L_k, 1 = H_k), 32-item tiles (csrc/imm_batch.cu)
  const double* facL[2];
  const double* facU[2];
  const unsigned char* dp[2];
  int NP;        // items: (nz-1+1)/2 * nx/2 when paired, else all modes
  int nu;        // stored superdiagonals (kl+1 or 2 kl)
  int paired;    // mirror mode (nz-1-s, kx) reads item (s, kx)'s factors
  int max_smem;  // per-CTA shared-memory limit of the device
  int* status;   // bit 1: bad pivot, bit 2: a substitution ring wait timed out
  int wait_limit;  // polls of a ring slot's mbarrier before the wait gives up
  double2* F;
  double2* R;
};
// Influence-matrix precompute (csrc/precompute.cu); every pointer is device
// memory, D1 / D2 dense (ny, ny) row-major, outputs in the reference's
// layouts ([nkz][nkx][...]).
struct ImmPrecomputeArgs {
  const double* D1;
  const double* D2;
  const double* kx;  // [nkx]
  const double* kz;  // [nkz]
  int nkx, nkz, ny, p;
  double dt, c, nu;
  double *p1, *p2, *v1, *v2, *q1, *q2;  // [nkz][nkx][ny]
  double* M_inv;                         // [nkz][nkx][2][2]
  double* Lk_ab;                         // [nkz][nkx][3p+1][ny]
  int* Lk_piv;                           // [nkz][nkx][ny], 0-based
  double* Hk_ab;
  int* Hk_piv;
  int* info;    // bit 1: zero pivot in some L_k, bit 2: in some H_k
  int* status;  // bit 0: a pivot out of range in a substitution
};
// bp: nkz*nkx*ny*2 doubles, bv: nkz*nkx*ny*4 doubles of workspace.
cudaError_t launch_imm_precompute(const ImmPrecomputeArgs& a, double* bp, double* bv,
                                  cudaStream_t st, int* launches);
// Learned corrector guess (csrc/learned.cu): BF16 MLP kernels.
cudaError_t launch_mlp_gemm(int ta, int tb, int M, int N, int K, const void* A, int lda,
                            const void* B, int ldb, const float* bias, int relu,
                            const void* mask, int ldm, float* Cf, void* Cb, int ldc, float* work,
                            long long work_elems, int* status, cudaStream_t st, int* launches);
// tcgen05 GEMM C = A B^T with K-contiguous BF16 operands (csrc/mlp_tc.cu).
bool tc_gemm_supported(const void* A, int lda, const void* B, int ldb);
cudaError_t launch_tc_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                           const float* bias, int relu, const void* mask, int ldm, float* Cf,
                           void* Cb, int ldc, float* work, long long work_elems, int* status,
                           cudaStream_t st, int* launches);
cudaError_t launch_bf16_transpose(const void* in, int R, int C, int ldi, void* out, int ldo,
                                  cudaStream_t st);
int colsum_groups(int M);
cudaError_t launch_colsum_det(const void* A, int bf16, int M, int N, int lda, float* out,
                              float* work, cudaStream_t st);
cudaError_t launch_learned_features(const double2* un, const double2* up, const double2* dprev,
                                    const double2* target, const double* kx, const double* kz,
                                    int NKX, int NZ1, int Ny, double kx_max, double kz_max,
                                    double s_floor, void* X, int ldx, float* T, int ldt,
                                    float* scale, cudaStream_t st);
cudaError_t launch_learned_guess(const double2* up, const float* Y, int ldy, const float* scale,
                                 int NM, int Ny, double2* out, cudaStream_t st);
cudaError_t launch_mlp_loss_grad(const float* Y, const float* T, int M, int N, int ld, float* dYf,
                                 void* dYb, float* err, float* ref, cudaStream_t st);
cudaError_t launch_mlp_adam(float* w, float* m, float* v, const float* grad, void* wb,
                            long long n, float lr, float b1, float b2, float eps, int step,
                            cudaStream_t st);
bool imm_batch_supported(int kl, int ny);
size_t imm_batch_stage_smem(int Ny);
int imm_nu(int kl, int row0);
bool imm_batch_fits(int kl, int nu, int max_smem);
cudaError_t launch_imm_repack(const double* ab, const int* piv, int Ny, int kl, int nu,
                              int row0, int NP, int ntiles, double* facL, double* facU,
                              unsigned char* dp, int* status, cudaStream_t st);
cudaError_t launch_imm_batch(const ImmArgs& a, const ImmBatch& bt, const double2* vel_n,
                             const double2* vel_j, const double2* nl_n,
                             const double2* nl_j, double2* vel_new, double2* corr_out,
                             double* partials, cudaStream_t st);
cudaError_t set_imm_batch_attributes(int max_smem);

// Simpson-weighted k_metric |v|^2 per block (Couette norm).
cudaError_t launch_couette_norm2(const ImmArgs& a, const double2* v,
                                 double* partials, cudaStream_t st);

// ---- library-wide error / launch bookkeeping (capi.cu) ----------------------
int set_last_error(int code, const std::string& msg);
void count_launches(int n);

// ---- standalone per-mode banded solve (PerModeBandedOperator.solve) -------
cudaError_t launch_banded_solve(const double* ab, const int* ipiv, double* b,
                                int nmodes, int ny, int kl, int ku,
                                int ncols, int* status, cudaStream_t st);

}  // namespace dnsb
