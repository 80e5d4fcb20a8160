// Axis-pass kernels of the dealiased transforms (declarations + arg blocks).
//
// A 3/2-dealiased transform is a sequence of axis passes; each pass reads
// one layout from HBM, transforms a tile of columns in shared memory and
// writes the next layout.  Zero-padding (inverse) and truncation (forward)
// happen on load/store, and the curl, the rotational nonlinear product and
// the pressure projection are fused into the passes that already hold the
// data they need.
#pragma once

#include "common.cuh"

namespace dnsb {

constexpr int kTile = 8;     // columns per CTA in the column passes
constexpr int kXRows = 4;    // physical rows per CTA in the x pass
constexpr int kPassThreads = 256;
constexpr int kX2Rows = 4;       // physical rows per CTA in the two-stage x pass
constexpr int kX2Threads = 96;   // one item per thread in every stage
size_t x_pass2_smem(int M, int nkx);

// Slab exchange (the reference's slab scheme over several GPUs): a pass
// that feeds the other layout stores each output straight into the
// buffer of the rank that owns it, through that rank's pointer (peer
// memory, or a buffer of this GPU when the ranks are emulated on one).
constexpr int kMaxRanks = 8;
struct SlabDest {
  double2* buf[kMaxRanks];  // receive buffer of each rank (null: no slab store)
  int blk;                  // extent of the split coordinate per rank
  long long fs, ts;         // destination field / split-coordinate strides
  long long off;            // offset of this rank's share in every destination
  long long so, si;         // x pass: destination row (outer + oo, inner + io)
  int oo, io;
  long long ks;             // x pass: destination kx stride
};

// Generic strided column pass: element (f, o, t, i) at
// base + f*fs + o*os + t*ts + i, with i the contiguous inner index.
struct ColPassArgs {
  const double2* in;
  double2* out;
  long long in_fs, out_fs, in_os, out_os, in_ts, out_ts;
  int nI;        // inner extent
  int nstored;   // stored (Nyquist-free) modes on the spectral side
  int inverse;   // 1: spectral -> padded, inverse FFT; 0: forward, truncate
  FFTPlan plan;  // transform length M = plan.L
  const double2* tw;
  int fp32;            // `in` and arithmetic in FP32 (compile-time sizes)
  int out32;           // with fp32: `out` is an FP32 pass buffer (always for inverse)
  int variant;         // 0: two-stage register pass when compiled for L, 1: Stockham
                       // stages (compile-time plan when compiled for L), 2: runtime plan
  // curl (inverse only, two-stage pass): `in` is the FP64 spectral state
  // [3][nstored][nO][nI] (component stride in_fs) and the 6 output fields are
  // u, v, w and i (k x u) with k = (kx[inner], ky[stored], kz[outer])
  int curl;
  const double* kx;
  const double* ky;
  const double* kz;
  int occ4;  // FP64 two-stage pass held to 4 CTAs per SM (128 registers)
  // Slab store (inverse, FP64 two-stage pass): position t goes to
  // slab.buf[t / blk] + f*fs + o*out_os + (t % blk)*ts + off + i, instead of
  // out + f*out_fs + o*out_os + t*out_ts + i.
  SlabDest slab;
  // Unrolled step-graph iterations: when non-null and *skip != 0 (the
  // corrector loop ended earlier in the step), the kernel returns at once.
  const int* skip = nullptr;
};

// x pass.  Rows are (outer, inner) pairs; row r = outer * inner_n + inner
// starts at outer*so + inner*si and its kx modes are ks apart.
struct XPassArgs {
  const double2* in;   // 6 fields (u, omega) of x-half-spectra
  double2* out;        // 3 fields of the forward x-transformed product
  long long in_fs, out_fs;
  int nrows, inner_n;
  long long so, si, ks;
  int nkx;             // stored kx modes (nx/2)
  int y_outer;         // y index = outer (1) or inner (0)
  int rows_fast;       // load mapping: rows contiguous (1) or kx (0)
  const double* U;     // base flow [3][ny_grid]
  const double* cU;    // curl of base flow
  const double* nU;    // U x curl U
  int ny_grid;
  FFTPlan plan;        // Mx
  const double2* tw;   // float2 table when fp32
  int fp32;            // pass buffer and arithmetic in FP32 (compile-time sizes)
  int variant;         // 0: two-stage register pass when compiled for L, 1: Stockham
                       // stages (compile-time plan when compiled for L), 2: runtime plan
  // Slab store (FP64 two-stage pass): mode k of field f of row (outer,
  // inner) goes to slab.buf[k / blk] + f*fs + (outer + oo)*so +
  // (inner + io)*si + (k % blk)*ks, instead of into `out`.
  SlabDest slab;
  // Unrolled step-graph iterations: when non-null and *skip != 0 (the
  // corrector loop ended earlier in the step), the kernel returns at once.
  const int* skip = nullptr;
};

// x pass to physical space only (3 fields -> real [c] at row offsets
// outer*pso + inner*psi, x contiguous).
struct XPhysArgs {
  const double2* in;
  double* out;
  long long in_fs, out_fs;
  int nrows, inner_n;
  long long so, si, ks, pso, psi;
  int nkx;
  int rows_fast;
  FFTPlan plan;
  const double2* tw;
};

// Periodic first inverse pass (y), curl fused: spectral u [3][NY1][NZ1][NKX]
// -> 6 (or 3) fields [f][My][NZ1][NKX].
struct YInvArgs {
  const double2* u;
  double2* out;
  int NY1, NZ1, NKX;
  int curl;
  const double* kx;
  const double* ky;
  const double* kz;
  FFTPlan plan;
  const double2* tw;
  int fp32;  // FP32 transform and output pass buffer (tw: float2 table)
  int variant;  // 0 / 1: compile-time plan when compiled for L, 2: runtime plan
};

// Periodic last forward pass (y), projection fused: [3][My][NZ1][NKX] ->
// spectral [3][NY1][NZ1][NKX].
struct YFwdArgs {
  const double2* in;
  double2* out;
  int NY1, NZ1, NKX;
  int project;
  const double* kx;
  const double* ky;
  const double* kz;
  const double* inv_lapl;  // [NY1][NZ1][NKX]
  FFTPlan plan;
  const double2* tw;
  int fp32;  // FP32 input pass buffer and transform (tw: float2 table)
  int variant;  // 0 / 1: compile-time plan when compiled for L, 2: runtime plan
};

// Couette first inverse pass (z), FD curl fused: spectral
// [3][NZ1][NKX][Ny] -> 6 (or 3) fields [f][Mz][NKX][Ny].
struct ZInvCurlArgs {
  const double2* u;
  double2* out;
  int NZ1, NKX, Ny;
  int curl;
  int s1;              // D1 stencil width (p + 1)
  const int* d1_j0;    // [Ny]
  const double* d1_w;  // [Ny][s1]
  const double* d1_wT; // [s1][Ny] (the same weights, tap-major)
  const double* kx;
  const double* kz;
  FFTPlan plan;
  const double2* tw;   // float2 table when fp32
  int fp32;            // output pass buffer and FFT in FP32 (compile-time sizes)
  int variant;         // 0: two-stage register pass when compiled for L, 1: Stockham
                       // stages (compile-time plan when compiled for L), 2: runtime plan
  // Slab store (FP64 two-stage pass): position t of column q goes to
  // slab.buf[t / blk] + f*fs + (t % blk)*ts + off + q.
  SlabDest slab;
  // Unrolled step-graph iterations: when non-null and *skip != 0 (the
  // corrector loop ended earlier in the step), the kernel returns at once.
  const int* skip = nullptr;
};

constexpr int kZTile = 8;  // y values per CTA in the Couette z passes

size_t col_pass_smem(int M);
size_t x_pass_smem(int Mx);
size_t x_phys_smem(int Mx);
size_t yinv_smem(int My, int NY1, int fp32);
size_t yfwd_smem(int My, int NY1, int fp32);
size_t zinv_curl_smem(int Mz, int NZ1, int span_max);
size_t zinv_curl2_smem(int M);

cudaError_t launch_col_pass(const ColPassArgs& a, int nfields, int nO,
                            cudaStream_t st);
cudaError_t launch_x_pass(const XPassArgs& a, cudaStream_t st);

// Work lists of the ensemble form (one launch per pass for every member;
// FP64 two-stage passes, padded lengths 48, 72, 96, 192).
struct EnsColItem {
  ColPassArgs a;
  int gx, gy;  // the member's grid (gx, gy, nfields), flattened bx fastest
  int member;
};
struct EnsXItem {
  XPassArgs a;
  int member;
};
bool ens_pass_supported(int L);
int ens_col_blocks(const ColPassArgs& a, int nO, int nfields, int* gx, int* gy);
int ens_x_blocks(const XPassArgs& a);
size_t ens_col_smem(int maxL);
size_t ens_x_smem(int maxL, int maxNKX);
// kind 0: inverse pass with the spectral curl, 1: inverse, 2: forward
// (column passes); 3: the x pass.  base[k]: first virtual block of item k.
int ens_pass_grid(int kind, size_t smem, int total, int max_smem);
cudaError_t launch_ens_pass(int kind, const void* items, const int* base, int n, int total,
                            const int* active, int grid, size_t smem, cudaStream_t st);
cudaError_t launch_x_phys(const XPhysArgs& a, cudaStream_t st);
// Forward x pass from physical rows (uses XPhysArgs with in_fs = spectral
// field stride, out_fs = physical field stride).
cudaError_t launch_x_fwd(const XPhysArgs& a, const double* phys, double2* spec,
                         cudaStream_t st);
size_t x_fwd_smem(int Mx);
cudaError_t set_pass_attributes(int max_smem);
cudaError_t launch_yinv(const YInvArgs& a, cudaStream_t st);
cudaError_t launch_yfwd(const YFwdArgs& a, cudaStream_t st);
cudaError_t launch_zinv_curl(const ZInvCurlArgs& a, int span_max,
                             cudaStream_t st);

FFTPlan make_plan(int L);  // host; L.nst == 0 when L is not 2^a 3^b

}  // namespace dnsb
