// C ABI of libdnsb.so (include/dnsb.h): contexts, workspace, and the
// launch sequences of the time-step operations.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/dnsb.h"
#include "passes.cuh"
#include "solver.cuh"

using namespace dnsb;

namespace {

thread_local std::string g_last_error;
std::atomic<long long> g_launches{0};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define DNSB_CUDA(call)                                                     \
  do {                                                                      \
    cudaError_t e_ = (call);                                                \
    if (e_ != cudaSuccess)                                                  \
      return fail(DNSB_ERR_CUDA, std::string(#call) + ": " +               \
                                     cudaGetErrorString(e_));               \
  } while (0)

// Counts one kernel launch and checks its launch status.
#define DNSB_LAUNCH(call)                                                   \
  do {                                                                      \
    g_launches.fetch_add(1, std::memory_order_relaxed);                     \
    DNSB_CUDA(call);                                                        \
  } while (0)

template <typename T>
int upload(T** dst, const T* src, size_t n) {
  *dst = nullptr;
  if (n == 0) return 0;
  if (!src) return fail(DNSB_ERR_ARG, "null host array");
  DNSB_CUDA(cudaMalloc((void**)dst, n * sizeof(T)));
  DNSB_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// tw[m] = exp(-2 pi i m / L), evaluated in long double.
int make_twiddles(double2** dst, int L) {
  std::vector<double2> h(L);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int m = 0; m < L; ++m) {
    const long double a = 2.0L * pi * (long double)m / (long double)L;
    h[m] = make_double2((double)cosl(a), (double)(-sinl(a)));
  }
  return upload(dst, h.data(), (size_t)L);
}

// The same table rounded to single precision (FP32 passes).
int make_twiddles32(float2** dst, int L) {
  std::vector<float2> h(L);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int m = 0; m < L; ++m) {
    const long double a = 2.0L * pi * (long double)m / (long double)L;
    h[m] = make_float2((float)cosl(a), (float)(-sinl(a)));
  }
  return upload(dst, h.data(), (size_t)L);
}

bool fft_size_ok(int L) { return L >= 1 && make_plan(L).nst > 0; }

int max_smem_optin() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

namespace dnsb {
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace dnsb

// Slab decomposition over several GPUs (the reference's scheme,
// fft.py:193-392 and sharding.py:107-129): a context of rank `rank` of
// `nranks` holds the kx modes [rank NKX, (rank + 1) NKX) of the NKXg of the
// whole problem (its NKX is the local count); the x pass works on a share
// of Mz / nranks padded-z rows with every kx mode, in Bx.  xdest / kdest:
// every rank's Bx and kx-sharded pass buffer, as this process addresses
// them.
struct SlabState {
  int nranks = 0, rank = 0, NKXg = 0;
  double2* Bx = nullptr;
  double2* xdest[kMaxRanks] = {};
  double2* kdest[kMaxRanks] = {};
  bool connected = false;
};

// ===========================================================================
// Triply periodic
// ===========================================================================
struct dnsb_periodic {
  int NY1, NZ1, NKX, My, Mz, Mx, S;
  double c;
  FFTPlan py, pz, px;
  double2 *twy = nullptr, *twz = nullptr, *twx = nullptr;
  float2 *twy32 = nullptr, *twz32 = nullptr, *twx32 = nullptr;
  double *kx = nullptr, *ky = nullptr, *kz = nullptr;
  double *U = nullptr, *cU = nullptr, *nU = nullptr;
  double *ldt1 = nullptr, *ildt2 = nullptr, *lapl = nullptr, *inv_lapl = nullptr;
  double2 *A = nullptr, *B = nullptr;
  double* partials = nullptr;
  size_t ws_bytes = 0;
  int rhs_fp32 = 0;  // RHS transforms and product in FP32 (pass buffers float2)
  int var[5] = {0, 0, 0, 0, 0};  // pass variants: y inverse, z inverse, x, z forward, y forward
  SlabState slab;                 // nranks > 0: a slab context
  int graph_unroll = 0;           // corrector iterations step graphs capture unrolled
  // set only while a step graph captures an unrolled iteration: the device
  // flag that makes the iteration's kernels return at once
  const int* skip = nullptr;

  PeriodicPointArgs point() const {
    PeriodicPointArgs a;
    a.S = S;
    a.NY1 = NY1;
    a.NZ1 = NZ1;
    a.NKX = NKX;
    a.ldt_1 = ldt1;
    a.ildt_2 = ildt2;
    a.kx = kx;
    a.ky = ky;
    a.kz = kz;
    a.inv_lapl = inv_lapl;
    a.lapl = lapl;
    a.c = c;
    a.kx0 = slab.rank == 0 ? 1 : 0;
    a.skip = skip;
    return a;
  }
};

static void periodic_free(dnsb_periodic* p) {
  void* ptrs[] = {p->twy, p->twz, p->twx, p->twy32, p->twz32, p->twx32, p->kx, p->ky,
                  p->kz, p->U, p->cU, p->nU, p->ldt1, p->ildt2, p->lapl, p->inv_lapl,
                  p->A, p->B, p->partials, p->slab.Bx};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete p;
}

extern "C" int dnsb_version(void) { return 1; }
extern "C" const char* dnsb_last_error(void) { return g_last_error.c_str(); }
extern "C" long long dnsb_launch_count(void) { return g_launches.load(); }

extern "C" int dnsb_periodic_create(const dnsb_periodic_desc* d,
                                    dnsb_periodic** out) {
  if (!d || !out) return fail(DNSB_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->nx < 2 || d->ny < 2 || d->nz < 2 || d->nx % 2 || d->ny % 2 || d->nz % 2)
    return fail(DNSB_ERR_ARG, "nx, ny, nz must be even and >= 2");
  if (!fft_size_ok(d->nx_p) || !fft_size_ok(d->ny_p) || !fft_size_ok(d->nz_p))
    return fail(DNSB_ERR_ARG, "padded sizes must be of the form 2^a 3^b");
  if (d->nx_p % 2 || d->nx_p < d->nx || d->ny_p < d->ny || d->nz_p < d->nz ||
      (d->ny_p - d->ny) % 2 || (d->nz_p - d->nz) % 2)
    return fail(DNSB_ERR_ARG, "padded sizes incompatible with the 3/2 rule");
  dnsb_periodic* p = new dnsb_periodic();
  p->NY1 = d->ny - 1;
  p->NZ1 = d->nz - 1;
  p->NKX = d->nx / 2;
  p->My = d->ny_p;
  p->Mz = d->nz_p;
  p->Mx = d->nx_p;
  p->S = p->NY1 * p->NZ1 * p->NKX;
  p->c = d->implicitness;
  p->py = make_plan(p->My);
  p->pz = make_plan(p->Mz);
  p->px = make_plan(p->Mx);
  const int smax = max_smem_optin();
  const size_t need[] = {col_pass_smem(p->Mz), x_pass_smem(p->Mx),
                         x_phys_smem(p->Mx), x_fwd_smem(p->Mx),
                         yinv_smem(p->My, p->NY1, 0), yfwd_smem(p->My, p->NY1, 0)};
  for (size_t n : need)
    if ((int)n > smax) {
      periodic_free(p);
      return fail(DNSB_ERR_ARG, "grid too large for shared-memory tiles");
    }
  int rc = 0;
  auto chk = [&](int r) {
    if (r && !rc) rc = r;
  };
  chk(make_twiddles(&p->twy, p->My));
  chk(make_twiddles(&p->twz, p->Mz));
  chk(make_twiddles(&p->twx, p->Mx));
  chk(make_twiddles32(&p->twy32, p->My));
  chk(make_twiddles32(&p->twz32, p->Mz));
  chk(make_twiddles32(&p->twx32, p->Mx));
  chk(upload(&p->kx, d->kx, p->NKX));
  chk(upload(&p->ky, d->ky, p->NY1));
  chk(upload(&p->kz, d->kz, p->NZ1));
  chk(upload(&p->U, d->base_flow, 3 * (size_t)p->My));
  chk(upload(&p->cU, d->curl_base_flow, 3 * (size_t)p->My));
  chk(upload(&p->nU, d->nonlin_base_flow, 3 * (size_t)p->My));
  chk(upload(&p->ldt1, d->ldt_1, p->S));
  chk(upload(&p->ildt2, d->ildt_2, p->S));
  if (!rc) {
    // lapl = -(kx^2 + ky^2 + kz^2), inv_lapl = 1/lapl off the mean mode
    // (triply_periodic.py:59-67).
    std::vector<double> l(p->S), il(p->S);
    for (int iy = 0; iy < p->NY1; ++iy)
      for (int iz = 0; iz < p->NZ1; ++iz)
        for (int ix = 0; ix < p->NKX; ++ix) {
          const double a = d->kx[ix], b = d->ky[iy], cc = d->kz[iz];
          const double v = -(a * a + b * b + cc * cc);
          const int s = (iy * p->NZ1 + iz) * p->NKX + ix;
          l[s] = v;
          il[s] = v < 0 ? 1.0 / v : 0.0;
        }
    chk(upload(&p->lapl, l.data(), p->S));
    chk(upload(&p->inv_lapl, il.data(), p->S));
  }
  const size_t nA = 6ull * p->My * p->NZ1 * p->NKX;
  const size_t nB = 6ull * p->My * p->Mz * p->NKX;
  if (!rc) {
    cudaError_t e1 = cudaMalloc(&p->A, nA * sizeof(double2));
    cudaError_t e2 = cudaMalloc(&p->B, nB * sizeof(double2));
    cudaError_t e3 = cudaMalloc(&p->partials, 2 * kRedBlocks * sizeof(double));
    if (e1 || e2 || e3) rc = fail(DNSB_ERR_CUDA, "workspace allocation failed");
  }
  if (!rc) {
    cudaError_t e = set_pass_attributes(smax);
    if (e == cudaSuccess) e = set_solver_attributes(smax);
    if (e != cudaSuccess)
      rc = fail(DNSB_ERR_CUDA, std::string("cudaFuncSetAttribute: ") +
                                   cudaGetErrorString(e));
  }
  if (rc) {
    periodic_free(p);
    return rc;
  }
  p->ws_bytes = (nA + nB) * sizeof(double2) + 2 * kRedBlocks * sizeof(double);
  *out = p;
  return 0;
}

extern "C" int dnsb_periodic_destroy(dnsb_periodic* p) {
  if (p) periodic_free(p);
  return 0;
}

extern "C" size_t dnsb_periodic_workspace_bytes(const dnsb_periodic* p) {
  return p ? p->ws_bytes : 0;
}

// Inverse z pass over nf fields: A[f][y][kz][kx] -> B[f][y][z][kx].
static ColPassArgs periodic_zinv(const dnsb_periodic* p) {
  ColPassArgs a{};
  a.in = p->A;
  a.out = p->B;
  a.in_fs = (long long)p->My * p->NZ1 * p->NKX;
  a.out_fs = (long long)p->My * p->Mz * p->NKX;
  a.in_os = (long long)p->NZ1 * p->NKX;
  a.out_os = (long long)p->Mz * p->NKX;
  a.in_ts = p->NKX;
  a.out_ts = p->NKX;
  a.nI = p->NKX;
  a.nstored = p->NZ1;
  a.inverse = 1;
  a.plan = p->pz;
  a.tw = p->twz;
  a.occ4 = 1;  // measured faster at 4 CTAs per SM
  return a;
}

// Forward z pass over 3 fields: B[f][y][z][kx] -> A[f][y][kz][kx].
static ColPassArgs periodic_zfwd(const dnsb_periodic* p) {
  ColPassArgs a{};
  a.in = p->B;
  a.out = p->A;
  a.in_fs = (long long)p->My * p->Mz * p->NKX;
  a.out_fs = (long long)p->My * p->NZ1 * p->NKX;
  a.in_os = (long long)p->Mz * p->NKX;
  a.out_os = (long long)p->NZ1 * p->NKX;
  a.in_ts = p->NKX;
  a.out_ts = p->NKX;
  a.nI = p->NKX;
  a.nstored = p->NZ1;
  a.inverse = 0;
  a.plan = p->pz;
  a.tw = p->twz;
  a.occ4 = 1;  // measured faster at 4 CTAs per SM
  return a;
}

// y inverse with the curl as a two-stage column pass: state
// [comp][ky][kz][kx] -> A[f][y][kz][kx] (FP64 fields; the FP32 form sets its
// flags and table on top).
static ColPassArgs periodic_ycurl(const dnsb_periodic* p, const void* state) {
  ColPassArgs yc{};
  yc.in = (const double2*)state;
  yc.out = p->A;
  yc.in_fs = (long long)p->NY1 * p->NZ1 * p->NKX;
  yc.out_fs = (long long)p->My * p->NZ1 * p->NKX;
  yc.in_os = p->NKX;
  yc.out_os = p->NKX;
  yc.in_ts = (long long)p->NZ1 * p->NKX;
  yc.out_ts = (long long)p->NZ1 * p->NKX;
  yc.nI = p->NKX;
  yc.nstored = p->NY1;
  yc.inverse = 1;
  yc.plan = p->py;
  yc.tw = p->twy;
  yc.curl = 1;
  yc.kx = p->kx;
  yc.ky = p->ky;
  yc.kz = p->kz;
  yc.occ4 = 1;  // measured faster at 4 CTAs per SM
  return yc;
}

// x pass with the rotational product, in place on B[f][y][z][kx].
static XPassArgs periodic_xpass(const dnsb_periodic* p) {
  XPassArgs xa{};
  xa.in = p->B;
  xa.out = p->B;
  xa.in_fs = xa.out_fs = (long long)p->My * p->Mz * p->NKX;
  xa.nrows = p->My * p->Mz;
  xa.inner_n = p->Mz;
  xa.so = (long long)p->Mz * p->NKX;
  xa.si = p->NKX;
  xa.ks = 1;
  xa.nkx = p->NKX;
  xa.y_outer = 1;
  xa.rows_fast = 0;
  xa.U = p->U;
  xa.cU = p->cU;
  xa.nU = p->nU;
  xa.ny_grid = p->My;
  xa.plan = p->px;
  xa.tw = p->twx;
  return xa;
}

// y forward as a two-stage column pass with truncation, A[f][y][kz][kx] ->
// rhs[comp][ky][kz][kx] (complex128); the projection follows in place.
static ColPassArgs periodic_yfwd_col(const dnsb_periodic* p, void* rhs) {
  ColPassArgs yc{};
  yc.in = p->A;
  yc.out = (double2*)rhs;
  yc.in_fs = (long long)p->My * p->NZ1 * p->NKX;
  yc.out_fs = p->S;
  yc.in_os = p->NKX;
  yc.out_os = p->NKX;
  yc.in_ts = (long long)p->NZ1 * p->NKX;
  yc.out_ts = (long long)p->NZ1 * p->NKX;
  yc.nI = p->NKX;
  yc.nstored = p->NY1;
  yc.inverse = 0;
  yc.plan = p->py;
  yc.tw = p->twy;
  yc.occ4 = 1;  // measured faster at 4 CTAs per SM
  return yc;
}

// The five passes of the periodic RHS; bit k of `mask` runs pass k (y
// inverse, z inverse, x, z forward, y forward), each with its variant.
static int periodic_rhs_impl(dnsb_periodic* p, const void* state, void* rhs, unsigned mask,
                             cudaStream_t st) {
  YInvArgs yi{};
  yi.u = (const double2*)state;
  yi.out = p->A;
  yi.NY1 = p->NY1;
  yi.NZ1 = p->NZ1;
  yi.NKX = p->NKX;
  yi.curl = 1;
  yi.kx = p->kx;
  yi.ky = p->ky;
  yi.kz = p->kz;
  yi.plan = p->py;
  const int f32 = p->rhs_fp32;
  yi.tw = f32 ? reinterpret_cast<const double2*>(p->twy32) : p->twy;
  yi.fp32 = f32;
  yi.variant = p->var[0];
  auto fixed = [](int L) { return L == 48 || L == 72 || L == 96 || L == 192; };
  if ((mask & 1u) && p->var[0] == 0 && fixed(p->My)) {
    // y inverse with the curl as a two-stage column pass: state
    // [comp][ky][kz][kx] -> A[f][y][kz][kx]
    ColPassArgs yc = periodic_ycurl(p, state);
    yc.skip = p->skip;
    yc.tw = yi.tw;
    yc.fp32 = yc.out32 = f32;
    DNSB_LAUNCH(launch_col_pass(yc, 6, p->NZ1, st));
  } else if (mask & 1u) {
    DNSB_LAUNCH(launch_yinv(yi, st));
  }
  ColPassArgs zi = periodic_zinv(p);
  zi.skip = p->skip;
  zi.fp32 = zi.out32 = f32;
  if (f32) zi.tw = reinterpret_cast<const double2*>(p->twz32);
  zi.variant = p->var[1];
  if (mask & 2u) DNSB_LAUNCH(launch_col_pass(zi, 6, p->My, st));
  XPassArgs xa = periodic_xpass(p);
  xa.skip = p->skip;
  xa.tw = f32 ? reinterpret_cast<const double2*>(p->twx32) : p->twx;
  xa.fp32 = f32;
  xa.variant = p->var[2];
  if (mask & 4u) DNSB_LAUNCH(launch_x_pass(xa, st));
  ColPassArgs zf = periodic_zfwd(p);
  zf.skip = p->skip;
  zf.fp32 = zf.out32 = f32;
  if (f32) zf.tw = reinterpret_cast<const double2*>(p->twz32);
  zf.variant = p->var[3];
  if (mask & 8u) DNSB_LAUNCH(launch_col_pass(zf, 3, p->My, st));
  YFwdArgs yf{};
  yf.in = p->A;
  yf.out = (double2*)rhs;
  yf.NY1 = p->NY1;
  yf.NZ1 = p->NZ1;
  yf.NKX = p->NKX;
  yf.project = 1;
  yf.kx = p->kx;
  yf.ky = p->ky;
  yf.kz = p->kz;
  yf.inv_lapl = p->inv_lapl;
  yf.plan = p->py;
  yf.tw = f32 ? reinterpret_cast<const double2*>(p->twy32) : p->twy;
  yf.fp32 = f32;
  yf.variant = p->var[4];
  if ((mask & 16u) && p->var[4] == 0 && fixed(p->My)) {
    // y forward as a two-stage column pass with truncation, A[f][y][kz][kx]
    // -> rhs[comp][ky][kz][kx] (complex128), then the projection in place
    ColPassArgs yc = periodic_yfwd_col(p, rhs);
    yc.skip = p->skip;
    yc.tw = yf.tw;
    yc.fp32 = f32;
    DNSB_LAUNCH(launch_col_pass(yc, 3, p->NZ1, st));
    DNSB_LAUNCH(launch_periodic_project(p->point(), (double2*)rhs, st));
  } else if (mask & 16u) {
    DNSB_LAUNCH(launch_yfwd(yf, st));
  }
  return 0;
}

extern "C" int dnsb_periodic_rhs(dnsb_periodic* p, const void* state, void* rhs,
                                 void* stream) {
  if (!p || !state || !rhs) return fail(DNSB_ERR_ARG, "null argument");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab context: the RHS runs in phases");
  return periodic_rhs_impl(p, state, rhs, 31u, as_stream(stream));
}

extern "C" int dnsb_periodic_set_rhs_precision(dnsb_periodic* p, int fp32) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  if (fp32 && p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts run the FP64 passes");
  if (fp32) {
    auto fixed = [](int L) { return L == 48 || L == 72 || L == 96 || L == 192; };
    if (!fixed(p->My) || !fixed(p->Mz) || !fixed(p->Mx) || 3 * p->NKX != p->Mx)
      return fail(DNSB_ERR_ARG,
                  "FP32 RHS passes need padded sizes in {48, 72, 96, 192} with nx_p = 3 nx / 2");
  }
  p->rhs_fp32 = fp32 < 0 ? 0 : (fp32 > 2 ? 2 : fp32);
  return 0;
}

extern "C" int dnsb_periodic_predict(dnsb_periodic* p, const void* state,
                                     const void* rhs, void* out,
                                     void* stream) {
  if (!p || !state || !rhs || !out) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_LAUNCH(launch_periodic_predict(p->point(), (const double2*)state,
                                      (const double2*)rhs, (double2*)out,
                                      as_stream(stream)));
  return 0;
}

extern "C" int dnsb_periodic_correct(dnsb_periodic* p, const void* pred,
                                     const void* rhs_prev,
                                     const void* rhs_next, void* pred_out,
                                     void* corr_out, double* err_dev,
                                     void* stream) {
  if (!p || !pred || !rhs_prev || !rhs_next || !pred_out)
    return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_LAUNCH(launch_periodic_correct(
      p->point(), (const double2*)pred, (const double2*)rhs_prev,
      (const double2*)rhs_next, (double2*)pred_out, (double2*)corr_out,
      err_dev ? p->partials : nullptr, st));
  // A slab rank returns its share of the squared norm (summed over the ranks
  // by the caller, who takes the square root).
  if (err_dev)
    DNSB_LAUNCH(launch_finalize(p->partials, kRedBlocks, err_dev, 1.0, p->slab.nranks ? 0 : 1,
                                st, p->skip));
  return 0;
}

extern "C" int dnsb_periodic_norm(dnsb_periodic* p, const void* v,
                                  double* out_dev, void* stream) {
  if (!p || !v || !out_dev) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_LAUNCH(launch_periodic_norm2(p->point(), (const double2*)v, p->partials, st));
  DNSB_LAUNCH(launch_finalize(p->partials, kRedBlocks, out_dev, 1.0, p->slab.nranks ? 0 : 1,
                              st));
  return 0;
}

extern "C" int dnsb_periodic_correct_velocity(dnsb_periodic* p, const void* v,
                                              void* out, int divergence,
                                              void* stream) {
  if (!p || !v || !out) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_LAUNCH(launch_periodic_correct_velocity(p->point(), (const double2*)v,
                                               (double2*)out, divergence,
                                               as_stream(stream)));
  return 0;
}

// ---------------------------------------------------------------------------
// One full time step as a CUDA graph: predictor and first correction, the
// corrector iterations as a device-controlled WHILE node (the reference
// driver's loop, __main__.py:166-180: iterate while error > tol and
// iterations < max_iter), then correct_velocity into the state.  Fixed
// buffers: the state (in / out) and the graph's own prediction, two RHS
// buffers and control words.  The WHILE body holds two iterations, the
// second inside an IF node, so the two RHS buffers alternate as previous
// and next without a copy: iteration A (RHS into Ra, previous Rb), then, if
// A did not end the loop, iteration B (RHS into Rb, previous Ra).
// ---------------------------------------------------------------------------
namespace dnsb {
// After a correction: count the iteration (first: the predictor's), keep
// the error, and set the loop's condition -- and, after iteration A, the IF
// node's (set_if) -- to "iterate again".
//
// skip (non-null for the first correction and the unrolled iterations): the
// flag of the unrolled iterations, set to "skip" once the loop has ended;
// after a skipped iteration the control kernel returns at once as well.
__global__ void step_ctl_kernel(cudaGraphConditionalHandle h, cudaGraphConditionalHandle h_if,
                                int set_if, const double* err, int* ctl, double* err_last,
                                double tol, int max_iter, int first, int* skip) {
  if (skip && !first && *skip) return;
  const int it = first ? 0 : ctl[0] + 1;
  const double e = err[0];
  const unsigned cont = (e > tol && it < max_iter) ? 1u : 0u;
  ctl[0] = it;
  err_last[0] = e;
  if (skip) *skip = cont ? 0 : 1;
  cudaGraphSetConditional(h, cont);
  if (set_if) cudaGraphSetConditional(h_if, cont);
}
}  // namespace dnsb

struct dnsb_step_graph {
  cudaGraphExec_t exec = nullptr;
  long long k_fixed = 0, k_iter = 0;  // kernels per step outside / per corrector iteration
  int unroll = 0;                     // corrector iterations captured unrolled
  double2 *P = nullptr, *Ra = nullptr, *Rb = nullptr;
  double* err = nullptr;  // [0] corrector error, [1] error of the last step
  int* ctl = nullptr;     // [0] corrector iterations of the last step, [1] skip flag
  // pinned host copies read by dnsb_step_graph_status (a copy into pageable
  // memory would not be asynchronous and could queue behind other copies)
  int* h_ctl = nullptr;
  double* h_err = nullptr;
};

static void step_graph_free(dnsb_step_graph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  void* ptrs[] = {g->P, g->Ra, g->Rb, g->err, g->ctl};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (g->h_ctl) cudaFreeHost(g->h_ctl);
  if (g->h_err) cudaFreeHost(g->h_err);
  delete g;
}

// Adds a conditional node of `type` to graph `gr` after the work captured so
// far on `st` (which captures into `gr`), makes it the stream's dependency,
// and returns the node's body graph (nullptr and rc set on failure).
static cudaGraph_t add_cond_node(cudaStream_t st, cudaGraph_t gr, cudaGraphConditionalHandle hd,
                                 cudaGraphConditionalNodeType type, int& rc) {
  if (rc) return nullptr;
  auto ck = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && !rc)
      rc = fail(DNSB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  cudaStreamCaptureStatus cst;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  ck(cudaStreamGetCaptureInfo(st, &cst, nullptr, nullptr, &deps, &ndeps), "capture info");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hd;
  cp.conditional.type = type;
  cp.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  if (!rc) ck(cudaGraphAddNode(&node, gr, deps, ndeps, &cp), "conditional node");
  if (!rc)
    ck(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies),
       "capture dependencies");
  return rc ? nullptr : cp.conditional.phGraph_out[0];
}

// Captures prologue (predictor and first correction, error into g->err),
// `unroll` corrector iterations as straight-line kernels
// (`body(stream, parity, skip)` with the skip flag, which their kernels check
// and which the control kernel sets once the loop has ended), the remaining
// iterations `body(stream, parity, nullptr)` (A) and the other parity (B)
// inside the WHILE node, and `epilogue`, with the control kernel after the
// prologue and after each iteration.  An unrolled iteration costs no
// conditional-node evaluation (measured about 30 us of idle GPU per WHILE
// or IF entry at 128x129x128); one after the loop has ended launches its
// kernels, which return at once.
static int build_step_graph(dnsb_step_graph* g, double tol, int max_iter,
                            const std::function<int(cudaStream_t)>& prologue,
                            const std::function<int(cudaStream_t, int, const int*)>& body,
                            const std::function<int(cudaStream_t)>& epilogue,
                            int unroll = 0) {
  cudaStream_t s = nullptr, sb = nullptr, si = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&si, cudaStreamNonBlocking);
  int rc = 0;
  auto ck = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && !rc)
      rc = fail(DNSB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  auto add_cond = [&](cudaStream_t st, cudaGraph_t gr, cudaGraphConditionalHandle hd,
                      cudaGraphConditionalNodeType type) {
    return add_cond_node(st, gr, hd, type, rc);
  };
  cudaGraph_t graph = nullptr;
  ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaStreamCaptureStatus cs;
  ck(cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, nullptr, nullptr), "capture info");
  cudaGraphConditionalHandle h = 0, h_if = 0;
  ck(cudaGraphConditionalHandleCreate(&h, graph, 0, 0), "conditional handle");
  // Captured calls count their launches; the graph's kernels are counted
  // when they run (dnsb_step_graph_status), so the capture's count is undone.
  const long long c0 = g_launches.load();
  int* skip = unroll > 0 ? g->ctl + 1 : nullptr;
  if (!rc) rc = prologue(s);
  dnsb::step_ctl_kernel<<<1, 1, 0, s>>>(h, 0, 0, g->err, g->ctl, g->err + 1, tol, max_iter, 1,
                                        skip);
  ck(cudaGetLastError(), "control kernel");
  for (int k = 0; k < unroll && !rc; ++k) {
    rc = body(s, k & 1, skip);
    dnsb::step_ctl_kernel<<<1, 1, 0, s>>>(h, 0, 0, g->err, g->ctl, g->err + 1, tol, max_iter,
                                          0, skip);
    ck(cudaGetLastError(), "control kernel");
  }
  g->unroll = unroll;
  const long long c1 = g_launches.load() + 1 + unroll;  // + the control kernels
  long long c2 = c1;
  cudaGraph_t bg = add_cond(s, graph, h, cudaGraphCondTypeWhile);
  if (!rc) {
    ck(cudaGraphConditionalHandleCreate(&h_if, bg, 0, 0), "conditional handle");
    ck(cudaStreamBeginCaptureToGraph(sb, bg, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal), "body capture");
    if (!rc) rc = body(sb, unroll & 1, nullptr);
    dnsb::step_ctl_kernel<<<1, 1, 0, sb>>>(h, h_if, 1, g->err, g->ctl, g->err + 1, tol,
                                           max_iter, 0, nullptr);
    ck(cudaGetLastError(), "control kernel");
    c2 = g_launches.load() + 1;  // + the control kernel of iteration A
    cudaGraph_t ig = add_cond(sb, bg, h_if, cudaGraphCondTypeIf);
    if (!rc) {
      ck(cudaStreamBeginCaptureToGraph(si, ig, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal), "IF body capture");
      if (!rc) rc = body(si, (unroll + 1) & 1, nullptr);
      dnsb::step_ctl_kernel<<<1, 1, 0, si>>>(h, 0, 0, g->err, g->ctl, g->err + 1, tol,
                                             max_iter, 0, nullptr);
      ck(cudaGetLastError(), "control kernel");
      cudaGraph_t iout = nullptr;
      ck(cudaStreamEndCapture(si, &iout), "end IF body capture");
    }
    cudaGraph_t bout = nullptr;
    ck(cudaStreamEndCapture(sb, &bout), "end body capture");
  }
  const long long c3 = g_launches.load();  // after both iterations
  if (!rc) rc = epilogue(s);
  const long long c4 = g_launches.load();
  g->k_iter = c2 - c1;                      // one iteration + its control kernel
  g->k_fixed = (c1 - c0) + (c4 - c3);       // prologue, unrolled iterations, epilogue
  g_launches.fetch_sub(c4 - c0, std::memory_order_relaxed);
  cudaGraph_t done = nullptr;
  ck(cudaStreamEndCapture(s, &done), "end capture");  // always end the capture
  if (!rc) ck(cudaGraphInstantiate(&g->exec, done, 0), "instantiate");
  if (done) cudaGraphDestroy(done);
  cudaStreamDestroy(s);
  cudaStreamDestroy(sb);
  cudaStreamDestroy(si);
  return rc;
}

static dnsb_step_graph* new_step_graph(size_t n) {
  auto* g = new dnsb_step_graph();
  if (cudaMalloc(&g->P, n * sizeof(double2)) || cudaMalloc(&g->Ra, n * sizeof(double2)) ||
      cudaMalloc(&g->Rb, n * sizeof(double2)) || cudaMalloc(&g->err, 2 * sizeof(double)) ||
      cudaMalloc(&g->ctl, 2 * sizeof(int)) || cudaMallocHost(&g->h_ctl, sizeof(int)) ||
      cudaMallocHost(&g->h_err, sizeof(double))) {
    step_graph_free(g);
    return nullptr;
  }
  return g;
}

// Corrector iterations a periodic step graph captures unrolled: the
// context's setting, when every kernel of an iteration checks the skip flag
// (the two-stage passes at the compiled sizes, the y forward as a column
// pass plus the projection), at most max_iter; otherwise none.
static int periodic_unroll(const dnsb_periodic* p, int max_iter) {
  auto fixed = [](int L) { return L == 48 || L == 72 || L == 96 || L == 192; };
  if (p->graph_unroll <= 0 || !fixed(p->My) || !fixed(p->Mz) || !fixed(p->Mx) ||
      3 * p->NKX != p->Mx)
    return 0;
  for (int k = 0; k < 5; ++k)
    if (p->var[k] != 0) return 0;
  return std::min(p->graph_unroll, std::max(max_iter, 0));
}

extern "C" int dnsb_periodic_set_graph_unroll(dnsb_periodic* p, int n) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  if (n < 0 || n > 64) return fail(DNSB_ERR_ARG, "unroll must be in [0, 64]");
  p->graph_unroll = n;
  return 0;
}

extern "C" int dnsb_periodic_step_graph_create(dnsb_periodic* p, void* state, double tol,
                                               int max_iter, int divergence,
                                               dnsb_step_graph** out) {
  if (!p || !state || !out) return fail(DNSB_ERR_ARG, "null argument");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts step through the host loop");
  const size_t n = 3 * (size_t)p->S;
  dnsb_step_graph* g = new_step_graph(n);
  if (!g) return fail(DNSB_ERR_CUDA, "step graph allocation failed");
  auto prologue = [&](cudaStream_t s) {
    int rc = dnsb_periodic_rhs(p, state, g->Ra, s);
    if (!rc) rc = dnsb_periodic_predict(p, state, g->Ra, g->P, s);
    if (!rc) rc = dnsb_periodic_rhs(p, g->P, g->Rb, s);
    if (!rc) rc = dnsb_periodic_correct(p, g->P, g->Ra, g->Rb, g->P, nullptr, g->err, s);
    return rc;
  };
  // one corrector iteration: A (parity 0) rhs_next -> Ra with rhs_prev Rb,
  // B (parity 1) the other way round
  auto body = [&](cudaStream_t s, int parity, const int* skip) {
    double2* nx = parity ? g->Rb : g->Ra;
    double2* pv = parity ? g->Ra : g->Rb;
    p->skip = skip;
    int rc = dnsb_periodic_rhs(p, g->P, nx, s);
    if (!rc) rc = dnsb_periodic_correct(p, g->P, pv, nx, g->P, nullptr, g->err, s);
    p->skip = nullptr;
    return rc;
  };
  auto epilogue = [&](cudaStream_t s) {
    return dnsb_periodic_correct_velocity(p, g->P, state, divergence, s);
  };
  const int rc = build_step_graph(g, tol, max_iter, prologue, body, epilogue,
                                 periodic_unroll(p, max_iter));
  if (rc) {
    step_graph_free(g);
    return rc;
  }
  *out = g;
  return 0;
}

extern "C" int dnsb_step_graph_launch(dnsb_step_graph* g, void* stream) {
  if (!g) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_CUDA(cudaGraphLaunch(g->exec, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_step_graph_status(dnsb_step_graph* g, int* iters, double* err,
                                      void* stream) {
  if (!g || !iters || !err) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_CUDA(cudaMemcpyAsync(g->h_ctl, g->ctl, sizeof(int), cudaMemcpyDeviceToHost, st));
  DNSB_CUDA(cudaMemcpyAsync(g->h_err, g->err + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
  DNSB_CUDA(cudaStreamSynchronize(st));
  *iters = *g->h_ctl;
  *err = *g->h_err;
  const long long looped = *iters > g->unroll ? *iters - g->unroll : 0;
  g_launches.fetch_add(g->k_fixed + looped * g->k_iter, std::memory_order_relaxed);
  return 0;
}

extern "C" int dnsb_step_graph_destroy(dnsb_step_graph* g) {
  if (!g) return fail(DNSB_ERR_ARG, "null argument");
  step_graph_free(g);
  return 0;
}

// ===========================================================================
// Ensembles as work lists: one launch per stage for every member
// ===========================================================================
namespace dnsb {
// After a correction of every active member: count the iteration (first: the
// predictor's correction), keep the errors, and set the loop's condition --
// and, after iteration A, the IF node's (set_if) -- to "some member iterates
// again", per member as step_ctl_kernel decides for one trajectory.
__global__ void ens_ctl_kernel(cudaGraphConditionalHandle h, cudaGraphConditionalHandle h_if,
                               int set_if, int n, const double* err, const double* tol,
                               const int* max_iter, int* iters, int* active, double* err_last,
                               int first) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    int act = 0;
    if (first || active[m]) {
      const int it = first ? 0 : iters[m] + 1;
      const double e = err[m];
      iters[m] = it;
      err_last[m] = e;
      act = (e > tol[m] && it < max_iter[m]) ? 1 : 0;
    }
    active[m] = act;
    if (act) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cudaGraphSetConditional(h, any ? 1u : 0u);
    if (set_if) cudaGraphSetConditional(h_if, any ? 1u : 0u);
  }
}
}  // namespace dnsb

struct dnsb_ensemble {
  int n = 0;
  cudaGraphExec_t exec = nullptr;
  std::vector<void*> bufs;  // device allocations owned by the ensemble
  long long k_fixed = 0, k_iter = 0;
  int* iters = nullptr;
  double* err_last = nullptr;
};

static void ensemble_free(dnsb_ensemble* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  for (void* q : e->bufs)
    if (q) cudaFree(q);
  delete e;
}

namespace {
// One stage's work list on the device: items, their first virtual blocks,
// the total and the persistent grid.
struct EnsStage {
  const void* items = nullptr;
  const int* base = nullptr;
  int n = 0, total = 0, grid = 0;
  size_t smem = 0;
  int kind = 0;
};

template <typename T>
int ens_upload(dnsb_ensemble* e, const std::vector<T>& h, T** d) {
  *d = nullptr;
  if (cudaMalloc((void**)d, h.size() * sizeof(T)) != cudaSuccess)
    return fail(DNSB_ERR_CUDA, "ensemble allocation failed");
  e->bufs.push_back(*d);
  if (cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(DNSB_ERR_CUDA, "ensemble upload failed");
  return 0;
}
}  // namespace

// Members: periodic contexts in FP64 with the default pass variants and
// padded lengths 48, 72, 96 or 192 with nx_p = 3 nx / 2; each bound to its
// state (updated in place by every step).
extern "C" int dnsb_ensemble_create(dnsb_periodic* const* ctxs, void* const* states, int n,
                                    const double* tol, const int* max_iter, int divergence,
                                    dnsb_ensemble** out) {
  using namespace dnsb;
  if (!ctxs || !states || !tol || !max_iter || !out || n < 1)
    return fail(DNSB_ERR_ARG, "null argument or no members");
  if (n > 1024) return fail(DNSB_ERR_ARG, "at most 1024 members");
  for (int m = 0; m < n; ++m) {
    const dnsb_periodic* p = ctxs[m];
    if (!p || !states[m]) return fail(DNSB_ERR_ARG, "null member");
    if (p->rhs_fp32) return fail(DNSB_ERR_ARG, "ensemble members run in FP64");
    for (int k = 0; k < 5; ++k)
      if (p->var[k] != 0) return fail(DNSB_ERR_ARG, "ensemble members use the default variants");
    if (p->slab.nranks) return fail(DNSB_ERR_ARG, "ensemble members are whole contexts");
    if (!ens_pass_supported(p->My) || !ens_pass_supported(p->Mz) ||
        !ens_pass_supported(p->Mx) || 3 * p->NKX != p->Mx)
      return fail(DNSB_ERR_ARG, "ensemble members need padded lengths 48, 72, 96 or 192 "
                                "with nx_p = 3 nx / 2");
  }
  auto* e = new dnsb_ensemble();
  e->n = n;
  int rc = 0;
  auto alloc = [&](size_t bytes) -> void* {
    void* q = nullptr;
    if (!rc && cudaMalloc(&q, bytes) != cudaSuccess)
      rc = fail(DNSB_ERR_CUDA, "ensemble allocation failed");
    if (q) e->bufs.push_back(q);
    return q;
  };
  std::vector<double2*> P(n), Ra(n), Rb(n);
  for (int m = 0; m < n && !rc; ++m) {
    const size_t b = 3 * (size_t)ctxs[m]->S * sizeof(double2);
    P[m] = (double2*)alloc(b);
    Ra[m] = (double2*)alloc(b);
    Rb[m] = (double2*)alloc(b);
  }
  auto* err = (double*)alloc(n * sizeof(double));
  e->err_last = (double*)alloc(n * sizeof(double));
  e->iters = (int*)alloc(n * sizeof(int));
  auto* active = (int*)alloc(n * sizeof(int));
  double* d_tol = nullptr;
  int* d_max = nullptr;
  if (!rc) rc = ens_upload(e, std::vector<double>(tol, tol + n), &d_tol);
  if (!rc) rc = ens_upload(e, std::vector<int>(max_iter, max_iter + n), &d_max);
  if (rc) {
    ensemble_free(e);
    return rc;
  }
  // members ordered by size, largest first, so the persistent CTAs start
  // on the longest blocks
  std::vector<int> order(n);
  for (int m = 0; m < n; ++m) order[m] = m;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return ctxs[a]->S > ctxs[b]->S; });
  const int smax = max_smem_optin();
  int maxL = 0, maxNKX = 0;
  for (int m = 0; m < n; ++m) {
    maxL = std::max({maxL, ctxs[m]->My, ctxs[m]->Mz, ctxs[m]->Mx});
    maxNKX = std::max(maxNKX, ctxs[m]->NKX);
  }
  // kind 0..3: col (curl), col (inverse), col (forward), x pass
  auto col_stage = [&](int kind, auto make, int nfields, auto nO) -> EnsStage {
    EnsStage st;
    st.kind = kind;
    std::vector<EnsColItem> items;
    std::vector<int> base;
    int total = 0;
    for (int m : order) {
      EnsColItem it{};
      it.a = make(ctxs[m], m);
      it.member = m;
      base.push_back(total);
      total += ens_col_blocks(it.a, nO(ctxs[m]), nfields, &it.gx, &it.gy);
      items.push_back(it);
    }
    EnsColItem* di = nullptr;
    int* db = nullptr;
    if (!rc) rc = ens_upload(e, items, &di);
    if (!rc) rc = ens_upload(e, base, &db);
    st.items = di;
    st.base = db;
    st.n = n;
    st.total = total;
    st.smem = ens_col_smem(maxL);
    st.grid = rc ? 0 : ens_pass_grid(kind, st.smem, total, smax);
    if (!rc && st.grid <= 0) rc = fail(DNSB_ERR_CUDA, "ensemble pass occupancy");
    return st;
  };
  auto x_stage = [&]() -> EnsStage {
    EnsStage st;
    st.kind = 3;
    std::vector<EnsXItem> items;
    std::vector<int> base;
    int total = 0;
    for (int m : order) {
      EnsXItem it{};
      it.a = periodic_xpass(ctxs[m]);
      it.member = m;
      base.push_back(total);
      total += ens_x_blocks(it.a);
      items.push_back(it);
    }
    EnsXItem* di = nullptr;
    int* db = nullptr;
    if (!rc) rc = ens_upload(e, items, &di);
    if (!rc) rc = ens_upload(e, base, &db);
    st.items = di;
    st.base = db;
    st.n = n;
    st.total = total;
    st.smem = ens_x_smem(maxL, maxNKX);
    st.grid = rc ? 0 : ens_pass_grid(3, st.smem, total, smax);
    if (!rc && st.grid <= 0) rc = fail(DNSB_ERR_CUDA, "ensemble pass occupancy");
    return st;
  };
  auto point_list = [&](auto fill) -> EnsPointItem* {
    std::vector<EnsPointItem> items;
    for (int m : order) {
      EnsPointItem it{};
      it.a = ctxs[m]->point();
      it.member = m;
      fill(it, m);
      items.push_back(it);
    }
    EnsPointItem* d = nullptr;
    if (!rc) rc = ens_upload(e, items, &d);
    return d;
  };
  // RHS work lists for (in, out) = (state, Ra), (P, Rb), (P, Ra)
  struct RhsLists {
    EnsStage yc, zi, x, zf, yf;
    EnsPointItem* proj = nullptr;
  } rl[3];
  for (int c = 0; c < 3; ++c) {
    auto in_of = [&](int m) -> const void* { return c == 0 ? states[m] : (const void*)P[m]; };
    auto out_of = [&](int m) -> void* { return c == 1 ? (void*)Rb[m] : (void*)Ra[m]; };
    rl[c].yc = col_stage(0, [&](const dnsb_periodic* q, int m) { return periodic_ycurl(q, in_of(m)); },
                         6, [](const dnsb_periodic* q) { return q->NZ1; });
    rl[c].zi = col_stage(1, [&](const dnsb_periodic* q, int) { return periodic_zinv(q); }, 6,
                         [](const dnsb_periodic* q) { return q->My; });
    rl[c].x = x_stage();
    rl[c].zf = col_stage(2, [&](const dnsb_periodic* q, int) { return periodic_zfwd(q); }, 3,
                         [](const dnsb_periodic* q) { return q->My; });
    rl[c].yf = col_stage(2, [&](const dnsb_periodic* q, int m) { return periodic_yfwd_col(q, out_of(m)); },
                         3, [](const dnsb_periodic* q) { return q->NZ1; });
    rl[c].proj = point_list([&](EnsPointItem& it, int m) {
      it.in0 = (const double2*)out_of(m);
      it.out = (double2*)out_of(m);
    });
  }
  EnsPointItem* pred = point_list([&](EnsPointItem& it, int m) {
    it.in0 = (const double2*)states[m];
    it.in1 = Ra[m];
    it.out = P[m];
  });
  // corrections: (prev, next) = (Ra, Rb) and (Rb, Ra)
  EnsPointItem* corr[2];
  for (int k = 0; k < 2; ++k)
    corr[k] = point_list([&](EnsPointItem& it, int m) {
      it.in0 = P[m];
      it.in1 = k == 0 ? Ra[m] : Rb[m];
      it.in2 = k == 0 ? Rb[m] : Ra[m];
      it.out = P[m];
      it.partials = ctxs[m]->partials;
    });
  EnsPointItem* cv = point_list([&](EnsPointItem& it, int m) {
    it.in0 = P[m];
    it.out = (double2*)states[m];
  });
  if (rc) {
    ensemble_free(e);
    return rc;
  }
  int nsm = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int pgrid = std::min(n * kRedBlocks, 4 * nsm);

  auto run_pass = [&](const EnsStage& st, const int* act, cudaStream_t s) {
    return launch_ens_pass(st.kind, st.items, st.base, st.n, st.total, act, st.grid, st.smem, s);
  };
  auto rhs = [&](int c, const int* act, cudaStream_t s) -> cudaError_t {
    cudaError_t r;
    const RhsLists& L = rl[c];
    if ((r = run_pass(L.yc, act, s)) != cudaSuccess) return r;
    if ((r = run_pass(L.zi, act, s)) != cudaSuccess) return r;
    if ((r = run_pass(L.x, act, s)) != cudaSuccess) return r;
    if ((r = run_pass(L.zf, act, s)) != cudaSuccess) return r;
    if ((r = run_pass(L.yf, act, s)) != cudaSuccess) return r;
    return launch_ens_point(L.proj, n, act, 2, 1, 0, pgrid, s);
  };
  auto correct = [&](int k, const int* act, cudaStream_t s) -> cudaError_t {
    cudaError_t r = launch_ens_point(corr[k], n, act, 1, 0, 0, pgrid, s);
    if (r == cudaSuccess) r = launch_ens_finalize(corr[k], n, act, err, s);
    return r;
  };

  // the graph: prologue, WHILE { A; IF { B } }, epilogue (as build_step_graph)
  cudaStream_t s = nullptr, sb = nullptr, si = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&si, cudaStreamNonBlocking);
  auto ck = [&](cudaError_t r, const char* what) {
    if (r != cudaSuccess && !rc)
      rc = fail(DNSB_ERR_CUDA, std::string("ensemble graph: ") + what + ": " +
                                   cudaGetErrorString(r));
  };
  auto add_cond = [&](cudaStream_t st, cudaGraph_t gr, cudaGraphConditionalHandle hd,
                      cudaGraphConditionalNodeType type) {
    return add_cond_node(st, gr, hd, type, rc);
  };
  cudaGraph_t graph = nullptr;
  ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaStreamCaptureStatus cs;
  ck(cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, nullptr, nullptr), "capture info");
  cudaGraphConditionalHandle h = 0, h_if = 0;
  ck(cudaGraphConditionalHandleCreate(&h, graph, 0, 0), "conditional handle");
  // prologue: every member
  ck(rhs(0, nullptr, s), "rhs");
  ck(launch_ens_point(pred, n, nullptr, 0, 0, 0, pgrid, s), "predict");
  ck(rhs(1, nullptr, s), "rhs");
  ck(correct(0, nullptr, s), "correct");
  ens_ctl_kernel<<<1, 1024, 0, s>>>(h, 0, 0, n, err, d_tol, d_max, e->iters, active,
                                    e->err_last, 1);
  ck(cudaGetLastError(), "control kernel");
  cudaGraph_t bg = add_cond(s, graph, h, cudaGraphCondTypeWhile);
  if (!rc) {
    ck(cudaGraphConditionalHandleCreate(&h_if, bg, 0, 0), "conditional handle");
    ck(cudaStreamBeginCaptureToGraph(sb, bg, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal), "body capture");
    // iteration A: rhs_next -> Ra, rhs_prev Rb
    ck(rhs(2, active, sb), "rhs");
    ck(correct(1, active, sb), "correct");
    ens_ctl_kernel<<<1, 1024, 0, sb>>>(h, h_if, 1, n, err, d_tol, d_max, e->iters, active,
                                       e->err_last, 0);
    ck(cudaGetLastError(), "control kernel");
    cudaGraph_t ig = add_cond(sb, bg, h_if, cudaGraphCondTypeIf);
    if (!rc) {
      ck(cudaStreamBeginCaptureToGraph(si, ig, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal), "IF body capture");
      // iteration B: rhs_next -> Rb, rhs_prev Ra
      ck(rhs(1, active, si), "rhs");
      ck(correct(0, active, si), "correct");
      ens_ctl_kernel<<<1, 1024, 0, si>>>(h, 0, 0, n, err, d_tol, d_max, e->iters, active,
                                         e->err_last, 0);
      ck(cudaGetLastError(), "control kernel");
      cudaGraph_t iout = nullptr;
      ck(cudaStreamEndCapture(si, &iout), "end IF body capture");
    }
    cudaGraph_t bout = nullptr;
    ck(cudaStreamEndCapture(sb, &bout), "end body capture");
  }
  ck(launch_ens_point(cv, n, nullptr, 2, divergence, 1, pgrid, s), "correct_velocity");
  cudaGraph_t done = nullptr;
  ck(cudaStreamEndCapture(s, &done), "end capture");  // always end the capture
  if (!rc) ck(cudaGraphInstantiate(&e->exec, done, 0), "instantiate");
  if (done) cudaGraphDestroy(done);
  cudaStreamDestroy(s);
  cudaStreamDestroy(sb);
  cudaStreamDestroy(si);
  if (rc) {
    ensemble_free(e);
    return rc;
  }
  // launches: prologue 2 RHS (6 each) + predict + correct + finalize +
  // control, epilogue 1; an iteration 6 + 3
  e->k_fixed = 2 * 6 + 4 + 1;
  e->k_iter = 6 + 3;
  *out = e;
  return 0;
}

extern "C" int dnsb_ensemble_step(dnsb_ensemble* e, void* stream) {
  if (!e) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_CUDA(cudaGraphLaunch(e->exec, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_ensemble_status(dnsb_ensemble* e, int* iters, double* errs, void* stream) {
  if (!e || !iters || !errs) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_CUDA(cudaMemcpyAsync(iters, e->iters, e->n * sizeof(int), cudaMemcpyDeviceToHost, st));
  DNSB_CUDA(cudaMemcpyAsync(errs, e->err_last, e->n * sizeof(double), cudaMemcpyDeviceToHost,
                            st));
  DNSB_CUDA(cudaStreamSynchronize(st));
  int most = 0;
  for (int m = 0; m < e->n; ++m) most = std::max(most, iters[m]);
  g_launches.fetch_add(e->k_fixed + (long long)most * e->k_iter, std::memory_order_relaxed);
  return 0;
}

extern "C" int dnsb_ensemble_destroy(dnsb_ensemble* e) {
  if (!e) return fail(DNSB_ERR_ARG, "null argument");
  ensemble_free(e);
  return 0;
}

extern "C" int dnsb_periodic_energy_sums(dnsb_periodic* p, const void* v,
                                         double* out_dev, void* stream) {
  if (!p || !v || !out_dev) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_LAUNCH(launch_periodic_stats(p->point(), (const double2*)v, p->partials, st));
  DNSB_LAUNCH(launch_finalize(p->partials, kRedBlocks, out_dev, 1.0, 0, st));
  DNSB_LAUNCH(launch_finalize(p->partials + kRedBlocks, kRedBlocks, out_dev + 1,
                              1.0, 0, st));
  return 0;
}

extern "C" int dnsb_periodic_spec_to_phys(dnsb_periodic* p, const void* spec,
                                          double* phys, void* stream) {
  if (!p || !spec || !phys) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  YInvArgs yi{};
  yi.u = (const double2*)spec;
  yi.out = p->A;
  yi.NY1 = p->NY1;
  yi.NZ1 = p->NZ1;
  yi.NKX = p->NKX;
  yi.curl = 0;
  yi.kx = p->kx;
  yi.ky = p->ky;
  yi.kz = p->kz;
  yi.plan = p->py;
  yi.tw = p->twy;
  DNSB_LAUNCH(launch_yinv(yi, st));
  DNSB_LAUNCH(launch_col_pass(periodic_zinv(p), 3, p->My, st));
  XPhysArgs xa{};
  xa.in = p->B;
  xa.out = phys;
  xa.in_fs = (long long)p->My * p->Mz * p->NKX;
  xa.out_fs = (long long)p->My * p->Mz * p->Mx;
  xa.nrows = p->My * p->Mz;
  xa.inner_n = p->Mz;
  xa.so = (long long)p->Mz * p->NKX;
  xa.si = p->NKX;
  xa.ks = 1;
  xa.pso = (long long)p->Mz * p->Mx;
  xa.psi = p->Mx;
  xa.nkx = p->NKX;
  xa.rows_fast = 0;
  xa.plan = p->px;
  xa.tw = p->twx;
  DNSB_LAUNCH(launch_x_phys(xa, st));
  return 0;
}

extern "C" int dnsb_periodic_phys_to_spec(dnsb_periodic* p, const double* phys,
                                          void* spec, void* stream) {
  if (!p || !spec || !phys) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  XPhysArgs xa{};
  xa.in_fs = (long long)p->My * p->Mz * p->NKX;
  xa.out_fs = (long long)p->My * p->Mz * p->Mx;
  xa.nrows = p->My * p->Mz;
  xa.inner_n = p->Mz;
  xa.so = (long long)p->Mz * p->NKX;
  xa.si = p->NKX;
  xa.ks = 1;
  xa.pso = (long long)p->Mz * p->Mx;
  xa.psi = p->Mx;
  xa.nkx = p->NKX;
  xa.rows_fast = 0;
  xa.plan = p->px;
  xa.tw = p->twx;
  DNSB_LAUNCH(launch_x_fwd(xa, phys, p->B, st));
  DNSB_LAUNCH(launch_col_pass(periodic_zfwd(p), 3, p->My, st));
  YFwdArgs yf{};
  yf.in = p->A;
  yf.out = (double2*)spec;
  yf.NY1 = p->NY1;
  yf.NZ1 = p->NZ1;
  yf.NKX = p->NKX;
  yf.project = 0;
  yf.kx = p->kx;
  yf.ky = p->ky;
  yf.kz = p->kz;
  yf.inv_lapl = p->inv_lapl;
  yf.plan = p->py;
  yf.tw = p->twy;
  DNSB_LAUNCH(launch_yfwd(yf, st));
  return 0;
}

// ===========================================================================
// Plane Couette
// ===========================================================================
struct dnsb_couette {
  int NZ1, NKX, Ny, Mz, Mx, p, s1, s2, span_max, NM;
  double dt, c, nu, ly;
  FFTPlan pz, px;
  double2 *twz = nullptr, *twx = nullptr;
  float2 *twz32 = nullptr, *twx32 = nullptr;
  int rhs_fp32 = 0;  // RHS passes in FP32 (dnsb_couette_set_rhs_precision)
  double *kx = nullptr, *kz = nullptr, *d1w = nullptr, *d2w = nullptr;
  double *d1wT = nullptr, *d2wT = nullptr;  // [tap][Ny]: lanes over y read contiguously
  int *d1j0 = nullptr, *d2j0 = nullptr;
  double *U = nullptr, *cU = nullptr, *nU = nullptr, *simpson = nullptr;
  double2* B = nullptr;
  double* partials = nullptr;
  int* status = nullptr;
  dnsb_imm_ops ops{};
  bool bound = false;
  int var[4] = {0, 0, 0, 0};  // variants: z inverse, x, z forward passes; IMM
  int ab_row0 = 0;
  int pair_modes = 0;
  size_t ws_bytes = 0;
  // five-kernel IMM: repacked factors and stage workspace (bind time)
  double* fac = nullptr;
  unsigned char* dp = nullptr;
  double2* Fw = nullptr;
  double2* Rw = nullptr;
  ImmBatch batch{};
  bool batch_ready = false;
  int wait_limit = 1 << 20;  // substitution ring: polls before a wait gives up
  SlabState slab;            // nranks > 0: a slab context
  int graph_unroll = 0;      // corrector iterations step graphs capture unrolled
  // set only while a step graph captures an unrolled iteration: the device
  // flag that makes the iteration's kernels return at once
  const int* skip = nullptr;

  ImmArgs imm() const {
    ImmArgs a{};
    a.NZ1 = NZ1;
    a.NKX = NKX;
    a.Ny = Ny;
    a.kl = a.ku = p;
    a.s1 = s1;
    a.s2 = s2;
    a.d1_j0 = d1j0;
    a.d1_w = d1w;
    a.d2_j0 = d2j0;
    a.d2_w = d2w;
    a.d1_wT = d1wT;
    a.d2_wT = d2wT;
    a.kx = kx;
    a.kz = kz;
    a.simpson = simpson;
    a.dt = dt;
    a.c = c;
    a.nu = nu;
    a.Lk_ab = ops.Lk_ab;
    a.Lk_piv = ops.Lk_piv;
    a.Hk_ab = ops.Hk_ab;
    a.Hk_piv = ops.Hk_piv;
    a.v1 = ops.v1;
    a.v2 = ops.v2;
    a.q1 = ops.q1;
    a.q2 = ops.q2;
    a.M_inv = ops.M_inv;
    a.status = status;
    a.ab_row0 = ab_row0;
    a.pair_modes = pair_modes;
    a.kx0 = slab.rank == 0 ? 1 : 0;
    return a;
  }
};

static void couette_free(dnsb_couette* p) {
  void* ptrs[] = {p->twz, p->twx, p->twz32, p->twx32, p->kx, p->kz, p->d1w, p->d2w, p->d1wT, p->d2wT, p->d1j0,
                  p->d2j0, p->U, p->cU, p->nU, p->simpson, p->B, p->partials,
                  p->status, p->fac, p->dp, p->Fw, p->Rw, p->slab.Bx};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete p;
}

// Composite Simpson weights on non-uniform panels (cartesian.py:106-140),
// expressed as the linear functional sum_y W_y f_y.
static std::vector<double> simpson_weights(const double* ys, int n) {
  std::vector<double> W(n, 0.0);
  for (int i = 0; i + 2 < n; i += 2) {
    const double h0 = ys[i + 1] - ys[i], h1 = ys[i + 2] - ys[i + 1];
    const double hs = h0 + h1, hp = h0 * h1, r = h0 / h1;
    W[i] += (hs / 6) * (2 - 1 / r);
    W[i + 1] += (hs / 6) * (hs * hs / hp);
    W[i + 2] += (hs / 6) * (2 - r);
  }
  return W;
}

static bool stencil_ok(const int* j0, int n, int s) {
  for (int i = 0; i < n; ++i) {
    if (j0[i] < 0 || j0[i] > i || j0[i] + s > n || j0[i] + s <= i) return false;
    if (i > 0 && (j0[i] < j0[i - 1] || j0[i] > j0[i - 1] + 1)) return false;
  }
  return true;
}

extern "C" int dnsb_couette_create(const dnsb_couette_desc* d,
                                   dnsb_couette** out) {
  if (!d || !out) return fail(DNSB_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->nx < 2 || d->nz < 2 || d->nx % 2 || d->nz % 2)
    return fail(DNSB_ERR_ARG, "nx, nz must be even and >= 2");
  if (d->ny < 3 || d->ny % 2 == 0)
    return fail(DNSB_ERR_ARG, "ny must be odd and >= 3 (Simpson rule)");
  if (d->fd_order < 2 || d->fd_order + 2 > d->ny)
    return fail(DNSB_ERR_ARG, "fd_order out of range");
  if (!fft_size_ok(d->nx_p) || !fft_size_ok(d->nz_p) || d->nx_p % 2 ||
      d->nx_p < d->nx || d->nz_p < d->nz || (d->nz_p - d->nz) % 2)
    return fail(DNSB_ERR_ARG, "padded sizes must be 2^a 3^b and >= modes");
  const int pord = d->fd_order;
  if (!d->d1_j0 || !d->d2_j0 || !stencil_ok(d->d1_j0, d->ny, pord + 1) ||
      !stencil_ok(d->d2_j0, d->ny, pord + 2))
    return fail(DNSB_ERR_ARG, "invalid FD stencil start columns");
  dnsb_couette* p = new dnsb_couette();
  p->NZ1 = d->nz - 1;
  p->NKX = d->nx / 2;
  p->Ny = d->ny;
  p->Mz = d->nz_p;
  p->Mx = d->nx_p;
  p->p = pord;
  p->s1 = pord + 1;
  p->s2 = pord + 2;
  p->span_max = kZTile + pord;
  p->NM = p->NZ1 * p->NKX;
  p->dt = d->dt;
  p->c = d->implicitness;
  p->nu = d->nu;
  p->ly = d->ly;
  p->pz = make_plan(p->Mz);
  p->px = make_plan(p->Mx);
  const int smax = max_smem_optin();
  const size_t need[] = {col_pass_smem(p->Mz), x_pass_smem(p->Mx),
                         x_phys_smem(p->Mx), x_fwd_smem(p->Mx),
                         zinv_curl_smem(p->Mz, p->NZ1, p->span_max),
                         zinv_curl2_smem(p->Mz), imm_smem(p->Ny),
                         imm_v2_supported(p->p, p->Ny) ? imm_v2_smem(p->Ny, p->p, 0) : 0,
                         imm_batch_supported(p->p, p->Ny) ? imm_batch_stage_smem(p->Ny) : 0};
  for (size_t n : need)
    if ((int)n > smax) {
      couette_free(p);
      return fail(DNSB_ERR_ARG, "grid too large for shared-memory tiles");
    }
  int rc = 0;
  auto chk = [&](int r) {
    if (r && !rc) rc = r;
  };
  chk(make_twiddles(&p->twz, p->Mz));
  chk(make_twiddles(&p->twx, p->Mx));
  chk(make_twiddles32(&p->twz32, p->Mz));
  chk(make_twiddles32(&p->twx32, p->Mx));
  chk(upload(&p->kx, d->kx, p->NKX));
  chk(upload(&p->kz, d->kz, p->NZ1));
  chk(upload(&p->d1j0, d->d1_j0, p->Ny));
  chk(upload(&p->d2j0, d->d2_j0, p->Ny));
  chk(upload(&p->d1w, d->d1_w, (size_t)p->Ny * p->s1));
  chk(upload(&p->d2w, d->d2_w, (size_t)p->Ny * p->s2));
  {
    std::vector<double> t1((size_t)p->Ny * p->s1), t2((size_t)p->Ny * p->s2);
    for (int y = 0; y < p->Ny; ++y) {
      for (int m = 0; m < p->s1; ++m) t1[(size_t)m * p->Ny + y] = d->d1_w[(size_t)y * p->s1 + m];
      for (int m = 0; m < p->s2; ++m) t2[(size_t)m * p->Ny + y] = d->d2_w[(size_t)y * p->s2 + m];
    }
    chk(upload(&p->d1wT, t1.data(), t1.size()));
    chk(upload(&p->d2wT, t2.data(), t2.size()));
  }
  chk(upload(&p->U, d->base_flow, 3 * (size_t)p->Ny));
  chk(upload(&p->cU, d->curl_base_flow, 3 * (size_t)p->Ny));
  chk(upload(&p->nU, d->nonlin_base_flow, 3 * (size_t)p->Ny));
  if (!rc) {
    if (!d->ys) rc = fail(DNSB_ERR_ARG, "null ys");
    else {
      std::vector<double> W = simpson_weights(d->ys, p->Ny);
      chk(upload(&p->simpson, W.data(), W.size()));
    }
  }
  const size_t nB = 6ull * p->Mz * p->NKX * p->Ny;
  const size_t npart = (size_t)std::max(p->NM, kRedBlocks);
  if (!rc) {
    cudaError_t e1 = cudaMalloc(&p->B, nB * sizeof(double2));
    cudaError_t e2 = cudaMalloc(&p->partials, npart * sizeof(double));
    cudaError_t e3 = cudaMalloc(&p->status, sizeof(int));
    if (e1 || e2 || e3) rc = fail(DNSB_ERR_CUDA, "workspace allocation failed");
    else if (cudaMemset(p->status, 0, sizeof(int)) != cudaSuccess)
      rc = fail(DNSB_ERR_CUDA, "cudaMemset failed");
  }
  if (!rc) {
    cudaError_t e = set_pass_attributes(smax);
    if (e == cudaSuccess) e = set_solver_attributes(smax);
    if (e == cudaSuccess) e = set_imm_v2_attributes(smax);
    if (e == cudaSuccess) e = set_imm_batch_attributes(smax);
    if (e != cudaSuccess)
      rc = fail(DNSB_ERR_CUDA, std::string("cudaFuncSetAttribute: ") +
                                   cudaGetErrorString(e));
  }
  if (rc) {
    couette_free(p);
    return rc;
  }
  p->ws_bytes = nB * sizeof(double2) + npart * sizeof(double) + sizeof(int);
  *out = p;
  return 0;
}

extern "C" int dnsb_couette_destroy(dnsb_couette* p) {
  if (p) couette_free(p);
  return 0;
}

extern "C" size_t dnsb_couette_workspace_bytes(const dnsb_couette* p) {
  return p ? p->ws_bytes : 0;
}

// Repack both operators' factors for the five-kernel IMM (items = modes
// (s, kx), s <= (nz-1)/2, when mirror modes share factors; 16-item tiles)
// and allocate its stage workspace; kept until the next bind or destroy.
// Returns 0 with batch_ready false when the ring of the substitution
// kernel does not fit in shared memory (the single-kernel IMM runs then).
static int bind_batch(dnsb_couette* p) {
  const int kl = p->p, nu = imm_nu(kl, p->ab_row0);
  const int smax = max_smem_optin();
  if (!imm_batch_fits(kl, nu, smax)) return 0;
  const int NP = p->pair_modes ? ((p->NZ1 + 1) / 2) * p->NKX : p->NM;
  const int tile = 16;  // items per substitution tile (csrc/imm_batch.cu)
  const int ntiles = (NP + tile - 1) / tile;
  const size_t nL = (size_t)ntiles * (p->Ny + kl + 1) * kl * tile;
  const size_t nU = (size_t)ntiles * (p->Ny + nu + 1) * ((nu + 2) & ~1) * tile;
  const size_t nP = (size_t)ntiles * (p->Ny + kl + 1) * tile;
  void* ptrs[] = {p->fac, p->dp, p->Fw, p->Rw};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  p->fac = nullptr;
  p->dp = nullptr;
  p->Fw = p->Rw = nullptr;
  const size_t fac_bytes = 2 * (nL + nU) * sizeof(double);
  cudaError_t e1 = cudaMalloc(&p->fac, fac_bytes);
  cudaError_t e2 = cudaMalloc(&p->dp, 2 * nP);
  cudaError_t e3 = cudaMalloc(&p->Fw, (size_t)p->NM * p->Ny * sizeof(double2));
  cudaError_t e4 = cudaMalloc(&p->Rw, 3 * (size_t)p->NM * p->Ny * sizeof(double2));
  if (e1 || e2 || e3 || e4) return fail(DNSB_ERR_CUDA, "IMM workspace allocation failed");
  if (cudaMemset(p->fac, 0, fac_bytes) != cudaSuccess || cudaMemset(p->dp, 0, 2 * nP) != cudaSuccess)
    return fail(DNSB_ERR_CUDA, "cudaMemset failed");
  ImmBatch& b = p->batch;
  const double* abs_[2] = {p->ops.Lk_ab, p->ops.Hk_ab};
  const int* pivs[2] = {p->ops.Lk_piv, p->ops.Hk_piv};
  for (int k = 0; k < 2; ++k) {
    double* fL = p->fac + k * (nL + nU);
    double* fU = fL + nL;
    unsigned char* d = p->dp + k * nP;
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (launch_imm_repack(abs_[k], pivs[k], p->Ny, kl, nu, p->ab_row0, NP, ntiles, fL, fU, d,
                          p->status, 0) != cudaSuccess)
      return fail(DNSB_ERR_CUDA, "IMM repack launch failed");
    b.facL[k] = fL;
    b.facU[k] = fU;
    b.dp[k] = d;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(DNSB_ERR_CUDA, "IMM repack failed");
  b.NP = NP;
  b.nu = nu;
  b.paired = p->pair_modes;
  b.max_smem = smax;
  b.status = p->status;
  b.wait_limit = p->wait_limit;
  b.F = p->Fw;
  b.R = p->Rw;
  p->batch_ready = true;
  return 0;
}

extern "C" int dnsb_couette_bind_imm(dnsb_couette* p, const dnsb_imm_ops* ops) {
  if (!p || !ops) return fail(DNSB_ERR_ARG, "null argument");
  if (!ops->Lk_ab || !ops->Lk_piv || !ops->Hk_ab || !ops->Hk_piv || !ops->v1 ||
      !ops->v2 || !ops->q1 || !ops->q2 || !ops->M_inv)
    return fail(DNSB_ERR_ARG, "null IMM operator");
  p->ops = *ops;
  // Rows of the LU factors above the first nonzero one (over all modes, both
  // operators) are skipped by the register-window kernel.
  const int kuu = 2 * p->p, rows = 3 * p->p + 1;
  int* d_row = nullptr;
  DNSB_CUDA(cudaMalloc(&d_row, sizeof(int)));
  int h_row = kuu;
  int rc = 0;
  if (cudaMemcpy(d_row, &h_row, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(DNSB_ERR_CUDA, "cudaMemcpy failed");
  const double* abs_[2] = {ops->Lk_ab, ops->Hk_ab};
  for (int k = 0; k < 2 && !rc; ++k) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (launch_ab_first_row(abs_[k], p->NM, rows, p->Ny, kuu, d_row, 0) != cudaSuccess)
      rc = fail(DNSB_ERR_CUDA, "ab scan launch failed");
  }
  if (!rc && cudaMemcpy(&h_row, d_row, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(DNSB_ERR_CUDA, "ab scan failed");
  // Modes (s, kx) and (nz-1-s, kx) share k^2; the kernel solves them together
  // when their factors are bit-identical (DNSB_IMM_PAIRS=0 disables this).
  int h_diff = 0;
  if (!rc && cudaMemcpy(d_row, &h_diff, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(DNSB_ERR_CUDA, "cudaMemcpy failed");
  const int* pivs[2] = {ops->Lk_piv, ops->Hk_piv};
  for (int k = 0; k < 2 && !rc; ++k) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (launch_ab_pair_check(abs_[k], pivs[k], p->NZ1, p->NKX, rows, p->Ny, d_row, 0) !=
        cudaSuccess)
      rc = fail(DNSB_ERR_CUDA, "ab pair check launch failed");
  }
  if (!rc && cudaMemcpy(&h_diff, d_row, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(DNSB_ERR_CUDA, "ab pair check failed");
  cudaFree(d_row);
  if (rc) return rc;
  const char* env = getenv("DNSB_IMM_PAIRS");
  const bool allow = !(env && env[0] == '0');
  p->pair_modes = (allow && h_diff == 0) ? 1 : 0;
  p->ab_row0 = h_row;
  p->bound = true;
  p->batch_ready = false;
  if (imm_batch_supported(p->p, p->Ny)) {
    rc = bind_batch(p);
    if (rc) return rc;
  }
  return 0;
}

// The three passes of the Couette RHS; bit k of `mask` runs pass k (z
// inverse with the curl, x, z forward), each with its variant.
static int couette_rhs_impl(dnsb_couette* p, const void* state, void* rhs, unsigned mask,
                            cudaStream_t st) {
  ZInvCurlArgs zi{};
  zi.u = (const double2*)state;
  zi.out = p->B;
  zi.NZ1 = p->NZ1;
  zi.NKX = p->NKX;
  zi.Ny = p->Ny;
  zi.curl = 1;
  zi.s1 = p->s1;
  zi.d1_j0 = p->d1j0;
  zi.d1_w = p->d1w;
  zi.d1_wT = p->d1wT;
  zi.kx = p->kx;
  zi.kz = p->kz;
  zi.plan = p->pz;
  zi.tw = p->rhs_fp32 ? reinterpret_cast<const double2*>(p->twz32) : p->twz;
  zi.fp32 = p->rhs_fp32;
  zi.variant = p->var[0];
  zi.skip = p->skip;
  if (mask & 1u) DNSB_LAUNCH(launch_zinv_curl(zi, p->span_max, st));
  XPassArgs xa{};
  xa.in = p->B;
  xa.out = p->B;
  xa.in_fs = xa.out_fs = (long long)p->Mz * p->NKX * p->Ny;
  xa.nrows = p->Mz * p->Ny;
  xa.inner_n = p->Ny;
  xa.so = (long long)p->NKX * p->Ny;
  xa.si = 1;
  xa.ks = p->Ny;
  xa.nkx = p->NKX;
  xa.y_outer = 0;
  xa.rows_fast = 1;
  xa.U = p->U;
  xa.cU = p->cU;
  xa.nU = p->nU;
  xa.ny_grid = p->Ny;
  xa.plan = p->px;
  xa.tw = p->rhs_fp32 ? reinterpret_cast<const double2*>(p->twx32) : p->twx;
  xa.fp32 = p->rhs_fp32;
  xa.variant = p->var[1];
  xa.skip = p->skip;
  if (mask & 2u) DNSB_LAUNCH(launch_x_pass(xa, st));
  ColPassArgs zf{};
  zf.in = p->B;
  zf.out = (double2*)rhs;
  zf.in_fs = (long long)p->Mz * p->NKX * p->Ny;
  zf.out_fs = (long long)p->NZ1 * p->NKX * p->Ny;
  zf.in_os = p->Ny;
  zf.out_os = p->Ny;
  zf.in_ts = (long long)p->NKX * p->Ny;
  zf.out_ts = (long long)p->NKX * p->Ny;
  zf.nI = p->Ny;
  zf.nstored = p->NZ1;
  zf.inverse = 0;
  zf.plan = p->pz;
  zf.tw = p->rhs_fp32 ? reinterpret_cast<const double2*>(p->twz32) : p->twz;
  zf.fp32 = p->rhs_fp32;
  zf.variant = p->var[2];
  zf.skip = p->skip;
  if (mask & 4u) DNSB_LAUNCH(launch_col_pass(zf, 3, p->NKX, st));
  return 0;
}

extern "C" int dnsb_couette_rhs(dnsb_couette* p, const void* state, void* rhs,
                                void* stream) {
  if (!p || !state || !rhs) return fail(DNSB_ERR_ARG, "null argument");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab context: the RHS runs in phases");
  return couette_rhs_impl(p, state, rhs, 7u, as_stream(stream));
}

// The FP32 passes are compiled for padded lengths 48, 72, 96 and 192 with
// 3/2 oversampling in x.
static bool couette_fp32_sizes(const dnsb_couette* p) {
  auto fixed = [](int L) { return L == 48 || L == 72 || L == 96 || L == 192; };
  return fixed(p->Mz) && fixed(p->Mx) && 3 * p->NKX == p->Mx;
}

extern "C" int dnsb_couette_set_rhs_precision(dnsb_couette* p, int fp32) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  if (fp32 && p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts run the FP64 passes");
  if (fp32 && !couette_fp32_sizes(p))
    return fail(DNSB_ERR_ARG,
                "FP32 RHS passes need padded sizes in {48, 72, 96, 192} with nx_p = 3 nx / 2");
  p->rhs_fp32 = fp32 < 0 ? 0 : (fp32 > 2 ? 2 : fp32);
  return 0;
}

extern "C" int dnsb_couette_imm(dnsb_couette* p, const void* vel_n,
                                const void* vel_j, const void* nl_n,
                                const void* nl_j, void* vel_new,
                                void* corr_out, double* err_dev,
                                void* stream) {
  if (!p || !vel_n || !vel_j || !nl_n || !nl_j || !vel_new)
    return fail(DNSB_ERR_ARG, "null argument");
  if (!p->bound) return fail(DNSB_ERR_ARG, "IMM operators not bound");
  if (vel_new == vel_n)
    return fail(DNSB_ERR_ARG, "vel_new must not alias vel_n");
  cudaStream_t st = as_stream(stream);
  if (p->skip && !(p->batch_ready && p->var[3] == 0))
    return fail(DNSB_ERR_ARG, "unrolled graph iterations need the batched IMM");
  if (p->batch_ready && p->var[3] == 0) {
    ImmArgs ia = p->imm();
    ia.skip = p->skip;
    DNSB_LAUNCH(launch_imm_batch(ia, p->batch, (const double2*)vel_n,
                                 (const double2*)vel_j, (const double2*)nl_n,
                                 (const double2*)nl_j, (double2*)vel_new,
                                 (double2*)corr_out, err_dev ? p->partials : nullptr, st));
    count_launches(4);  // five kernels
  } else if (imm_v2_supported(p->p, p->Ny) && p->var[3] <= 1) {
    DNSB_LAUNCH(launch_imm_v2(p->imm(), (const double2*)vel_n, (const double2*)vel_j,
                              (const double2*)nl_n, (const double2*)nl_j,
                              (double2*)vel_new, (double2*)corr_out,
                              err_dev ? p->partials : nullptr, st));
  } else {
    DNSB_LAUNCH(launch_imm(p->imm(), (const double2*)vel_n, (const double2*)vel_j,
                           (const double2*)nl_n, (const double2*)nl_j,
                           (double2*)vel_new, (double2*)corr_out,
                           err_dev ? p->partials : nullptr, st));
  }
  // A slab rank returns its share of the squared norm.
  if (err_dev)
    DNSB_LAUNCH(launch_finalize(p->partials, p->NM, err_dev, 1.0 / p->ly,
                                p->slab.nranks ? 0 : 1, st, p->skip));
  return 0;
}

static int couette_norm_impl(dnsb_couette* p, const void* v, double* out_dev,
                             int do_sqrt, void* stream) {
  if (!p || !v || !out_dev) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_LAUNCH(launch_couette_norm2(p->imm(), (const double2*)v, p->partials, st));
  DNSB_LAUNCH(launch_finalize(p->partials, kRedBlocks, out_dev, 1.0 / p->ly,
                              p->slab.nranks ? 0 : do_sqrt, st));
  return 0;
}

extern "C" int dnsb_couette_norm(dnsb_couette* p, const void* v,
                                 double* out_dev, void* stream) {
  return couette_norm_impl(p, v, out_dev, 1, stream);
}

extern "C" int dnsb_couette_norm2(dnsb_couette* p, const void* v,
                                  double* out_dev, void* stream) {
  return couette_norm_impl(p, v, out_dev, 0, stream);
}

extern "C" int dnsb_couette_spec_to_phys(dnsb_couette* p, const void* spec,
                                         double* phys, void* stream) {
  if (!p || !spec || !phys) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  ZInvCurlArgs zi{};
  zi.u = (const double2*)spec;
  zi.out = p->B;
  zi.NZ1 = p->NZ1;
  zi.NKX = p->NKX;
  zi.Ny = p->Ny;
  zi.curl = 0;
  zi.s1 = p->s1;
  zi.d1_j0 = p->d1j0;
  zi.d1_w = p->d1w;
  zi.d1_wT = p->d1wT;
  zi.kx = p->kx;
  zi.kz = p->kz;
  zi.plan = p->pz;
  zi.tw = p->twz;
  DNSB_LAUNCH(launch_zinv_curl(zi, p->span_max, st));
  XPhysArgs xa{};
  xa.in = p->B;
  xa.out = phys;
  xa.in_fs = (long long)p->Mz * p->NKX * p->Ny;
  xa.out_fs = (long long)p->Ny * p->Mz * p->Mx;
  xa.nrows = p->Mz * p->Ny;
  xa.inner_n = p->Ny;
  xa.so = (long long)p->NKX * p->Ny;
  xa.si = 1;
  xa.ks = p->Ny;
  xa.pso = p->Mx;
  xa.psi = (long long)p->Mz * p->Mx;
  xa.nkx = p->NKX;
  xa.rows_fast = 1;
  xa.plan = p->px;
  xa.tw = p->twx;
  DNSB_LAUNCH(launch_x_phys(xa, st));
  return 0;
}

extern "C" int dnsb_couette_phys_to_spec(dnsb_couette* p, const double* phys,
                                         void* spec, void* stream) {
  if (!p || !spec || !phys) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  XPhysArgs xa{};
  xa.in_fs = (long long)p->Mz * p->NKX * p->Ny;
  xa.out_fs = (long long)p->Ny * p->Mz * p->Mx;
  xa.nrows = p->Mz * p->Ny;
  xa.inner_n = p->Ny;
  xa.so = (long long)p->NKX * p->Ny;
  xa.si = 1;
  xa.ks = p->Ny;
  xa.pso = p->Mx;
  xa.psi = (long long)p->Mz * p->Mx;
  xa.nkx = p->NKX;
  xa.rows_fast = 1;
  xa.plan = p->px;
  xa.tw = p->twx;
  DNSB_LAUNCH(launch_x_fwd(xa, phys, p->B, st));
  ColPassArgs zf{};
  zf.in = p->B;
  zf.out = (double2*)spec;
  zf.in_fs = (long long)p->Mz * p->NKX * p->Ny;
  zf.out_fs = (long long)p->NZ1 * p->NKX * p->Ny;
  zf.in_os = p->Ny;
  zf.out_os = p->Ny;
  zf.in_ts = (long long)p->NKX * p->Ny;
  zf.out_ts = (long long)p->NKX * p->Ny;
  zf.nI = p->Ny;
  zf.nstored = p->NZ1;
  zf.inverse = 0;
  zf.plan = p->pz;
  zf.tw = p->twz;
  DNSB_LAUNCH(launch_col_pass(zf, 3, p->NKX, st));
  return 0;
}

// Corrector iterations a step graph captures unrolled: the context's
// setting, when every kernel of an iteration checks the skip flag (the
// two-stage passes at the compiled sizes and the batched IMM), at most
// max_iter; otherwise none.
static int couette_unroll(const dnsb_couette* p, int max_iter) {
  if (p->graph_unroll <= 0 || !couette_fp32_sizes(p) || !p->batch_ready) return 0;
  for (int k = 0; k < 4; ++k)
    if (p->var[k] != 0) return 0;
  return std::min(p->graph_unroll, std::max(max_iter, 0));
}

extern "C" int dnsb_couette_set_graph_unroll(dnsb_couette* p, int n) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  if (n < 0 || n > 64) return fail(DNSB_ERR_ARG, "unroll must be in [0, 64]");
  p->graph_unroll = n;
  return 0;
}

// One full plane-Couette time step as a CUDA graph (see
// dnsb_periodic_step_graph_create): the predictor is the influence-matrix
// iteration with (u^n, u^n, N^n, N^n), each correction the iteration with
// (u^n, u^j, N_prev, N^j) (plane_couette.py:507-540); correct_velocity is
// the identity (:575-582), so the epilogue copies the converged iterate
// into the state.
extern "C" int dnsb_couette_step_graph_create(dnsb_couette* p, void* state, double tol,
                                              int max_iter, dnsb_step_graph** out) {
  if (!p || !state || !out) return fail(DNSB_ERR_ARG, "null argument");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts step through the host loop");
  if (!p->bound) return fail(DNSB_ERR_ARG, "IMM operators not bound");
  const size_t n = 3 * (size_t)p->NM * p->Ny;
  dnsb_step_graph* g = new_step_graph(n);
  if (!g) return fail(DNSB_ERR_CUDA, "step graph allocation failed");
  auto prologue = [&](cudaStream_t s) {
    int rc = dnsb_couette_rhs(p, state, g->Ra, s);
    if (!rc) rc = dnsb_couette_imm(p, state, state, g->Ra, g->Ra, g->P, nullptr, nullptr, s);
    if (!rc) rc = dnsb_couette_rhs(p, g->P, g->Rb, s);
    if (!rc) rc = dnsb_couette_imm(p, state, g->P, g->Ra, g->Rb, g->P, nullptr, g->err, s);
    return rc;
  };
  auto body = [&](cudaStream_t s, int parity, const int* skip) {
    double2* nx = parity ? g->Rb : g->Ra;
    double2* pv = parity ? g->Ra : g->Rb;
    p->skip = skip;
    int rc = dnsb_couette_rhs(p, g->P, nx, s);
    if (!rc) rc = dnsb_couette_imm(p, state, g->P, pv, nx, g->P, nullptr, g->err, s);
    p->skip = nullptr;
    return rc;
  };
  auto epilogue = [&](cudaStream_t s) {
    if (cudaMemcpyAsync(state, g->P, n * sizeof(double2), cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess)
      return fail(DNSB_ERR_CUDA, "state copy");
    return 0;
  };
  const int rc = build_step_graph(g, tol, max_iter, prologue, body, epilogue,
                                 couette_unroll(p, max_iter));
  if (rc) {
    step_graph_free(g);
    return rc;
  }
  *out = g;
  return 0;
}

// ---------------------------------------------------------------------------
// The restarted, mixed-precision corrector step as two CUDA graphs (no
// counterpart in the reference: the device form of the learned corrector
// step of dnsjax_b200.learned, whose corrector is the reference's
// iterate_correction, plane_couette.py:522-540, started from a guessed
// iterate).
//   "predict": the RHS of u^n (into Rb) and the predictor (the IMM
//     iteration with (u^n, u^n, N^n, N^n)) into `up`, copied into the
//     iterate `cur`.  Between the two launches the caller may overwrite
//     `cur` with a guessed start.
//   "correct": the first correction from `cur` (restart != 0: the start's
//     own RHS in both RHS slots; else N^n as the previous RHS), then the
//     corrector iterations in a WHILE node while error > tol and iterations
//     < max_iter, as in build_step_graph, and the converged iterate copied
//     into `state`.
// With mixed != 0 the RHS runs at precision mode `mixed` (1 FP32, 2 FP32
// with compensated butterflies) until the error after a correction is at or
// below switch_tol, or the iteration stops contracting (error > stall x the
// error two corrections back: the errors fall in pairs); from then on it
// runs in FP64 for the rest of the step.
// The control kernel makes that choice on the device after every
// correction, and each iteration selects one of two IF nodes holding the RHS
// passes captured at each precision.
// ---------------------------------------------------------------------------
namespace dnsb {
struct MixedCtl {
  int it;         // corrector iterations of the step so far
  int fp32;       // the next RHS runs at the reduced precision
  int n32, n64;   // RHS evaluations of the step at reduced precision / FP64
  double e_prev;   // error of the previous correction (+inf before the first)
  double e_prev2;  // and of the one before it
  double first;   // error of the first correction
  double err;     // error of the latest correction
};

__global__ void mixed_init_kernel(MixedCtl* c, int mixed) {
  c->it = 0;
  c->fp32 = mixed ? 1 : 0;
  c->n32 = mixed ? 2 : 0;  // the RHS of u^n and of the start
  c->n64 = mixed ? 0 : 2;
  c->e_prev = __longlong_as_double(0x7ff0000000000000LL);  // +inf
  c->e_prev2 = c->e_prev;
  c->first = 0.0;
  c->err = 0.0;
}

// After a correction: count the iteration (first: the start's correction),
// keep the errors, choose the next RHS's precision, and set the loop's
// condition (and, after iteration A, the IF node's) to "iterate again".
//
// flags (non-null for the first correction and the unrolled iterations): [0]
// skip the next unrolled iteration (the loop has ended), [1] / [2] skip its
// reduced-precision / FP64 RHS; count_next: the next iteration is an unrolled
// one, so its RHS is counted here (the WHILE body's precision kernel counts
// its own).  After a skipped iteration the kernel returns at once.
__global__ void mixed_ctl_kernel(cudaGraphConditionalHandle h, cudaGraphConditionalHandle h_if,
                                 int set_if, const double* err, MixedCtl* c, double tol,
                                 int max_iter, double switch_tol, double stall, int first,
                                 int* flags, int count_next) {
  if (flags && !first && flags[0]) return;
  const int it = first ? 0 : c->it + 1;
  const double e = err[0];
  const unsigned cont = (e > tol && it < max_iter) ? 1u : 0u;
  if (first) c->first = e;
  if (c->fp32 && (e <= switch_tol || e > stall * c->e_prev2)) c->fp32 = 0;
  c->e_prev2 = c->e_prev;
  c->e_prev = e;
  c->it = it;
  c->err = e;
  if (flags) {
    flags[0] = cont ? 0 : 1;
    flags[1] = (cont && c->fp32) ? 0 : 1;
    flags[2] = (cont && !c->fp32) ? 0 : 1;
    if (cont && count_next) {
      if (c->fp32)
        c->n32 += 1;
      else
        c->n64 += 1;
    }
  }
  cudaGraphSetConditional(h, cont);
  if (set_if) cudaGraphSetConditional(h_if, cont);
}

// Top of a corrector iteration of the mixed form: run the RHS of the chosen
// precision (one of the two IF nodes) and count it.
__global__ void mixed_prec_kernel(cudaGraphConditionalHandle h32, cudaGraphConditionalHandle h64,
                                  MixedCtl* c) {
  const int f = c->fp32;
  if (f)
    c->n32 += 1;
  else
    c->n64 += 1;
  cudaGraphSetConditional(h32, f ? 1u : 0u);
  cudaGraphSetConditional(h64, f ? 0u : 1u);
}
}  // namespace dnsb

struct dnsb_mixed_graph {
  cudaGraphExec_t pre = nullptr, post = nullptr;
  long long k_pre = 0, k_post = 0, k_iter = 0;  // kernels per graph / per iteration
  int mixed = 0;
  int unroll = 0;  // corrector iterations captured unrolled
  double2 *Ra = nullptr, *Rb = nullptr;
  double* err = nullptr;
  int* flags = nullptr;  // skip flags of the unrolled iterations (mixed_ctl_kernel)
  dnsb::MixedCtl* ctl = nullptr;
  dnsb::MixedCtl* h_ctl = nullptr;  // pinned copy read by dnsb_mixed_graph_status
};

static void mixed_graph_free(dnsb_mixed_graph* g) {
  if (g->pre) cudaGraphExecDestroy(g->pre);
  if (g->post) cudaGraphExecDestroy(g->post);
  void* ptrs[] = {g->Ra, g->Rb, g->err, g->ctl, g->flags};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (g->h_ctl) cudaFreeHost(g->h_ctl);
  delete g;
}

extern "C" int dnsb_couette_mixed_graph_create(dnsb_couette* p, void* state, void* up,
                                               void* cur, double tol, int max_iter, int mixed,
                                               double switch_tol, double stall, int restart,
                                               dnsb_mixed_graph** out) {
  if (!p || !state || !up || !cur || !out) return fail(DNSB_ERR_ARG, "null argument");
  if (state == up || state == cur || up == cur)
    return fail(DNSB_ERR_ARG, "state, up and cur must be distinct buffers");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts step through the host loop");
  if (!p->bound) return fail(DNSB_ERR_ARG, "IMM operators not bound");
  if (mixed < 0 || mixed > 2) return fail(DNSB_ERR_ARG, "mixed must be 0, 1 or 2");
  if (mixed && !couette_fp32_sizes(p))
    return fail(DNSB_ERR_ARG,
                "FP32 RHS passes need padded sizes in {48, 72, 96, 192} with nx_p = 3 nx / 2");
  const size_t n = 3 * (size_t)p->NM * p->Ny;
  auto* g = new dnsb_mixed_graph();
  g->mixed = mixed;
  if (cudaMalloc(&g->Ra, n * sizeof(double2)) || cudaMalloc(&g->Rb, n * sizeof(double2)) ||
      cudaMalloc(&g->err, sizeof(double)) || cudaMalloc(&g->ctl, sizeof(dnsb::MixedCtl)) ||
      cudaMalloc(&g->flags, 4 * sizeof(int)) ||
      cudaMallocHost(&g->h_ctl, sizeof(dnsb::MixedCtl))) {
    mixed_graph_free(g);
    return fail(DNSB_ERR_CUDA, "mixed step graph allocation failed");
  }
  const int keep = p->rhs_fp32;
  // the RHS passes of one precision (the context's own setting is restored)
  auto rhs = [&](const void* in, void* o, int prec, cudaStream_t s) {
    p->rhs_fp32 = prec;
    const int r = couette_rhs_impl(p, in, o, 7u, s);
    p->rhs_fp32 = keep;
    return r;
  };
  cudaStream_t s = nullptr, sb = nullptr, si = nullptr, sp = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&si, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&sp, cudaStreamNonBlocking);
  int rc = 0;
  auto ck = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && !rc)
      rc = fail(DNSB_ERR_CUDA, std::string("mixed step graph: ") + what + ": " +
                                   cudaGetErrorString(e));
  };
  const long long c0 = g_launches.load();

  // -- predict
  cudaGraph_t done = nullptr;
  ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
  dnsb::mixed_init_kernel<<<1, 1, 0, s>>>(g->ctl, mixed);
  ck(cudaGetLastError(), "init kernel");
  if (!rc) rc = rhs(state, g->Rb, mixed, s);
  if (!rc) rc = dnsb_couette_imm(p, state, state, g->Rb, g->Rb, up, nullptr, nullptr, s);
  ck(cudaMemcpyAsync(cur, up, n * sizeof(double2), cudaMemcpyDeviceToDevice, s), "copy");
  g->k_pre = g_launches.load() - c0 + 1;  // + the init kernel
  ck(cudaStreamEndCapture(s, &done), "end capture");  // always end the capture
  if (!rc) ck(cudaGraphInstantiate(&g->pre, done, 0), "instantiate");
  if (done) cudaGraphDestroy(done);
  done = nullptr;

  // -- correct
  // one corrector iteration captured on `st` into graph `gr`: the RHS of
  // `cur` into nx (both precisions behind IF nodes in the mixed form), then
  // the correction with rhs_prev pv
  long long k_rhs = 0, k_imm = 0;
  auto iteration = [&](cudaStream_t st, cudaGraph_t gr, double2* nx, double2* pv) {
    if (rc) return;
    if (mixed) {
      cudaGraphConditionalHandle h32 = 0, h64 = 0;
      ck(cudaGraphConditionalHandleCreate(&h32, gr, 0, 0), "conditional handle");
      ck(cudaGraphConditionalHandleCreate(&h64, gr, 0, 0), "conditional handle");
      dnsb::mixed_prec_kernel<<<1, 1, 0, st>>>(h32, h64, g->ctl);
      ck(cudaGetLastError(), "precision kernel");
      for (int f = 0; f < 2 && !rc; ++f) {
        cudaGraph_t ib = add_cond_node(st, gr, f ? h64 : h32, cudaGraphCondTypeIf, rc);
        if (rc) break;
        ck(cudaStreamBeginCaptureToGraph(sp, ib, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal), "RHS capture");
        const long long a = g_launches.load();
        if (!rc) rc = rhs(cur, nx, f ? 0 : mixed, sp);
        k_rhs = g_launches.load() - a;
        cudaGraph_t o = nullptr;
        ck(cudaStreamEndCapture(sp, &o), "end RHS capture");
      }
    } else {
      const long long a = g_launches.load();
      rc = rhs(cur, nx, 0, st);
      k_rhs = g_launches.load() - a;
    }
    const long long b = g_launches.load();
    if (!rc) rc = dnsb_couette_imm(p, state, cur, pv, nx, cur, nullptr, g->err, st);
    k_imm = g_launches.load() - b;
  };
  ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaStreamCaptureStatus cs;
  cudaGraph_t graph = nullptr;
  ck(cudaStreamGetCaptureInfo(s, &cs, nullptr, &graph, nullptr, nullptr), "capture info");
  cudaGraphConditionalHandle h = 0, h_if = 0;
  ck(cudaGraphConditionalHandleCreate(&h, graph, 0, 0), "conditional handle");
  const long long c1 = g_launches.load();
  if (!rc) rc = rhs(cur, g->Ra, mixed, s);
  if (!rc) rc = dnsb_couette_imm(p, state, cur, restart ? g->Ra : g->Rb, g->Ra, cur, nullptr,
                                 g->err, s);
  const int U = couette_unroll(p, max_iter);
  g->unroll = U;
  int* flags = U > 0 ? g->flags : nullptr;
  dnsb::mixed_ctl_kernel<<<1, 1, 0, s>>>(h, 0, 0, g->err, g->ctl, tol, max_iter, switch_tol,
                                         stall, 1, flags, U > 0 ? 1 : 0);
  ck(cudaGetLastError(), "control kernel");
  // the unrolled iterations: both RHS precisions in line, each skipped by its
  // own flag, so no conditional node is entered while the loop runs in them
  for (int k = 0; k < U && !rc; ++k) {
    double2* nx = (k & 1) ? g->Ra : g->Rb;
    double2* pv = (k & 1) ? g->Rb : g->Ra;
    if (mixed) {
      p->skip = flags + 1;
      rc = rhs(cur, nx, mixed, s);
      p->skip = flags + 2;
      if (!rc) rc = rhs(cur, nx, 0, s);
    } else {
      p->skip = flags;
      rc = rhs(cur, nx, 0, s);
    }
    p->skip = flags;
    if (!rc) rc = dnsb_couette_imm(p, state, cur, pv, nx, cur, nullptr, g->err, s);
    p->skip = nullptr;
    dnsb::mixed_ctl_kernel<<<1, 1, 0, s>>>(h, 0, 0, g->err, g->ctl, tol, max_iter, switch_tol,
                                           stall, 0, flags, k + 1 < U ? 1 : 0);
    ck(cudaGetLastError(), "control kernel");
  }
  g->k_post = g_launches.load() - c1 + 1 + U;  // + the control kernels
  // the WHILE body's iteration A continues the alternation of the RHS buffers
  double2* na = (U & 1) ? g->Ra : g->Rb;
  double2* nb = (U & 1) ? g->Rb : g->Ra;
  cudaGraph_t bg = add_cond_node(s, graph, h, cudaGraphCondTypeWhile, rc);
  if (!rc) {
    ck(cudaGraphConditionalHandleCreate(&h_if, bg, 0, 0), "conditional handle");
    ck(cudaStreamBeginCaptureToGraph(sb, bg, nullptr, nullptr, 0,
                                     cudaStreamCaptureModeThreadLocal), "body capture");
    iteration(sb, bg, na, nb);  // A: rhs_next -> na, rhs_prev nb
    dnsb::mixed_ctl_kernel<<<1, 1, 0, sb>>>(h, h_if, 1, g->err, g->ctl, tol, max_iter,
                                            switch_tol, stall, 0, nullptr, 0);
    ck(cudaGetLastError(), "control kernel");
    cudaGraph_t ig = add_cond_node(sb, bg, h_if, cudaGraphCondTypeIf, rc);
    if (!rc) {
      ck(cudaStreamBeginCaptureToGraph(si, ig, nullptr, nullptr, 0,
                                       cudaStreamCaptureModeThreadLocal), "IF body capture");
      iteration(si, ig, nb, na);  // B: rhs_next -> nb, rhs_prev na
      dnsb::mixed_ctl_kernel<<<1, 1, 0, si>>>(h, 0, 0, g->err, g->ctl, tol, max_iter,
                                              switch_tol, stall, 0, nullptr, 0);
      ck(cudaGetLastError(), "control kernel");
      cudaGraph_t iout = nullptr;
      ck(cudaStreamEndCapture(si, &iout), "end IF body capture");
    }
    cudaGraph_t bout = nullptr;
    ck(cudaStreamEndCapture(sb, &bout), "end body capture");
  }
  ck(cudaMemcpyAsync(state, cur, n * sizeof(double2), cudaMemcpyDeviceToDevice, s), "copy");
  ck(cudaStreamEndCapture(s, &done), "end capture");
  if (!rc) ck(cudaGraphInstantiate(&g->post, done, 0), "instantiate");
  if (done) cudaGraphDestroy(done);
  // a mixed iteration: precision kernel, one RHS, the IMM, the control kernel
  g->k_iter = (mixed ? 1 : 0) + k_rhs + k_imm + 1;
  g_launches.fetch_sub(g_launches.load() - c0, std::memory_order_relaxed);
  cudaStreamDestroy(s);
  cudaStreamDestroy(sb);
  cudaStreamDestroy(si);
  cudaStreamDestroy(sp);
  if (rc) {
    mixed_graph_free(g);
    return rc;
  }
  *out = g;
  return 0;
}

extern "C" int dnsb_mixed_graph_predict(dnsb_mixed_graph* g, void* stream) {
  if (!g) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_CUDA(cudaGraphLaunch(g->pre, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_mixed_graph_correct(dnsb_mixed_graph* g, void* stream) {
  if (!g) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_CUDA(cudaGraphLaunch(g->post, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_mixed_graph_status(dnsb_mixed_graph* g, int* iters, double* err,
                                       double* first_err, int* n32, int* n64, void* stream) {
  if (!g || !iters || !err) return fail(DNSB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  DNSB_CUDA(cudaMemcpyAsync(g->h_ctl, g->ctl, sizeof(dnsb::MixedCtl), cudaMemcpyDeviceToHost,
                            st));
  DNSB_CUDA(cudaStreamSynchronize(st));
  const dnsb::MixedCtl c = *g->h_ctl;
  *iters = c.it;
  *err = c.err;
  if (first_err) *first_err = c.first;
  // the FP64 form has no precision kernel: every RHS of the step is FP64
  if (n32) *n32 = g->mixed ? c.n32 : 0;
  if (n64) *n64 = g->mixed ? c.n64 : 2 + c.it;
  const long long looped = c.it > g->unroll ? c.it - g->unroll : 0;
  g_launches.fetch_add(g->k_pre + g->k_post + looped * g->k_iter, std::memory_order_relaxed);
  return 0;
}

extern "C" int dnsb_mixed_graph_destroy(dnsb_mixed_graph* g) {
  if (!g) return fail(DNSB_ERR_ARG, "null argument");
  mixed_graph_free(g);
  return 0;
}

extern "C" int dnsb_couette_set_wait_limit(dnsb_couette* p, int polls) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  if (polls < 0) return fail(DNSB_ERR_ARG, "polls must be >= 0");
  p->wait_limit = polls;
  p->batch.wait_limit = polls;
  return 0;
}

extern "C" int dnsb_couette_clear_status(dnsb_couette* p, void* stream) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_CUDA(cudaMemsetAsync(p->status, 0, sizeof(int), as_stream(stream)));
  return 0;
}

extern "C" int dnsb_couette_check(dnsb_couette* p, void* stream) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  int h = 0;
  DNSB_CUDA(cudaMemcpyAsync(&h, p->status, sizeof(int), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
  DNSB_CUDA(cudaStreamSynchronize(as_stream(stream)));
  if (h & 1) return fail(DNSB_ERR_PIVOT, "pivot index outside [j, j+kl]");
  if (h & 2) return fail(DNSB_ERR_CUDA, "IMM substitution: a shared-memory ring wait timed out");
  return 0;
}

// ===========================================================================
// Autotuning: per-pass kernel variants picked by timing on the context's
// own sizes and buffers
// ===========================================================================
namespace {
// Mean milliseconds of `reps` calls of f on st (after one untimed call).
template <typename F>
int time_calls(F&& f, int reps, cudaStream_t st, float* ms) {
  int rc = f();
  if (rc) return rc;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, st);
  for (int r = 0; r < reps && !rc; ++r) rc = f();
  cudaEventRecord(b, st);
  const cudaError_t e = cudaEventSynchronize(b);
  float t = 0.0f;
  if (!rc && e == cudaSuccess) cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (!rc && e != cudaSuccess) rc = fail(DNSB_ERR_CUDA, cudaGetErrorString(e));
  *ms = t / (float)(reps > 0 ? reps : 1);
  return rc;
}

// Tunes pass k over `variants` (count nv, the default first): for each,
// `prefix` rebuilds the pass's input, then the pass alone is timed; var[k]
// keeps the fastest, but the default unless another is 5% faster (timing
// noise does not move a pass to a variant of about the same speed).
template <typename Prefix, typename Pass>
int tune_one(int* var, int k, const int* variants, int nv, int reps, cudaStream_t st,
             float* ms_out, Prefix&& prefix, Pass&& pass) {
  float best = 0.0f;
  int pick = var[k];
  for (int i = 0; i < nv; ++i) {
    var[k] = variants[i];
    int rc = prefix();
    float t = 0.0f;
    if (!rc) rc = time_calls(pass, reps, st, &t);
    if (rc) return rc;
    ms_out[variants[i]] = t;
    if (i == 0 || t < best) {
      best = t;
      pick = variants[i];
    }
  }
  if (pick != variants[0] && best > 0.95f * ms_out[variants[0]]) pick = variants[0];
  var[k] = pick;
  return 0;
}
}  // namespace

extern "C" int dnsb_periodic_set_variants(dnsb_periodic* p, const int* var) {
  if (!p || !var) return fail(DNSB_ERR_ARG, "null argument");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts run the default pass variants");
  for (int k = 0; k < 5; ++k)
    if (var[k] < 0 || var[k] > 2 || (p->rhs_fp32 && var[k] != 0))
      return fail(DNSB_ERR_ARG, "pass variants are 0, 1 or 2 (0 only in FP32)");
  for (int k = 0; k < 5; ++k) p->var[k] = var[k];
  return 0;
}

extern "C" int dnsb_couette_set_variants(dnsb_couette* p, const int* var) {
  if (!p || !var) return fail(DNSB_ERR_ARG, "null argument");
  if (p->slab.nranks && (var[0] || var[1] || var[2]))
    return fail(DNSB_ERR_ARG, "slab contexts run the default pass variants");
  for (int k = 0; k < 4; ++k)
    if (var[k] < 0 || var[k] > 2 || (k < 3 && p->rhs_fp32 && var[k] != 0))
      return fail(DNSB_ERR_ARG, "variants are 0, 1 or 2 (passes: 0 only in FP32)");
  if (var[3] == 1 && !imm_v2_supported(p->p, p->Ny))
    return fail(DNSB_ERR_ARG, "the register-window IMM does not cover these sizes");
  for (int k = 0; k < 4; ++k) p->var[k] = var[k];
  return 0;
}

extern "C" int dnsb_periodic_autotune(dnsb_periodic* p, const void* state, int reps,
                                      int* chosen, float* ms, void* stream) {
  if (!p || !state || !chosen || !ms) return fail(DNSB_ERR_ARG, "null argument");
  if (reps < 1) return fail(DNSB_ERR_ARG, "reps must be positive");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts run the default pass variants");
  cudaStream_t st = as_stream(stream);
  for (int i = 0; i < 15; ++i) ms[i] = -1.0f;
  double2* rhs = nullptr;
  DNSB_CUDA(cudaMallocAsync(&rhs, 3 * (size_t)p->S * sizeof(double2), st));
  const int all[] = {0, 1, 2}, only0[] = {0};
  int rc = 0;
  for (int k = 0; k < 5 && !rc; ++k) {
    const int* vs = p->rhs_fp32 ? only0 : all;
    const int nv = p->rhs_fp32 ? 1 : 3;
    const unsigned before = (1u << k) - 1u, self = 1u << k;
    rc = tune_one(
        p->var, k, vs, nv, reps, st, ms + 3 * k,
        [&] { return before ? periodic_rhs_impl(p, state, rhs, before, st) : 0; },
        [&] { return periodic_rhs_impl(p, state, rhs, self, st); });
  }
  cudaFreeAsync(rhs, st);
  for (int k = 0; k < 5; ++k) chosen[k] = p->var[k];
  return rc;
}

extern "C" int dnsb_couette_autotune(dnsb_couette* p, const void* state, int reps, int* chosen,
                                     float* ms, void* stream) {
  if (!p || !state || !chosen || !ms) return fail(DNSB_ERR_ARG, "null argument");
  if (reps < 1) return fail(DNSB_ERR_ARG, "reps must be positive");
  if (p->slab.nranks) return fail(DNSB_ERR_ARG, "slab contexts run the default pass variants");
  cudaStream_t st = as_stream(stream);
  for (int i = 0; i < 12; ++i) ms[i] = -1.0f;
  const size_t n = 3 * (size_t)p->NM * p->Ny;
  double2 *rhs = nullptr, *out = nullptr;
  double* err = nullptr;
  DNSB_CUDA(cudaMallocAsync(&rhs, n * sizeof(double2), st));
  DNSB_CUDA(cudaMallocAsync(&out, n * sizeof(double2), st));
  DNSB_CUDA(cudaMallocAsync(&err, sizeof(double), st));
  const int all[] = {0, 1, 2}, only0[] = {0};
  int rc = 0;
  for (int k = 0; k < 3 && !rc; ++k) {
    const unsigned before = (1u << k) - 1u, self = 1u << k;
    rc = tune_one(
        p->var, k, p->rhs_fp32 ? only0 : all, p->rhs_fp32 ? 1 : 3, reps, st, ms + 3 * k,
        [&] { return before ? couette_rhs_impl(p, state, rhs, before, st) : 0; },
        [&] { return couette_rhs_impl(p, state, rhs, self, st); });
  }
  if (!rc && p->bound) {
    // the IMM with the correction norm, as a corrector iteration calls it
    int vs[3], nv = 0;
    if (p->batch_ready) vs[nv++] = 0;
    if (imm_v2_supported(p->p, p->Ny)) vs[nv++] = 1;
    vs[nv++] = 2;
    rc = couette_rhs_impl(p, state, rhs, 7u, st);
    if (!rc)
      rc = tune_one(
          p->var, 3, vs, nv, reps, st, ms + 9, [] { return 0; },
          [&] { return dnsb_couette_imm(p, state, state, rhs, rhs, out, nullptr, err, st); });
  }
  cudaFreeAsync(rhs, st);
  cudaFreeAsync(out, st);
  cudaFreeAsync(err, st);
  for (int k = 0; k < 4; ++k) chosen[k] = p->var[k];
  return rc;
}

// ===========================================================================
// Learned corrector guess (plane Couette): BF16 MLP kernels
// ===========================================================================
extern "C" int dnsb_mlp_gemm(int ta, int tb, int M, int N, int K, const void* A, int lda,
                             const void* B, int ldb, const float* bias, int relu,
                             const void* mask, int ldm, float* Cf, void* Cb, int ldc,
                             float* work, long long work_elems, int* status, void* stream) {
  if (!A || !B || (!Cf && !Cb)) return fail(DNSB_ERR_ARG, "null argument");
  if (M < 1 || N < 1 || K < 1 || lda < 1 || ldb < 1 || ldc < N || (mask && ldm < N))
    return fail(DNSB_ERR_ARG, "invalid GEMM sizes");
  if ((ta ? lda < M : lda < K) || (tb ? ldb < N : ldb < K))
    return fail(DNSB_ERR_ARG, "leading dimension smaller than the operand");
  if (work_elems < 0 || (work_elems > 0 && !work))
    return fail(DNSB_ERR_ARG, "invalid workspace");
  int n = 1;
  const cudaError_t e = launch_mlp_gemm(ta, tb, M, N, K, A, lda, B, ldb, bias, relu, mask, ldm,
                                        Cf, Cb, ldc, work_elems > 0 ? work : nullptr, work_elems,
                                        status, as_stream(stream), &n);
  count_launches(n);
  if (e != cudaSuccess) return fail(DNSB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return 0;
}

extern "C" int dnsb_mlp_transpose(const void* A, int R, int C, int lda, void* out, int ldo,
                                  void* stream) {
  if (!A || !out) return fail(DNSB_ERR_ARG, "null argument");
  if (R < 1 || C < 1 || lda < C || ldo < R) return fail(DNSB_ERR_ARG, "invalid sizes");
  DNSB_LAUNCH(launch_bf16_transpose(A, R, C, lda, out, ldo, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_learned_features(dnsb_couette* p, const void* un, const void* up,
                                     const void* dprev, const void* target, double kx_max,
                                     double kz_max, double s_floor, void* X, int ldx, float* T,
                                     int ldt, float* scale, void* stream) {
  if (!p || !un || !up || !X || !scale || (target && !T)) return fail(DNSB_ERR_ARG, "null argument");
  if (ldx < 12 * p->Ny + 2 || (target && ldt < 6 * p->Ny) || !(kx_max > 0.0) || !(kz_max > 0.0))
    return fail(DNSB_ERR_ARG, "invalid feature sizes");
  DNSB_LAUNCH(launch_learned_features(
      (const double2*)un, (const double2*)up, (const double2*)dprev, (const double2*)target,
      p->kx, p->kz, p->NKX, p->NZ1, p->Ny, kx_max, kz_max, s_floor, X, ldx, T, ldt, scale,
      as_stream(stream)));
  return 0;
}

extern "C" int dnsb_learned_guess(dnsb_couette* p, const void* up, const float* Y, int ldy,
                                  const float* scale, void* out, void* stream) {
  if (!p || !up || !Y || !scale || !out) return fail(DNSB_ERR_ARG, "null argument");
  if (ldy < 6 * p->Ny) return fail(DNSB_ERR_ARG, "invalid output stride");
  DNSB_LAUNCH(launch_learned_guess((const double2*)up, Y, ldy, scale, p->NM, p->Ny,
                                   (double2*)out, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_mlp_loss_grad(const float* Y, const float* T, int M, int N, int ld,
                                  float* dYf, void* dYb, float* err, float* ref, void* stream) {
  if (!Y || !T || !dYf || !dYb || !err || !ref) return fail(DNSB_ERR_ARG, "null argument");
  if (M < 1 || N < 1 || ld < N) return fail(DNSB_ERR_ARG, "invalid sizes");
  DNSB_LAUNCH(launch_mlp_loss_grad(Y, T, M, N, ld, dYf, dYb, err, ref, as_stream(stream)));
  return 0;
}

extern "C" int dnsb_mlp_colsum(const void* A, int bf16, int M, int N, int lda, float* out,
                               float* work, long long work_elems, void* stream) {
  if (!A || !out || !work) return fail(DNSB_ERR_ARG, "null argument");
  if (M < 1 || N < 1 || lda < N) return fail(DNSB_ERR_ARG, "invalid sizes");
  if (work_elems < (long long)colsum_groups(M) * N)
    return fail(DNSB_ERR_ARG, "colsum workspace smaller than min(M, 128) x N floats");
  const cudaError_t e = launch_colsum_det(A, bf16, M, N, lda, out, work, as_stream(stream));
  count_launches(2);
  if (e != cudaSuccess) return fail(DNSB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return 0;
}

extern "C" int dnsb_mlp_adam(float* w, float* m, float* v, const float* grad, void* wb,
                             long long n, float lr, float b1, float b2, float eps, int step,
                             void* stream) {
  if (!w || !m || !v || !grad) return fail(DNSB_ERR_ARG, "null argument");
  if (n < 1 || step < 1) return fail(DNSB_ERR_ARG, "invalid sizes");
  DNSB_LAUNCH(launch_mlp_adam(w, m, v, grad, wb, n, lr, b1, b2, eps, step, as_stream(stream)));
  return 0;
}

// ===========================================================================
// Influence-matrix precompute on the GPU
// ===========================================================================
extern "C" int dnsb_imm_precompute(const double* D1, const double* D2, const double* kx,
                                   int nkx, const double* kz, int nkz, int ny, int p,
                                   double dt, double c, double nu, double* p1, double* p2,
                                   double* v1, double* v2, double* q1, double* q2,
                                   double* M_inv, double* Lk_ab, int* Lk_piv, double* Hk_ab,
                                   int* Hk_piv, int* info_dev, void* stream) {
  if (!D1 || !D2 || !kx || !kz || !p1 || !p2 || !v1 || !v2 || !q1 || !q2 || !M_inv ||
      !Lk_ab || !Lk_piv || !Hk_ab || !Hk_piv || !info_dev)
    return fail(DNSB_ERR_ARG, "null argument");
  if (nkx < 1 || nkz < 1 || ny < 3 || p < 1 || p >= ny || !(dt > 0.0))
    return fail(DNSB_ERR_ARG, "invalid sizes");
  cudaStream_t st = as_stream(stream);
  const size_t nmy = (size_t)nkx * nkz * ny;
  double* bp = nullptr;
  double* bv = nullptr;
  DNSB_CUDA(cudaMallocAsync(&bp, nmy * 2 * sizeof(double), st));
  if (cudaMallocAsync(&bv, nmy * 4 * sizeof(double), st) != cudaSuccess) {
    cudaFreeAsync(bp, st);
    return fail(DNSB_ERR_CUDA, "precompute workspace allocation failed");
  }
  ImmPrecomputeArgs a{D1, D2, kx, kz, nkx, nkz, ny, p, dt, c, nu, p1, p2, v1, v2, q1, q2,
                      M_inv, Lk_ab, Lk_piv, Hk_ab, Hk_piv, info_dev, info_dev};
  int nl = 0;
  const cudaError_t e = launch_imm_precompute(a, bp, bv, st, &nl);
  g_launches.fetch_add(nl, std::memory_order_relaxed);
  cudaFreeAsync(bp, st);
  cudaFreeAsync(bv, st);
  if (e != cudaSuccess)
    return fail(DNSB_ERR_CUDA, std::string("IMM precompute: ") + cudaGetErrorString(e));
  return 0;
}

// ===========================================================================
// Standalone banded solve
// ===========================================================================
extern "C" int dnsb_banded_solve(const double* ab, const int* ipiv, double* b,
                                 int nmodes, int ny, int kl, int ku, int ncols,
                                 int* status_dev, void* stream) {
  if (!ab || !ipiv || !b) return fail(DNSB_ERR_ARG, "null argument");
  if (nmodes < 0 || ny < 1 || kl < 0 || ku < 0 || ncols < 1)
    return fail(DNSB_ERR_ARG, "invalid sizes");
  if (nmodes == 0) return 0;
  DNSB_LAUNCH(launch_banded_solve(ab, ipiv, b, nmodes, ny, kl, ku, ncols,
                                  status_dev, as_stream(stream)));
  return 0;
}

// ===========================================================================
// Slab decomposition over several GPUs (fft.py:193-392, sharding.py:107-129
// of the reference).  Spectral arrays are sharded on kx; between the column
// passes and the x pass the padded grid is sharded on z.  The two passes
// that feed the other layout (the z inverse, the x pass) store every output
// straight into the receive buffer of the rank that owns it, through that
// rank's pointer (peer memory over NVLink, or a buffer of the same GPU when
// the ranks are emulated in one process): the exchange is fused into the
// pass kernels.  The RHS runs in three phases; between them the caller
// makes every rank's previous phase complete before any rank starts the
// next one (a collective on the stream, or plain stream order when the
// ranks share one).
// ===========================================================================
static bool slab_sizes_ok(int nx_p, int nz_p, int nkxg, int nranks, int rank,
                          const char** why) {
  auto fixed = [](int L) { return L == 48 || L == 72 || L == 96 || L == 192; };
  if (nranks < 1 || nranks > kMaxRanks || rank < 0 || rank >= nranks) {
    *why = "nranks must be 1..8 and 0 <= rank < nranks";
    return false;
  }
  if (nkxg % nranks || nz_p % nranks) {
    *why = "nx/2 and nz_p must be multiples of nranks";
    return false;
  }
  if (!fixed(nx_p) || !fixed(nz_p) || 3 * nkxg != nx_p) {
    *why = "slab passes need padded sizes in {48, 72, 96, 192} with nx_p = 3 nx / 2";
    return false;
  }
  return true;
}

extern "C" int dnsb_periodic_create_slab(const dnsb_periodic_desc* d, int nranks, int rank,
                                         dnsb_periodic** out) {
  if (!d || !out || !d->kx || !d->ldt_1 || !d->ildt_2) return fail(DNSB_ERR_ARG, "null argument");
  *out = nullptr;
  const int nkxg = d->nx / 2;
  const char* why = nullptr;
  if (!slab_sizes_ok(d->nx_p, d->nz_p, nkxg, nranks, rank, &why)) return fail(DNSB_ERR_ARG, why);
  auto fixed = [](int L) { return L == 48 || L == 72 || L == 96 || L == 192; };
  if (!fixed(d->ny_p)) return fail(DNSB_ERR_ARG, "slab passes need ny_p in {48, 72, 96, 192}");
  // This rank's kx columns of the per-mode coefficients ([ky][kz][kx]).
  const int nkx = nkxg / nranks, ny1 = d->ny - 1, nz1 = d->nz - 1;
  std::vector<double> l1((size_t)ny1 * nz1 * nkx), l2(l1.size());
  for (size_t r = 0; r < (size_t)ny1 * nz1; ++r)
    for (int ix = 0; ix < nkx; ++ix) {
      l1[r * nkx + ix] = d->ldt_1[r * nkxg + (size_t)rank * nkx + ix];
      l2[r * nkx + ix] = d->ildt_2[r * nkxg + (size_t)rank * nkx + ix];
    }
  dnsb_periodic_desc ld = *d;
  ld.nx = 2 * nkx;
  ld.kx = d->kx + (size_t)rank * nkx;
  ld.ldt_1 = l1.data();
  ld.ildt_2 = l2.data();
  dnsb_periodic* p = nullptr;
  int rc = dnsb_periodic_create(&ld, &p);
  if (rc) return rc;
  p->slab.nranks = nranks;
  p->slab.rank = rank;
  p->slab.NKXg = nkxg;
  const size_t nx = 6ull * p->My * (p->Mz / nranks) * nkxg;
  if (cudaMalloc(&p->slab.Bx, nx * sizeof(double2)) != cudaSuccess) {
    periodic_free(p);
    return fail(DNSB_ERR_CUDA, "slab buffer allocation failed");
  }
  p->ws_bytes += nx * sizeof(double2);
  *out = p;
  return 0;
}

extern "C" int dnsb_couette_create_slab(const dnsb_couette_desc* d, int nranks, int rank,
                                        dnsb_couette** out) {
  if (!d || !out || !d->kx) return fail(DNSB_ERR_ARG, "null argument");
  *out = nullptr;
  const int nkxg = d->nx / 2;
  const char* why = nullptr;
  if (!slab_sizes_ok(d->nx_p, d->nz_p, nkxg, nranks, rank, &why)) return fail(DNSB_ERR_ARG, why);
  const int nkx = nkxg / nranks;
  dnsb_couette_desc ld = *d;
  ld.nx = 2 * nkx;
  ld.kx = d->kx + (size_t)rank * nkx;
  dnsb_couette* p = nullptr;
  int rc = dnsb_couette_create(&ld, &p);
  if (rc) return rc;
  p->slab.nranks = nranks;
  p->slab.rank = rank;
  p->slab.NKXg = nkxg;
  const size_t nx = 6ull * (p->Mz / nranks) * nkxg * p->Ny;
  if (cudaMalloc(&p->slab.Bx, nx * sizeof(double2)) != cudaSuccess) {
    couette_free(p);
    return fail(DNSB_ERR_CUDA, "slab buffer allocation failed");
  }
  p->ws_bytes += nx * sizeof(double2);
  *out = p;
  return 0;
}

static int slab_buffers(const SlabState& s, double2* B, void** bx, void** bk) {
  if (!s.nranks) return fail(DNSB_ERR_ARG, "not a slab context");
  if (!bx || !bk) return fail(DNSB_ERR_ARG, "null argument");
  *bx = s.Bx;
  *bk = B;
  return 0;
}

static int slab_connect(SlabState& s, void* const* bx, void* const* bk) {
  if (!s.nranks) return fail(DNSB_ERR_ARG, "not a slab context");
  if (!bx || !bk) return fail(DNSB_ERR_ARG, "null argument");
  for (int r = 0; r < s.nranks; ++r)
    if (!bx[r] || !bk[r]) return fail(DNSB_ERR_ARG, "null rank buffer");
  for (int r = 0; r < s.nranks; ++r) {
    s.xdest[r] = (double2*)bx[r];
    s.kdest[r] = (double2*)bk[r];
  }
  s.connected = true;
  return 0;
}

extern "C" int dnsb_periodic_slab_buffers(dnsb_periodic* p, void** bx, void** bk) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  return slab_buffers(p->slab, p->B, bx, bk);
}

extern "C" int dnsb_periodic_slab_connect(dnsb_periodic* p, void* const* bx, void* const* bk) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  return slab_connect(p->slab, bx, bk);
}

extern "C" int dnsb_couette_slab_buffers(dnsb_couette* p, void** bx, void** bk) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  return slab_buffers(p->slab, p->B, bx, bk);
}

extern "C" int dnsb_couette_slab_connect(dnsb_couette* p, void* const* bx, void* const* bk) {
  if (!p) return fail(DNSB_ERR_ARG, "null argument");
  return slab_connect(p->slab, bx, bk);
}

static int slab_ready(const SlabState& s, int fp32, const int* var, int nvar) {
  if (!s.nranks) return fail(DNSB_ERR_ARG, "not a slab context");
  if (!s.connected) return fail(DNSB_ERR_ARG, "slab context not connected");
  if (fp32) return fail(DNSB_ERR_ARG, "slab contexts run the FP64 passes");
  for (int k = 0; k < nvar; ++k)
    if (var[k] != 0) return fail(DNSB_ERR_ARG, "slab contexts run the default pass variants");
  return 0;
}

// Phase 0: y inverse with the curl, z inverse into every rank's Bx (its
// padded-z share).  Phase 1: the x pass with the product over this rank's
// Bx into every rank's pass buffer (its kx share).  Phase 2: z forward, y
// forward and the projection into `rhs`.
extern "C" int dnsb_periodic_rhs_phase(dnsb_periodic* p, const void* state, void* rhs,
                                       int phase, void* stream) {
  if (!p || !state || !rhs) return fail(DNSB_ERR_ARG, "null argument");
  int rc = slab_ready(p->slab, p->rhs_fp32, p->var, 5);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const SlabState& s = p->slab;
  const int mzl = p->Mz / s.nranks;
  if (phase == 0) {
    rc = periodic_rhs_impl(p, state, rhs, 1u, st);
    if (rc) return rc;
    ColPassArgs zi = periodic_zinv(p);
    for (int r = 0; r < s.nranks; ++r) zi.slab.buf[r] = s.xdest[r];
    zi.slab.blk = mzl;
    zi.slab.fs = (long long)p->My * mzl * s.NKXg;
    zi.out_os = (long long)mzl * s.NKXg;
    zi.slab.ts = s.NKXg;
    zi.slab.off = (long long)s.rank * p->NKX;
    DNSB_LAUNCH(launch_col_pass(zi, 6, p->My, st));
    return 0;
  }
  if (phase == 1) {
    XPassArgs xa{};
    xa.in = xa.out = s.Bx;
    xa.in_fs = xa.out_fs = (long long)p->My * mzl * s.NKXg;
    xa.nrows = p->My * mzl;
    xa.inner_n = mzl;
    xa.so = (long long)mzl * s.NKXg;
    xa.si = s.NKXg;
    xa.ks = 1;
    xa.nkx = s.NKXg;
    xa.y_outer = 1;
    xa.rows_fast = 0;
    xa.U = p->U;
    xa.cU = p->cU;
    xa.nU = p->nU;
    xa.ny_grid = p->My;
    xa.plan = p->px;
    xa.tw = p->twx;
    for (int r = 0; r < s.nranks; ++r) xa.slab.buf[r] = s.kdest[r];
    xa.slab.blk = p->NKX;
    xa.slab.fs = (long long)p->My * p->Mz * p->NKX;
    xa.slab.so = (long long)p->Mz * p->NKX;
    xa.slab.si = p->NKX;
    xa.slab.oo = 0;
    xa.slab.io = s.rank * mzl;
    xa.slab.ks = 1;
    DNSB_LAUNCH(launch_x_pass(xa, st));
    return 0;
  }
  if (phase == 2) return periodic_rhs_impl(p, state, rhs, 8u | 16u, st);
  return fail(DNSB_ERR_ARG, "phase must be 0, 1 or 2");
}

// Phase 0: z inverse with the FD curl into every rank's Bx.  Phase 1: the x
// pass over this rank's Bx into every rank's pass buffer.  Phase 2: z
// forward into `rhs`.
extern "C" int dnsb_couette_rhs_phase(dnsb_couette* p, const void* state, void* rhs, int phase,
                                      void* stream) {
  if (!p || !state || !rhs) return fail(DNSB_ERR_ARG, "null argument");
  int rc = slab_ready(p->slab, p->rhs_fp32, p->var, 3);
  if (rc) return rc;
  cudaStream_t st = as_stream(stream);
  const SlabState& s = p->slab;
  const int mzl = p->Mz / s.nranks;
  if (phase == 0) {
    ZInvCurlArgs zi{};
    zi.u = (const double2*)state;
    zi.out = p->B;
    zi.NZ1 = p->NZ1;
    zi.NKX = p->NKX;
    zi.Ny = p->Ny;
    zi.curl = 1;
    zi.s1 = p->s1;
    zi.d1_j0 = p->d1j0;
    zi.d1_w = p->d1w;
    zi.d1_wT = p->d1wT;
    zi.kx = p->kx;
    zi.kz = p->kz;
    zi.plan = p->pz;
    zi.tw = p->twz;
    for (int r = 0; r < s.nranks; ++r) zi.slab.buf[r] = s.xdest[r];
    zi.slab.blk = mzl;
    zi.slab.fs = (long long)mzl * s.NKXg * p->Ny;
    zi.slab.ts = (long long)s.NKXg * p->Ny;
    zi.slab.off = (long long)s.rank * p->NKX * p->Ny;
    DNSB_LAUNCH(launch_zinv_curl(zi, p->span_max, st));
    return 0;
  }
  if (phase == 1) {
    XPassArgs xa{};
    xa.in = xa.out = s.Bx;
    xa.in_fs = xa.out_fs = (long long)mzl * s.NKXg * p->Ny;
    xa.nrows = mzl * p->Ny;
    xa.inner_n = p->Ny;
    xa.so = (long long)s.NKXg * p->Ny;
    xa.si = 1;
    xa.ks = p->Ny;
    xa.nkx = s.NKXg;
    xa.y_outer = 0;
    xa.rows_fast = 1;
    xa.U = p->U;
    xa.cU = p->cU;
    xa.nU = p->nU;
    xa.ny_grid = p->Ny;
    xa.plan = p->px;
    xa.tw = p->twx;
    for (int r = 0; r < s.nranks; ++r) xa.slab.buf[r] = s.kdest[r];
    xa.slab.blk = p->NKX;
    xa.slab.fs = (long long)p->Mz * p->NKX * p->Ny;
    xa.slab.so = (long long)p->NKX * p->Ny;
    xa.slab.si = 1;
    xa.slab.oo = s.rank * mzl;
    xa.slab.io = 0;
    xa.slab.ks = p->Ny;
    DNSB_LAUNCH(launch_x_pass(xa, st));
    return 0;
  }
  if (phase == 2) return couette_rhs_impl(p, state, rhs, 4u, st);
  return fail(DNSB_ERR_ARG, "phase must be 0, 1 or 2");
}

// CUDA IPC of a device allocation (the slab buffers of another process's
// rank): a 64-byte handle, opened with peer access.
extern "C" int dnsb_ipc_handle(const void* dev_ptr, void* handle) {
  if (!dev_ptr || !handle) return fail(DNSB_ERR_ARG, "null argument");
  cudaIpcMemHandle_t h;
  DNSB_CUDA(cudaIpcGetMemHandle(&h, const_cast<void*>(dev_ptr)));
  static_assert(sizeof(h) == 64, "CUDA IPC handles are 64 bytes");
  std::memcpy(handle, &h, sizeof(h));
  return 0;
}

extern "C" int dnsb_ipc_open(const void* handle, void** dev_ptr) {
  if (!handle || !dev_ptr) return fail(DNSB_ERR_ARG, "null argument");
  cudaIpcMemHandle_t h;
  std::memcpy(&h, handle, sizeof(h));
  DNSB_CUDA(cudaIpcOpenMemHandle(dev_ptr, h, cudaIpcMemLazyEnablePeerAccess));
  return 0;
}

extern "C" int dnsb_ipc_close(void* dev_ptr) {
  if (!dev_ptr) return fail(DNSB_ERR_ARG, "null argument");
  DNSB_CUDA(cudaIpcCloseMemHandle(dev_ptr));
  return 0;
}
