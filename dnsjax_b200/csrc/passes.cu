// Axis-pass kernels of the 3/2-dealiased transforms.
//
// Index maps follow the reference's pad/truncate helpers
// (src/dnsjax/fft.py:41-190) and transform order (fft.py:193-408); the
// fused products follow src/dnsjax/rhs.py:77-90 (rotational form),
// src/dnsjax/geometries/triply_periodic.py:122-132 (curl),
// src/dnsjax/flows/plane_couette.py:251-271 (FD curl) and
// src/dnsjax/flows/monochromatic.py:366-386 (projection).
#include "passes.cuh"

namespace dnsb {

// Transform lengths with a compile-time FFT plan; others use the runtime
// plan (template argument 0).
#define DNSB_DISPATCH(L, KERNEL, GRID, SMEM, ST, ...)                         \
  switch (L) {                                                              \
    case 48: KERNEL<48><<<GRID, kPassThreads, SMEM, ST>>>(__VA_ARGS__); break; \
    case 72: KERNEL<72><<<GRID, kPassThreads, SMEM, ST>>>(__VA_ARGS__); break; \
    case 96: KERNEL<96><<<GRID, kPassThreads, SMEM, ST>>>(__VA_ARGS__); break; \
    case 192: KERNEL<192><<<GRID, kPassThreads, SMEM, ST>>>(__VA_ARGS__); break; \
    default: KERNEL<0><<<GRID, kPassThreads, SMEM, ST>>>(__VA_ARGS__); break; \
  }
// Variant 2 (runtime-planned stages) takes KERNEL<0> whatever L is.
#define DNSB_DISPATCH_V(VAR, L, KERNEL, GRID, SMEM, ST, ...)                  \
  do {                                                                      \
    if ((VAR) == 2)                                                         \
      KERNEL<0><<<GRID, kPassThreads, SMEM, ST>>>(__VA_ARGS__);             \
    else                                                                    \
      DNSB_DISPATCH(L, KERNEL, GRID, SMEM, ST, __VA_ARGS__);                \
  } while (0)
#define DNSB_ALL_SIZES(KERNEL)                                                \
  (const void*)KERNEL<0>, (const void*)KERNEL<48>, (const void*)KERNEL<72>,   \
      (const void*)KERNEL<96>, (const void*)KERNEL<192>

FFTPlan make_plan(int L) {
  FFTPlan P{};
  P.L = L;
  P.nst = 0;
  int n = L;
  if (L < 1) return P;
  while (n % 8 == 0 && n != 8 && P.nst < DNSB_MAX_STAGES) {
    P.radix[P.nst++] = 8;
    n /= 8;
  }
  while (n % 4 == 0 && n > 1 && P.nst < DNSB_MAX_STAGES) {
    P.radix[P.nst++] = 4;
    n /= 4;
  }
  while (n % 2 == 0 && n > 1 && P.nst < DNSB_MAX_STAGES) {
    P.radix[P.nst++] = 2;
    n /= 2;
  }
  while (n % 3 == 0 && n > 1 && P.nst < DNSB_MAX_STAGES) {
    P.radix[P.nst++] = 3;
    n /= 3;
  }
  if (n == 8 && P.nst < DNSB_MAX_STAGES) {
    P.radix[P.nst++] = 8;
    n = 1;
  }
  if (n != 1) P.nst = 0;
  return P;
}

// ---------------------------------------------------------------------------
// Generic strided column pass.
// ---------------------------------------------------------------------------
size_t col_pass_smem(int M) {
  return sizeof(double2) * (size_t)(2 * M * kTile + M);
}

template <int ML>
__global__ void __launch_bounds__(kPassThreads)
col_pass_kernel(ColPassArgs a) {
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int C = kTile;
  double2* bufA = sm;
  double2* bufB = sm + M * C;
  double2* tw = sm + 2 * M * C;
  const int i0 = blockIdx.x * C;
  const long long o = blockIdx.y;
  const long long f = blockIdx.z;
  const double2* in = a.in + f * a.in_fs + o * a.in_os + i0;
  double2* out = a.out + f * a.out_fs + o * a.out_os + i0;
  const int ni = min(C, a.nI - i0);
  load_twiddles(tw, a.tw, M);
  if (a.inverse) {
    for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
      const int c = idx % C, t = idx / C;
      const int s = pos_to_stored(t, a.nstored, M);
      double2 v = make_double2(0.0, 0.0);
      if (s >= 0 && c < ni) v = in[s * a.in_ts + c];
      bufA[idx] = v;
    }
  } else {
    for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
      const int c = idx % C, t = idx / C;
      double2 v = make_double2(0.0, 0.0);
      if (c < ni) v = in[t * a.in_ts + c];
      bufA[idx] = v;
    }
  }
  __syncthreads();
  const double2* res = fft_cols<ML, C, kPassThreads>(bufA, bufB, a.plan, a.inverse ? 1 : -1, tw);
  if (a.inverse) {
    for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
      const int c = idx % C, t = idx / C;
      if (c < ni) out[t * a.out_ts + c] = res[idx];
    }
  } else {
    const double sc = 1.0 / M;
    for (int idx = threadIdx.x; idx < a.nstored * C; idx += blockDim.x) {
      const int c = idx % C, s = idx / C;
      const int t = stored_to_pos(s, a.nstored, M);
      if (c < ni) out[s * a.out_ts + c] = cscale(res[t * C + c], sc);
    }
  }
}

// ---------------------------------------------------------------------------
// Column pass, two register stages (M = 8 R1): stage 1 (radix R1, Ns = 1)
// loads its inputs from global memory (zero-padding applied on load),
// stage 2 (radix 8, Ns = R1) stores its outputs to global memory
// (truncation applied on store); one shared buffer in between.
// ---------------------------------------------------------------------------
constexpr int kC2Cols = 16;
constexpr int kC2Threads = 128;

size_t col_pass2_smem(int M) {
  return sizeof(double2) * (size_t)(M * kC2Cols + M);
}

// T: the compute type and the element type of `in` (double, or float for the
// FP32 forms, whose pass buffers hold float2); `out` is complex128, or with
// OUT32 (FP32 only) an FP32 pass buffer.  CURL (inverse): `in` is the FP64
// spectral state and field f of the 6 is u, v, w (f < 3) or the spectral
// curl i (k x u) (triply_periodic.py:122-132), formed in FP64 at the load.
template <int ML, int SIGN, typename T = double, bool OUT32 = false, bool CURL = false,
          bool SLAB = false>
__device__ __forceinline__ void col_pass2_body(const ColPassArgs& a, int bx, int by, int bz) {
  using CT = typename pass_types<T>::C;
  using RT = typename pass_types<T>::R;
  constexpr int M = ML, R1 = M / 8, C = kC2Cols;
  extern __shared__ double2 sm_[];
  CT* X = reinterpret_cast<CT*>(sm_);  // [t][C]
  CT* tw = X + M * C;
  const int tid = threadIdx.x;
  const int i0 = bx * C;
  const long long o = by;
  const long long f = bz;
  const CT* in = reinterpret_cast<const CT*>(a.in) + f * a.in_fs + o * a.in_os + i0;
  // FP64 output, or (OUT32, FP32 arithmetic) an FP32 pass buffer
  double2* out = a.out + f * a.out_fs + o * a.out_os + i0;
  CT* out_c = reinterpret_cast<CT*>(a.out) + f * a.out_fs + o * a.out_os + i0;
  const int ni = min(C, a.nI - i0);
  const unsigned long long drop = l2_drop();
  load_twiddles(tw, reinterpret_cast<const CT*>(a.tw), M);
  __syncthreads();
  for (int it = tid; it < 8 * C; it += kC2Threads) {
    const int c = it % C, j = it / C;
    CT v[R1];
#pragma unroll
    for (int i = 0; i < R1; ++i) {
      const int t = j + 8 * i;
      CT z = cmake<CT>(0, 0);
      if (c < ni) {
        if (SIGN > 0) {
          const int sidx = pos_to_stored(t, a.nstored, M);
          if (sidx >= 0) {
            if constexpr (CURL) {
              // f is the same for the whole CTA: load only the components
              // the field needs
              const double2* st = reinterpret_cast<const double2*>(a.in) + o * a.in_os + i0 +
                                  (long long)sidx * a.in_ts + c;
              const long long fs = a.in_fs;
              double2 q;
              switch (f) {
                case 0: q = st[0]; break;
                case 1: q = st[fs]; break;
                case 2: q = st[2 * fs]; break;
                case 3: {
                  const double2 vv = st[fs], w = st[2 * fs];
                  const double ky = a.ky[sidx], kz = a.kz[o];
                  q = ci(make_double2(ky * w.x - kz * vv.x, ky * w.y - kz * vv.y));
                  break;
                }
                case 4: {
                  const double2 u = st[0], w = st[2 * fs];
                  const double kx = a.kx[i0 + c], kz = a.kz[o];
                  q = ci(make_double2(kz * u.x - kx * w.x, kz * u.y - kx * w.y));
                  break;
                }
                default: {
                  const double2 u = st[0], vv = st[fs];
                  const double kx = a.kx[i0 + c], ky = a.ky[sidx];
                  q = ci(make_double2(kx * vv.x - ky * u.x, kx * vv.y - ky * u.y));
                  break;
                }
              }
              z = to_c(q, (CT*)nullptr);
            } else {
              z = in[sidx * a.in_ts + c];
            }
          }
        } else {
          z = ld_l2(in + t * a.in_ts + c, drop);  // the input's last use
        }
      }
      v[i] = z;
    }
    dft_3p<R1, SIGN>(v, tw, 8);
#pragma unroll
    for (int i = 0; i < R1; ++i) X[(j * R1 + i) * C + c] = v[i];
  }
  __syncthreads();
  const double sc = 1.0 / M;
  for (int it = tid; it < R1 * C; it += kC2Threads) {
    const int c = it % C, k = it / C;
    CT z[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) z[i] = X[(k + R1 * i) * C + c];
#pragma unroll
    for (int i = 1; i < 8; ++i) {
      CT w = tw[i * k];
      if (SIGN > 0) w.y = -w.y;
      z[i] = cmul(z[i], w);
    }
    dft8(z, SIGN);
    if (c < ni) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int t = k + R1 * i;
        if (SIGN > 0) {
          if constexpr (SLAB) {
            // position t belongs to rank t / blk (its padded-z share)
            const int q = t / a.slab.blk;
            a.slab.buf[q][f * a.slab.fs + o * a.out_os + (t - q * a.slab.blk) * a.slab.ts +
                          a.slab.off + i0 + c] = to_d(z[i]);
          } else if (OUT32) {
            out_c[t * a.out_ts + c] = z[i];
          } else {
            out[t * a.out_ts + c] = to_d(z[i]);
          }
        } else {
          const int sidx = pos_to_stored(t, a.nstored, M);
          if (sidx >= 0) {
            if (OUT32) out_c[sidx * a.out_ts + c] = cscale(z[i], (RT)sc);
            else out[sidx * a.out_ts + c] = cscale(to_d(z[i]), sc);
          }
        }
      }
    }
  }
}

// Block (bx, by, bz) = (column tile, outer index, field) of the grid
// ((nI + 15) / 16, nO, nfields); the work-list ensemble kernels call the body
// with their own block numbering.
template <int ML, int SIGN, typename T = double, bool OUT32 = false, bool CURL = false,
          bool SLAB = false>
__global__ void __launch_bounds__(kC2Threads)
col_pass2_kernel(ColPassArgs a) {
  if (a.skip && *a.skip) return;
  col_pass2_body<ML, SIGN, T, OUT32, CURL, SLAB>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// The FP64 pass held to 128 registers, so 4 CTAs fit per SM instead of 3
// (ColPassArgs::occ4: the periodic flows' column passes, measured faster so;
// the Couette z forward measured slower).
template <int ML, int SIGN, bool CURL>
__global__ void __launch_bounds__(kC2Threads, 4)
col_pass2_occ4_kernel(ColPassArgs a) {
  if (a.skip && *a.skip) return;
  col_pass2_body<ML, SIGN, double, false, CURL, false>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

cudaError_t launch_col_pass(const ColPassArgs& a, int nfields, int nO,
                            cudaStream_t st) {
  const int L = a.plan.L;
  if (a.variant == 0 && (L == 48 || L == 72 || L == 96 || L == 192)) {
    dim3 g2((a.nI + kC2Cols - 1) / kC2Cols, nO, nfields);
    const size_t sm2 = a.fp32 ? col_pass2_smem(L) / 2 : col_pass2_smem(L);
    if (a.fp32 && a.inverse && !a.out32) return cudaErrorInvalidValue;
    const bool slab = a.slab.buf[0] != nullptr;
    if (slab && (a.fp32 || a.curl || !a.inverse)) return cudaErrorInvalidValue;
#define DNSB_C2(LL)                                                                     \
  case LL:                                                                              \
    if (slab)                                                                           \
      col_pass2_kernel<LL, 1, double, false, false, true><<<g2, kC2Threads, sm2, st>>>(a); \
    else if (a.curl && a.fp32 == 2)                                                     \
      col_pass2_kernel<LL, 1, fcomp, true, true><<<g2, kC2Threads, sm2, st>>>(a);       \
    else if (a.fp32 == 2 && a.inverse)                                                  \
      col_pass2_kernel<LL, 1, fcomp, true><<<g2, kC2Threads, sm2, st>>>(a);             \
    else if (a.fp32 == 2 && a.out32)                                                    \
      col_pass2_kernel<LL, -1, fcomp, true><<<g2, kC2Threads, sm2, st>>>(a);            \
    else if (a.fp32 == 2)                                                               \
      col_pass2_kernel<LL, -1, fcomp><<<g2, kC2Threads, sm2, st>>>(a);                  \
    else if (a.curl && a.fp32)                                                          \
      col_pass2_kernel<LL, 1, float, true, true><<<g2, kC2Threads, sm2, st>>>(a);       \
    else if (a.occ4 && !a.fp32 && a.curl)                                               \
      col_pass2_occ4_kernel<LL, 1, true><<<g2, kC2Threads, sm2, st>>>(a);               \
    else if (a.occ4 && !a.fp32 && a.inverse)                                            \
      col_pass2_occ4_kernel<LL, 1, false><<<g2, kC2Threads, sm2, st>>>(a);              \
    else if (a.occ4 && !a.fp32)                                                         \
      col_pass2_occ4_kernel<LL, -1, false><<<g2, kC2Threads, sm2, st>>>(a);             \
    else if (a.curl)                                                                    \
      col_pass2_kernel<LL, 1, double, false, true><<<g2, kC2Threads, sm2, st>>>(a);     \
    else if (a.fp32 && a.inverse)                                                       \
      col_pass2_kernel<LL, 1, float, true><<<g2, kC2Threads, sm2, st>>>(a);             \
    else if (a.fp32 && a.out32)                                                         \
      col_pass2_kernel<LL, -1, float, true><<<g2, kC2Threads, sm2, st>>>(a);            \
    else if (a.fp32)                                                                    \
      col_pass2_kernel<LL, -1, float><<<g2, kC2Threads, sm2, st>>>(a);                  \
    else if (a.inverse)                                                                 \
      col_pass2_kernel<LL, 1><<<g2, kC2Threads, sm2, st>>>(a);                          \
    else                                                                                \
      col_pass2_kernel<LL, -1><<<g2, kC2Threads, sm2, st>>>(a);                         \
    break;
    switch (L) { DNSB_C2(48) DNSB_C2(72) DNSB_C2(96) DNSB_C2(192) }
#undef DNSB_C2
    return cudaGetLastError();
  }
  // two-stage compile-time passes only
  if (a.fp32 || a.curl || a.slab.buf[0]) return cudaErrorInvalidValue;
  dim3 grid((a.nI + kTile - 1) / kTile, nO, nfields);
  size_t sm = col_pass_smem(a.plan.L);
  DNSB_DISPATCH_V(a.variant, a.plan.L, col_pass_kernel, grid, sm, st, a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// x pass: two real fields per complex transform (z = a + i b).
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long row_offset(int r, int inner_n,
                                                long long so, long long si) {
  return (long long)(r / inner_n) * so + (long long)(r % inner_n) * si;
}

size_t x_pass_smem(int Mx) {
  return sizeof(double2) * (size_t)(2 * Mx * 3 * kXRows + Mx);
}

template <int ML>
__global__ void __launch_bounds__(kPassThreads)
x_pass_kernel(XPassArgs a) {
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int R = kXRows;
  const int CI = 3 * R;  // inverse columns
  const int CF = 2 * R;  // forward columns
  double2* bufA = sm;
  double2* bufB = sm + M * CI;
  double2* tw = sm + 2 * M * CI;
  const int r0 = blockIdx.x * R;
  const int nr = min(R, a.nrows - r0);
  const int nkx = ML > 0 ? ML / 3 : a.nkx;  // launcher guarantees nx/2 = M/3
  __shared__ long long s_off[kXRows];
  __shared__ int s_y[kXRows];
  if (threadIdx.x < R) {
    const int row = r0 + threadIdx.x;
    const int outer = row / a.inner_n, inner = row % a.inner_n;
    s_off[threadIdx.x] = (long long)outer * a.so + (long long)inner * a.si;
    s_y[threadIdx.x] = a.y_outer ? outer : inner;
  }
  load_twiddles(tw, a.tw, M);
  __syncthreads();
  // Stage the 6 half spectra: stage[(f * nkx + k) * R + r] in bufB.
  double2* stage = bufB;
  const int nload = 6 * nkx * R;
  for (int idx = threadIdx.x; idx < nload; idx += blockDim.x) {
    int r, k, f;
    if (a.rows_fast) {
      r = idx % R;
      k = (idx / R) % nkx;
      f = idx / (R * nkx);
    } else {
      k = idx % nkx;
      r = (idx / nkx) % R;
      f = idx / (R * nkx);
    }
    double2 v = make_double2(0.0, 0.0);
    if (r < nr) v = a.in[f * a.in_fs + s_off[r] + k * a.ks];
    stage[(f * nkx + k) * R + r] = v;
  }
  __syncthreads();
  // Build the 3 complex inputs per row: (u_x,u_y), (u_z,w_x), (w_y,w_z).
  for (int idx = threadIdx.x; idx < M * CI; idx += blockDim.x) {
    const int q = idx % CI, t = idx / CI;
    const int r = q / 3, pr = q % 3;
    const int fa = 2 * pr, fb = 2 * pr + 1;
    double2 z = make_double2(0.0, 0.0);
    if (t == 0) {
      z = make_double2(stage[(fa * nkx) * R + r].x, stage[(fb * nkx) * R + r].x);
    } else if (t < nkx) {
      const double2 A = stage[(fa * nkx + t) * R + r];
      const double2 B = stage[(fb * nkx + t) * R + r];
      z = make_double2(A.x - B.y, A.y + B.x);
    } else if (M - t < nkx) {
      const int k = M - t;
      const double2 A = stage[(fa * nkx + k) * R + r];
      const double2 B = stage[(fb * nkx + k) * R + r];
      z = make_double2(A.x + B.y, -A.y + B.x);
    }
    bufA[idx] = z;
  }
  __syncthreads();
  double2* res = fft_cols<ML, CI, kPassThreads>(bufA, bufB, a.plan, 1, tw);
  double2* nl = (res == bufA) ? bufB : bufA;
  // Rotational nonlinear product at every physical point of the rows.
  for (int idx = threadIdx.x; idx < M * R; idx += blockDim.x) {
    const int r = idx % R, t = idx / R;
    double2 o0 = make_double2(0.0, 0.0), o1 = make_double2(0.0, 0.0);
    if (r < nr) {
      const double2 z0 = res[t * CI + 3 * r + 0];
      const double2 z1 = res[t * CI + 3 * r + 1];
      const double2 z2 = res[t * CI + 3 * r + 2];
      const double u0 = z0.x, u1 = z0.y, u2 = z1.x;
      const double w0 = z1.y, w1 = z2.x, w2 = z2.y;
      const int y = s_y[r];
      const int ny = a.ny_grid;
      const double U0 = a.U[y], U1 = a.U[ny + y], U2 = a.U[2 * ny + y];
      const double C0 = a.cU[y], C1 = a.cU[ny + y], C2 = a.cU[2 * ny + y];
      const double N0 = a.nU[y], N1 = a.nU[ny + y], N2 = a.nU[2 * ny + y];
      // u x w
      const double n0 = u1 * w2 - u2 * w1;
      const double n1 = u2 * w0 - u0 * w2;
      const double n2 = u0 * w1 - u1 * w0;
      // u x curl U + U x w + U x curl U
      const double b0 = (u1 * C2 - u2 * C1) + (U1 * w2 - U2 * w1) + N0;
      const double b1 = (u2 * C0 - u0 * C2) + (U2 * w0 - U0 * w2) + N1;
      const double b2 = (u0 * C1 - u1 * C0) + (U0 * w1 - U1 * w0) + N2;
      o0 = make_double2(n0 + b0, n1 + b1);
      o1 = make_double2(n2 + b2, 0.0);
    }
    nl[t * CF + 2 * r + 0] = o0;
    nl[t * CF + 2 * r + 1] = o1;
  }
  __syncthreads();
  double2* other = (nl == bufA) ? bufB : bufA;
  double2* fres = fft_cols<ML, CF, kPassThreads>(nl, other, a.plan, -1, tw);
  // Unpack the real-field spectra, truncate to nkx, scale 1/M, store.
  const double h = 0.5 / M;
  const int nst = 3 * nkx * R;
  for (int idx = threadIdx.x; idx < nst; idx += blockDim.x) {
    int r, k, f;
    if (a.rows_fast) {
      r = idx % R;
      k = (idx / R) % nkx;
      f = idx / (R * nkx);
    } else {
      k = idx % nkx;
      r = (idx / nkx) % R;
      f = idx / (R * nkx);
    }
    if (r >= nr) continue;
    const int col = 2 * r + (f == 2 ? 1 : 0);
    const double2 Z = fres[k * CF + col];
    const double2 Zm = fres[((M - k) % M) * CF + col];
    double2 v;
    if (f == 1) {
      v = make_double2((Z.y + Zm.y) * h, (Zm.x - Z.x) * h);
    } else {
      v = make_double2((Z.x + Zm.x) * h, (Z.y - Zm.y) * h);
    }
    a.out[f * a.out_fs + s_off[r] + k * a.ks] = v;
  }
}

template <int ML, typename T = double, bool SLAB = false>
__global__ void __launch_bounds__(kX2Threads, std::is_same<T, float>::value ? 8 : 5)
x_pass2_kernel(XPassArgs a);

cudaError_t launch_x_pass(const XPassArgs& a, cudaStream_t st) {
  dim3 grid((a.nrows + kXRows - 1) / kXRows);
  // The compile-time variants assume nx/2 = M/3 (3/2 oversampling).
  const int L = (a.nkx * 3 == a.plan.L) ? a.plan.L : -1;
  const bool slab = a.slab.buf[0] != nullptr;
  if (slab && (a.fp32 || a.variant != 0 || L < 0)) return cudaErrorInvalidValue;
  if (a.variant == 0 && (L == 48 || L == 72 || L == 96 || L == 192)) {
    dim3 g2((a.nrows + kX2Rows - 1) / kX2Rows);
    if (slab) {
      const size_t sm2 = x_pass2_smem(L, a.nkx);
      switch (L) {
        case 48: x_pass2_kernel<48, double, true><<<g2, kX2Threads, sm2, st>>>(a); break;
        case 72: x_pass2_kernel<72, double, true><<<g2, kX2Threads, sm2, st>>>(a); break;
        case 96: x_pass2_kernel<96, double, true><<<g2, kX2Threads, sm2, st>>>(a); break;
        default: x_pass2_kernel<192, double, true><<<g2, kX2Threads, sm2, st>>>(a); break;
      }
      return cudaGetLastError();
    }
    if (a.fp32 == 2) {
      const size_t sm2 = x_pass2_smem(L, a.nkx) / 2;
      switch (L) {
        case 48: x_pass2_kernel<48, fcomp><<<g2, kX2Threads, sm2, st>>>(a); break;
        case 72: x_pass2_kernel<72, fcomp><<<g2, kX2Threads, sm2, st>>>(a); break;
        case 96: x_pass2_kernel<96, fcomp><<<g2, kX2Threads, sm2, st>>>(a); break;
        default: x_pass2_kernel<192, fcomp><<<g2, kX2Threads, sm2, st>>>(a); break;
      }
      return cudaGetLastError();
    }
    if (a.fp32) {
      const size_t sm2 = x_pass2_smem(L, a.nkx) / 2;
      switch (L) {
        case 48: x_pass2_kernel<48, float><<<g2, kX2Threads, sm2, st>>>(a); break;
        case 72: x_pass2_kernel<72, float><<<g2, kX2Threads, sm2, st>>>(a); break;
        case 96: x_pass2_kernel<96, float><<<g2, kX2Threads, sm2, st>>>(a); break;
        default: x_pass2_kernel<192, float><<<g2, kX2Threads, sm2, st>>>(a); break;
      }
      return cudaGetLastError();
    }
    const size_t sm2 = x_pass2_smem(L, a.nkx);
    switch (L) {
      case 48: x_pass2_kernel<48><<<g2, kX2Threads, sm2, st>>>(a); break;
      case 72: x_pass2_kernel<72><<<g2, kX2Threads, sm2, st>>>(a); break;
      case 96: x_pass2_kernel<96><<<g2, kX2Threads, sm2, st>>>(a); break;
      default: x_pass2_kernel<192><<<g2, kX2Threads, sm2, st>>>(a); break;
    }
    return cudaGetLastError();
  }
  if (a.fp32) return cudaErrorInvalidValue;  // two-stage compile-time passes only
  DNSB_DISPATCH_V(a.variant, L, x_pass_kernel, grid, x_pass_smem(a.plan.L), st, a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// x pass, two register stages (M = 8 R1, R1 = M/8 = 3P): inverse radix-R1
// stage straight from the staged half spectra; inverse radix-8 stage, the
// rotational product and the first forward radix-8 stage fused in one
// thread (the 8 positions k + R1 i a radix-8 output holds are the inputs of
// the forward radix-8 stage); forward radix-R1 stage; unpack and store.
// ---------------------------------------------------------------------------
// One work region holds, in turn, the staged half spectra, the inverse
// stage-A output, the forward stage-1 output and the stage-C output: each
// stage reads its input into registers, waits for every thread, then writes
// its output over it.
size_t x_pass2_smem(int M, int nkx) {
  // the stage-B output: M / 8 blocks of 8 * CF + 16 slots (CF = 2 rows x 4)
  const size_t S = (size_t)6 * nkx * kX2Rows, Y = (size_t)(M / 8) * (8 * 2 * kX2Rows + 16);
  const size_t X = (size_t)M * 3 * kX2Rows + 4 * 8;  // + the stage-A skew
  size_t W = S > Y ? S : Y;
  W = W > X ? W : X;
  return sizeof(double2) * (W + M);
}

// T: the compute type and the element type of the pass buffer (double, or
// float for the FP32 form of the Couette RHS).
template <int ML, typename T, bool SLAB = false>
__device__ __forceinline__ void x_pass2_body(const XPassArgs& a, int bx) {
  using CT = typename pass_types<T>::C;
  using RT = typename pass_types<T>::R;
  constexpr int M = ML, R1 = M / 8, R = kX2Rows, NKX = ML / 3;
  constexpr int CI = 3 * R, CF = 2 * R;
  // Shared-memory layouts keep the stages' accesses free of bank conflicts
  // for 16-byte (FP64, 8 lanes per 128-byte wavefront) and 8-byte (FP32, 16
  // lanes) elements alike:
  //  * the stage-A output carries a skew of XS slots per block of R1
  //    positions;
  //  * the stage-B output, position t = 8 k + i, lives in blocks of YB
  //    slots (a multiple of 16, so the banks depend on the skew alone), with
  //    a skew of (k & 1) + 8 ((k >> 1) & 1) slots per block;
  //  * the stage-C output's row t starts at slot 9 t, which the final
  //    unpack reads without conflicts, rows or modes fastest (for 8-byte
  //    elements unpacked rows fastest, rows of CF slots measured faster).
  constexpr int XS = 4;
  constexpr int YB = 8 * CF + 16;
  static_assert(R == 4, "the stage-A lane map assumes 4 rows");
  static_assert(YB % 16 == 0 && YB >= 8 * CF + 10, "stage-B blocks hold their skew");
  constexpr int SZ_S = 6 * NKX * R, SZ_Y = R1 * YB, SZ_X = M * CI + XS * 8;
  static_assert(9 * M <= SZ_X, "the stage-C rows fit the work region");
  // 9 slots per row, except 8-byte elements unpacked rows fastest (CF:
  // 1% faster there); the mapping is fixed per launch
  const int xstride = (sizeof(CT) == 16 || !a.rows_fast) ? 9 : CF;
  auto xrow = [xstride](int t) { return xstride * t; };
  constexpr int SZ_SY = SZ_S > SZ_Y ? SZ_S : SZ_Y;
  constexpr int SZ_W = SZ_SY > SZ_X ? SZ_SY : SZ_X;
  // every stage has at most one item per thread, so a thread can hold its
  // item's inputs in registers across the barrier before the in-place write
  static_assert(8 * CI <= kX2Threads && R1 * R <= kX2Threads && 8 * CF <= kX2Threads,
                "one item per thread in every stage");
  extern __shared__ double2 sm_[];
  CT* sm = reinterpret_cast<CT*>(sm_);
  CT* S = sm;                 // staged half spectra, S[(f*NKX + k)*R + r]
  CT* X = sm;                 // inverse stage-A output [t][CI] (over S); later [t][CF]
  CT* Y = sm;                 // forward stage-1 output [t][CF] (over X)
  CT* tw = sm + SZ_W;
  const CT* gin = reinterpret_cast<const CT*>(a.in);
  const CT* gtw = reinterpret_cast<const CT*>(a.tw);
  CT* gout = reinterpret_cast<CT*>(a.out);
  const int tid = threadIdx.x;
  const int r0 = bx * R;
  const int nr = min(R, a.nrows - r0);
  __shared__ long long s_off[kX2Rows];
  __shared__ long long s_doff[kX2Rows];  // SLAB: the row in the destination layout
  __shared__ int s_y[kX2Rows];
  if (tid < R) {
    const int row = r0 + tid;
    const int outer = row / a.inner_n, inner = row % a.inner_n;
    s_off[tid] = (long long)outer * a.so + (long long)inner * a.si;
    s_y[tid] = a.y_outer ? outer : inner;
    if (SLAB)
      s_doff[tid] = (long long)(outer + a.slab.oo) * a.slab.so +
                    (long long)(inner + a.slab.io) * a.slab.si;
  }
  for (int i = tid; i < M; i += kX2Threads) cp_async_elem(tw + i, gtw + i);
  __syncthreads();
  // The input's last use (evict_first); the output is the next pass's input
  // (evict_last).
  const unsigned long long drop = l2_drop(), keep = l2_keep();
  for (int idx = tid; idx < 6 * NKX * R; idx += kX2Threads) {
    int r, k, f;
    if (a.rows_fast) {
      r = idx % R;
      k = (idx / R) % NKX;
      f = idx / (R * NKX);
    } else {
      k = idx % NKX;
      r = (idx / NKX) % R;
      f = idx / (R * NKX);
    }
    CT* dst = S + (f * NKX + k) * R + r;
    if (r < nr) cp_async_elem_l2(dst, gin + f * a.in_fs + s_off[r] + k * a.ks, drop);
    else *dst = cmake<CT>(0, 0);
  }
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  // Stage A: inverse radix R1 (Ns = 1) on Z = A + iB, built on the fly.
  {
    // lanes of a half warp: 4 rows x 4 values of j, one field pair, where
    // the stage-A output's stride per j (R1 CI + XS slots) spreads the four
    // j over the banks; else (M = 72) 4 rows x 2 values of j x 2 pairs
    constexpr bool J4 = (R1 * CI + XS) % 16 != 0;
    const int it = tid;
    const bool act = it < 8 * CI;
    const int r = it & 3, rest = J4 ? it >> 4 : it >> 3;
    const int pr = rest % 3;
    const int j = J4 ? ((it >> 2) & 3) + 4 * (rest / 3) : ((it >> 2) & 1) + 2 * (rest / 3);
    const int col = 3 * r + pr;
    CT v[R1];
    if (act) {
      const CT* A = S + (2 * pr) * NKX * R + r;
      const CT* B = S + (2 * pr + 1) * NKX * R + r;
#pragma unroll
      for (int i = 0; i < R1; ++i) {
        const int t = j + 8 * i;
        CT z = cmake<CT>(0, 0);
        if (t == 0) {
          z = cmake<CT>(A[0].x, B[0].x);
        } else if (t < NKX) {
          const CT av = A[t * R], bv = B[t * R];
          z = cmake<CT>(av.x - bv.y, av.y + bv.x);
        } else if (M - t < NKX) {
          const CT av = A[(M - t) * R], bv = B[(M - t) * R];
          z = cmake<CT>(av.x + bv.y, -av.y + bv.x);
        }
        v[i] = z;
      }
    }
    __syncthreads();  // S read by every thread before X is written over it
    if (act) {
      dft_3p<R1, 1, CT, true>(v, tw, 8);
#pragma unroll
      for (int i = 0; i < R1; ++i) X[(j * R1 + i) * CI + col + XS * j] = v[i];
    }
  }
  __syncthreads();
  // Stage B: inverse radix 8 (Ns = R1) -> physical values at t = k + R1 i;
  // rotational product there; forward radix-8 stage (Ns = 1) on the same t.
  {
    const int it = tid;
    const bool act = it < R1 * R;
    const int r = it % R, k = it / R;
    CT F0[8], F1[8];
    if (act) {
      CT z[3][8];
#pragma unroll
      for (int pr = 0; pr < 3; ++pr) {
#pragma unroll
        for (int i = 0; i < 8; ++i) z[pr][i] = X[(k + R1 * i) * CI + 3 * r + pr + XS * i];
#pragma unroll
        for (int i = 1; i < 8; ++i) {
          CT w = tw[i * k];
          w.y = -w.y;
          z[pr][i] = cmul(z[pr][i], w);
        }
        dft8(z[pr], 1);
      }
      const bool live = r < nr;
      const int y = s_y[r];
      const int ny = a.ny_grid;
      const RT U0 = live ? (RT)a.U[y] : RT(0), U1 = live ? (RT)a.U[ny + y] : RT(0),
              U2 = live ? (RT)a.U[2 * ny + y] : RT(0);
      const RT C0 = live ? (RT)a.cU[y] : RT(0), C1 = live ? (RT)a.cU[ny + y] : RT(0),
              C2 = live ? (RT)a.cU[2 * ny + y] : RT(0);
      const RT N0 = live ? (RT)a.nU[y] : RT(0), N1 = live ? (RT)a.nU[ny + y] : RT(0),
              N2 = live ? (RT)a.nU[2 * ny + y] : RT(0);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const RT u0 = z[0][i].x, u1 = z[0][i].y, u2 = z[1][i].x;
        const RT w0 = z[1][i].y, w1 = z[2][i].x, w2 = z[2][i].y;
        const RT n0 = u1 * w2 - u2 * w1;
        const RT n1 = u2 * w0 - u0 * w2;
        const RT n2 = u0 * w1 - u1 * w0;
        const RT b0 = (u1 * C2 - u2 * C1) + (U1 * w2 - U2 * w1) + N0;
        const RT b1 = (u2 * C0 - u0 * C2) + (U2 * w0 - U0 * w2) + N1;
        const RT b2 = (u0 * C1 - u1 * C0) + (U0 * w1 - U1 * w0) + N2;
        F0[i] = live ? cmake<CT>(n0 + b0, n1 + b1) : cmake<CT>(0, 0);
        F1[i] = live ? cmake<CT>(n2 + b2, 0) : cmake<CT>(0, 0);
      }
      dft8(F0, -1);
      dft8(F1, -1);
    }
    __syncthreads();  // X read by every thread before Y is written over it
    if (act) {
      CT* yk = Y + k * YB + (k & 1) + 8 * ((k >> 1) & 1);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        yk[i * CF + 2 * r] = F0[i];
        yk[i * CF + 2 * r + 1] = F1[i];
      }
    }
  }
  __syncthreads();
  // Stage C: forward radix R1 (Ns = 8), natural order into X[t][CF].
  {
    const int it = tid;
    const bool act = it < 8 * CF;
    const int col = it % CF, j = it / CF;
    CT v[R1];
    if (act) {
      // position t = j + 8 i is entry j of stage-B block i
#pragma unroll
      for (int i = 0; i < R1; ++i)
        v[i] = Y[i * YB + (i & 1) + 8 * ((i >> 1) & 1) + j * CF + col];
    }
    __syncthreads();  // Y read by every thread before X is written over it
    if (act) {
#pragma unroll
      for (int i = 1; i < R1; ++i) v[i] = cmul(v[i], tw[i * j]);
      dft_3p<R1, -1, CT, true>(v, tw, 8);
#pragma unroll
      for (int i = 0; i < R1; ++i) X[xrow(j + 8 * i) + col] = v[i];
    }
  }
  __syncthreads();
  // Unpack the real-field spectra, truncate to NKX, scale 1/M, store.
  const RT h = (RT)0.5 / M;
  for (int idx = tid; idx < 3 * NKX * R; idx += kX2Threads) {
    int r, k, f;
    if (a.rows_fast) {
      r = idx % R;
      k = (idx / R) % NKX;
      f = idx / (R * NKX);
    } else {
      k = idx % NKX;
      r = (idx / NKX) % R;
      f = idx / (R * NKX);
    }
    if (r >= nr) continue;
    const int col = 2 * r + (f == 2 ? 1 : 0);
    const CT Z = X[xrow(k) + col];
    const CT Zm = X[xrow((M - k) % M) + col];
    CT v;
    if (f == 1) {
      v = cmake<CT>((Z.y + Zm.y) * h, (Zm.x - Z.x) * h);
    } else {
      v = cmake<CT>((Z.x + Zm.x) * h, (Z.y - Zm.y) * h);
    }
    if constexpr (SLAB) {
      // mode k belongs to rank k / blk (its kx share)
      const int q = k / a.slab.blk;
      a.slab.buf[q][f * a.slab.fs + s_doff[r] + (k - q * a.slab.blk) * a.slab.ks] = to_d(v);
    } else {
      st_l2(gout + f * a.out_fs + s_off[r] + k * a.ks, v, keep);
    }
  }
}

template <int ML, typename T, bool SLAB>
__global__ void __launch_bounds__(kX2Threads, std::is_same<T, float>::value ? 8 : 5)
x_pass2_kernel(XPassArgs a) {
  if (a.skip && *a.skip) return;
  x_pass2_body<ML, T, SLAB>(a, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Work-list forms for ensembles (csrc/capi.cu, dnsb_ensemble_*): one launch
// runs the two-stage pass of every member.  Item k covers the member's blocks
// base_k .. base_k + blocks_k - 1 of the flattened grid (bx fastest); every
// CTA walks the virtual blocks blockIdx.x, blockIdx.x + gridDim.x, ... and
// runs the member's body on its block, so each member computes exactly what
// its own launch computes.  Members whose `active` flag is 0 are skipped.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int ens_find(const int* __restrict__ base, int n, int vb) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= vb) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int SIGN, bool CURL>
__global__ void __launch_bounds__(kC2Threads)
ens_col_pass2_kernel(const EnsColItem* __restrict__ items, const int* __restrict__ base, int n,
                     int total, const int* __restrict__ active) {
  __shared__ int s_k;
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    if (threadIdx.x == 0) s_k = ens_find(base, n, vb);
    __syncthreads();
    const int k = s_k;
    const int m = items[k].member;
    if (!active || active[m]) {
      const ColPassArgs a = items[k].a;
      const int local = vb - base[k], gx = items[k].gx, gy = items[k].gy;
      const int bx = local % gx, by = (local / gx) % gy, bz = local / (gx * gy);
      switch (a.plan.L) {
        case 48: col_pass2_body<48, SIGN, double, false, CURL>(a, bx, by, bz); break;
        case 72: col_pass2_body<72, SIGN, double, false, CURL>(a, bx, by, bz); break;
        case 96: col_pass2_body<96, SIGN, double, false, CURL>(a, bx, by, bz); break;
        default: col_pass2_body<192, SIGN, double, false, CURL>(a, bx, by, bz); break;
      }
    }
    __syncthreads();  // shared memory and s_k are reused by the next block
  }
}

__global__ void __launch_bounds__(kX2Threads)
ens_x_pass2_kernel(const EnsXItem* __restrict__ items, const int* __restrict__ base, int n,
                   int total, const int* __restrict__ active) {
  __shared__ int s_k;
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    if (threadIdx.x == 0) s_k = ens_find(base, n, vb);
    __syncthreads();
    const int k = s_k;
    const int m = items[k].member;
    if (!active || active[m]) {
      const XPassArgs a = items[k].a;
      const int bx = vb - base[k];
      switch (a.plan.L) {
        case 48: x_pass2_body<48, double>(a, bx); break;
        case 72: x_pass2_body<72, double>(a, bx); break;
        case 96: x_pass2_body<96, double>(a, bx); break;
        default: x_pass2_body<192, double>(a, bx); break;
      }
    }
    __syncthreads();
  }
}

bool ens_pass_supported(int L) { return L == 48 || L == 72 || L == 96 || L == 192; }

int ens_col_blocks(const ColPassArgs& a, int nO, int nfields, int* gx, int* gy) {
  *gx = (a.nI + kC2Cols - 1) / kC2Cols;
  *gy = nO;
  return *gx * nO * nfields;
}

int ens_x_blocks(const XPassArgs& a) { return (a.nrows + kX2Rows - 1) / kX2Rows; }

size_t ens_col_smem(int maxL) { return col_pass2_smem(maxL); }
size_t ens_x_smem(int maxL, int maxNKX) { return x_pass2_smem(maxL, maxNKX); }

// kind 0: inverse with the curl, 1: inverse, 2: forward (col_pass2); 3: x pass.
static const void* ens_kernel(int kind) {
  switch (kind) {
    case 0: return (const void*)ens_col_pass2_kernel<1, true>;
    case 1: return (const void*)ens_col_pass2_kernel<1, false>;
    case 2: return (const void*)ens_col_pass2_kernel<-1, false>;
    default: return (const void*)ens_x_pass2_kernel;
  }
}

// Persistent grid of a work-list pass kernel: resident CTAs per SM x SMs,
// at most `total`; also raises the kernel's dynamic shared-memory limit.
int ens_pass_grid(int kind, size_t smem, int total, int max_smem) {
  const void* f = ens_kernel(kind);
  if (allow_dynamic_smem(f, max_smem) != cudaSuccess) return 0;
  int per_sm = 0, dev = 0, nsm = 0;
  const int threads = kind == 3 ? kX2Threads : kC2Threads;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, smem) != cudaSuccess)
    return 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  const int g = per_sm * nsm;
  return g < total ? g : total;
}

cudaError_t launch_ens_pass(int kind, const void* items, const int* base, int n, int total,
                            const int* active, int grid, size_t smem, cudaStream_t st) {
  switch (kind) {
    case 0:
      ens_col_pass2_kernel<1, true><<<grid, kC2Threads, smem, st>>>(
          static_cast<const EnsColItem*>(items), base, n, total, active);
      break;
    case 1:
      ens_col_pass2_kernel<1, false><<<grid, kC2Threads, smem, st>>>(
          static_cast<const EnsColItem*>(items), base, n, total, active);
      break;
    case 2:
      ens_col_pass2_kernel<-1, false><<<grid, kC2Threads, smem, st>>>(
          static_cast<const EnsColItem*>(items), base, n, total, active);
      break;
    default:
      ens_x_pass2_kernel<<<grid, kX2Threads, smem, st>>>(static_cast<const EnsXItem*>(items),
                                                          base, n, total, active);
  }
  return cudaGetLastError();
}

// x pass to physical values only (spec_to_phys of 3 fields).
size_t x_phys_smem(int Mx) {
  return sizeof(double2) * (size_t)(2 * Mx * 2 * kXRows + Mx);
}

template <int ML>
__global__ void __launch_bounds__(kPassThreads)
x_phys_kernel(XPhysArgs a) {
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int R = kXRows;
  const int CI = 2 * R;
  double2* bufA = sm;
  double2* bufB = sm + M * CI;
  double2* tw = sm + 2 * M * CI;
  const int r0 = blockIdx.x * R;
  const int nr = min(R, a.nrows - r0);
  const int nkx = a.nkx;
  load_twiddles(tw, a.tw, M);
  double2* stage = bufB;
  for (int idx = threadIdx.x; idx < 3 * nkx * R; idx += blockDim.x) {
    int r, k, f;
    if (a.rows_fast) {
      r = idx % R;
      k = (idx / R) % nkx;
      f = idx / (R * nkx);
    } else {
      k = idx % nkx;
      r = (idx / nkx) % R;
      f = idx / (R * nkx);
    }
    double2 v = make_double2(0.0, 0.0);
    if (r < nr) {
      const long long off = row_offset(r0 + r, a.inner_n, a.so, a.si);
      v = a.in[f * a.in_fs + off + k * a.ks];
    }
    stage[(f * nkx + k) * R + r] = v;
  }
  // Zero partner of the third field lives past the staged block.
  double2* zeros = stage + 3 * nkx * R;
  for (int idx = threadIdx.x; idx < nkx * R; idx += blockDim.x)
    zeros[idx] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int idx = threadIdx.x; idx < M * CI; idx += blockDim.x) {
    const int q = idx % CI, t = idx / CI;
    const int r = q / 2, pr = q % 2;
    const double2* A = stage + ((2 * pr) * nkx) * R + r;
    const double2* B = (pr == 0) ? stage + (1 * nkx) * R + r : zeros + r;
    double2 z = make_double2(0.0, 0.0);
    if (t == 0) {
      z = make_double2(A[0].x, B[0].x);
    } else if (t < nkx) {
      const double2 Av = A[t * R], Bv = B[t * R];
      z = make_double2(Av.x - Bv.y, Av.y + Bv.x);
    } else if (M - t < nkx) {
      const int k = M - t;
      const double2 Av = A[k * R], Bv = B[k * R];
      z = make_double2(Av.x + Bv.y, -Av.y + Bv.x);
    }
    bufA[idx] = z;
  }
  __syncthreads();
  const double2* res = fft_cols<ML, CI, kPassThreads>(bufA, bufB, a.plan, 1, tw);
  for (int idx = threadIdx.x; idx < M * R * 3; idx += blockDim.x) {
    const int t = idx % M;
    const int r = (idx / M) % R;
    const int f = idx / (M * R);
    if (r >= nr) continue;
    const double2 z = res[t * CI + 2 * r + (f == 2 ? 1 : 0)];
    const double v = (f == 1) ? z.y : z.x;
    const long long off = row_offset(r0 + r, a.inner_n, a.pso, a.psi);
    a.out[f * a.out_fs + off + t] = v;
  }
}

cudaError_t launch_x_phys(const XPhysArgs& a, cudaStream_t st) {
  dim3 grid((a.nrows + kXRows - 1) / kXRows);
  DNSB_DISPATCH(a.plan.L, x_phys_kernel, grid, x_phys_smem(a.plan.L), st, a);
  return cudaGetLastError();
}

// Forward x pass from physical values (phys_to_spec of 3 fields): rows of
// real samples at outer*pso + inner*psi -> x half spectra at outer*so +
// inner*si, kx modes ks apart, truncated to nkx, scaled 1/Mx.
template <int ML>
__global__ void __launch_bounds__(kPassThreads)
x_fwd_kernel(XPhysArgs a, const double* phys, double2* spec) {
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int R = kXRows;
  const int CF = 2 * R;
  double2* bufA = sm;
  double2* bufB = sm + M * CF;
  double2* tw = sm + 2 * M * CF;
  const int r0 = blockIdx.x * R;
  const int nr = min(R, a.nrows - r0);
  const int nkx = a.nkx;
  load_twiddles(tw, a.tw, M);
  for (int idx = threadIdx.x; idx < M * CF; idx += blockDim.x) {
    const int t = idx % M;
    const int q = idx / M;
    const int r = q / 2, pr = q % 2;
    double re = 0.0, im = 0.0;
    if (r < nr) {
      const long long off = row_offset(r0 + r, a.inner_n, a.pso, a.psi);
      if (pr == 0) {
        re = phys[0 * a.out_fs + off + t];
        im = phys[1 * a.out_fs + off + t];
      } else {
        re = phys[2 * a.out_fs + off + t];
      }
    }
    bufA[t * CF + q] = make_double2(re, im);
  }
  __syncthreads();
  const double2* fres = fft_cols<ML, CF, kPassThreads>(bufA, bufB, a.plan, -1, tw);
  const double h = 0.5 / M;
  for (int idx = threadIdx.x; idx < 3 * nkx * R; idx += blockDim.x) {
    int r, k, f;
    if (a.rows_fast) {
      r = idx % R;
      k = (idx / R) % nkx;
      f = idx / (R * nkx);
    } else {
      k = idx % nkx;
      r = (idx / nkx) % R;
      f = idx / (R * nkx);
    }
    if (r >= nr) continue;
    const int col = 2 * r + (f == 2 ? 1 : 0);
    const double2 Z = fres[k * CF + col];
    const double2 Zm = fres[((M - k) % M) * CF + col];
    double2 v;
    if (f == 1) {
      v = make_double2((Z.y + Zm.y) * h, (Zm.x - Z.x) * h);
    } else {
      v = make_double2((Z.x + Zm.x) * h, (Z.y - Zm.y) * h);
    }
    const long long off = row_offset(r0 + r, a.inner_n, a.so, a.si);
    spec[f * a.in_fs + off + k * a.ks] = v;
  }
}

size_t x_fwd_smem(int Mx) {
  return sizeof(double2) * (size_t)(2 * Mx * 2 * kXRows + Mx);
}

cudaError_t launch_x_fwd(const XPhysArgs& a, const double* phys, double2* spec,
                         cudaStream_t st) {
  dim3 grid((a.nrows + kXRows - 1) / kXRows);
  DNSB_DISPATCH(a.plan.L, x_fwd_kernel, grid, x_fwd_smem(a.plan.L), st, a, phys, spec);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Periodic first inverse pass (y) with the spectral curl fused.
// ---------------------------------------------------------------------------
// FP32 form: the state columns and the curl stay FP64 (su); the transform
// buffers, twiddles and the output pass buffer are FP32.
size_t yinv_smem(int My, int NY1, int fp32) {
  const size_t cb = fp32 ? sizeof(float2) : sizeof(double2);
  return sizeof(double2) * (size_t)(3 * NY1 * kTile) + cb * (size_t)(2 * My * kTile + My);
}

template <int ML, typename T = double>
__global__ void __launch_bounds__(kPassThreads)
yinv_kernel(YInvArgs a) {
  using CT = typename pass_types<T>::C;
  using RT = typename pass_types<T>::R;
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int C = kTile;
  const int NY1 = a.NY1, NZ1 = a.NZ1, NKX = a.NKX;
  double2* su = sm;                       // [3][NY1][C]
  CT* bufA = reinterpret_cast<CT*>(su + 3 * NY1 * C);
  CT* bufB = bufA + M * C;
  CT* tw = bufB + M * C;
  const int i0 = blockIdx.x * C;
  const int iz = blockIdx.y;
  const int ni = min(C, NKX - i0);
  const long long cs = (long long)NY1 * NZ1 * NKX;
  load_twiddles(tw, reinterpret_cast<const CT*>(a.tw), M);
  for (int idx = threadIdx.x; idx < 3 * NY1 * C; idx += blockDim.x) {
    const int c = idx % C, s = (idx / C) % NY1, comp = idx / (C * NY1);
    double2 v = make_double2(0.0, 0.0);
    if (c < ni) v = a.u[comp * cs + ((long long)s * NZ1 + iz) * NKX + i0 + c];
    su[idx] = v;
  }
  __syncthreads();
  const double kz = a.kz[iz];
  const int nf = a.curl ? 6 : 3;
  const long long fs = (long long)M * NZ1 * NKX;
  for (int f = 0; f < nf; ++f) {
    for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
      const int c = idx % C, t = idx / C;
      const int s = pos_to_stored(t, NY1, M);
      double2 v = make_double2(0.0, 0.0);
      if (s >= 0 && c < ni) {
        const double2 u = su[(0 * NY1 + s) * C + c];
        const double2 vv = su[(1 * NY1 + s) * C + c];
        const double2 w = su[(2 * NY1 + s) * C + c];
        const double kx = a.kx[i0 + c], ky = a.ky[s];
        switch (f) {
          case 0: v = u; break;
          case 1: v = vv; break;
          case 2: v = w; break;
          // curl = 1j * (k x u), triply_periodic.py:122-132
          case 3: v = ci(make_double2(ky * w.x - kz * vv.x, ky * w.y - kz * vv.y)); break;
          case 4: v = ci(make_double2(kz * u.x - kx * w.x, kz * u.y - kx * w.y)); break;
          default: v = ci(make_double2(kx * vv.x - ky * u.x, kx * vv.y - ky * u.y)); break;
        }
      }
      bufA[idx] = to_c(v, (CT*)nullptr);
    }
    __syncthreads();
    const CT* res = fft_cols<ML, C, kPassThreads, CT>(bufA, bufB, a.plan, 1, tw);
    CT* out = reinterpret_cast<CT*>(a.out) + f * fs + (long long)iz * NKX + i0;
    for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
      const int c = idx % C, t = idx / C;
      if (c < ni) out[(long long)t * NZ1 * NKX + c] = res[idx];
    }
    __syncthreads();
  }
}

cudaError_t launch_yinv(const YInvArgs& a, cudaStream_t st) {
  dim3 grid((a.NKX + kTile - 1) / kTile, a.NZ1);
  if (a.fp32 == 2) return cudaErrorInvalidValue;  // compensated: two-stage passes only
  if (a.fp32) {
    const size_t sm = yinv_smem(a.plan.L, a.NY1, 1);
    switch (a.plan.L) {
      case 48: yinv_kernel<48, float><<<grid, kPassThreads, sm, st>>>(a); break;
      case 72: yinv_kernel<72, float><<<grid, kPassThreads, sm, st>>>(a); break;
      case 96: yinv_kernel<96, float><<<grid, kPassThreads, sm, st>>>(a); break;
      case 192: yinv_kernel<192, float><<<grid, kPassThreads, sm, st>>>(a); break;
      default: return cudaErrorInvalidValue;  // compile-time sizes only
    }
    return cudaGetLastError();
  }
  DNSB_DISPATCH_V(a.variant, a.plan.L, yinv_kernel, grid, yinv_smem(a.plan.L, a.NY1, 0), st, a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Periodic last forward pass (y) with the pressure projection fused.
// ---------------------------------------------------------------------------
// FP32 form: the input pass buffer, transform buffers and twiddles are
// FP32; the transformed rows are scaled into FP64 (snl) and the projection
// and the output RHS are FP64.
size_t yfwd_smem(int My, int NY1, int fp32) {
  const size_t cb = fp32 ? sizeof(float2) : sizeof(double2);
  return sizeof(double2) * (size_t)(3 * NY1 * kTile) + cb * (size_t)(2 * My * kTile + My);
}

template <int ML, typename T = double>
__global__ void __launch_bounds__(kPassThreads)
yfwd_kernel(YFwdArgs a) {
  using CT = typename pass_types<T>::C;
  using RT = typename pass_types<T>::R;
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int C = kTile;
  const int NY1 = a.NY1, NZ1 = a.NZ1, NKX = a.NKX;
  double2* snl = sm;  // [3][NY1][C]
  CT* bufA = reinterpret_cast<CT*>(snl + 3 * NY1 * C);
  CT* bufB = bufA + M * C;
  CT* tw = bufB + M * C;
  const int i0 = blockIdx.x * C;
  const int iz = blockIdx.y;
  const int ni = min(C, NKX - i0);
  load_twiddles(tw, reinterpret_cast<const CT*>(a.tw), M);
  const long long fs = (long long)M * NZ1 * NKX;
  const double sc = 1.0 / M;
  for (int f = 0; f < 3; ++f) {
    const CT* in = reinterpret_cast<const CT*>(a.in) + f * fs + (long long)iz * NKX + i0;
    for (int idx = threadIdx.x; idx < M * C; idx += blockDim.x) {
      const int c = idx % C, t = idx / C;
      CT v = cmake<CT>(0, 0);
      if (c < ni) v = in[(long long)t * NZ1 * NKX + c];
      bufA[idx] = v;
    }
    __syncthreads();
    const CT* res = fft_cols<ML, C, kPassThreads, CT>(bufA, bufB, a.plan, -1, tw);
    for (int idx = threadIdx.x; idx < NY1 * C; idx += blockDim.x) {
      const int c = idx % C, s = idx / C;
      const int t = stored_to_pos(s, NY1, M);
      snl[(f * NY1 + s) * C + c] = cscale(to_d(res[t * C + c]), sc);
    }
    __syncthreads();
  }
  const long long cs = (long long)NY1 * NZ1 * NKX;
  const double kz = a.kz[iz];
  for (int idx = threadIdx.x; idx < NY1 * C; idx += blockDim.x) {
    const int c = idx % C, s = idx / C;
    if (c >= ni) continue;
    const double2 n0 = snl[(0 * NY1 + s) * C + c];
    const double2 n1 = snl[(1 * NY1 + s) * C + c];
    const double2 n2 = snl[(2 * NY1 + s) * C + c];
    const long long off = ((long long)s * NZ1 + iz) * NKX + i0 + c;
    double2 r0 = n0, r1 = n1, r2 = n2;
    if (a.project) {
      const double kx = a.kx[i0 + c], ky = a.ky[s];
      // NL - grad(inv_lapl * div NL), monochromatic.py:377-385
      const double2 div = cadd(cadd(cik(kx, n0), cik(ky, n1)), cik(kz, n2));
      const double il = a.inv_lapl[off];
      const double2 p = cscale(div, il);
      r0 = csub(n0, cik(kx, p));
      r1 = csub(n1, cik(ky, p));
      r2 = csub(n2, cik(kz, p));
    }
    a.out[off] = r0;
    a.out[cs + off] = r1;
    a.out[2 * cs + off] = r2;
  }
}

cudaError_t launch_yfwd(const YFwdArgs& a, cudaStream_t st) {
  dim3 grid((a.NKX + kTile - 1) / kTile, a.NZ1);
  if (a.fp32 == 2) return cudaErrorInvalidValue;  // compensated: two-stage passes only
  if (a.fp32) {
    const size_t sm = yfwd_smem(a.plan.L, a.NY1, 1);
    switch (a.plan.L) {
      case 48: yfwd_kernel<48, float><<<grid, kPassThreads, sm, st>>>(a); break;
      case 72: yfwd_kernel<72, float><<<grid, kPassThreads, sm, st>>>(a); break;
      case 96: yfwd_kernel<96, float><<<grid, kPassThreads, sm, st>>>(a); break;
      case 192: yfwd_kernel<192, float><<<grid, kPassThreads, sm, st>>>(a); break;
      default: return cudaErrorInvalidValue;  // compile-time sizes only
    }
    return cudaGetLastError();
  }
  DNSB_DISPATCH_V(a.variant, a.plan.L, yfwd_kernel, grid, yfwd_smem(a.plan.L, a.NY1, 0), st, a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Couette first inverse pass (z) with the FD curl fused.
// ---------------------------------------------------------------------------
size_t zinv_curl_smem(int Mz, int NZ1, int span_max) {
  (void)NZ1;
  (void)span_max;
  return sizeof(double2) * (size_t)(2 * Mz * kZTile + Mz);
}

// D1 along y of column x (complex, stride 1) at row y: sum_m w[m] x[j0 + m].
// Up to kD1Unroll taps are unrolled (predicated), so the loads of several
// rows can be in flight together; wider stencils take the plain loop.
constexpr int kD1Unroll = 9;

__device__ __forceinline__ double2 d1_row(const double2* x, const ZInvCurlArgs& a, int y) {
  const int j0 = a.d1_j0[y];
  const double* w = a.d1_wT + y;  // tap m at w[m * Ny]: consecutive y contiguous
  const int Ny = a.Ny;
  double2 d = make_double2(0.0, 0.0);
  if (a.s1 <= kD1Unroll) {
#pragma unroll
    for (int m = 0; m < kD1Unroll; ++m) {
      if (m < a.s1) {
        const double2 q = x[j0 + m];
        d.x += w[m * Ny] * q.x;
        d.y += w[m * Ny] * q.y;
      }
    }
  } else {
    for (int m = 0; m < a.s1; ++m) {
      const double2 q = x[j0 + m];
      d.x += w[m * Ny] * q.x;
      d.y += w[m * Ny] * q.y;
    }
  }
  return d;
}

// Field F of the z-inverse input at stored z mode s (column base b) and row
// y: 0 u, 1 v, 2 w, 3 dy w - dz v, 4 dz u - dx w, 5 dx v - dy u
// (plane_couette.py:251-271).
template <int F>
__device__ __forceinline__ double2 zinv_field(const ZInvCurlArgs& a, const double2* U,
                                              const double2* V, const double2* Wc,
                                              long long b, int s, int y, double kx) {
  if (F == 0) return U[b + y];
  if (F == 1) return V[b + y];
  if (F == 2) return Wc[b + y];
  const double kz = a.kz[s];
  if (F == 3) return csub(d1_row(Wc + b, a, y), cik(kz, V[b + y]));
  if (F == 4) return csub(cik(kz, U[b + y]), cik(kx, Wc[b + y]));
  return csub(cik(kx, V[b + y]), d1_row(U + b, a, y));
}

// Fill buf[t][c] with field F over the tile.  Every element of a thread is
// computed into registers before any is stored, so the global loads of all
// of a thread's elements are in flight together.
template <int M, int F>
__device__ __forceinline__ void zinv_fill(const ZInvCurlArgs& a, double2* buf,
                                          const double2* U, const double2* V,
                                          const double2* Wc, long long sstride,
                                          int y0, int y1, double kx) {
  constexpr int C = kZTile;
  constexpr int NE = (M * C + kPassThreads - 1) / kPassThreads;
  double2 v[NE];
#pragma unroll
  for (int e = 0; e < NE; ++e) {
    const int idx = threadIdx.x + e * kPassThreads;
    const int c = idx % C, t = idx / C;
    const int s = (idx < M * C) ? pos_to_stored(t, a.NZ1, M) : -1;
    const int y = y0 + c;
    v[e] = make_double2(0.0, 0.0);
    if (s >= 0 && y < y1) v[e] = zinv_field<F>(a, U, V, Wc, s * sstride, s, y, kx);
  }
#pragma unroll
  for (int e = 0; e < NE; ++e) {
    const int idx = threadIdx.x + e * kPassThreads;
    if (idx < M * C) buf[idx] = v[e];
  }
}

// Runtime-length variant of the fill (no compile-time plan).
__device__ __forceinline__ void zinv_fill_rt(const ZInvCurlArgs& a, double2* buf, int M, int f,
                                             const double2* U, const double2* V,
                                             const double2* Wc, long long sstride,
                                             int y0, int y1, double kx) {
  const int C = kZTile;
  for (int idx = threadIdx.x; idx < M * C; idx += kPassThreads) {
    const int c = idx % C, t = idx / C;
    const int s = pos_to_stored(t, a.NZ1, M);
    const int y = y0 + c;
    double2 v = make_double2(0.0, 0.0);
    if (s >= 0 && y < y1) {
      const long long b = s * sstride;
      switch (f) {
        case 0: v = zinv_field<0>(a, U, V, Wc, b, s, y, kx); break;
        case 1: v = zinv_field<1>(a, U, V, Wc, b, s, y, kx); break;
        case 2: v = zinv_field<2>(a, U, V, Wc, b, s, y, kx); break;
        case 3: v = zinv_field<3>(a, U, V, Wc, b, s, y, kx); break;
        case 4: v = zinv_field<4>(a, U, V, Wc, b, s, y, kx); break;
        default: v = zinv_field<5>(a, U, V, Wc, b, s, y, kx); break;
      }
    }
    buf[idx] = v;
  }
}

// Fills read the spectral state straight from global memory (the y-stencil
// neighbours of a tile come from L1/L2), so only the FFT buffers occupy
// shared memory and four CTAs fit per SM.
template <int ML>
__global__ void __launch_bounds__(kPassThreads)
zinv_curl_kernel(ZInvCurlArgs a, int span_max) {
  (void)span_max;
  extern __shared__ double2 sm[];
  const int M = ML > 0 ? ML : a.plan.L;
  const int C = kZTile;
  const int NZ1 = a.NZ1;
  const int NKX = a.NKX, Ny = a.Ny;
  double2* bufA = sm;
  double2* bufB = bufA + M * C;
  double2* tw = bufB + M * C;
  const int y0 = blockIdx.x * C;
  const int ix = blockIdx.y;
  const int y1 = min(y0 + C, Ny);
  const long long cs = (long long)NZ1 * NKX * Ny;
  const double2* U = a.u + (long long)ix * Ny;
  const double2* V = U + cs;
  const double2* Wc = U + 2 * cs;
  const long long sstride = (long long)NKX * Ny;
  load_twiddles(tw, a.tw, M);
  const double kx = a.kx[ix];
  const int nf = a.curl ? 6 : 3;
  const long long fs = (long long)M * NKX * Ny;
  for (int f = 0; f < nf; ++f) {
    if (ML > 0) {
      constexpr int MC = ML > 0 ? ML : 1;
      switch (f) {
        case 0: zinv_fill<MC, 0>(a, bufA, U, V, Wc, sstride, y0, y1, kx); break;
        case 1: zinv_fill<MC, 1>(a, bufA, U, V, Wc, sstride, y0, y1, kx); break;
        case 2: zinv_fill<MC, 2>(a, bufA, U, V, Wc, sstride, y0, y1, kx); break;
        case 3: zinv_fill<MC, 3>(a, bufA, U, V, Wc, sstride, y0, y1, kx); break;
        case 4: zinv_fill<MC, 4>(a, bufA, U, V, Wc, sstride, y0, y1, kx); break;
        default: zinv_fill<MC, 5>(a, bufA, U, V, Wc, sstride, y0, y1, kx); break;
      }
    } else {
      zinv_fill_rt(a, bufA, M, f, U, V, Wc, sstride, y0, y1, kx);
    }
    __syncthreads();
    const double2* res = fft_cols<ML, C, kPassThreads>(bufA, bufB, a.plan, 1, tw);
    double2* out = a.out + f * fs + (long long)ix * Ny + y0;
    for (int idx = threadIdx.x; idx < M * C; idx += kPassThreads) {
      const int c = idx % C, t = idx / C;
      if (y0 + c < y1) out[(long long)t * NKX * Ny + c] = res[idx];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Couette z-inverse pass, two register stages (M = 8 R1): a CTA takes 16
// consecutive (kx, y) columns -- contiguous in the (nz-1, nx/2, ny) layout --
// fills each field's zero-padded z column into shared memory (all of a
// thread's loads of a batch in flight together), runs the inverse radix-R1
// stage in registers, exchanges once through shared memory, and stores the
// inverse radix-8 stage's outputs straight to global memory.
// ---------------------------------------------------------------------------
constexpr int kZ2Cols = 16;
constexpr int kZ2Threads = 8 * kZ2Cols;  // stage 1: one thread per (j, column)

size_t zinv_curl2_smem(int M) {
  return sizeof(double2) * (size_t)(M * kZ2Cols + M);
}

template <int M, int F, typename CT>
__device__ __forceinline__ void zinv2_fill(const ZInvCurlArgs& a, CT* X,
                                           const double2* U, const double2* V,
                                           const double2* Wc, long long sstride,
                                           int y, double kx, bool live) {
  constexpr int NE = M * kZ2Cols / kZ2Threads;  // elements per thread (= M / 8)
  constexpr int B = (NE % 6 == 0) ? 6 : ((NE % 3 == 0) ? 3 : 1);
  const int tid = threadIdx.x;
  for (int e0 = 0; e0 < NE; e0 += B) {
    double2 v[B];
#pragma unroll
    for (int e = 0; e < B; ++e) {
      const int t = (tid + (e0 + e) * kZ2Threads) / kZ2Cols;
      const int s = pos_to_stored(t, a.NZ1, M);
      v[e] = make_double2(0.0, 0.0);
      if (live && s >= 0) v[e] = zinv_field<F>(a, U, V, Wc, s * sstride, s, y, kx);
    }
#pragma unroll
    for (int e = 0; e < B; ++e) X[tid + (e0 + e) * kZ2Threads] = to_c(v[e], (CT*)nullptr);
  }
}

// T: the compute type and the element type of the output pass buffer
// (double, or float for the FP32 form of the Couette RHS); the state is
// read, and the curl's fill computed, in FP64.
template <int ML, typename T = double, bool SLAB = false>
__global__ void __launch_bounds__(kZ2Threads, std::is_same<T, float>::value ? 6 : 4)
zinv_curl2_kernel(ZInvCurlArgs a) {
  if (a.skip && *a.skip) return;
  using CT = typename pass_types<T>::C;
  using RT = typename pass_types<T>::R;
  constexpr int M = ML, R1 = M / 8, C = kZ2Cols;
  extern __shared__ double2 sm_[];
  CT* X = reinterpret_cast<CT*>(sm_);  // [t][C]
  CT* tw = X + M * C;
  const CT* gtw = reinterpret_cast<const CT*>(a.tw);
  CT* gout = reinterpret_cast<CT*>(a.out);
  const int tid = threadIdx.x;
  const int NZ1 = a.NZ1, NKX = a.NKX, Ny = a.Ny;
  const long long ncol = (long long)NKX * Ny;
  const long long q0 = (long long)blockIdx.x * C;
  const int nq = (int)min((long long)C, ncol - q0);
  const long long cs = (long long)NZ1 * ncol;
  for (int i = tid; i < M; i += kZ2Threads) cp_async_elem(tw + i, gtw + i);
  cp_async_commit();
  // The fill column of this thread (the same for all its elements).
  const int cf = tid % C;
  const bool live = cf < nq;
  const long long q = q0 + (live ? cf : 0);
  const int ix = (int)(q / Ny), y = (int)(q % Ny);
  const double kx = a.kx[ix];
  const double2* U = a.u + (long long)ix * Ny;
  const double2* V = U + cs;
  const double2* Wc = U + 2 * cs;
  const int nf = a.curl ? 6 : 3;
  const long long fs = (long long)M * ncol;
  // Half of the pass buffer's lines stay in L2 for the x pass that reads
  // them next (all of them would not fit beside the rest).
  const unsigned long long keep = l2_keep_half();
  // the fields of this CTA: blockIdx.y, blockIdx.y + gridDim.y, ...
  for (int f = blockIdx.y; f < nf; f += gridDim.y) {
    switch (f) {
      case 0: zinv2_fill<M, 0>(a, X, U, V, Wc, ncol, y, kx, live); break;
      case 1: zinv2_fill<M, 1>(a, X, U, V, Wc, ncol, y, kx, live); break;
      case 2: zinv2_fill<M, 2>(a, X, U, V, Wc, ncol, y, kx, live); break;
      case 3: zinv2_fill<M, 3>(a, X, U, V, Wc, ncol, y, kx, live); break;
      case 4: zinv2_fill<M, 4>(a, X, U, V, Wc, ncol, y, kx, live); break;
      default: zinv2_fill<M, 5>(a, X, U, V, Wc, ncol, y, kx, live); break;
    }
    cp_async_wait_all();  // twiddles
    __syncthreads();
    // Stage 1: inverse radix R1 (Ns = 1) on positions t = j + 8 i of column c.
    {
      const int c = tid % C, j = tid / C;
      CT v[R1];
#pragma unroll
      for (int i = 0; i < R1; ++i) v[i] = X[(j + 8 * i) * C + c];
      dft_3p<R1, 1>(v, tw, 8);
      __syncthreads();  // every read done before the in-place writes
#pragma unroll
      for (int i = 0; i < R1; ++i) X[(j * R1 + i) * C + c] = v[i];
    }
    __syncthreads();
    // Stage 2: inverse radix 8 (Ns = R1) -> positions t = k + R1 i.
    for (int it = tid; it < R1 * C; it += kZ2Threads) {
      const int c = it % C, k = it / C;
      CT z[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) z[i] = X[(k + R1 * i) * C + c];
#pragma unroll
      for (int i = 1; i < 8; ++i) {
        CT w = tw[i * k];
        w.y = -w.y;
        z[i] = cmul(z[i], w);
      }
      dft8(z, 1);
      if (c < nq) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          if constexpr (SLAB) {
            // position t belongs to rank t / blk (its padded-z share)
            const int t = k + R1 * i, r = t / a.slab.blk;
            a.slab.buf[r][f * a.slab.fs + (long long)(t - r * a.slab.blk) * a.slab.ts +
                          a.slab.off + q0 + c] = to_d(z[i]);
          } else {
            st_l2(gout + f * fs + (long long)(k + R1 * i) * ncol + q0 + c, z[i], keep);
          }
        }
      }
    }
    __syncthreads();  // X is refilled by the next field
  }
}

cudaError_t launch_zinv_curl(const ZInvCurlArgs& a, int span_max,
                             cudaStream_t st) {
  const int L = a.plan.L;
  const bool slab = a.slab.buf[0] != nullptr;
  const bool fixed = L == 48 || L == 72 || L == 96 || L == 192;
  if (slab && (a.fp32 || a.variant != 0 || !fixed)) return cudaErrorInvalidValue;
  if (a.variant == 0 && fixed) {
    const long long ncol = (long long)a.NKX * a.Ny;
    // one field per CTA along y
    const dim3 grid((unsigned)((ncol + kZ2Cols - 1) / kZ2Cols), a.curl ? 6 : 3);
    if (slab) {
      const size_t sm = zinv_curl2_smem(L);
      switch (L) {
        case 48: zinv_curl2_kernel<48, double, true><<<grid, kZ2Threads, sm, st>>>(a); break;
        case 72: zinv_curl2_kernel<72, double, true><<<grid, kZ2Threads, sm, st>>>(a); break;
        case 96: zinv_curl2_kernel<96, double, true><<<grid, kZ2Threads, sm, st>>>(a); break;
        default: zinv_curl2_kernel<192, double, true><<<grid, kZ2Threads, sm, st>>>(a); break;
      }
      return cudaGetLastError();
    }
    if (a.fp32 == 2) {
      const size_t sm = zinv_curl2_smem(L) / 2;
      switch (L) {
        case 48: zinv_curl2_kernel<48, fcomp><<<grid, kZ2Threads, sm, st>>>(a); break;
        case 72: zinv_curl2_kernel<72, fcomp><<<grid, kZ2Threads, sm, st>>>(a); break;
        case 96: zinv_curl2_kernel<96, fcomp><<<grid, kZ2Threads, sm, st>>>(a); break;
        default: zinv_curl2_kernel<192, fcomp><<<grid, kZ2Threads, sm, st>>>(a); break;
      }
      return cudaGetLastError();
    }
    if (a.fp32) {
      const size_t sm = zinv_curl2_smem(L) / 2;
      switch (L) {
        case 48: zinv_curl2_kernel<48, float><<<grid, kZ2Threads, sm, st>>>(a); break;
        case 72: zinv_curl2_kernel<72, float><<<grid, kZ2Threads, sm, st>>>(a); break;
        case 96: zinv_curl2_kernel<96, float><<<grid, kZ2Threads, sm, st>>>(a); break;
        default: zinv_curl2_kernel<192, float><<<grid, kZ2Threads, sm, st>>>(a); break;
      }
      return cudaGetLastError();
    }
    const size_t sm = zinv_curl2_smem(L);
    switch (L) {
      case 48: zinv_curl2_kernel<48><<<grid, kZ2Threads, sm, st>>>(a); break;
      case 72: zinv_curl2_kernel<72><<<grid, kZ2Threads, sm, st>>>(a); break;
      case 96: zinv_curl2_kernel<96><<<grid, kZ2Threads, sm, st>>>(a); break;
      default: zinv_curl2_kernel<192><<<grid, kZ2Threads, sm, st>>>(a); break;
    }
    return cudaGetLastError();
  }
  if (a.fp32) return cudaErrorInvalidValue;  // two-stage compile-time passes only
  dim3 grid((a.Ny + kZTile - 1) / kZTile, a.NKX);
  DNSB_DISPATCH_V(a.variant, a.plan.L, zinv_curl_kernel, grid,
                  zinv_curl_smem(a.plan.L, a.NZ1, span_max), st, a, span_max);
  return cudaGetLastError();
}

cudaError_t set_pass_attributes(int max_smem) {
  cudaError_t e = cudaSuccess;
  const void* fns[] = {DNSB_ALL_SIZES(col_pass_kernel), DNSB_ALL_SIZES(x_pass_kernel),
                       DNSB_ALL_SIZES(x_phys_kernel), DNSB_ALL_SIZES(x_fwd_kernel),
                       DNSB_ALL_SIZES(yinv_kernel), DNSB_ALL_SIZES(yfwd_kernel),
                       DNSB_ALL_SIZES(zinv_curl_kernel),
                       (const void*)zinv_curl2_kernel<48>, (const void*)zinv_curl2_kernel<72>,
                       (const void*)zinv_curl2_kernel<96>, (const void*)zinv_curl2_kernel<192>,
                       (const void*)zinv_curl2_kernel<48, float>,
                       (const void*)zinv_curl2_kernel<72, float>,
                       (const void*)zinv_curl2_kernel<96, float>,
                       (const void*)zinv_curl2_kernel<192, float>,
                       (const void*)zinv_curl2_kernel<48, double, true>,
                       (const void*)zinv_curl2_kernel<72, double, true>,
                       (const void*)zinv_curl2_kernel<96, double, true>,
                       (const void*)zinv_curl2_kernel<192, double, true>,
                       (const void*)x_pass2_kernel<48, double, true>,
                       (const void*)x_pass2_kernel<72, double, true>,
                       (const void*)x_pass2_kernel<96, double, true>,
                       (const void*)x_pass2_kernel<192, double, true>,
                       (const void*)x_pass2_kernel<48>, (const void*)x_pass2_kernel<72>,
                       (const void*)x_pass2_kernel<96>, (const void*)x_pass2_kernel<192>,
                       (const void*)x_pass2_kernel<48, float>, (const void*)x_pass2_kernel<72, float>,
                       (const void*)x_pass2_kernel<96, float>, (const void*)x_pass2_kernel<192, float>,
                       (const void*)col_pass2_kernel<48, -1, float>,
                       (const void*)col_pass2_kernel<72, -1, float>,
                       (const void*)col_pass2_kernel<96, -1, float>,
                       (const void*)col_pass2_kernel<192, -1, float>,
                       (const void*)col_pass2_kernel<48, 1>, (const void*)col_pass2_kernel<48, -1>,
                       (const void*)col_pass2_kernel<72, 1>, (const void*)col_pass2_kernel<72, -1>,
                       (const void*)col_pass2_kernel<96, 1>, (const void*)col_pass2_kernel<96, -1>,
                       (const void*)col_pass2_kernel<192, 1>, (const void*)col_pass2_kernel<192, -1>,
#define DNSB_OCC4_PASSES(L)                                                         \
  (const void*)col_pass2_occ4_kernel<L, 1, true>,                                   \
      (const void*)col_pass2_occ4_kernel<L, 1, false>,                              \
      (const void*)col_pass2_occ4_kernel<L, -1, false>
                       DNSB_OCC4_PASSES(48), DNSB_OCC4_PASSES(72), DNSB_OCC4_PASSES(96),
                       DNSB_OCC4_PASSES(192),
#undef DNSB_OCC4_PASSES
#define DNSB_F32_PASSES(L)                                                          \
  (const void*)yinv_kernel<L, float>, (const void*)yfwd_kernel<L, float>,           \
      (const void*)col_pass2_kernel<L, 1, float, true>,                             \
      (const void*)col_pass2_kernel<L, -1, float, true>,                            \
      (const void*)col_pass2_kernel<L, 1, float, true, true>,                       \
      (const void*)col_pass2_kernel<L, 1, double, false, true>,                     \
      (const void*)col_pass2_kernel<L, 1, double, false, false, true>
                       DNSB_F32_PASSES(48), DNSB_F32_PASSES(72), DNSB_F32_PASSES(96),
                       DNSB_F32_PASSES(192)};
#undef DNSB_F32_PASSES
  for (const void* f : fns) {
    cudaError_t r = allow_dynamic_smem(f, max_smem);
    if (r != cudaSuccess) e = r;
  }
  return e;
}

}  // namespace dnsb
