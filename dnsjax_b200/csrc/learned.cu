// Learned corrector guess for plane Couette: kernels of a per-(kz, kx)-mode
// MLP with BF16 weights and activations and FP32 accumulation.
//
// The network maps, for every mode, the predictor increment u_p - u^n and
// the previous step's converged correction (3 components x Ny complex
// values each, scaled by the mode's rms of u_p - u^n) plus (kx, kz) to the
// guessed converged correction u^{n+1} - u_p (3 x Ny complex, same scale):
//   h = relu(W1 x + b1),  y = W2 h + b2.
// Training is online on the pairs the solver generates (mean squared error,
// Adam).  The kernels:
//   gemm        C[M][N] = sum_k A(m, k) B(n, k): with both operands
//               K-contiguous, the tcgen05 kernel of csrc/mlp_tc.cu (TMA,
//               TMEM accumulator); operands stored transposed take the
//               mma.sync m16n8k16 BF16 -> FP32 kernels below; epilogue with
//               bias, relu, a relu-derivative mask, FP32 and / or BF16 output
//   features    x and the target from the spectral fields
//   guess       u_p + scale * y
//   loss_grad   dy = 2 (y - t) / M as BF16 and FP32 copies, per-row error
//   colsum      bias gradients (fixed-order two-stage sums, csrc/mlp_tc.cu)
//   adam        FP32 master weights, BF16 copies
#include <cuda_bf16.h>

#include <cmath>
#include <algorithm>
#include <cstdint>

#include "solver.cuh"

namespace dnsb {

namespace {

constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;

__device__ __forceinline__ unsigned pack_bf16(const __nv_bfloat16* p) {
  return *reinterpret_cast<const unsigned*>(p);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4],
                                         const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A(m, k) = TA ? A[k lda + m] : A[m lda + k]; B(n, k) = TB ? B[k ldb + n] :
// B[n ldb + k].  Epilogue per element: v = acc + bias[n]; relu; times
// (mask[m ldm + n] > 0) when mask is given; Cf / Cb at [m ldc + n].
template <bool TA, bool TB>
__global__ void __launch_bounds__(128)
gemm_bf16_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                 const __nv_bfloat16* __restrict__ B, int ldb, const float* __restrict__ bias,
                 int relu, const __nv_bfloat16* __restrict__ mask, int ldm, float* Cf,
                 __nv_bfloat16* Cb, int ldc) {
  __shared__ __align__(16) __nv_bfloat16 As[kBM][kBK + kPad];
  __shared__ __align__(16) __nv_bfloat16 Bs[kBN][kBK + kPad];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  float acc[2][4][4] = {};
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  for (int k0 = 0; k0 < K; k0 += kBK) {
    // tiles: As[i][kk] = A(m0 + i, k0 + kk), Bs[j][kk] = B(n0 + j, k0 + kk)
    for (int e = tid; e < kBM * kBK; e += 128) {
      int i, kk;
      if (TA) {
        i = e % kBM;
        kk = e / kBM;
      } else {
        kk = e % kBK;
        i = e / kBK;
      }
      const int m = m0 + i, k = k0 + kk;
      As[i][kk] = (m < M && k < K) ? (TA ? A[(long long)k * lda + m] : A[(long long)m * lda + k])
                                   : zero;
    }
    for (int e = tid; e < kBN * kBK; e += 128) {
      int j, kk;
      if (TB) {
        j = e % kBN;
        kk = e / kBN;
      } else {
        kk = e % kBK;
        j = e / kBK;
      }
      const int n = n0 + j, k = k0 + kk;
      Bs[j][kk] = (n < N && k < K) ? (TB ? B[(long long)k * ldb + n] : B[(long long)n * ldb + k])
                                   : zero;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kBK; ks += 16) {
      unsigned af[2][4], bf[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const int r = wm * 32 + mt * 16 + g;
        af[mt][0] = pack_bf16(&As[r][ks + 2 * t]);
        af[mt][1] = pack_bf16(&As[r + 8][ks + 2 * t]);
        af[mt][2] = pack_bf16(&As[r][ks + 2 * t + 8]);
        af[mt][3] = pack_bf16(&As[r + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int c = wn * 32 + nt * 8 + g;
        bf[nt][0] = pack_bf16(&Bs[c][ks + 2 * t]);
        bf[nt][1] = pack_bf16(&Bs[c][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], af[mt], bf[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm * 32 + mt * 16 + g + (q >= 2 ? 8 : 0);
        const int n = n0 + wn * 32 + nt * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        float v = acc[mt][nt][q];
        if (bias) v += bias[n];
        if (relu) v = fmaxf(v, 0.0f);
        if (mask && !(__bfloat162float(mask[(long long)m * ldm + n]) > 0.0f)) v = 0.0f;
        if (Cf) Cf[(long long)m * ldc + n] = v;
        if (Cb) Cb[(long long)m * ldc + n] = __float2bfloat16(v);
      }
}

// The same product with 128 x 128 CTA tiles (8 warps of 64 x 32), 16-byte
// operand loads (8 consecutive BF16 along the operand's contiguous index,
// which needs lda, ldb multiples of 8 and 16-byte aligned bases) staged
// through registers one k-tile ahead of the tensor-core loop.
constexpr int kBM2 = 128, kBN2 = 128, kBK2 = 32;

template <bool T_, int ROWS>
struct TileLoad {
  // One k-tile of an operand X(r, k) (r < ROWS tile rows, k < kBK2): two
  // 16-byte chunks per thread.  !T_: X[r ld + k] (k contiguous); T_:
  // X[k ld + r] (r contiguous).
  uint4 v[2];
  int r[2], k[2];
  bool full[2];
  __device__ __forceinline__ void load(const __nv_bfloat16* X, int ld, int R0, int K0, int nR,
                                       int nK) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int c = threadIdx.x + q * 256;
      if (!T_) {
        r[q] = c / (kBK2 / 8);
        k[q] = (c % (kBK2 / 8)) * 8;
      } else {
        // a warp's 32 chunks: 32 different k at one r, so the transposing
        // shared-memory stores of a warp fall in 16 different banks
        k[q] = c % kBK2;
        r[q] = (c / kBK2) * 8;
      }
      const int gr = R0 + r[q], gk = K0 + k[q];
      full[q] = !T_ ? (gr < nR && gk + 8 <= nK) : (gk < nK && gr + 8 <= nR);
      if (full[q]) {
        const __nv_bfloat16* src = !T_ ? X + (long long)gr * ld + gk : X + (long long)gk * ld + gr;
        v[q] = *reinterpret_cast<const uint4*>(src);
      } else {
        // ragged edge: element loads, zero outside the operand
        union {
          uint4 u;
          __nv_bfloat16 h[8];
        } e;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int rr = !T_ ? gr : gr + i, kk = !T_ ? gk + i : gk;
          e.h[i] = (rr < nR && kk < nK)
                       ? (!T_ ? X[(long long)rr * ld + kk] : X[(long long)kk * ld + rr])
                       : __float2bfloat16(0.0f);
        }
        v[q] = e.u;
      }
    }
  }
  __device__ __forceinline__ void store(__nv_bfloat16 (*S)[kBK2 + kPad]) const {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      if (!T_) {
        *reinterpret_cast<uint4*>(&S[r[q]][k[q]]) = v[q];
      } else {
        union {
          uint4 u;
          __nv_bfloat16 h[8];
        } e;
        e.u = v[q];
#pragma unroll
        for (int i = 0; i < 8; ++i) S[r[q] + i][k[q]] = e.h[i];
      }
    }
  }
};

template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
gemm_bf16_v2_kernel(int M, int N, int K, const __nv_bfloat16* __restrict__ A, int lda,
                    const __nv_bfloat16* __restrict__ B, int ldb, const float* __restrict__ bias,
                    int relu, const __nv_bfloat16* __restrict__ mask, int ldm, float* Cf,
                    __nv_bfloat16* Cb, int ldc) {
  __shared__ __align__(16) __nv_bfloat16 As[kBM2][kBK2 + kPad];
  __shared__ __align__(16) __nv_bfloat16 Bs[kBN2][kBK2 + kPad];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps, 64 x 32 each
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.y * kBM2, n0 = blockIdx.x * kBN2;
  float acc[4][4][4] = {};
  const int kb = 0, ke = K;
  TileLoad<TA, kBM2> la;
  TileLoad<TB, kBN2> lb;
  if (kb < ke) {
    la.load(A, lda, m0, kb, M, ke);
    lb.load(B, ldb, n0, kb, N, ke);
  }
  for (int k0 = kb; k0 < ke; k0 += kBK2) {
    la.store(As);
    lb.store(Bs);
    __syncthreads();
    if (k0 + kBK2 < ke) {  // next tile in flight during this one's products
      la.load(A, lda, m0, k0 + kBK2, M, ke);
      lb.load(B, ldb, n0, k0 + kBK2, N, ke);
    }
#pragma unroll
    for (int ks = 0; ks < kBK2; ks += 16) {
      unsigned af[4][4], bf[4][2];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int r = wm * 64 + mt * 16 + g;
        af[mt][0] = pack_bf16(&As[r][ks + 2 * t]);
        af[mt][1] = pack_bf16(&As[r + 8][ks + 2 * t]);
        af[mt][2] = pack_bf16(&As[r][ks + 2 * t + 8]);
        af[mt][3] = pack_bf16(&As[r + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int c = wn * 32 + nt * 8 + g;
        bf[nt][0] = pack_bf16(&Bs[c][ks + 2 * t]);
        bf[nt][1] = pack_bf16(&Bs[c][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], af[mt], bf[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = m0 + wm * 64 + mt * 16 + g + (q >= 2 ? 8 : 0);
        const int n = n0 + wn * 32 + nt * 8 + 2 * t + (q & 1);
        if (m >= M || n >= N) continue;
        float v = acc[mt][nt][q];
        if (bias) v += bias[n];
        if (relu) v = fmaxf(v, 0.0f);
        if (mask && !(__bfloat162float(mask[(long long)m * ldm + n]) > 0.0f)) v = 0.0f;
        if (Cf) Cf[(long long)m * ldc + n] = v;
        if (Cb) Cb[(long long)m * ldc + n] = __float2bfloat16(v);
      }
}

// Feature row of mode m (Couette spectral layout [3][NM][Ny], complex):
//   x[((F * 3 + c) * Ny + y) * 2 + part], F = 0: (u_p - u^n) / s,
//   F = 1: d_prev / s; then kx / kx_max, kz / kz_max;
//   t[(c * Ny + y) * 2 + part] = target / s when target is given;
//   s = rms over the mode of u_p - u^n, at least s_floor (and 1e-30).
__global__ void features_kernel(const double2* __restrict__ un, const double2* __restrict__ up,
                                const double2* __restrict__ dprev,
                                const double2* __restrict__ target,
                                const double* __restrict__ kx, const double* __restrict__ kz,
                                int NKX, int NZ1, int Ny, double kx_max, double kz_max,
                                double s_floor, __nv_bfloat16* X, int ldx, float* T, int ldt,
                                float* scale) {
  const int m = blockIdx.x;
  const int NM = NKX * NZ1;
  const long long CS = (long long)NM * Ny, mo = (long long)m * Ny;
  __shared__ double s_red[32];
  double ss = 0.0;
  for (int e = threadIdx.x; e < 3 * Ny; e += blockDim.x) {
    const int c = e / Ny, y = e % Ny;
    const double2 a = up[c * CS + mo + y], b = un[c * CS + mo + y];
    const double dx = a.x - b.x, dy = a.y - b.y;
    ss += dx * dx + dy * dy;
  }
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_down_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) t += s_red[w];
    s_red[0] = fmax(fmax(sqrt(t / (6.0 * Ny)), s_floor), 1e-30);
  }
  __syncthreads();
  const double s = s_red[0], is = 1.0 / s;
  if (threadIdx.x == 0) scale[m] = (float)s;
  __nv_bfloat16* xr = X + (long long)m * ldx;
  for (int e = threadIdx.x; e < 3 * Ny; e += blockDim.x) {
    const int c = e / Ny, y = e % Ny;
    const long long i = c * CS + mo + y;
    const double2 a = up[i], b = un[i];
    const double2 d = dprev ? dprev[i] : make_double2(0.0, 0.0);
    const int f0 = ((0 * 3 + c) * Ny + y) * 2, f1 = ((1 * 3 + c) * Ny + y) * 2;
    xr[f0] = __double2bfloat16((a.x - b.x) * is);
    xr[f0 + 1] = __double2bfloat16((a.y - b.y) * is);
    xr[f1] = __double2bfloat16(d.x * is);
    xr[f1 + 1] = __double2bfloat16(d.y * is);
    if (target) {
      const double2 q = target[i];
      float* tr = T + (long long)m * ldt + (c * Ny + y) * 2;
      tr[0] = (float)(q.x * is);
      tr[1] = (float)(q.y * is);
    }
  }
  if (threadIdx.x == 0) {
    const int iz = m / NKX, ix = m % NKX;
    xr[12 * Ny] = __double2bfloat16(kx[ix] / kx_max);
    xr[12 * Ny + 1] = __double2bfloat16(kz[iz] / kz_max);
  }
}

// out = up + s_m * y (the guessed prediction), FP64.
__global__ void guess_kernel(const double2* __restrict__ up, const float* __restrict__ Y, int ldy,
                             const float* __restrict__ scale, int NM, int Ny, double2* out) {
  const long long n = 3LL * NM * Ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i / ((long long)NM * Ny));
    const long long r = i % ((long long)NM * Ny);
    const int m = (int)(r / Ny), y = (int)(r % Ny);
    const float* yr = Y + (long long)m * ldy + (c * Ny + y) * 2;
    const double s = scale[m];
    const double2 a = up[i];
    out[i] = make_double2(a.x + s * (double)yr[0], a.y + s * (double)yr[1]);
  }
}

// dy = 2 (y - t) / M (FP32 and BF16); err[m] = sum over the row of (y - t)^2
// and ref[m] = sum of t^2 (so the relative error of the guess is
// sum(err) / sum(ref)).
__global__ void loss_grad_kernel(const float* __restrict__ Y, const float* __restrict__ T,
                                 int M, int N, int ld, float* dYf, __nv_bfloat16* dYb,
                                 float* err, float* ref) {
  const int m = blockIdx.x;
  if (m >= M) return;
  float e = 0.0f, r = 0.0f;
  const float k = 2.0f / (float)M;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const long long i = (long long)m * ld + n;
    const float d = Y[i] - T[i];
    e += d * d;
    r += T[i] * T[i];
    dYf[i] = k * d;
    dYb[i] = __float2bfloat16(k * d);
  }
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, o);
    r += __shfl_down_sync(0xffffffffu, r, o);
  }
  __shared__ float se[32], sr[32];
  if ((threadIdx.x & 31) == 0) {
    se[threadIdx.x >> 5] = e;
    sr[threadIdx.x >> 5] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.0f, b = 0.0f;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) {
      a += se[w];
      b += sr[w];
    }
    err[m] = a;
    ref[m] = b;
  }
}

// Adam on FP32 master weights w with moments mo, ve; BF16 copy wb.
__global__ void adam_kernel(float* w, float* mo, float* ve, const float* __restrict__ grad,
                            __nv_bfloat16* wb, long long n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float m1 = b1 * mo[i] + (1.0f - b1) * gi;
    const float v1 = b2 * ve[i] + (1.0f - b2) * gi * gi;
    mo[i] = m1;
    ve[i] = v1;
    const float wi = w[i] - lr * (m1 / c1) / (sqrtf(v1 / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

}  // namespace

cudaError_t launch_mlp_gemm(int ta, int tb, int M, int N, int K, const void* A, int lda,
                            const void* B, int ldb, const float* bias, int relu,
                            const void* mask, int ldm, float* Cf, void* Cb, int ldc, float* work,
                            long long work_elems, int* status, cudaStream_t st, int* launches) {
  if (!ta && !tb && tc_gemm_supported(A, lda, B, ldb))
    return launch_tc_gemm(M, N, K, A, lda, B, ldb, bias, relu, mask, ldm, Cf, Cb, ldc, work,
                          work_elems, status, st, launches);
  if (launches) *launches = 1;
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* b = static_cast<const __nv_bfloat16*>(B);
  const auto* mk = static_cast<const __nv_bfloat16*>(mask);
  auto* cb = static_cast<__nv_bfloat16*>(Cb);
  const bool vec = lda % 8 == 0 && ldb % 8 == 0 && reinterpret_cast<uintptr_t>(A) % 16 == 0 &&
                   reinterpret_cast<uintptr_t>(B) % 16 == 0;
  if (vec) {
    const dim3 g2((N + kBN2 - 1) / kBN2, (M + kBM2 - 1) / kBM2);
#define DNSB_V2(TA_, TB_)                                                                      \
  gemm_bf16_v2_kernel<TA_, TB_><<<g2, 256, 0, st>>>(M, N, K, a, lda, b, ldb, bias, relu, mk,  \
                                                    ldm, Cf, cb, ldc)
    if (!ta && !tb) DNSB_V2(false, false);
    else if (ta && tb) DNSB_V2(true, true);
    else if (!ta && tb) DNSB_V2(false, true);
    else DNSB_V2(true, false);
#undef DNSB_V2
    return cudaGetLastError();
  }
  const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
  if (!ta && !tb)
    gemm_bf16_kernel<false, false><<<grid, 128, 0, st>>>(M, N, K, a, lda, b, ldb, bias, relu, mk,
                                                         ldm, Cf, cb, ldc);
  else if (ta && tb)
    gemm_bf16_kernel<true, true><<<grid, 128, 0, st>>>(M, N, K, a, lda, b, ldb, bias, relu, mk,
                                                       ldm, Cf, cb, ldc);
  else if (!ta && tb)
    gemm_bf16_kernel<false, true><<<grid, 128, 0, st>>>(M, N, K, a, lda, b, ldb, bias, relu, mk,
                                                        ldm, Cf, cb, ldc);
  else
    gemm_bf16_kernel<true, false><<<grid, 128, 0, st>>>(M, N, K, a, lda, b, ldb, bias, relu, mk,
                                                        ldm, Cf, cb, ldc);
  return cudaGetLastError();
}

cudaError_t launch_learned_features(const double2* un, const double2* up, const double2* dprev,
                                    const double2* target, const double* kx, const double* kz,
                                    int NKX, int NZ1, int Ny, double kx_max, double kz_max,
                                    double s_floor, void* X, int ldx, float* T, int ldt,
                                    float* scale, cudaStream_t st) {
  features_kernel<<<NKX * NZ1, 128, 0, st>>>(un, up, dprev, target, kx, kz, NKX, NZ1, Ny,
                                             kx_max, kz_max, s_floor,
                                             static_cast<__nv_bfloat16*>(X), ldx, T, ldt, scale);
  return cudaGetLastError();
}

cudaError_t launch_learned_guess(const double2* up, const float* Y, int ldy, const float* scale,
                                 int NM, int Ny, double2* out, cudaStream_t st) {
  guess_kernel<<<1184, 256, 0, st>>>(up, Y, ldy, scale, NM, Ny, out);
  return cudaGetLastError();
}

cudaError_t launch_mlp_loss_grad(const float* Y, const float* T, int M, int N, int ld, float* dYf,
                                 void* dYb, float* err, float* ref, cudaStream_t st) {
  loss_grad_kernel<<<M, 256, 0, st>>>(Y, T, M, N, ld, dYf, static_cast<__nv_bfloat16*>(dYb),
                                      err, ref);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* w, float* m, float* v, const float* grad, void* wb,
                            long long n, float lr, float b1, float b2, float eps, int step,
                            cudaStream_t st) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  adam_kernel<<<592, 256, 0, st>>>(w, m, v, grad, static_cast<__nv_bfloat16*>(wb), n, lr, b1,
                                   b2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace dnsb
