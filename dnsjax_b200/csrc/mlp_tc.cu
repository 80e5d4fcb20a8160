// BF16 GEMM of the learned corrector guess on the 5th-generation tensor
// cores (tcgen05), plus the deterministic reductions around it.
//
//   C[m][n] = sum_k A[m][k] B[n][k]        A: M x K, B: N x K, both K-contiguous
//
// A persistent grid (one CTA per SM) walks the 128 x 128 output tiles (or,
// split along K, partial tiles); each CTA runs six warps:
//   warp 0     TMA producer: 128 x 64 tiles of A and B (128-byte swizzle)
//              into a 6-stage shared-memory ring, completing on the stage's
//              "full" mbarrier;
//   warp 1     allocates 256 TMEM columns, two FP32 accumulators; one
//              elected lane issues tcgen05.mma (M 128, N 128, K 16; 4 per
//              stage) into the tile's accumulator, releases each stage with
//              tcgen05.commit on its "empty" mbarrier and commits the tile's
//              "accumulator full" one;
//   warps 2-5  epilogue: tcgen05.ld of their 32 TMEM lanes (rows), bias,
//              relu, relu-derivative mask, FP32 and / or BF16 stores; the
//              accumulator is handed back as soon as it is read, so the
//              next tile's main loop runs under this tile's stores.
// Split along K (gridDim.z > 1) each CTA stores its raw partial tile in a
// caller-given workspace and a second kernel sums the partials in a fixed
// order and applies the epilogue, so results do not depend on scheduling.
//
// Every mbarrier wait is bounded; a wait that gives up sets bit 0 of the
// status word and the CTA still drains its copies and frees its TMEM.
// Operands come from this GPU's memory only (no multicast).
#include <cuda.h>  // CUtensorMap and the encode function's types; the function
                   // itself is fetched at run time (the library does not link libcuda)
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "solver.cuh"

namespace dnsb {

namespace {

constexpr int kTcBM = 128, kTcBN = 128, kTcBK = 64, kTcStages = 6;
constexpr int kTcTileBytes = kTcBM * kTcBK * 2;            // 16 KB per operand tile
constexpr int kTcStageBytes = 2 * kTcTileBytes;            // A + B
constexpr int kTcSmem = kTcStages * kTcStageBytes + 1024;  // + alignment slack
constexpr int kTcThreads = 192;
constexpr int kTcWaitLimit = 1 << 22;

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and B
// BF16 (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at
// bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                              ((uint32_t)(kTcBN >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void bar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void bar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; false (and bit 0 of *status set) if the phase never completed.
__device__ __forceinline__ bool bar_wait(uint64_t* b, uint32_t parity, int* status) {
  for (int it = 0; it < kTcWaitLimit; ++it)
    if (bar_try_wait(b, parity)) return true;
  if (status) atomicOr(status, 1);
  return false;
}

// 2D tiled TMA load (this GPU's memory, no multicast); x = inner (K)
// coordinate, a multiple of 64 elements = 128 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}

// Shared-memory matrix descriptor of a K-major tile with 128-byte swizzle:
// rows of 64 BF16 (128 bytes), 8-row groups 1024 bytes apart (SBO = 64 in
// 16-byte units), LBO = 1 (unused for swizzled K-major), version 1 (bits
// 46-47), layout SWIZZLE_128B = 2 (bits 61-63).  The tile base is 1024-byte
// aligned; advancing K by 16 elements adds 32 bytes to the start address.
__device__ __forceinline__ uint64_t kmajor_sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 32 lanes x 16 columns of 32-bit TMEM cells: this thread's row, columns
// col .. col + 15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32"
      " {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct TcEpilogue {
  const float* bias;
  int relu;
  const __nv_bfloat16* mask;
  int ldm;
  float* Cf;
  __nv_bfloat16* Cb;
  int ldc;
  int vec;  // rows and pointers allow 16-byte vector loads and stores
};

// 16 consecutive outputs n .. n + 15 of row m (n + 16 <= N, 16-byte aligned
// rows and pointers): vector loads of bias and mask, vector stores.
__device__ __forceinline__ void epilogue_store16(const TcEpilogue& e, int m, int n,
                                                 float (&v)[16]) {
  if (e.bias) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 b = *reinterpret_cast<const float4*>(e.bias + n + 4 * q);
      v[4 * q] += b.x;
      v[4 * q + 1] += b.y;
      v[4 * q + 2] += b.z;
      v[4 * q + 3] += b.w;
    }
  }
  if (e.relu) {
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.0f);
  }
  if (e.mask) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      union {
        uint4 u;
        __nv_bfloat16 h[8];
      } mk;
      mk.u = *reinterpret_cast<const uint4*>(e.mask + (long long)m * e.ldm + n + 8 * q);
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (!(__bfloat162float(mk.h[j]) > 0.0f)) v[8 * q + j] = 0.0f;
    }
  }
  if (e.Cf) {
    float4* dst = reinterpret_cast<float4*>(e.Cf + (long long)m * e.ldc + n);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
  if (e.Cb) {
    uint4* dst = reinterpret_cast<uint4*>(e.Cb + (long long)m * e.ldc + n);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      union {
        uint4 u;
        __nv_bfloat162 h[4];
      } o;
#pragma unroll
      for (int j = 0; j < 4; ++j) o.h[j] = __floats2bfloat162_rn(v[8 * q + 2 * j], v[8 * q + 2 * j + 1]);
      dst[q] = o.u;
    }
  }
}

__device__ __forceinline__ void epilogue_store(const TcEpilogue& e, int m, int n, float v) {
  if (e.bias) v += e.bias[n];
  if (e.relu) v = fmaxf(v, 0.0f);
  if (e.mask && !(__bfloat162float(e.mask[(long long)m * e.ldm + n]) > 0.0f)) v = 0.0f;
  if (e.Cf) e.Cf[(long long)m * e.ldc + n] = v;
  if (e.Cb) e.Cb[(long long)m * e.ldc + n] = __float2bfloat16(v);
}

__device__ __forceinline__ void bar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}

// Persistent form: CTA c takes the work units c, c + gridDim.x, ...; unit u
// is output tile u / splits, K split u % splits (kps k-blocks of 64 each).
// The k-block stream of all its units runs through the 6-stage ring without
// a break, and the accumulator alternates between two 128-column halves of
// TMEM, so the epilogue of one unit runs under the main loop of the next:
//   acc_full[b]   MMA -> epilogue: the unit in half b is complete
//   acc_empty[b]  epilogue -> MMA: half b has been read (one arrive per
//                 epilogue warp)
// work: splits partial tiles of M x N (row stride N) when splits > 1.
__global__ void __launch_bounds__(kTcThreads, 1)
gemm_tn_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                  int M, int N, int K, int kps, int splits, TcEpilogue ep, float* work,
                  int* status) {
  extern __shared__ uint8_t tc_smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kTcStages];
  __shared__ __align__(8) uint64_t empty_bar[kTcStages];
  __shared__ __align__(8) uint64_t acc_full[2];
  __shared__ __align__(8) uint64_t acc_empty[2];
  __shared__ uint32_t tmem_slot;

  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntn = (N + kTcBN - 1) / kTcBN, ntm = (M + kTcBM - 1) / kTcBM;
  const int nunits = ntm * ntn * splits;
  const int nkb = (K + kTcBK - 1) / kTcBK;
  auto unit_k = [&](int u, int* kb0) {
    *kb0 = (u % splits) * kps;
    return max(0, min(nkb, *kb0 + kps) - *kb0);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      bar_init(&full_bar[s], 1);
      bar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      bar_init(&acc_full[b], 1);
      bar_init(&acc_empty[b], 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(&tmem_slot)),
                 "r"(2 * kTcBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // producer: the k-blocks of every unit of this CTA, one stream
      int g = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        const int tile = u / splits;
        const int m0 = (tile / ntn) * kTcBM, n0 = (tile % ntn) * kTcBN;
        int kb0;
        const int nk = unit_k(u, &kb0);
        for (int i = 0; i < nk; ++i, ++g) {
          const int s = g % kTcStages;
          if (g >= kTcStages) ok = bar_wait(&empty_bar[s], ((g / kTcStages) - 1) & 1, status);
          if (!ok) break;
          uint8_t* sa = smem + s * kTcStageBytes;
          bar_expect_tx(&full_bar[s], kTcStageBytes);
          const int kx = (kb0 + i) * kTcBK;
          tma_load_2d(sa, &mapA, kx, m0, &full_bar[s]);
          tma_load_2d(sa + kTcTileBytes, &mapB, kx, n0, &full_bar[s]);
        }
      }
      // drain: every issued copy has landed before the CTA can exit
      for (int h = max(0, g - kTcStages); h < g; ++h)
        bar_wait(&full_bar[h % kTcStages], (h / kTcStages) & 1, status);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      int g = 0, j = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x, ++j) {
        const int b = j & 1;
        if (j >= 2) ok = bar_wait(&acc_empty[b], ((j >> 1) - 1) & 1, status);
        if (!ok) break;
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(b * kTcBN);
        int kb0;
        const int nk = unit_k(u, &kb0);
        for (int i = 0; i < nk && ok; ++i, ++g) {
          const int s = g % kTcStages;
          ok = bar_wait(&full_bar[s], (g / kTcStages) & 1, status);
          if (!ok) break;
          tc_fence_after();
          const uint32_t sa = su32(smem + s * kTcStageBytes);
          const uint32_t sb = sa + kTcTileBytes;
#pragma unroll
          for (int kk = 0; kk < kTcBK / 16; ++kk)
            tc_mma(acc, kmajor_sw128_desc(sa + kk * 32), kmajor_sw128_desc(sb + kk * 32),
                   (i > 0 || kk > 0) ? 1u : 0u);
          tc_commit(&empty_bar[s]);
        }
        if (ok) tc_commit(&acc_full[b]);
      }
    }
  } else {
    // epilogue: warps 2..5 own TMEM lanes 32 (warp % 4) .. + 31
    const int q = warp & 3;
    int j = 0;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x, ++j) {
      const int b = j & 1;
      bool ok = bar_wait(&acc_full[b], (j >> 1) & 1, status);
      ok = __all_sync(0xffffffffu, ok);  // the TMEM loads below are warp-collective
      if (!ok) break;
      tc_fence_after();
      const int tile = u / splits;
      const int m0 = (tile / ntn) * kTcBM, n0 = (tile % ntn) * kTcBN;
      const int m = m0 + q * 32 + lane;
      const bool split = splits > 1;
      float* part = split ? work + (long long)(u % splits) * M * N : nullptr;
      const bool pvec = (N % 4) == 0;
#pragma unroll 1
      for (int c0 = 0; c0 < kTcBN; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcBN + c0), v);
        if (c0 + 16 == kTcBN) {
          // the half is read: hand it back to the MMA warp
          tc_fence_before();
          __syncwarp();
          if (lane == 0) bar_arrive(&acc_empty[b]);
        }
        const int nb = n0 + c0;
        if (m < M && nb < N) {
          if (split && pvec && nb + 16 <= N) {
            float4* dst = reinterpret_cast<float4*>(part + (long long)m * N + nb);
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
              dst[jj] = make_float4(v[4 * jj], v[4 * jj + 1], v[4 * jj + 2], v[4 * jj + 3]);
          } else if (!split && ep.vec && nb + 16 <= N) {
            epilogue_store16(ep, m, nb, v);
          } else {
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
              const int n = nb + jj;
              if (n < N) {
                if (split)
                  part[(long long)m * N + n] = v[jj];
                else
                  epilogue_store(ep, m, n, v[jj]);
              }
            }
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * kTcBN)
                 : "memory");
  }
}

// Sum of the split partial tiles in the order z = 0, 1, ..., then the epilogue.
__global__ void split_reduce_kernel(const float* __restrict__ work, int splits, int M, int N,
                                    TcEpilogue ep) {
  const long long total = (long long)M * N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += work[z * total + i];
    epilogue_store(ep, (int)(i / N), (int)(i % N), s);
  }
}

// out[c][r] = in[r][c] (BF16), 32 x 32 tiles through shared memory.
__global__ void transpose_bf16_kernel(const __nv_bfloat16* __restrict__ in, int R, int Cn, int ldi,
                                      __nv_bfloat16* __restrict__ out, int ldo) {
  __shared__ __nv_bfloat16 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    if (r < R && c < Cn) t[j][threadIdx.x] = in[(long long)r * ldi + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (r < R && c < Cn) out[(long long)c * ldo + r] = t[threadIdx.x][j];
  }
}

// Column sums in two fixed-order stages: partial[g][n] = sum over rows
// m = g, g + G, ... (stage 1), out[n] = sum_g partial[g][n] (stage 2).
template <typename T>
__global__ void colsum_partial_kernel(const T* __restrict__ A, int M, int N, int lda,
                                      float* __restrict__ partial) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = blockIdx.y; m < M; m += gridDim.y) {
    if constexpr (sizeof(T) == 4)
      s += A[(long long)m * lda + n];
    else
      s += __bfloat162float(A[(long long)m * lda + n]);
  }
  partial[(long long)blockIdx.y * N + n] = s;
}

__global__ void colsum_final_kernel(const float* __restrict__ partial, int G, int N,
                                    float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int g = 0; g < G; ++g) s += partial[(long long)g * N + n];
  out[n] = s;
}

// ---- host side ------------------------------------------------------------

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault,
                                         &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  });
  return fn;
}

// rows x cols BF16 matrix, row stride ld elements; 64 x 128 (cols x rows) box.
bool make_map(CUtensorMap* map, const void* base, int rows, int cols, int ld) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {kTcBK, kTcBM};
  const cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool tc_gemm_supported(const void* A, int lda, const void* B, int ldb) {
  return encode_fn() != nullptr && lda % 8 == 0 && ldb % 8 == 0 &&
         reinterpret_cast<uintptr_t>(A) % 16 == 0 && reinterpret_cast<uintptr_t>(B) % 16 == 0;
}

cudaError_t launch_tc_gemm(int M, int N, int K, const void* A, int lda, const void* B, int ldb,
                           const float* bias, int relu, const void* mask, int ldm, float* Cf,
                           void* Cb, int ldc, float* work, long long work_elems, int* status,
                           cudaStream_t st, int* launches) {
  static std::once_flag attr_once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once, [] {
    attr_err = cudaFuncSetAttribute(gemm_tn_tc_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
  });
  if (attr_err != cudaSuccess) return attr_err;
  CUtensorMap ma, mb;
  if (!make_map(&ma, A, M, K, lda) || !make_map(&mb, B, N, K, ldb)) return cudaErrorInvalidValue;
  auto al16 = [](const void* q) { return reinterpret_cast<uintptr_t>(q) % 16 == 0; };
  const int vec = ldc % 8 == 0 && al16(Cf) && al16(Cb) && al16(bias) &&
                  (!mask || (ldm % 8 == 0 && al16(mask)));
  TcEpilogue ep{bias, relu, static_cast<const __nv_bfloat16*>(mask), ldm, Cf,
                static_cast<__nv_bfloat16*>(Cb), ldc, vec};
  const int nkb = (K + kTcBK - 1) / kTcBK;
  const int tiles = ((N + kTcBN - 1) / kTcBN) * ((M + kTcBM - 1) / kTcBM);
  // split K when the tiles cannot fill the GPU: about one CTA per SM, at
  // least 8 k-blocks per split, within the workspace
  int splits = 1;
  if (work && tiles < 148) {
    splits = std::max(1, std::min(148 / tiles, nkb / 8));
    const long long per = (long long)M * N;
    splits = (int)std::max(1LL, std::min<long long>(splits, work_elems / std::max(1LL, per)));
  }
  const int kps = (nkb + splits - 1) / splits;
  splits = (nkb + kps - 1) / kps;  // every split has at least one k-block
  // one persistent CTA per SM (the ring takes most of its shared memory)
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      nsm = 148;
  }
  const int units = tiles * splits;
  const int grid = units < nsm ? units : nsm;
  gemm_tn_tc_kernel<<<grid, kTcThreads, kTcSmem, st>>>(ma, mb, M, N, K, kps, splits, ep, work,
                                                       status);
  cudaError_t e = cudaGetLastError();
  if (launches) *launches = 1;
  if (e != cudaSuccess || splits == 1) return e;
  split_reduce_kernel<<<592, 256, 0, st>>>(work, splits, M, N, ep);
  if (launches) *launches = 2;
  return cudaGetLastError();
}

cudaError_t launch_bf16_transpose(const void* in, int R, int C, int ldi, void* out, int ldo,
                                  cudaStream_t st) {
  const dim3 grid((C + 31) / 32, (R + 31) / 32);
  transpose_bf16_kernel<<<grid, dim3(32, 8), 0, st>>>(static_cast<const __nv_bfloat16*>(in), R, C,
                                                      ldi, static_cast<__nv_bfloat16*>(out), ldo);
  return cudaGetLastError();
}

int colsum_groups(int M) { return std::max(1, std::min(M, 128)); }

cudaError_t launch_colsum_det(const void* A, int bf16, int M, int N, int lda, float* out,
                              float* work, cudaStream_t st) {
  const int G = colsum_groups(M);
  const dim3 grid((N + 127) / 128, G);
  if (bf16)
    colsum_partial_kernel<__nv_bfloat16><<<grid, 128, 0, st>>>(
        static_cast<const __nv_bfloat16*>(A), M, N, lda, work);
  else
    colsum_partial_kernel<float><<<grid, 128, 0, st>>>(static_cast<const float*>(A), M, N, lda,
                                                       work);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  colsum_final_kernel<<<(N + 127) / 128, 128, 0, st>>>(work, G, N, out);
  return cudaGetLastError();
}

}  // namespace dnsb
