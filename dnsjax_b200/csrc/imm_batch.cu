// Plane Couette influence-matrix iteration as five bandwidth-shaped kernels.
//
// Follows src/dnsjax/flows/plane_couette.py:376-504 (six stages) and the
// dgbtrs-'N' substitution of src/dnsjax/geometries/cartesian.py:360-441.
//
//   stages 0-1   one warp per (kz, kx) mode: d_hat = div u^n, then f_hat
//   (+ 3)        (D1 / D2 along y from shared memory) -> F      [NM][Ny],
//                and in the same pass the part of stage 3 that does not
//                need p_P, Q = H_k^- u^n + c N_j + (1-c) N_n -> R [3][NM][Ny]
//   L_k solve    p_P = L_k^-1 f_hat in place in F: a CTA per 16 items, one
//                warp per component, lane = side * 16 + item (side 1 is the
//                mirror mode (nz-1-s, kx) of item (s, kx) when it shares the
//                item's factors), each lane one complex column
//   stage 3      one warp per mode: R = Q - grad p_P (interior rows)
//   H_k solve    as the L_k solve, three components, in place in R
//   stages 4-6   one warp per mode: wall divergence, influence-matrix
//                weights, u^{j+1}, the correction and its Simpson norm
//
// The LU factors are repacked once, when the operators are bound, into
// 16-item tiles whose rows are contiguous (layout below), so a block of
// substitution steps of one tile is one bulk copy into shared memory; the
// substitution kernels stream those blocks through a ring of slots, each
// lane fetching its own entering rows with cp.async.
// An item is mode (s, kx) with s <= (nz-1)/2; when the factors of (s, kx)
// and its mirror (nz-1-s, kx) are bit-identical (same k^2; checked at bind
// time) the mirror reads the item's records, else every mode is an item.
#include "solver.cuh"

namespace dnsb {

namespace {

constexpr int kTile = 16;       // items per substitution CTA (two sides per item)
constexpr int kStageWarps = 4;  // modes per CTA in the stage kernels
constexpr int kSYM = 5;         // y values per lane: y = lane + 32 k, Ny <= 160

// L2 residency of the workspaces F and R (K Ny and 3 K Ny complex, 67 MB at
// 128x129x128, each touched about three times per call): their writes and
// the substitutions' accesses carry an evict_last policy, and their last
// reads (F in the gradient kernel, R in stage 6) evict_first, so the streamed
// inputs do not push them out of the 126 MB L2 between the kernels of one call
// (l2_keep / l2_drop and the hinted accesses are in common.cuh).

// Banded stencil row y applied to x: sum_m w[m][y] x[j0[y] + m], with the
// weights stored tap-major ([S][Ny]) so the lanes of a warp (consecutive y)
// read each tap's weights contiguously.
template <int S>
__device__ __forceinline__ double2 band_row(const double2* x, const int* __restrict__ j0,
                                            const double* __restrict__ wT, int Ny, int y) {
  const int j = j0[y];
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const double wm = wT[m * Ny + y];
    const double2 v = x[j + m];
    acc.x += wm * v.x;
    acc.y += wm * v.y;
  }
  return acc;
}

}  // namespace

// ---------------------------------------------------------------------------
// Bind time: repack one operator's factors into 16-item tiles, each tile's
// rows contiguous so a block of substitution steps is one contiguous copy:
//   facL[tile][j][i/2][16][2]       (rows j < Ny, then W zero rows)  L
//                                   multipliers of rows j+1..j+kl
//   facU[tile][j + WB][i/2][16][2]  (WB zero rows first; NUP = NU+1 rounded
//                                   up to even) i = 0: 1/U_jj, i > 0:
//                                   U_{j-i,j} / U_jj
//   dp[tile][j][16]            ipiv[j] - j, validated (a bad pivot is flagged
//                              and replaced by 0)
// Item p is mode p (modes (s, kx) with s <= (nz-1)/2 when mirrors share
// factors).  The arrays must be zeroed before the call (padding rows and
// items).
// ---------------------------------------------------------------------------
__global__ void imm_repack_kernel(const double* __restrict__ ab, const int* __restrict__ piv,
                                  int Ny, int kl, int nu, int row0, int NP, int ntiles,
                                  double* facL, double* facU, unsigned char* dp, int* status) {
  const int rows = 3 * kl + 1, kuu = 2 * kl, W = kl + 1, WB = nu + 1;
  const int nup = (nu + 2) & ~1;  // U record length, even
  const long long NyF = Ny + W, NyB = Ny + WB;
  const long long n = (long long)NP * Ny;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(idx % NP), j = (int)(idx / NP);
    const int tile = p / kTile, it = p % kTile;
    const double* abm = ab + (long long)p * rows * Ny;
    const double r = 1.0 / abm[(long long)kuu * Ny + j];
    // element i of row j: [tile][j][i / 2][it][i % 2]
    double* L = facL + (tile * NyF + j) * kl * kTile + 2 * it;
    for (int i = 1; i <= kl; ++i) {
      const int e = i - 1;
      L[(e >> 1) * 2 * kTile + (e & 1)] = abm[(long long)(kuu + i) * Ny + j];
    }
    double* U = facU + (tile * NyB + j + WB) * nup * kTile + 2 * it;
    U[0] = r;
    for (int i = 1; i <= nu; ++i) {
      const int row = kuu - i;
      const double u = (row >= row0) ? abm[(long long)row * Ny + j] : 0.0;
      U[(i >> 1) * 2 * kTile + (i & 1)] = u * r;
    }
    int d = piv[(long long)p * Ny + j] - j;
    if (d < 0 || d > kl || j + d >= Ny) {  // never follow a bad pivot
      atomicOr(status, 1);
      d = 0;
    }
    dp[(tile * NyF + j) * kTile + it] = (unsigned char)d;
  }
  (void)ntiles;
}

cudaError_t launch_imm_repack(const double* ab, const int* piv, int Ny, int kl, int nu,
                              int row0, int NP, int ntiles, double* facL, double* facU,
                              unsigned char* dp, int* status, cudaStream_t st) {
  imm_repack_kernel<<<592, 256, 0, st>>>(ab, piv, Ny, kl, nu, row0, NP, ntiles, facL, facU,
                                         dp, status);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Stages 0-1 and the pressure-free part of stage 3, in one pass over the
// inputs: f_hat -> F, and Q = H_k^- u^n + c N_j + (1-c) N_n -> R (wall rows
// zero), so u^n, N_j and N_n are read once per call.
// ---------------------------------------------------------------------------
template <int KL>
__global__ void __launch_bounds__(32 * kStageWarps)
imm_stage013_kernel(ImmArgs a, const double2* __restrict__ vel_n,
                    const double2* __restrict__ nl_n, const double2* __restrict__ nl_j,
                    double2* __restrict__ F, double2* __restrict__ R) {
  if (a.skip && *a.skip) return;
  constexpr int S1 = KL + 1, S2 = KL + 2, YM = kSYM;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int NKX = a.NKX, Ny = a.Ny, NM = a.NZ1 * a.NKX;
  const int m = blockIdx.x * kStageWarps + wq;
  if (m >= NM) return;  // no CTA-wide barrier below
  double2* T = sm + wq * 6 * Ny;  // u^n, v^n, w^n, N^j_v, N^n_v, d_hat^n
  double2* D = T + 5 * Ny;
  const long long CS = (long long)NM * Ny, mo = (long long)m * Ny;
  for (int y = lane; y < Ny; y += 32) {
    cp_async16(T + y, vel_n + mo + y);
    cp_async16(T + Ny + y, vel_n + CS + mo + y);
    cp_async16(T + 2 * Ny + y, vel_n + 2 * CS + mo + y);
    cp_async16(T + 3 * Ny + y, nl_j + CS + mo + y);
    cp_async16(T + 4 * Ny + y, nl_n + CS + mo + y);
  }
  cp_async_commit();
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  const double c = a.c, dt = a.dt, omc = 1.0 - c, omc_nu = omc * a.nu, idt = 1.0 / dt;
  const unsigned long long keep = l2_keep();
  double2 nj[3][YM], nn[3][YM];
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny) {
#pragma unroll
      for (int cpt = 0; cpt < 3; ++cpt) {
        nj[cpt][k] = nl_j[cpt * CS + mo + y];
        nn[cpt][k] = nl_n[cpt * CS + mo + y];
      }
    }
  }
  cp_async_wait_all();
  __syncwarp();
  // Stage 0: d_hat^n = div u^n
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny)
      D[y] = cadd(cadd(cik(kx, T[y]), band_row<S1>(T + Ny, a.d1_j0, a.d1_wT, Ny, y)),
                  cik(kz, T[2 * Ny + y]));
  }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y >= Ny) continue;
    double2 fy = make_double2(0.0, 0.0), qu = fy, qv = fy, qw = fy;
    if (y > 0 && y < Ny - 1) {
      // Stage 1: f_hat
      const double2 divNj = cadd(cadd(cik(kx, nj[0][k]),
                                      band_row<S1>(T + 3 * Ny, a.d1_j0, a.d1_wT, Ny, y)),
                                 cik(kz, nj[2][k]));
      const double2 divNn = cadd(cadd(cik(kx, nn[0][k]),
                                      band_row<S1>(T + 4 * Ny, a.d1_j0, a.d1_wT, Ny, y)),
                                 cik(kz, nn[2][k]));
      const double2 dy = D[y];
      const double2 Lkd = csub(band_row<S2>(D, a.d2_j0, a.d2_wT, Ny, y), cscale(dy, k2));
      const double2 dd = make_double2(dy.x / dt, dy.y / dt);
      fy = cadd(cadd(cadd(dd, cscale(divNj, c)), cscale(divNn, omc)), cscale(Lkd, omc_nu));
      // Stage 3 without the pressure gradient
      const double2 u = T[y], v = T[Ny + y], w = T[2 * Ny + y];
      const double2 D2u = band_row<S2>(T, a.d2_j0, a.d2_wT, Ny, y);
      const double2 D2v = band_row<S2>(T + Ny, a.d2_j0, a.d2_wT, Ny, y);
      const double2 D2w = band_row<S2>(T + 2 * Ny, a.d2_j0, a.d2_wT, Ny, y);
      const double2 hu = cadd(cscale(u, idt), cscale(csub(D2u, cscale(u, k2)), omc_nu));
      const double2 hv = cadd(cscale(v, idt), cscale(csub(D2v, cscale(v, k2)), omc_nu));
      const double2 hw = cadd(cscale(w, idt), cscale(csub(D2w, cscale(w, k2)), omc_nu));
      qu = cadd(cadd(hu, cscale(nj[0][k], c)), cscale(nn[0][k], omc));
      qv = cadd(cadd(hv, cscale(nj[1][k], c)), cscale(nn[1][k], omc));
      qw = cadd(cadd(hw, cscale(nj[2][k], c)), cscale(nn[2][k], omc));
    }
    st_l2(F + mo + y, fy, keep);
    st_l2(R + mo + y, qu, keep);
    st_l2(R + CS + mo + y, qv, keep);
    st_l2(R + 2 * CS + mo + y, qw, keep);
  }
}

// ---------------------------------------------------------------------------
// Stage 3's pressure gradient: R -= grad p_P on the interior rows (the wall
// rows of R stay zero), p_P = L_k^-1 f_hat from the L_k substitution in F.
// ---------------------------------------------------------------------------
template <int KL>
__global__ void __launch_bounds__(32 * kStageWarps)
imm_grad_kernel(ImmArgs a, const double2* __restrict__ P, double2* __restrict__ R) {
  if (a.skip && *a.skip) return;
  constexpr int S1 = KL + 1, YM = kSYM;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int NKX = a.NKX, Ny = a.Ny, NM = a.NZ1 * a.NKX;
  const int m = blockIdx.x * kStageWarps + wq;
  if (m >= NM) return;
  double2* Pp = sm + wq * Ny;
  const long long CS = (long long)NM * Ny, mo = (long long)m * Ny;
  const unsigned long long keep = l2_keep(), drop = l2_drop();
  for (int y = lane; y < Ny; y += 32) cp_async16_l2(Pp + y, P + mo + y, drop);
  cp_async_commit();
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  double2 q[3][YM];
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y > 0 && y < Ny - 1) {
#pragma unroll
      for (int cpt = 0; cpt < 3; ++cpt) q[cpt][k] = ld_l2(R + cpt * CS + mo + y, keep);
    }
  }
  cp_async_wait_all();
  __syncwarp();
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y <= 0 || y >= Ny - 1) continue;
    const double2 p = Pp[y];
    st_l2(R + mo + y, csub(q[0][k], cik(kx, p)), keep);
    st_l2(R + CS + mo + y, csub(q[1][k], band_row<S1>(Pp, a.d1_j0, a.d1_wT, Ny, y)), keep);
    st_l2(R + 2 * CS + mo + y, csub(q[2][k], cik(kz, p)), keep);
  }
}

// ---------------------------------------------------------------------------
// Stages 4-6: vel_new, correction, per-mode norm partial.
// ---------------------------------------------------------------------------
template <int KL>
__global__ void __launch_bounds__(32 * kStageWarps)
imm_stage6_kernel(ImmArgs a, const double2* __restrict__ R, const double2* vel_j,
                  double2* vel_new, double2* __restrict__ corr_out,
                  double* __restrict__ partials) {
  if (a.skip && *a.skip) return;
  constexpr int S1 = KL + 1, YM = kSYM;
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int NKX = a.NKX, Ny = a.Ny, NM = a.NZ1 * a.NKX;
  const int m = blockIdx.x * kStageWarps + wq;
  if (m >= NM) return;
  const long long CS = (long long)NM * Ny, mo = (long long)m * Ny;
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  double2 vj[3][YM], ra[3][YM];
  double c1[YM], c2[YM], e1[YM], e2[YM];
  const unsigned long long drop = l2_drop();
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny) {
#pragma unroll
      for (int cpt = 0; cpt < 3; ++cpt) {
        vj[cpt][k] = vel_j[cpt * CS + mo + y];
        ra[cpt][k] = ld_l2(R + cpt * CS + mo + y, drop);
      }
      c1[k] = a.v1[mo + y];
      c2[k] = a.v2[mo + y];
      e1[k] = a.q1[mo + y];
      e2[k] = a.q2[mo + y];
    }
  }
  // Stages 4-5: wall divergence and influence-matrix weights
  const double2* va = R + CS + mo;
  double2 dw0 = band_row<S1>(va, a.d1_j0, a.d1_wT, Ny, 0);
  const double2 dw1 = band_row<S1>(va, a.d1_j0, a.d1_wT, Ny, Ny - 1);
  if (k2 == 0.0) dw0 = make_double2(0.0, 0.0);
  const double* Mi = a.M_inv + (long long)m * 4;
  const double2 a1 = make_double2(-(Mi[0] * dw0.x + Mi[1] * dw1.x),
                                  -(Mi[0] * dw0.y + Mi[1] * dw1.y));
  const double2 a2 = make_double2(-(Mi[2] * dw0.x + Mi[3] * dw1.x),
                                  -(Mi[2] * dw0.y + Mi[3] * dw1.y));
  // Stage 6: assemble, store, correction norm
  const double km = (ix == 0 && a.kx0) ? 1.0 : 2.0;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y >= Ny) continue;
    const double2 vnew = cadd(cadd(ra[1][k], cscale(a1, c1[k])), cscale(a2, c2[k]));
    const double2 qq = cadd(cscale(a1, e1[k]), cscale(a2, e2[k]));
    const double2 unew = csub(ra[0][k], cik(kx, qq));
    const double2 wnew = csub(ra[2][k], cik(kz, qq));
    const double2 cu = csub(unew, vj[0][k]);
    const double2 cv = csub(vnew, vj[1][k]);
    const double2 cw = csub(wnew, vj[2][k]);
    vel_new[mo + y] = unew;
    vel_new[CS + mo + y] = vnew;
    vel_new[2 * CS + mo + y] = wnew;
    if (corr_out) {
      corr_out[mo + y] = cu;
      corr_out[CS + mo + y] = cv;
      corr_out[2 * CS + mo + y] = cw;
    }
    acc += a.simpson[y] * km *
           ((cu.x * cu.x + cu.y * cu.y) + (cv.x * cv.x + cv.y * cv.y) +
            (cw.x * cw.x + cw.y * cw.y));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0 && partials) partials[m] = acc;
}

// ---------------------------------------------------------------------------
// Batched banded substitution: one CTA per tile of 16 items, one warp per
// component (1 for L_k: p_P; 3 for H_k); lane = (side, item) (lanes 0-15 the
// items' own modes, 16-31 their mirrors), and each thread solves both real
// columns (re, im) of its mode's component as two recurrences sharing every
// factor load; the warps share the tile's factor stream.  Lane 0 streams each block of
// steps' factors (and pivots) for the tile -- one contiguous chunk each --
// into a ring of shared-memory slots with bulk copies completing on the
// slot's mbarrier; every thread copies the right-hand-side rows entering its
// windows during the block into the same slot with cp.async.  Both run
// ring-1 blocks ahead of the block being computed.
//
// Forward elimination (dgbtrs 'N'): windows b[j..j+KL] in registers,
// slot(o, ph) = (o + ph) % W, W = KL + 1; the row interchange is chosen per
// block for the warp: none, with the next row only (two selects), or
// general (switch).  Back substitution: windows b[j-NU..j], slot(o, ph) =
// (o - ph) mod WB, WB = NU + 1, one FMA deep per step (U pre-scaled).
// A ring wait that does not complete within its bound sets bit 2 of the
// status word and the CTA stops computing.
// ---------------------------------------------------------------------------

struct SolveArgs {
  const double* facL;
  const double* facU;
  const unsigned char* dp;
  double2* X;  // [ncomp][NM][Ny]
  int* status;
  int NP, NM, Ny, NKX, NZ1, paired, ring, slot_bytes;
  int wait_limit;  // polls before a ring wait gives up (the drain after it uses kDrainPolls)
  const int* skip;  // non-null and *skip != 0: return at once (ImmArgs::skip)
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Global -> shared bulk copy (this GPU's memory, no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for a ring slot: false if it did not complete within
// `limit` polls.
constexpr int kDrainPolls = 1 << 20;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int limit) {
  for (int it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Mode of item p on side q and whether its columns are solved.
__device__ __forceinline__ bool item_mode(const SolveArgs& a, int p, int q, int* m) {
  bool live = p < a.NP;
  int mm = min(p, a.NP - 1);
  if (q == 1) {
    const int s = mm / a.NKX, ix = mm % a.NKX;
    live = live && a.paired && s != 0;
    if (live) mm = (a.NZ1 - s) * a.NKX + ix;
  }
  *m = mm;
  return live;
}

// Row interchange of step ph (pivot offset d) on one window.
template <int KL, int MODE>
__device__ __forceinline__ double pivot_take(double (&w)[KL + 1], int ph, int d) {
  constexpr int W = KL + 1;
  double bpj = w[ph % W];
  if (MODE == 1) {
    const double x1 = w[(1 + ph) % W];
    const bool p = d != 0;
    w[(1 + ph) % W] = p ? bpj : x1;
    bpj = p ? x1 : bpj;
  } else if (MODE == 2) {
    switch (d) {
#define DNSB_PIV(I)                  \
  case I:                            \
    if (I <= KL) {                   \
      bpj = w[(I + ph) % W];         \
      w[(I + ph) % W] = w[ph % W];   \
    }                                \
    break;
      DNSB_PIV(1) DNSB_PIV(2) DNSB_PIV(3) DNSB_PIV(4)
      DNSB_PIV(5) DNSB_PIV(6) DNSB_PIV(7) DNSB_PIV(8)
#undef DNSB_PIV
      default: break;
    }
  }
  return bpj;
}

template <int KL, int NCP, int MW, int MODE, bool TAIL>
__device__ __forceinline__ void tile_fwd_block(double2* const (&col)[NCP], int j0, int nsteps,
                                               int Ny, bool live, double (&w)[2 * NCP][KL + 1],
                                               const double2* Lp, const int (&dr)[KL + 1],
                                               const double2* ent, int ES,
                                               unsigned long long pol) {
  constexpr int W = KL + 1;
#pragma unroll
  for (int ph = 0; ph < W; ++ph) {
    const int j = j0 + ph;
    if (!TAIL || j < nsteps) {
      double L[KL];
#pragma unroll
      for (int i2 = 0; i2 < KL / 2; ++i2) {
        const double2 t = Lp[(ph * (KL / 2) + i2) * kTile];
        L[2 * i2] = t.x;
        L[2 * i2 + 1] = t.y;
      }
      double bp[2 * NCP];
#pragma unroll
      for (int c = 0; c < 2 * NCP; ++c) bp[c] = pivot_take<KL, MODE>(w[c], ph, dr[ph]);
      if (live) {
#pragma unroll
        for (int cc = 0; cc < NCP; ++cc)
          st_l2(col[cc] + j, make_double2(bp[2 * cc], bp[2 * cc + 1]), pol);
      }
#pragma unroll
      for (int c = 0; c < 2 * NCP; ++c) {
#pragma unroll
        for (int i = 1; i <= KL; ++i) w[c][(i + ph) % W] -= L[i - 1] * bp[c];
      }
      // b[j+W] enters at offset KL (0 past the last row)
      const bool in = j + W < Ny;
#pragma unroll
      for (int cc = 0; cc < NCP; ++cc) {
        const double2 e = in ? ent[(cc * MW + ph) * ES] : make_double2(0.0, 0.0);
        w[2 * cc][ph % W] = e.x;
        w[2 * cc + 1][ph % W] = e.y;
      }
    }
  }
}

template <int NU, int NCP, int MW, bool TAIL>
__device__ __forceinline__ void tile_bwd_block(double2* const (&col)[NCP], int j0, bool live,
                                               double (&w)[2 * NCP][NU + 1], const double2* Up,
                                               const double2* ent, int ES,
                                               unsigned long long pol) {
  constexpr int WB = NU + 1, NUP = (NU + 2) & ~1;
#pragma unroll
  for (int ph = 0; ph < WB; ++ph) {
    const int j = j0 - ph;
    if (!TAIL || j >= 0) {
      const double2* u = Up + (WB - 1 - ph) * (NUP / 2) * kTile;
      double U[NUP];
#pragma unroll
      for (int i2 = 0; i2 < NUP / 2; ++i2) {
        const double2 t = u[i2 * kTile];
        U[2 * i2] = t.x;
        U[2 * i2 + 1] = t.y;
      }
      const int st = ((NU - ph) % WB + WB) % WB;
      double bj[2 * NCP];
#pragma unroll
      for (int c = 0; c < 2 * NCP; ++c) bj[c] = w[c][st];
      if (live) {
#pragma unroll
        for (int cc = 0; cc < NCP; ++cc)
          st_l2(col[cc] + j, make_double2(bj[2 * cc] * U[0], bj[2 * cc + 1] * U[0]), pol);
      }
#pragma unroll
      for (int i = 1; i <= NU; ++i) {
        const int si = ((NU - i - ph) % WB + WB) % WB;
#pragma unroll
        for (int c = 0; c < 2 * NCP; ++c) w[c][si] -= U[i] * bj[c];
      }
      // b[j-WB] enters at offset 0 (0 below row 0)
      const bool in = j - WB >= 0;
#pragma unroll
      for (int cc = 0; cc < NCP; ++cc) {
        const double2 e = in ? ent[(cc * MW + ph) * ES] : make_double2(0.0, 0.0);
        w[2 * cc][st] = e.x;
        w[2 * cc + 1][st] = e.y;
      }
    }
  }
}

template <int KL, int NU>
__global__ void __launch_bounds__(96)
imm_solve_kernel(SolveArgs a) {
  if (a.skip && *a.skip) return;  // before any barrier is set up
  constexpr int NCP = 1;  // components per thread (one warp per component)
  constexpr int W = KL + 1, WB = NU + 1, NUP = (NU + 2) & ~1;
  constexpr int LB = W * KL * kTile * 8, PB = W * kTile, UB = WB * NUP * kTile * 8;
  constexpr int MW = W > WB ? W : WB;  // rows per (component, lane) in a slot
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ __align__(8) unsigned long long bars[3];
  __shared__ int s_fail;
  const int tid = threadIdx.x, lane = tid & 31, cw = tid >> 5;  // warp = component
  const int side = lane >> 4, it = lane & (kTile - 1);
  const int tile = blockIdx.x;
  const int Ny = a.Ny, R = a.ring, SB = a.slot_bytes, nthr = blockDim.x;
  const int EB = MW * nthr * 16;  // entering rows of every thread, at the slot's end
  const long long NyF = Ny + W, NyB = Ny + WB;
  int m;
  const bool live = item_mode(a, tile * kTile + it, side, &m);
  const unsigned long long keep = l2_keep();
  double2* col[NCP];
#pragma unroll
  for (int cc = 0; cc < NCP; ++cc) col[cc] = a.X + ((long long)(cw + cc) * a.NM + m) * Ny;
  const int nsteps = Ny - 1;
  const int nbf = (nsteps + W - 1) / W;  // forward blocks
  const int nbb = (Ny + WB - 1) / WB;    // back-substitution blocks
  const int nblk = nbf + nbb;

  if (tid == 0) {
    for (int r = 0; r < R; ++r) mbar_init(&bars[r], 1);
    mbar_fence_init();
    s_fail = 0;
  }
  __syncthreads();
  // Block g of the combined sequence into slot g % R: factors by lane 0
  // (bulk, mbarrier), this lane's entering rows by every lane (cp.async
  // group g).  Entering rows of component cc at ent[(cc * MW + ph) * 32 +
  // lane]: forward row j0+W+ph, back substitution row j0-WB-ph.
  int hi_issued = -1;
  auto issue = [&](int g) {
    if (g < nblk) {
      hi_issued = g;
      unsigned char* slot = ring + (g % R) * SB;
      unsigned long long* bar = &bars[g % R];
      double2* ent = reinterpret_cast<double2*>(slot + SB - EB) + tid;
      if (g < nbf) {
        const int j0 = g * W;
        if (tid == 0) {
          mbar_arrive_tx(bar, LB + PB);
          bulk_g2s(slot, a.facL + (tile * NyF + j0) * KL * kTile, LB, bar);
          bulk_g2s(slot + LB, a.dp + (tile * NyF + j0) * kTile, PB, bar);
        }
        if (live) {
#pragma unroll
          for (int ph = 0; ph < W; ++ph) {
            const int e = j0 + W + ph;
            if (e < Ny)
              for (int cc = 0; cc < NCP; ++cc) cp_async16_l2(ent + (cc * MW + ph) * nthr, col[cc] + e, keep);
          }
        }
      } else {
        const int j0 = Ny - 1 - (g - nbf) * WB;
        if (tid == 0) {
          mbar_arrive_tx(bar, UB);
          bulk_g2s(slot, a.facU + (tile * NyB + j0 + 1) * NUP * kTile, UB, bar);
        }
        if (live) {
#pragma unroll
          for (int ph = 0; ph < WB; ++ph) {
            const int e = j0 - WB - ph;
            if (e >= 0)
              for (int cc = 0; cc < NCP; ++cc) cp_async16_l2(ent + (cc * MW + ph) * nthr, col[cc] + e, keep);
          }
        }
      }
    }
    cp_async_commit();
  };
  auto wait_block = [&](int g) {
    if (R == 3) cp_async_wait_2(); else cp_async_wait_1();  // this lane's rows of block g
    if (!mbar_wait(&bars[g % R], (g / R) & 1, a.wait_limit)) s_fail = 1;
    __syncthreads();
  };
  // The back substitution reads the forward results: its blocks are issued
  // only after every forward result is stored.
  for (int h = 0; h < R - 1; ++h) issue(h < nbf ? h : nblk);
  int g = 0;
  bool ok = true;

  // ---- forward elimination, steps j = 0 .. Ny-2 ----
  {
    double w[2 * NCP][W];
#pragma unroll
    for (int cc = 0; cc < NCP; ++cc) {
#pragma unroll
      for (int o = 0; o < W; ++o) {
        const double2 v = (o < Ny) ? ld_l2(col[cc] + o, keep) : make_double2(0.0, 0.0);
        w[2 * cc][o] = v.x;
        w[2 * cc + 1][o] = v.y;
      }
    }
    for (int k = 0; k < nbf; ++k, ++g) {
      issue(g + R - 1 < nbf ? g + R - 1 : nblk);
      wait_block(g);
      const unsigned char* slot = ring + (g % R) * SB;
      const double2* Lp = reinterpret_cast<const double2*>(slot) + it;
      const unsigned char* Ps = slot + LB;
      const double2* ent = reinterpret_cast<const double2*>(slot + SB - EB) + tid;
      int dr[W];
      int dm = 0;
#pragma unroll
      for (int ph = 0; ph < W; ++ph) {
        dr[ph] = Ps[ph * kTile + it];
        dm = max(dm, dr[ph]);
      }
      dm = __reduce_max_sync(0xffffffffu, dm);
      const int j0 = k * W;
      if (j0 + W > nsteps)
        tile_fwd_block<KL, NCP, MW, 2, true>(col, j0, nsteps, Ny, live, w, Lp, dr, ent, nthr, keep);
      else if (dm == 0)
        tile_fwd_block<KL, NCP, MW, 0, false>(col, j0, nsteps, Ny, live, w, Lp, dr, ent, nthr, keep);
      else if (dm == 1)
        tile_fwd_block<KL, NCP, MW, 1, false>(col, j0, nsteps, Ny, live, w, Lp, dr, ent, nthr, keep);
      else
        tile_fwd_block<KL, NCP, MW, 2, false>(col, j0, nsteps, Ny, live, w, Lp, dr, ent, nthr, keep);
      __syncthreads();  // the slot is refilled by the next issue
      if (s_fail) {
        ok = false;
        break;
      }
    }
    // b[Ny-1] sits at offset 0 after the last step: slot nsteps % W.
    const int last = nsteps % W;
#pragma unroll
    for (int cc = 0; cc < NCP; ++cc) {
      double v0 = w[2 * cc][0], v1 = w[2 * cc + 1][0];
#pragma unroll
      for (int s = 1; s < W; ++s)
        if (last == s) {
          v0 = w[2 * cc][s];
          v1 = w[2 * cc + 1][s];
        }
      if (live && ok) st_l2(col[cc] + Ny - 1, make_double2(v0, v1), keep);
    }
  }

  // ---- back substitution, rows j = Ny-1 .. 0 (this lane's own forward
  // results, read back in program order) ----
  if (ok) {
    for (int h = nbf; h < nbf + R - 1; ++h) issue(h);
    double w[2 * NCP][WB];
#pragma unroll
    for (int cc = 0; cc < NCP; ++cc) {
#pragma unroll
      for (int o = 0; o < WB; ++o) {
        const int idx = Ny - 1 - NU + o;
        const double2 v = (idx >= 0) ? ld_l2(col[cc] + idx, keep) : make_double2(0.0, 0.0);
        w[2 * cc][o] = v.x;
        w[2 * cc + 1][o] = v.y;
      }
    }
    for (int k = 0; k < nbb; ++k, ++g) {
      issue(g + R - 1);
      wait_block(g);
      const unsigned char* slot = ring + (g % R) * SB;
      const double2* Up = reinterpret_cast<const double2*>(slot) + it;
      const double2* ent = reinterpret_cast<const double2*>(slot + SB - EB) + tid;
      const int j0 = Ny - 1 - k * WB;
      if (j0 - WB + 1 < 0)
        tile_bwd_block<NU, NCP, MW, true>(col, j0, live, w, Up, ent, nthr, keep);
      else
        tile_bwd_block<NU, NCP, MW, false>(col, j0, live, w, Up, ent, nthr, keep);
      __syncthreads();
      if (s_fail) {
        ok = false;
        break;
      }
    }
  }
  cp_async_wait_all();
  if (!ok && tid == 0) {
    // Leave no bulk copy in flight: blocks g .. hi_issued were issued
    // (block g is the one that timed out).
    for (int h = g; h <= hi_issued; ++h) mbar_wait(&bars[h % R], (h / R) & 1, kDrainPolls);
    atomicOr(a.status, 2);
  }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
size_t imm_batch_stage_smem(int Ny) {
  return sizeof(double2) * (size_t)(6 * Ny * kStageWarps);
}

static size_t imm_batch_grad_smem(int Ny) {
  return sizeof(double2) * (size_t)(Ny * kStageWarps);
}

bool imm_batch_supported(int kl, int ny) {
  return (kl == 2 || kl == 4 || kl == 6 || kl == 8) && ny <= 32 * kSYM;
}

// Ring slot bytes of one substitution launch: the larger of a forward block
// (factors, pivots) and a back-substitution block (U records), plus the
// entering rows of every lane; and the ring depth that fits.
static int solve_slot_bytes(int kl, int nu, int ncomp) {
  const int W = kl + 1, WB = nu + 1, nup = (nu + 2) & ~1;
  const int MW = W > WB ? W : WB;
  const int f = W * kl * kTile * 8 + W * kTile;
  const int b = WB * nup * kTile * 8;
  return (((f > b ? f : b) + 127) & ~127) + ncomp * MW * 32 * 16;
}

static int solve_ring(int kl, int nu, int ncomp, int max_smem) {
  const int sb = solve_slot_bytes(kl, nu, ncomp);
  if (3 * sb <= max_smem && 3 * sb <= 100 * 1024) return 3;
  if (2 * sb <= max_smem) return 2;
  return 0;
}

bool imm_batch_fits(int kl, int nu, int max_smem) {
  return solve_ring(kl, nu, 3, max_smem) > 0 && solve_ring(kl, nu, 1, max_smem) > 0;
}

template <int KL>
static cudaError_t solve_launch(const ImmBatch& bt, int op, double2* X, int ncomp, int NM,
                                int Ny, int NKX, int NZ1, const int* skip, cudaStream_t st) {
  SolveArgs s{};
  s.skip = skip;
  s.facL = bt.facL[op];
  s.facU = bt.facU[op];
  s.dp = bt.dp[op];
  s.X = X;
  s.status = bt.status;
  s.NP = bt.NP;
  s.NM = NM;
  s.Ny = Ny;
  s.NKX = NKX;
  s.NZ1 = NZ1;
  s.paired = bt.paired;
  s.ring = solve_ring(KL, bt.nu, ncomp, bt.max_smem);
  s.slot_bytes = solve_slot_bytes(KL, bt.nu, ncomp);
  s.wait_limit = bt.wait_limit;
  if (s.ring == 0) return cudaErrorInvalidValue;
  const size_t sm = (size_t)s.ring * s.slot_bytes;
  const int grid = (bt.NP + kTile - 1) / kTile;
  if (bt.nu == KL + 1)
    imm_solve_kernel<KL, KL + 1><<<grid, 32 * ncomp, sm, st>>>(s);
  else
    imm_solve_kernel<KL, 2 * KL><<<grid, 32 * ncomp, sm, st>>>(s);
  return cudaGetLastError();
}

template <int K>
static cudaError_t pipeline(const ImmArgs& a, const ImmBatch& bt, const double2* vel_n,
                           const double2* vel_j, const double2* nl_n, const double2* nl_j,
                           double2* vel_new, double2* corr_out, double* partials,
                           cudaStream_t st) {
  const int NM = a.NZ1 * a.NKX, Ny = a.Ny;
  const int grid = (NM + kStageWarps - 1) / kStageWarps;
  const size_t sm = imm_batch_stage_smem(Ny);
  cudaError_t e;
  imm_stage013_kernel<K><<<grid, 32 * kStageWarps, sm, st>>>(a, vel_n, nl_n, nl_j, bt.F, bt.R);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = solve_launch<K>(bt, 0, bt.F, 1, NM, Ny, a.NKX, a.NZ1, a.skip, st);
  if (e != cudaSuccess) return e;
  imm_grad_kernel<K><<<grid, 32 * kStageWarps, imm_batch_grad_smem(Ny), st>>>(a, bt.F, bt.R);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = solve_launch<K>(bt, 1, bt.R, 3, NM, Ny, a.NKX, a.NZ1, a.skip, st);
  if (e != cudaSuccess) return e;
  imm_stage6_kernel<K><<<grid, 32 * kStageWarps, 0, st>>>(a, bt.R, vel_j, vel_new, corr_out,
                                                          partials);
  return cudaGetLastError();
}

// Five launches: stages 0-1, L_k solve, stage 3, H_k solve, stages 4-6.
cudaError_t launch_imm_batch(const ImmArgs& a, const ImmBatch& bt, const double2* vel_n,
                             const double2* vel_j, const double2* nl_n,
                             const double2* nl_j, double2* vel_new, double2* corr_out,
                             double* partials, cudaStream_t st) {
  switch (a.kl) {
    case 2: return pipeline<2>(a, bt, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials, st);
    case 4: return pipeline<4>(a, bt, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials, st);
    case 6: return pipeline<6>(a, bt, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials, st);
    case 8: return pipeline<8>(a, bt, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t set_imm_batch_attributes(int max_smem) {
  const void* fns[] = {
      (const void*)imm_stage013_kernel<2>, (const void*)imm_stage013_kernel<4>,
      (const void*)imm_stage013_kernel<6>, (const void*)imm_stage013_kernel<8>,
      (const void*)imm_grad_kernel<2>,     (const void*)imm_grad_kernel<4>,
      (const void*)imm_grad_kernel<6>,     (const void*)imm_grad_kernel<8>,
#define DNSB_SOLVE_FNS(K) \
  (const void*)imm_solve_kernel<K, K + 1>, (const void*)imm_solve_kernel<K, 2 * K>
      DNSB_SOLVE_FNS(2), DNSB_SOLVE_FNS(4), DNSB_SOLVE_FNS(6), DNSB_SOLVE_FNS(8)};
#undef DNSB_SOLVE_FNS
  cudaError_t e = cudaSuccess;
  for (const void* f : fns) {
    cudaError_t r = allow_dynamic_smem(f, max_smem);
    if (r != cudaSuccess) e = r;
  }
  return e;
}

}  // namespace dnsb
