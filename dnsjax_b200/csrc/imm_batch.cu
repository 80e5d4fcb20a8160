// Plane Couette influence-matrix iteration as five bandwidth-shaped kernels.
//
// Follows src/dnsjax/flows/plane_couette.py:376-504 (six stages) and the
// dgbtrs-'N' substitution of src/dnsjax/geometries/cartesian.py:360-441.
//
//   stages 0-1   one warp per (kz, kx) mode: d_hat = div u^n, then f_hat
//                (D1 / D2 along y from shared memory) -> F      [NM][Ny]
//   L_k solve    one thread per (mode, real column): p_P = L_k^-1 f_hat,
//                in place in F
//   stage 3      one warp per mode: R = H_k^- u^n - grad p_P + c N_j +
//                (1-c) N_n -> R                                  [3][NM][Ny]
//   H_k solve    one thread per (mode, real column), in place in R
//   stages 4-6   one warp per mode: wall divergence, influence-matrix
//                weights, u^{j+1}, the correction and its Simpson norm
//
// The LU factors are repacked once, when the operators are bound, into a
// record-major layout with the item index fastest, so a warp of 32 items
// reads each factor of a substitution step with one coalesced load:
//   fac[(j * RS + slot) * NP + item],  slots [0, kl) L multipliers of rows
//   j+1..j+kl, [kl] 1/U_jj, [kl+i] U_{j-i,j}/U_jj (i = 1..NU);
//   piv[j * NP + item] = ipiv[j] - j (validated, 0..kl).
// An item is mode (s, kx) with s <= (nz-1)/2; when the factors of (s, kx)
// and its mirror (nz-1-s, kx) are bit-identical (same k^2; checked at bind
// time) the mirror reads the item's records, else every mode is an item.
#include "solver.cuh"

namespace dnsb {

namespace {

constexpr int kStageWarps = 4;  // modes per CTA in the stage kernels
constexpr int kSYM = 5;         // y values per lane: y = lane + 32 k, Ny <= 160

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
// Bind time: repack one operator's factors into 32-item tiles, each tile's
// rows contiguous so a block of substitution steps is one contiguous copy:
//   facL[tile][j][i/2][32][2]       (rows j < Ny, then W zero rows)  L
//                                   multipliers of rows j+1..j+kl
//   facU[tile][j + WB][i/2][32][2]  (WB zero rows first; NUP = NU+1 rounded
//                                   up to even) i = 0: 1/U_jj, i > 0:
//                                   U_{j-i,j} / U_jj
//   dp[tile][j][32]            ipiv[j] - j, validated (a bad pivot is flagged
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
    const int tile = p >> 5, lane = p & 31;
    const double* abm = ab + (long long)p * rows * Ny;
    const double r = 1.0 / abm[(long long)kuu * Ny + j];
    // element i of row j: [tile][j][i / 2][lane][i % 2]
    double* L = facL + (tile * NyF + j) * kl * 32 + 2 * lane;
    for (int i = 1; i <= kl; ++i) {
      const int e = i - 1;
      L[(e >> 1) * 64 + (e & 1)] = abm[(long long)(kuu + i) * Ny + j];
    }
    double* U = facU + (tile * NyB + j + WB) * nup * 32 + 2 * lane;
    U[0] = r;
    for (int i = 1; i <= nu; ++i) {
      const int row = kuu - i;
      const double u = (row >= row0) ? abm[(long long)row * Ny + j] : 0.0;
      U[(i >> 1) * 64 + (i & 1)] = u * r;
    }
    int d = piv[(long long)p * Ny + j] - j;
    if (d < 0 || d > kl || j + d >= Ny) {  // never follow a bad pivot
      atomicOr(status, 1);
      d = 0;
    }
    dp[(tile * NyF + j) * 32 + lane] = (unsigned char)d;
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
// Stages 0-1: f_hat -> F.
// ---------------------------------------------------------------------------
template <int KL>
__global__ void __launch_bounds__(32 * kStageWarps)
imm_stage01_kernel(ImmArgs a, const double2* __restrict__ vel_n,
                   const double2* __restrict__ nl_n, const double2* __restrict__ nl_j,
                   double2* __restrict__ F) {
  constexpr int S1 = KL + 1, S2 = KL + 2, YM = kSYM;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int NKX = a.NKX, Ny = a.Ny, NM = a.NZ1 * a.NKX;
  const int m = blockIdx.x * kStageWarps + wq;
  if (m >= NM) return;  // no CTA-wide barrier below
  double2* T = sm + wq * 4 * Ny;  // v^n, N^j_v, N^n_v
  double2* D = T + 3 * Ny;        // d_hat^n
  const long long CS = (long long)NM * Ny, mo = (long long)m * Ny;
  for (int y = lane; y < Ny; y += 32) {
    cp_async16(T + y, vel_n + CS + mo + y);
    cp_async16(T + Ny + y, nl_j + CS + mo + y);
    cp_async16(T + 2 * Ny + y, nl_n + CS + mo + y);
  }
  cp_async_commit();
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  const double c = a.c, dt = a.dt, omc = 1.0 - c, omc_nu = omc * a.nu;
  double2 ua[YM], wa[YM], uj[YM], wj[YM], un[YM], wn[YM];
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny) {
      ua[k] = vel_n[mo + y];
      wa[k] = vel_n[2 * CS + mo + y];
      uj[k] = nl_j[mo + y];
      wj[k] = nl_j[2 * CS + mo + y];
      un[k] = nl_n[mo + y];
      wn[k] = nl_n[2 * CS + mo + y];
    }
  }
  cp_async_wait_all();
  __syncwarp();
  // Stage 0: d_hat^n = div u^n
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny)
      D[y] = cadd(cadd(cik(kx, ua[k]), band_row<S1>(T, a.d1_j0, a.d1_wT, Ny, y)), cik(kz, wa[k]));
  }
  __syncwarp();
  // Stage 1: f_hat (wall rows zero)
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y >= Ny) continue;
    double2 fy = make_double2(0.0, 0.0);
    if (y > 0 && y < Ny - 1) {
      const double2 divNj =
          cadd(cadd(cik(kx, uj[k]), band_row<S1>(T + Ny, a.d1_j0, a.d1_wT, Ny, y)), cik(kz, wj[k]));
      const double2 divNn =
          cadd(cadd(cik(kx, un[k]), band_row<S1>(T + 2 * Ny, a.d1_j0, a.d1_wT, Ny, y)), cik(kz, wn[k]));
      const double2 dy = D[y];
      const double2 Lkd = csub(band_row<S2>(D, a.d2_j0, a.d2_wT, Ny, y), cscale(dy, k2));
      const double2 dd = make_double2(dy.x / dt, dy.y / dt);
      fy = cadd(cadd(cadd(dd, cscale(divNj, c)), cscale(divNn, omc)), cscale(Lkd, omc_nu));
    }
    F[mo + y] = fy;
  }
}

// ---------------------------------------------------------------------------
// Stage 3: R -> R (3 components).
// ---------------------------------------------------------------------------
template <int KL>
__global__ void __launch_bounds__(32 * kStageWarps)
imm_stage3_kernel(ImmArgs a, const double2* __restrict__ vel_n,
                  const double2* __restrict__ nl_n, const double2* __restrict__ nl_j,
                  const double2* __restrict__ P, double2* __restrict__ R) {
  constexpr int S1 = KL + 1, S2 = KL + 2, YM = kSYM;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const int NKX = a.NKX, Ny = a.Ny, NM = a.NZ1 * a.NKX;
  const int m = blockIdx.x * kStageWarps + wq;
  if (m >= NM) return;
  double2* T = sm + wq * 4 * Ny;  // u^n, v^n, w^n
  double2* Pp = T + 3 * Ny;       // p_P
  const long long CS = (long long)NM * Ny, mo = (long long)m * Ny;
  for (int y = lane; y < Ny; y += 32) {
    cp_async16(T + y, vel_n + mo + y);
    cp_async16(T + Ny + y, vel_n + CS + mo + y);
    cp_async16(T + 2 * Ny + y, vel_n + 2 * CS + mo + y);
    cp_async16(Pp + y, P + mo + y);
  }
  cp_async_commit();
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  const double c = a.c, omc = 1.0 - c, omc_nu = omc * a.nu, idt = 1.0 / a.dt;
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
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y >= Ny) continue;
    double2 ru = make_double2(0.0, 0.0), rv = ru, rw = ru;
    if (y > 0 && y < Ny - 1) {
      const double2 p = Pp[y];
      const double2 dxp = cik(kx, p);
      const double2 dyp = band_row<S1>(Pp, a.d1_j0, a.d1_wT, Ny, y);
      const double2 dzp = cik(kz, p);
      const double2 u = T[y], v = T[Ny + y], w = T[2 * Ny + y];
      const double2 D2u = band_row<S2>(T, a.d2_j0, a.d2_wT, Ny, y);
      const double2 D2v = band_row<S2>(T + Ny, a.d2_j0, a.d2_wT, Ny, y);
      const double2 D2w = band_row<S2>(T + 2 * Ny, a.d2_j0, a.d2_wT, Ny, y);
      const double2 hu = cadd(cscale(u, idt), cscale(csub(D2u, cscale(u, k2)), omc_nu));
      const double2 hv = cadd(cscale(v, idt), cscale(csub(D2v, cscale(v, k2)), omc_nu));
      const double2 hw = cadd(cscale(w, idt), cscale(csub(D2w, cscale(w, k2)), omc_nu));
      ru = cadd(cadd(csub(hu, dxp), cscale(nj[0][k], c)), cscale(nn[0][k], omc));
      rv = cadd(cadd(csub(hv, dyp), cscale(nj[1][k], c)), cscale(nn[1][k], omc));
      rw = cadd(cadd(csub(hw, dzp), cscale(nj[2][k], c)), cscale(nn[2][k], omc));
    }
    R[mo + y] = ru;
    R[CS + mo + y] = rv;
    R[2 * CS + mo + y] = rw;
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
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny) {
#pragma unroll
      for (int cpt = 0; cpt < 3; ++cpt) {
        vj[cpt][k] = vel_j[cpt * CS + mo + y];
        ra[cpt][k] = R[cpt * CS + mo + y];
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
  const double km = (ix == 0) ? 1.0 : 2.0;
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
// Batched banded substitution: one CTA per (tile of 32 items, side), one
// warp per real column (2 for L_k: re / im of p_P; 6 for H_k), one thread
// per (item, column).  One thread streams each block of steps -- the tile's
// factors (and pivots) for that block, one contiguous chunk each -- into a
// ring of shared-memory slots with bulk copies that complete on the slot's
// mbarrier, ring-1 blocks ahead of the block being computed; every thread
// runs its column's recurrence from registers and the ring, loading the
// right-hand-side rows that enter its window one block ahead.
//
// Forward elimination (dgbtrs 'N'): window b[j..j+KL] in registers,
// slot(o, ph) = (o + ph) % W, W = KL + 1; the row interchange is chosen per
// block for the warp: none, with the next row only (two selects), or
// general (switch).  Back substitution: window b[j-NU..j], slot(o, ph) =
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
  int NP, ncomp, NM, Ny, NKX, NZ1, paired, ring, slot_bytes;
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
// Bounded wait for a ring slot: false if it did not complete.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  for (int it = 0; it < (1 << 20); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Mode of item p on side q and whether its column is solved.
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

template <int KL, int MODE, bool TAIL>
__device__ __forceinline__ void ring_fwd_steps(double* b, int j0, int nsteps, bool live,
                                               double (&w)[KL + 1], const double2* Lp,
                                               const int (&dr)[KL + 1],
                                               const double (&be)[KL + 1]) {
  constexpr int W = KL + 1;
#pragma unroll
  for (int ph = 0; ph < W; ++ph) {
    const int j = j0 + ph;
    if (!TAIL || j < nsteps) {
      double L[KL];
#pragma unroll
      for (int i2 = 0; i2 < KL / 2; ++i2) {
        const double2 t = Lp[(ph * (KL / 2) + i2) * 32];
        L[2 * i2] = t.x;
        L[2 * i2 + 1] = t.y;
      }
      double bpj = w[ph % W];
      if (MODE == 1) {
        const double x1 = w[(1 + ph) % W];
        const bool p = dr[ph] != 0;
        w[(1 + ph) % W] = p ? bpj : x1;
        bpj = p ? x1 : bpj;
      } else if (MODE == 2) {
        switch (dr[ph]) {
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
      if (live) b[2 * j] = bpj;
#pragma unroll
      for (int i = 1; i <= KL; ++i) w[(i + ph) % W] -= L[i - 1] * bpj;
      w[ph % W] = be[ph];  // b[j+W] enters at offset KL
    }
  }
}

template <int NU, bool TAIL>
__device__ __forceinline__ void ring_bwd_steps(double* b, int j0, bool live,
                                               double (&w)[NU + 1], const double2* Up,
                                               const double (&be)[NU + 1]) {
  constexpr int WB = NU + 1, NUP = (NU + 2) & ~1;
#pragma unroll
  for (int ph = 0; ph < WB; ++ph) {
    const int j = j0 - ph;
    if (!TAIL || j >= 0) {
      const double2* u = Up + (WB - 1 - ph) * (NUP / 2) * 32;
      double U[NUP];
#pragma unroll
      for (int i2 = 0; i2 < NUP / 2; ++i2) {
        const double2 t = u[i2 * 32];
        U[2 * i2] = t.x;
        U[2 * i2 + 1] = t.y;
      }
      const int st = ((NU - ph) % WB + WB) % WB;
      const double bj = w[st];
      if (live) b[2 * j] = bj * U[0];
#pragma unroll
      for (int i = 1; i <= NU; ++i) {
        const int si = ((NU - i - ph) % WB + WB) % WB;
        w[si] -= U[i] * bj;
      }
      w[st] = be[ph];  // b[j-WB] enters at offset 0
    }
  }
}

template <int KL, int NU>
__global__ void __launch_bounds__(192)
imm_solve_kernel(SolveArgs a) {
  constexpr int W = KL + 1, WB = NU + 1, NUP = (NU + 2) & ~1;
  constexpr int LB = W * KL * 32 * 8, PB = W * 32, UB = WB * NUP * 32 * 8;
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ __align__(8) unsigned long long bars[3];
  __shared__ int s_fail;
  const int tid = threadIdx.x;
  const int lane = tid & 31, c = tid >> 5;
  const int comp = c >> 1, reim = c & 1;
  const int tile = blockIdx.x, q = blockIdx.y;
  const int Ny = a.Ny, R = a.ring, SB = a.slot_bytes;
  const long long NyF = Ny + W, NyB = Ny + WB;
  int m;
  const bool live = item_mode(a, tile * 32 + lane, q, &m);
  double* b = reinterpret_cast<double*>(a.X + ((long long)comp * a.NM + m) * Ny) + reim;
  const int nsteps = Ny - 1;
  const int nbf = (nsteps + W - 1) / W;   // forward blocks
  const int nbb = (Ny + WB - 1) / WB;     // back-substitution blocks
  const int nblk = nbf + nbb;

  if (tid == 0) {
    for (int r = 0; r < R; ++r) mbar_init(&bars[r], 1);
    mbar_fence_init();
    s_fail = 0;
  }
  __syncthreads();
  // Producer (thread 0): block g of the combined sequence into slot g % R.
  auto issue = [&](int g) {
    if (g >= nblk) return;
    unsigned char* slot = ring + (g % R) * SB;
    unsigned long long* bar = &bars[g % R];
    if (g < nbf) {
      const int j0 = g * W;
      mbar_arrive_tx(bar, LB + PB);
      bulk_g2s(slot, a.facL + (tile * NyF + j0) * KL * 32, LB, bar);
      bulk_g2s(slot + LB, a.dp + (tile * NyF + j0) * 32, PB, bar);
    } else {
      const int j0 = Ny - 1 - (g - nbf) * WB;  // rows j0-WB+1 .. j0
      mbar_arrive_tx(bar, UB);
      bulk_g2s(slot, a.facU + (tile * NyB + j0 + 1) * NUP * 32, UB, bar);
    }
  };
  if (tid == 0)
    for (int g = 0; g < R - 1; ++g) issue(g);
  int g = 0;
  bool ok = true;

  // ---- forward elimination, steps j = 0 .. Ny-2 ----
  {
    double w[W], be[W], bn[W];
#pragma unroll
    for (int o = 0; o < W; ++o) w[o] = (o < Ny) ? b[2 * o] : 0.0;
#pragma unroll
    for (int ph = 0; ph < W; ++ph) bn[ph] = (W + ph < Ny) ? b[2 * (W + ph)] : 0.0;
    for (int k = 0; k < nbf; ++k, ++g) {
      if (tid == 0) issue(g + R - 1);
#pragma unroll
      for (int ph = 0; ph < W; ++ph) be[ph] = bn[ph];
      const int j0 = k * W;
#pragma unroll
      for (int ph = 0; ph < W; ++ph) {
        const int e = j0 + 2 * W + ph;  // entering rows of the next block
        bn[ph] = (e < Ny) ? b[2 * e] : 0.0;
      }
      if (!mbar_wait(&bars[g % R], (g / R) & 1)) s_fail = 1;
      const unsigned char* slot = ring + (g % R) * SB;
      const double2* Lp = reinterpret_cast<const double2*>(slot) + lane;
      const unsigned char* Ps = slot + LB;
      int dr[W];
      int dm = 0;
#pragma unroll
      for (int ph = 0; ph < W; ++ph) {
        dr[ph] = Ps[ph * 32 + lane];
        dm = max(dm, dr[ph]);
      }
      dm = __reduce_max_sync(0xffffffffu, dm);
      if (j0 + W > nsteps)
        ring_fwd_steps<KL, 2, true>(b, j0, nsteps, live, w, Lp, dr, be);
      else if (dm == 0)
        ring_fwd_steps<KL, 0, false>(b, j0, nsteps, live, w, Lp, dr, be);
      else if (dm == 1)
        ring_fwd_steps<KL, 1, false>(b, j0, nsteps, live, w, Lp, dr, be);
      else
        ring_fwd_steps<KL, 2, false>(b, j0, nsteps, live, w, Lp, dr, be);
      __syncthreads();  // the slot is refilled by the next issue
      if (s_fail) {
        ok = false;
        break;
      }
    }
    // b[Ny-1] sits at offset 0 after the last step: slot nsteps % W.
    const int last = nsteps % W;
    double v = w[0];
#pragma unroll
    for (int s = 1; s < W; ++s)
      if (last == s) v = w[s];
    if (live && ok) b[2 * (Ny - 1)] = v;
  }

  // ---- back substitution, rows j = Ny-1 .. 0 (this thread's forward
  // results, read back in program order) ----
  if (ok) {
    double w[WB], be[WB], bn[WB];
#pragma unroll
    for (int o = 0; o < WB; ++o) {
      const int idx = Ny - 1 - NU + o;
      w[o] = (idx >= 0) ? b[2 * idx] : 0.0;
    }
#pragma unroll
    for (int ph = 0; ph < WB; ++ph) {
      const int e = Ny - 1 - ph - WB;
      bn[ph] = (e >= 0) ? b[2 * e] : 0.0;
    }
    for (int k = 0; k < nbb; ++k, ++g) {
      if (tid == 0) issue(g + R - 1);
#pragma unroll
      for (int ph = 0; ph < WB; ++ph) be[ph] = bn[ph];
      const int j0 = Ny - 1 - k * WB;
#pragma unroll
      for (int ph = 0; ph < WB; ++ph) {
        const int e = j0 - WB - ph - WB;  // entering rows of the next block
        bn[ph] = (e >= 0) ? b[2 * e] : 0.0;
      }
      if (!mbar_wait(&bars[g % R], (g / R) & 1)) s_fail = 1;
      const double2* Up = reinterpret_cast<const double2*>(ring + (g % R) * SB) + lane;
      if (j0 - WB + 1 < 0)
        ring_bwd_steps<NU, true>(b, j0, live, w, Up, be);
      else
        ring_bwd_steps<NU, false>(b, j0, live, w, Up, be);
      __syncthreads();
      if (s_fail) {
        ok = false;
        break;
      }
    }
  }
  if (!ok) {
    // Leave no bulk copy in flight: wait (bounded) for every issued block
    // not yet consumed, then report.
    if (tid == 0) {
      // blocks g .. g+R-1 were issued (block g is the one that timed out)
      const int last = min(g + R - 1, nblk - 1);
      for (int h = g; h <= last; ++h) mbar_wait(&bars[h % R], (h / R) & 1);
      atomicOr(a.status, 2);
    }
  }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
size_t imm_batch_stage_smem(int Ny) {
  return sizeof(double2) * (size_t)(4 * Ny * kStageWarps);
}

bool imm_batch_supported(int kl, int ny) {
  return (kl == 2 || kl == 4 || kl == 6 || kl == 8) && ny <= 32 * kSYM;
}

// Ring slot bytes of one solve launch (the larger of a forward and a back-
// substitution block) and the ring depth that fits.
static int solve_slot_bytes(int kl, int nu, int ncomp) {
  (void)ncomp;
  const int W = kl + 1, WB = nu + 1, nup = (nu + 2) & ~1;
  const int f = W * kl * 32 * 8 + W * 32;
  const int b = WB * nup * 32 * 8;
  return ((f > b ? f : b) + 127) & ~127;
}

static int solve_ring(int kl, int nu, int ncomp, int max_smem) {
  const int sb = solve_slot_bytes(kl, nu, ncomp);
  if (3 * sb <= max_smem && 3 * sb <= 110 * 1024) return 3;
  if (2 * sb <= max_smem) return 2;
  return 0;
}

bool imm_batch_fits(int kl, int nu, int max_smem) {
  return solve_ring(kl, nu, 3, max_smem) > 0 && solve_ring(kl, nu, 1, max_smem) > 0;
}

template <int KL>
static cudaError_t solve_launch(const ImmBatch& bt, int op, double2* X, int ncomp, int NM,
                                int Ny, int NKX, int NZ1, cudaStream_t st) {
  SolveArgs s{};
  s.facL = bt.facL[op];
  s.facU = bt.facU[op];
  s.dp = bt.dp[op];
  s.X = X;
  s.NP = bt.NP;
  s.ncomp = ncomp;
  s.NM = NM;
  s.Ny = Ny;
  s.NKX = NKX;
  s.NZ1 = NZ1;
  s.paired = bt.paired;
  s.status = bt.status;
  s.ring = solve_ring(KL, bt.nu, ncomp, bt.max_smem);
  s.slot_bytes = solve_slot_bytes(KL, bt.nu, ncomp);
  if (s.ring == 0) return cudaErrorInvalidValue;
  const size_t sm = (size_t)s.ring * s.slot_bytes;
  dim3 grid((bt.NP + 31) / 32, bt.paired ? 2 : 1);
  const int threads = 64 * ncomp;
  if (bt.nu == KL + 1)
    imm_solve_kernel<KL, KL + 1><<<grid, threads, sm, st>>>(s);
  else
    imm_solve_kernel<KL, 2 * KL><<<grid, threads, sm, st>>>(s);
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
  imm_stage01_kernel<K><<<grid, 32 * kStageWarps, sm, st>>>(a, vel_n, nl_n, nl_j, bt.F);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = solve_launch<K>(bt, 0, bt.F, 1, NM, Ny, a.NKX, a.NZ1, st);
  if (e != cudaSuccess) return e;
  imm_stage3_kernel<K><<<grid, 32 * kStageWarps, sm, st>>>(a, vel_n, nl_n, nl_j, bt.F, bt.R);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = solve_launch<K>(bt, 1, bt.R, 3, NM, Ny, a.NKX, a.NZ1, st);
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
      (const void*)imm_stage01_kernel<2>, (const void*)imm_stage01_kernel<4>,
      (const void*)imm_stage01_kernel<6>, (const void*)imm_stage01_kernel<8>,
      (const void*)imm_stage3_kernel<2>,  (const void*)imm_stage3_kernel<4>,
      (const void*)imm_stage3_kernel<6>,  (const void*)imm_stage3_kernel<8>,
      (const void*)imm_solve_kernel<2, 3>, (const void*)imm_solve_kernel<2, 4>,
      (const void*)imm_solve_kernel<4, 5>, (const void*)imm_solve_kernel<4, 8>,
      (const void*)imm_solve_kernel<6, 7>, (const void*)imm_solve_kernel<6, 12>,
      (const void*)imm_solve_kernel<8, 9>, (const void*)imm_solve_kernel<8, 16>};
  cudaError_t e = cudaSuccess;
  for (const void* f : fns) {
    cudaError_t r = allow_dynamic_smem(f, max_smem);
    if (r != cudaSuccess) e = r;
  }
  return e;
}

}  // namespace dnsb
