// Plane Couette influence-matrix iteration, one warp per (kz, kx) mode,
// with the banded LU substitutions run as register-window recurrences.
//
// Follows src/dnsjax/flows/plane_couette.py:376-504 (six stages) and the
// dgbtrs-'N' substitution of src/dnsjax/geometries/cartesian.py:360-441.
//
// Per mode (one 32-thread CTA):
//   * the mode's LAPACK `ab` factors are staged with cp.async into a
//     per-column record  [L multipliers (kl) | 1/U_jj | U_{j-1,j} ..
//     U_{j-NU,j}]  so a substitution step reads one contiguous record;
//     rows above `ab_row0` (zero for every mode -- checked when the
//     operators are bound) are neither read nor applied;
//   * each real right-hand-side column is one lane.  Forward elimination
//     keeps b[j..j+kl] in a circular register window (row interchange =
//     select; skipped by a warp-uniform branch when the pivot is the
//     diagonal), back substitution keeps b[j-2kl..j]; both loops are
//     unrolled by the window length so the window never moves between
//     registers, and the inputs entering the window are loaded one block
//     ahead;
//   * stencil inputs (D1, D2 along y) are staged in shared memory.
#include "solver.cuh"

namespace dnsb {

// Banded stencil row y applied to x (S taps from column j0[y]).
template <int S>
__device__ __forceinline__ double2 sband(const double2* x, const int* __restrict__ j0,
                                         const double* __restrict__ w, int y) {
  const int j = j0[y];
  const double* wy = w + y * S;
  double2 acc = make_double2(0.0, 0.0);
#pragma unroll
  for (int m = 0; m < S; ++m) {
    const double2 v = x[j + m];
    acc.x += wy[m] * v.x;
    acc.y += wy[m] * v.y;
  }
  return acc;
}

// Column record of the staged factors: [0, KL) L multipliers of rows
// j+1..j+KL, [KL] 1/U_jj, [KL+1, KL+1+NU) U_{j-1,j} .. U_{j-NU,j}.
template <int KL, int NU>
struct Rec {
  static constexpr int kLen = KL + 1 + NU;
  static constexpr int kStride = (kLen + 1) & ~1;  // even: 16-B records
};

// Forward elimination (row interchange + L update, dgbtrs 'N') on one real
// column b (stride 2) of length Ny.  dpiv[j] = ipiv[j] - j in [0, KL].
// The window holds b[j..j+KL] in registers, slot(o, ph) = (o + ph) % W; the
// loop is unrolled by W so slots are compile-time.  Each block of W steps
// first loads its multipliers (16-byte pairs), pivots and entering values
// into registers, then runs the recurrence from registers.  The row
// interchange is chosen once per block (warp-uniform: every lane solves
// the same factors): no interchange, interchanges with the next row only
// (two selects per step), or the general case (a switch per step).  Full
// blocks carry no per-step bounds test; the last, partial block does.
template <int KL, int MODE, bool TAIL>
__device__ __forceinline__ void forward_steps(double* __restrict__ b, int j0, int nsteps,
                                              double (&w)[KL + 1],
                                              const double (&Lr)[KL + 1][KL],
                                              const int (&dr)[KL + 1],
                                              const double (&be)[KL + 1]) {
  constexpr int W = KL + 1;
#pragma unroll
  for (int ph = 0; ph < W; ++ph) {
    const int j = j0 + ph;
    if (!TAIL || j < nsteps) {
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
      b[2 * j] = bpj;
#pragma unroll
      for (int i = 1; i <= KL; ++i) w[(i + ph) % W] -= Lr[ph][i - 1] * bpj;
      w[ph % W] = be[ph];  // offset 0 leaves; b[j+W] enters at offset KL
    }
  }
}

template <int KL, int RS, bool TAIL>
__device__ __forceinline__ void forward_load(const double* __restrict__ AB,
                                             const int* __restrict__ dpiv,
                                             const double* __restrict__ b, int j0,
                                             int nsteps, int Ny,
                                             double (&Lr)[KL + 1][KL], int (&dr)[KL + 1],
                                             double (&be)[KL + 1]) {
  constexpr int W = KL + 1;
  static_assert(KL % 2 == 0, "multipliers are loaded in pairs");
#pragma unroll
  for (int ph = 0; ph < W; ++ph) {
    const int j = TAIL ? min(j0 + ph, nsteps - 1) : j0 + ph;
    const double2* rec = reinterpret_cast<const double2*>(AB + j * RS);
#pragma unroll
    for (int i = 0; i < KL / 2; ++i) {
      const double2 t = rec[i];
      Lr[ph][2 * i] = t.x;
      Lr[ph][2 * i + 1] = t.y;
    }
    dr[ph] = dpiv[j];
    const int e = j0 + ph + W;
    be[ph] = (e < Ny) ? b[2 * e] : 0.0;
  }
}

template <int KL, int RS>
__device__ __forceinline__ void forward_chain(const double* __restrict__ AB,
                                              const int* __restrict__ dpiv,
                                              double* __restrict__ b, int Ny) {
  constexpr int W = KL + 1;
  double w[W];
#pragma unroll
  for (int o = 0; o < W; ++o) w[o] = (o < Ny) ? b[2 * o] : 0.0;
  const int nsteps = Ny - 1;
  const int jfull = (nsteps / W) * W;
  double Lr[W][KL];
  int dr[W];
  double be[W];
  for (int j0 = 0; j0 < jfull; j0 += W) {
    forward_load<KL, RS, false>(AB, dpiv, b, j0, nsteps, Ny, Lr, dr, be);
    int dm = 0;
#pragma unroll
    for (int ph = 0; ph < W; ++ph) dm = max(dm, dr[ph]);
    if (dm == 0)
      forward_steps<KL, 0, false>(b, j0, nsteps, w, Lr, dr, be);
    else if (dm == 1)
      forward_steps<KL, 1, false>(b, j0, nsteps, w, Lr, dr, be);
    else
      forward_steps<KL, 2, false>(b, j0, nsteps, w, Lr, dr, be);
  }
  if (jfull < nsteps) {
    forward_load<KL, RS, true>(AB, dpiv, b, jfull, nsteps, Ny, Lr, dr, be);
    forward_steps<KL, 2, true>(b, jfull, nsteps, w, Lr, dr, be);
  }
  // b[Ny-1] sits at offset 0 after the last step: slot nsteps % W.
  const int last = nsteps % W;
  double v = w[0];
#pragma unroll
  for (int s = 1; s < W; ++s)
    if (last == s) v = w[s];
  b[2 * (Ny - 1)] = v;
}

// Phases PH0 <= ph < PH1 of a back-substitution block starting at row j0
// (row j = j0 - ph).  Record slot KL holds 1/U_jj and slots KL+i hold
// U_{j-i,j}/U_jj (i = 1..NU), so the recurrence is one FMA deep:
// b[j-i] -= that * b[j]; x_j = b[j] / U_jj is stored off the dependency
// chain.  The window holds b[j-NU..j], slot(o, ph) = (o - ph) mod W with
// W = NU + 1: superdiagonals beyond NU are zero and never applied.
template <int KL, int NU, int RS, int PH0, int PH1, bool TAIL>
__device__ __forceinline__ void backward_part(const double* __restrict__ AB,
                                              double* __restrict__ b, int j0,
                                              double (&w)[NU + 1]) {
  constexpr int W = NU + 1;
  constexpr int H = PH1 - PH0;
  constexpr int NP = (NU + 2) / 2;  // 16-byte pairs covering slots KL..KL+NU
  static_assert(KL % 2 == 0, "U records are loaded in pairs");
  double Ur[H][2 * NP];
  double be[H];
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const int j = TAIL ? max(j0 - (PH0 + h), 0) : j0 - (PH0 + h);
    const double2* rec = reinterpret_cast<const double2*>(AB + j * RS + KL);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double2 t = rec[i];
      Ur[h][2 * i] = t.x;
      Ur[h][2 * i + 1] = t.y;
    }
    const int e = j0 - (PH0 + h) - W;
    be[h] = (e >= 0) ? b[2 * e] : 0.0;
  }
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const int ph = PH0 + h;
    const int j = j0 - ph;
    if (!TAIL || j >= 0) {
      const int st = ((NU - ph) % W + W) % W;
      const double bj = w[st];
      b[2 * j] = bj * Ur[h][0];
#pragma unroll
      for (int i = 1; i <= NU; ++i) {
        const int si = ((NU - i - ph) % W + W) % W;
        w[si] -= Ur[h][i] * bj;
      }
      w[st] = be[h];  // b[j-NU-1] enters at offset 0
    }
  }
}

// Back substitution with U (its NU nearest superdiagonals) on one real
// column b (stride 2), in blocks of W = NU + 1 rows, each loaded in two
// register halves.
template <int KL, int NU, int RS>
__device__ __forceinline__ void backward_chain(const double* __restrict__ AB,
                                               double* __restrict__ b, int Ny) {
  constexpr int W = NU + 1;
  constexpr int H = (W + 1) / 2;
  double w[W];
#pragma unroll
  for (int o = 0; o < W; ++o) {
    const int idx = Ny - 1 - NU + o;
    w[o] = (idx >= 0) ? b[2 * idx] : 0.0;
  }
  const int nfull = Ny / W;
  int j0 = Ny - 1;
  for (int blk = 0; blk < nfull; ++blk, j0 -= W) {
    backward_part<KL, NU, RS, 0, H, false>(AB, b, j0, w);
    backward_part<KL, NU, RS, H, W, false>(AB, b, j0, w);
  }
  if (j0 >= 0) {
    backward_part<KL, NU, RS, 0, H, true>(AB, b, j0, w);
    backward_part<KL, NU, RS, H, W, true>(AB, b, j0, w);
  }
}

// Both substitutions on one real column.  Kept out of line: the L_k and
// H_k solves share one copy of the fully unrolled recurrences, which keeps
// the kernel's hot code within the instruction cache.
template <int KL, int NU, int RS>
__device__ __noinline__ void lu_solve_column(const double* __restrict__ AB,
                                             const int* __restrict__ dpiv,
                                             double* __restrict__ b, int Ny) {
  forward_chain<KL, RS>(AB, dpiv, b, Ny);
  backward_chain<KL, NU, RS>(AB, b, Ny);
}

// Shared memory of one work item (1 or 2 modes sharing factors): per mode
// T[3][Ny] staged stencil inputs, f[Ny], R[3][Ny] (double2); factor records
// Ny x RS (double); pivot offsets Ny.
size_t imm_mode_smem(int Ny, int kl, int nu, int qmax) {
  const int rs = (kl + 1 + nu + 1) & ~1;
  return sizeof(double2) * (size_t)(7 * qmax * Ny) +
         sizeof(double) * (size_t)(Ny * rs) + sizeof(int) * (size_t)Ny;
}

// y values per lane: y = lane + 32 k, k < kYM (Ny <= 32 kYM).
constexpr int kYM = 5;

// Stage one operator's factors of mode m into the record layout and its
// pivots (threads tid = 0..nthr-1 of the CTA share the copies).
template <int KL, int NU, int RS>
__device__ __forceinline__ void stage_factors(double* AB, int* dpiv,
                                              const double* __restrict__ ab,
                                              const int* __restrict__ piv,
                                              int Ny, int row0, int tid, int nthr) {
  constexpr int KUU = 2 * KL;
  // L multipliers: rows KUU+1 .. KUU+KL -> record slots 0..KL-1
#pragma unroll
  for (int i = 1; i <= KL; ++i)
    for (int j = tid; j < Ny; j += nthr)
      cp_async8(AB + j * RS + (i - 1), ab + (KUU + i) * Ny + j);
  // diagonal -> slot KL (inverted after arrival)
  for (int j = tid; j < Ny; j += nthr) cp_async8(AB + j * RS + KL, ab + KUU * Ny + j);
  // U rows KUU-i for i = 1..NU -> slots KL+i; rows above row0 are zero
#pragma unroll
  for (int i = 1; i <= NU; ++i) {
    const int r = KUU - i;
    for (int j = tid; j < Ny; j += nthr) {
      if (r >= row0) cp_async8(AB + j * RS + KL + i, ab + r * Ny + j);
      else AB[j * RS + KL + i] = 0.0;
    }
  }
  for (int j = tid; j < Ny; j += nthr) cp_async4(dpiv + j, piv + j);
  cp_async_commit();
}

// After the staged factors arrived: slot KL <- 1/U_jj, U slots scaled by it,
// pivots turned into validated offsets (a pivot outside [j, j+KL] is flagged
// and not followed).
template <int KL, int NU>
__device__ __forceinline__ void finish_factors(double* AB, int* dpiv, int RS,
                                               int Ny, int tid, int nthr, int* status) {
  for (int j = tid; j < Ny; j += nthr) {
    const double r = 1.0 / AB[j * RS + KL];
    AB[j * RS + KL] = r;
#pragma unroll
    for (int i = 1; i <= NU; ++i) AB[j * RS + KL + i] *= r;
    int d = dpiv[j] - j;
    if (d < 0 || d > KL || j + d >= Ny) {  // never follow a bad pivot
      if (status) atomicOr(status, 1);
      d = 0;
    }
    dpiv[j] = d;
  }
}

// One work item: mode (s, kx), and, when `paired`, also its mirror
// (nz-1-s, kx) -- the same k^2 = kx^2 + kz^2 and therefore bit-identical L_k
// and H_k factors (checked when the operators are bound).  The CTA has one
// warp per mode of the item: all its threads stage each operator's factors
// once, then every warp runs its own mode's stages and substitution chains
// (2 / 6 lanes).  Stencil inputs are staged with cp.async (the stage-3
// staging overlaps the L_k substitution); pointwise inputs are loaded into
// registers for all of a lane's y values before they are used.
template <int KL, int NU>
__global__ void __launch_bounds__(64)
imm_mode_kernel(ImmArgs a, const double2* __restrict__ vel_n,
                const double2* vel_j, const double2* __restrict__ nl_n,
                const double2* __restrict__ nl_j, double2* vel_new,
                double2* corr_out, double* __restrict__ partials, int paired) {
  constexpr int ROWS = 3 * KL + 1;
  constexpr int RS = Rec<KL, NU>::kStride;
  constexpr int S1 = KL + 1, S2 = KL + 2;
  constexpr int YM = kYM;
  extern __shared__ double2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int q = tid >> 5;  // this warp's mode of the item
  const int lane = tid & 31;
  const int NKX = a.NKX, Ny = a.Ny, NZ1 = a.NZ1;
  const int NM = NZ1 * NKX;
  const int item = blockIdx.x;
  const int row0 = a.ab_row0;
  int m0 = item, m = item;
  bool mine = true;  // warp-uniform: the (s = 0, kx) items have one mode
  if (paired) {
    const int ixp = item % NKX, s = item / NKX;
    m0 = s * NKX + ixp;
    m = (q == 0) ? m0 : (NZ1 - s) * NKX + ixp;
    mine = (q == 0) || (s != 0);
  }
  const int qmax = nthr >> 5;
  double2* T = sm + q * 7 * Ny;  // staged stencil inputs [3][Ny]
  double2* F = T + 3 * Ny;       // f_hat, then p_P
  double2* R = F + Ny;           // d_hat^n, then R / (u, v, w)_arb
  double* AB = reinterpret_cast<double*>(sm + 7 * qmax * Ny);
  int* dpiv = reinterpret_cast<int*>(AB + Ny * RS);

  const double c = a.c, dt = a.dt, nu = a.nu;
  const double omc = 1.0 - c;
  const double omc_nu = omc * nu;
  const double idt = 1.0 / dt;
  const long long CS = (long long)NM * Ny;
  const int* d1j = a.d1_j0;
  const double* d1w = a.d1_w;
  const int* d2j = a.d2_j0;
  const double* d2w = a.d2_w;
  const long long abase = (long long)m0 * ROWS * Ny;
  const long long pbase = (long long)m0 * Ny;
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  const long long mo = (long long)m * Ny;

  // group: stencil inputs of stages 0-1 (v^n, N^j_v, N^n_v)
  if (mine) {
    for (int y = lane; y < Ny; y += 32) {
      cp_async16(T + y, vel_n + CS + mo + y);
      cp_async16(T + Ny + y, nl_j + CS + mo + y);
      cp_async16(T + 2 * Ny + y, nl_n + CS + mo + y);
    }
  }
  cp_async_commit();
  // group: L_k factors
  stage_factors<KL, NU, RS>(AB, dpiv, a.Lk_ab + abase, a.Lk_piv + pbase, Ny, row0, tid, nthr);
  cp_async_wait_1();
  __syncwarp();

  if (mine) {
    // Stage 0: d_hat^n = div u^n (kept in R until stage 3)
    {
      double2 ua[YM], wa[YM];
#pragma unroll
      for (int k = 0; k < YM; ++k) {
        const int y = lane + 32 * k;
        if (y < Ny) {
          ua[k] = vel_n[mo + y];
          wa[k] = vel_n[2 * CS + mo + y];
        }
      }
#pragma unroll
      for (int k = 0; k < YM; ++k) {
        const int y = lane + 32 * k;
        if (y < Ny)
          R[y] = cadd(cadd(cik(kx, ua[k]), sband<S1>(T, d1j, d1w, y)), cik(kz, wa[k]));
      }
    }
    __syncwarp();
    // Stage 1: f_hat (wall rows zero)
    double2 uj[YM], wj[YM], un_[YM], wn_[YM];
#pragma unroll
    for (int k = 0; k < YM; ++k) {
      const int y = lane + 32 * k;
      if (y < Ny) {
        uj[k] = nl_j[mo + y];
        wj[k] = nl_j[2 * CS + mo + y];
        un_[k] = nl_n[mo + y];
        wn_[k] = nl_n[2 * CS + mo + y];
      }
    }
#pragma unroll
    for (int k = 0; k < YM; ++k) {
      const int y = lane + 32 * k;
      if (y >= Ny) continue;
      double2 fy = make_double2(0.0, 0.0);
      if (y > 0 && y < Ny - 1) {
        const double2 divNj = cadd(cadd(cik(kx, uj[k]), sband<S1>(T + Ny, d1j, d1w, y)),
                                   cik(kz, wj[k]));
        const double2 divNn = cadd(cadd(cik(kx, un_[k]), sband<S1>(T + 2 * Ny, d1j, d1w, y)),
                                   cik(kz, wn_[k]));
        const double2 dy = R[y];
        const double2 Lkd = csub(sband<S2>(R, d2j, d2w, y), cscale(dy, k2));
        const double2 dd = make_double2(dy.x / dt, dy.y / dt);
        fy = cadd(cadd(cadd(dd, cscale(divNj, c)), cscale(divNn, omc)),
                  cscale(Lkd, omc_nu));
      }
      F[y] = fy;
    }
  }
  __syncwarp();
  // group: stencil inputs of stage 3 (u^n, v^n, w^n); overlaps the L_k solve
  if (mine) {
    for (int y = lane; y < Ny; y += 32) {
      cp_async16(T + y, vel_n + mo + y);
      cp_async16(T + Ny + y, vel_n + CS + mo + y);
      cp_async16(T + 2 * Ny + y, vel_n + 2 * CS + mo + y);
    }
  }
  cp_async_commit();
  cp_async_wait_1();  // L_k factors complete
  __syncthreads();
  finish_factors<KL, NU>(AB, dpiv, RS, Ny, tid, nthr, a.status);
  __syncthreads();
  // Stage 2: p_P = Lk^-1 f_hat (real / imaginary columns)
  if (mine && lane < 2) {
    double* col = reinterpret_cast<double*>(F) + lane;
    lu_solve_column<KL, NU, RS>(AB, dpiv, col, Ny);
  }
  __syncthreads();  // every warp is done with the L_k factors
  // group: H_k factors; overlaps stage 3
  stage_factors<KL, NU, RS>(AB, dpiv, a.Hk_ab + abase, a.Hk_piv + pbase, Ny, row0, tid, nthr);
  cp_async_wait_1();  // stage-3 stencil inputs complete
  __syncwarp();
  if (mine) {
    // Stage 3: R = Hk^- u^n - grad p_P + c N_j + (1-c) N_n (wall rows zero)
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
#pragma unroll
    for (int k = 0; k < YM; ++k) {
      const int y = lane + 32 * k;
      if (y >= Ny) continue;
      double2 ru = make_double2(0.0, 0.0), rv = ru, rw = ru;
      if (y > 0 && y < Ny - 1) {
        const double2 p = F[y];
        const double2 dxp = cik(kx, p);
        const double2 dyp = sband<S1>(F, d1j, d1w, y);
        const double2 dzp = cik(kz, p);
        const double2 u = T[y], v = T[Ny + y], w = T[2 * Ny + y];
        const double2 D2u = sband<S2>(T, d2j, d2w, y);
        const double2 D2v = sband<S2>(T + Ny, d2j, d2w, y);
        const double2 D2w = sband<S2>(T + 2 * Ny, d2j, d2w, y);
        const double2 hu = cadd(cscale(u, idt), cscale(csub(D2u, cscale(u, k2)), omc_nu));
        const double2 hv = cadd(cscale(v, idt), cscale(csub(D2v, cscale(v, k2)), omc_nu));
        const double2 hw = cadd(cscale(w, idt), cscale(csub(D2w, cscale(w, k2)), omc_nu));
        ru = cadd(cadd(csub(hu, dxp), cscale(nj[0][k], c)), cscale(nn[0][k], omc));
        rv = cadd(cadd(csub(hv, dyp), cscale(nj[1][k], c)), cscale(nn[1][k], omc));
        rw = cadd(cadd(csub(hw, dzp), cscale(nj[2][k], c)), cscale(nn[2][k], omc));
      }
      R[y] = ru;
      R[Ny + y] = rv;
      R[2 * Ny + y] = rw;
    }
  }
  cp_async_wait_all();  // H_k factors complete
  __syncthreads();
  finish_factors<KL, NU>(AB, dpiv, RS, Ny, tid, nthr, a.status);
  __syncthreads();
  // Helmholtz solves for u_arb, v_arb, w_arb (6 real columns)
  if (mine && lane < 6) {
    double* b = reinterpret_cast<double*>(R + (lane >> 1) * Ny) + (lane & 1);
    lu_solve_column<KL, NU, RS>(AB, dpiv, b, Ny);
  }
  __syncwarp();
  if (!mine) return;
  double2 vj[3][YM];
  double c1[YM], c2[YM], e1[YM], e2[YM];
#pragma unroll
  for (int k = 0; k < YM; ++k) {
    const int y = lane + 32 * k;
    if (y < Ny) {
#pragma unroll
      for (int cpt = 0; cpt < 3; ++cpt) vj[cpt][k] = vel_j[cpt * CS + mo + y];
      c1[k] = a.v1[mo + y];
      c2[k] = a.v2[mo + y];
      e1[k] = a.q1[mo + y];
      e2[k] = a.q2[mo + y];
    }
  }
  // Stages 4-5: wall divergence and influence-matrix weights
  const double2* va = R + Ny;
  double2 dw0 = sband<S1>(va, d1j, d1w, 0);
  const double2 dw1 = sband<S1>(va, d1j, d1w, Ny - 1);
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
    const double2 vnew = cadd(cadd(R[Ny + y], cscale(a1, c1[k])), cscale(a2, c2[k]));
    const double2 qq = cadd(cscale(a1, e1[k]), cscale(a2, e2[k]));
    const double2 unew = csub(R[y], cik(kx, qq));
    const double2 wnew = csub(R[2 * Ny + y], cik(kz, qq));
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

bool imm_v2_supported(int kl, int ny) {
  return (kl == 2 || kl == 4 || kl == 6 || kl == 8) && ny <= 32 * kYM;
}

// Stored U rows: the nearest NU superdiagonals; NU = kl+1 when the rows
// above ab_row0 leave at most that many, else all 2 kl.
int imm_nu(int kl, int row0) {
  const int nu = 2 * kl - row0;
  return nu <= kl + 1 ? kl + 1 : 2 * kl;
}

size_t imm_v2_smem(int Ny, int kl, int row0) {
  return imm_mode_smem(Ny, kl, imm_nu(kl, row0), 2);
}

#define DNSB_IMM_CASE(KL_)                                                      \
  case KL_:                                                                     \
    if (nuv == KL_ + 1)                                                         \
      imm_mode_kernel<KL_, KL_ + 1><<<items, threads, sm, st>>>(                     \
          a, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials, paired);    \
    else                                                                        \
      imm_mode_kernel<KL_, 2 * KL_><<<items, threads, sm, st>>>(                     \
          a, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials, paired);    \
    break;

cudaError_t launch_imm_v2(const ImmArgs& a, const double2* vel_n,
                          const double2* vel_j, const double2* nl_n,
                          const double2* nl_j, double2* vel_new,
                          double2* corr_out, double* partials, cudaStream_t st) {
  const int NM = a.NZ1 * a.NKX;
  const int paired = a.pair_modes ? 1 : 0;
  // paired: items (s, kx) with s in [0, (nz-1+1)/2); s = 0 is alone
  const int items = paired ? ((a.NZ1 + 1) / 2) * a.NKX : NM;
  const int nuv = imm_nu(a.kl, a.ab_row0);
  const size_t sm = imm_mode_smem(a.Ny, a.kl, nuv, paired ? 2 : 1);
  const int threads = paired ? 64 : 32;  // one warp per mode of an item
  switch (a.kl) {
    DNSB_IMM_CASE(2)
    DNSB_IMM_CASE(4)
    DNSB_IMM_CASE(6)
    DNSB_IMM_CASE(8)
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// Whether mode (s, kx) and its mirror (nz-1-s, kx) have bit-identical LU
// factors and pivots for every s in [1, (nz-1)/2] and kx: out[0] |= 1 on
// any difference.
__global__ void ab_pair_check_kernel(const double* __restrict__ ab,
                                     const int* __restrict__ piv, int nz1,
                                     int nkx, int rows, int ny, int* out) {
  const int npos = (nz1 - 1) / 2;  // s = 1 .. npos
  const long long per = (long long)(rows + 1) * ny;
  const long long n = (long long)npos * nkx * per;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long item = i / per;
    const long long e = i % per;
    const int s = 1 + (int)(item / nkx), ix = (int)(item % nkx);
    const long long ma = (long long)s * nkx + ix;
    const long long mb = (long long)(nz1 - s) * nkx + ix;
    bool same;
    if (e < (long long)rows * ny) {
      same = __double_as_longlong(ab[ma * rows * ny + e]) ==
             __double_as_longlong(ab[mb * rows * ny + e]);
    } else {
      const long long j = e - (long long)rows * ny;
      same = piv[ma * ny + j] == piv[mb * ny + j];
    }
    if (!same) atomicOr(out, 1);
  }
}

cudaError_t launch_ab_pair_check(const double* ab, const int* piv, int nz1,
                                 int nkx, int rows, int ny, int* out,
                                 cudaStream_t st) {
  ab_pair_check_kernel<<<592, 256, 0, st>>>(ab, piv, nz1, nkx, rows, ny, out);
  return cudaGetLastError();
}

// First ab row (below the kl+ku diagonal offset) holding a nonzero entry in
// any mode; rows above it are skipped by the register-window kernel.  out[0]
// starts at kuu (the diagonal row) and is lowered atomically.
__global__ void ab_first_row_kernel(const double* __restrict__ ab, long long nmodes,
                                    int rows, int ny, int kuu, int* out) {
  const long long per = (long long)kuu * ny;
  const long long n = nmodes * per;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long mm = i / per;
    const long long r = (i % per) / ny;
    const long long j = i % ny;
    const double v = ab[(mm * rows + r) * ny + j];
    if (!(v == 0.0)) atomicMin(out, (int)r);
  }
}

cudaError_t launch_ab_first_row(const double* ab, long long nmodes, int rows,
                                int ny, int kuu, int* out, cudaStream_t st) {
  ab_first_row_kernel<<<592, 256, 0, st>>>(ab, nmodes, rows, ny, kuu, out);
  return cudaGetLastError();
}

cudaError_t set_imm_v2_attributes(int max_smem) {
  cudaError_t e = cudaSuccess;
  const void* fns[] = {
      (const void*)imm_mode_kernel<2, 3>,  (const void*)imm_mode_kernel<2, 4>,
      (const void*)imm_mode_kernel<4, 5>,  (const void*)imm_mode_kernel<4, 8>,
      (const void*)imm_mode_kernel<6, 7>,  (const void*)imm_mode_kernel<6, 12>,
      (const void*)imm_mode_kernel<8, 9>,  (const void*)imm_mode_kernel<8, 16>};
  for (const void* f : fns) {
    cudaError_t r = allow_dynamic_smem(f, max_smem);
    if (r != cudaSuccess) e = r;
  }
  return e;
}

}  // namespace dnsb
