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

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

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
template <int KL, int RS>
__device__ __forceinline__ void forward_chain(const double* __restrict__ AB,
                                              const int* __restrict__ dpiv,
                                              double* __restrict__ b, int Ny) {
  constexpr int W = KL + 1;  // window b[j .. j+KL]; slot(o, ph) = (o+ph) % W
  double w[W];
#pragma unroll
  for (int o = 0; o < W; ++o) w[o] = (o < Ny) ? b[2 * o] : 0.0;
  const int nsteps = Ny - 1;
  double bb[W];  // element entering the window at each step of the block
#pragma unroll
  for (int ph = 0; ph < W; ++ph) {
    const int e = ph + W;
    bb[ph] = (e < Ny) ? b[2 * e] : 0.0;
  }
  for (int j0 = 0; j0 < nsteps; j0 += W) {
    double bn[W];
#pragma unroll
    for (int ph = 0; ph < W; ++ph) {
      const int e = j0 + 2 * W + ph;
      bn[ph] = (e < Ny) ? b[2 * e] : 0.0;
    }
#pragma unroll
    for (int ph = 0; ph < W; ++ph) {
      const int j = j0 + ph;
      if (j < nsteps) {
        const int d = dpiv[j];
        double bpj = w[ph % W];
        if (d != 0) {  // warp-uniform: every lane solves the same mode
#pragma unroll
          for (int i = 1; i <= KL; ++i)
            if (d == i) bpj = w[(i + ph) % W];
#pragma unroll
          for (int i = 1; i <= KL; ++i)
            if (d == i) w[(i + ph) % W] = w[ph % W];
        }
        b[2 * j] = bpj;
        const double* L = AB + j * RS;
#pragma unroll
        for (int i = 1; i <= KL; ++i) w[(i + ph) % W] -= L[i - 1] * bpj;
        w[ph % W] = bb[ph];  // offset 0 leaves; b[j+KL+1] enters at offset KL
      }
    }
#pragma unroll
    for (int ph = 0; ph < W; ++ph) bb[ph] = bn[ph];
  }
  // b[Ny-1] sits at offset 0 after the last step: slot nsteps % W.
  const int last = nsteps % W;
  double v = w[0];
#pragma unroll
  for (int s = 1; s < W; ++s)
    if (last == s) v = w[s];
  b[2 * (Ny - 1)] = v;
}

// Back substitution with U (2*KL superdiagonals, the NU nearest stored).
template <int KL, int NU, int RS>
__device__ __forceinline__ void backward_chain(const double* __restrict__ AB,
                                               double* __restrict__ b, int Ny) {
  constexpr int KUU = 2 * KL;
  constexpr int W = KUU + 1;  // window b[j-KUU .. j]; slot(o, ph) = (o-ph) mod W
  double w[W];
#pragma unroll
  for (int o = 0; o < W; ++o) {
    const int idx = Ny - 1 - KUU + o;
    w[o] = (idx >= 0) ? b[2 * idx] : 0.0;
  }
  double bb[W];
#pragma unroll
  for (int ph = 0; ph < W; ++ph) {
    const int e = Ny - 1 - ph - W;
    bb[ph] = (e >= 0) ? b[2 * e] : 0.0;
  }
  for (int j0 = Ny - 1; j0 >= 0; j0 -= W) {
    double bn[W];
#pragma unroll
    for (int ph = 0; ph < W; ++ph) {
      const int e = j0 - 2 * W - ph;
      bn[ph] = (e >= 0) ? b[2 * e] : 0.0;
    }
#pragma unroll
    for (int ph = 0; ph < W; ++ph) {
      const int j = j0 - ph;
      if (j >= 0) {
        const double* r = AB + j * RS;
        const int st = ((KUU - ph) % W + W) % W;
        const double xj = w[st] * r[KL];
        b[2 * j] = xj;
#pragma unroll
        for (int i = 1; i <= NU; ++i) {
          const int si = ((KUU - i - ph) % W + W) % W;
          w[si] -= r[KL + i] * xj;
        }
        w[st] = bb[ph];  // b[j-KUU-1] enters at offset 0
      }
    }
#pragma unroll
    for (int ph = 0; ph < W; ++ph) bb[ph] = bn[ph];
  }
}

// Shared memory of one mode: T[3][Ny] staged stencil inputs, f[Ny],
// R[3][Ny] (double2), factor records Ny x RS (double), pivot offsets Ny.
size_t imm_mode_smem(int Ny, int kl, int nu) {
  const int rs = (kl + 1 + nu + 1) & ~1;
  return sizeof(double2) * (size_t)(7 * Ny) + sizeof(double) * (size_t)(Ny * rs) +
         sizeof(int) * (size_t)Ny;
}

// Stage one operator's factors of mode m into the record layout and its
// validated pivot offsets; flags a pivot outside [j, j+KL].
template <int KL, int NU, int RS>
__device__ __forceinline__ void stage_factors(double* AB, int* dpiv,
                                              const double* __restrict__ ab,
                                              const int* __restrict__ piv,
                                              int Ny, int row0, int lane) {
  constexpr int KUU = 2 * KL;
  // L multipliers: rows KUU+1 .. KUU+KL -> record slots 0..KL-1
#pragma unroll
  for (int i = 1; i <= KL; ++i)
    for (int j = lane; j < Ny; j += 32)
      cp_async8(AB + j * RS + (i - 1), ab + (KUU + i) * Ny + j);
  // diagonal -> slot KL (inverted after arrival)
  for (int j = lane; j < Ny; j += 32) cp_async8(AB + j * RS + KL, ab + KUU * Ny + j);
  // U rows KUU-i for i = 1..NU -> slots KL+i; rows above row0 are zero
#pragma unroll
  for (int i = 1; i <= NU; ++i) {
    const int r = KUU - i;
    for (int j = lane; j < Ny; j += 32) {
      if (r >= row0) cp_async8(AB + j * RS + KL + i, ab + r * Ny + j);
      else AB[j * RS + KL + i] = 0.0;
    }
  }
  for (int j = lane; j < Ny; j += 32) cp_async4(dpiv + j, piv + j);
  cp_async_commit();
}

template <int KL>
__device__ __forceinline__ void finish_factors(double* AB, int* dpiv, int RS,
                                               int Ny, int lane, int* status) {
  for (int j = lane; j < Ny; j += 32) {
    AB[j * RS + KL] = 1.0 / AB[j * RS + KL];
    int d = dpiv[j] - j;
    if (d < 0 || d > KL || j + d >= Ny) {  // never follow a bad pivot
      if (status) atomicOr(status, 1);
      d = 0;
    }
    dpiv[j] = d;
  }
}

template <int KL, int NU>
__global__ void __launch_bounds__(32)
imm_mode_kernel(ImmArgs a, const double2* __restrict__ vel_n,
                const double2* vel_j, const double2* __restrict__ nl_n,
                const double2* __restrict__ nl_j, double2* vel_new,
                double2* corr_out, double* __restrict__ partials) {
  constexpr int ROWS = 3 * KL + 1;
  constexpr int RS = Rec<KL, NU>::kStride;
  constexpr int S1 = KL + 1, S2 = KL + 2;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x;
  const int NKX = a.NKX, Ny = a.Ny;
  const int NM = a.NZ1 * NKX;
  const int m = blockIdx.x;
  const int row0 = a.ab_row0;
  double2* T = sm;          // [3][Ny]
  double2* f = T + 3 * Ny;  // f_hat -> p_P
  double2* R = f + Ny;      // [3][Ny] R -> (u, v, w)_arb
  double* AB = reinterpret_cast<double*>(R + 3 * Ny);
  int* dpiv = reinterpret_cast<int*>(AB + Ny * RS);

  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  const bool k2zero = (k2 == 0.0);
  const double c = a.c, dt = a.dt, nu = a.nu;
  const double omc = 1.0 - c;
  const double omc_nu = omc * nu;
  const long long CS = (long long)NM * Ny;
  const long long mo = (long long)m * Ny;
  const long long abase = (long long)m * ROWS * Ny;
  const int* d1j = a.d1_j0;
  const double* d1w = a.d1_w;
  const int* d2j = a.d2_j0;
  const double* d2w = a.d2_w;
  const double2 *un = vel_n + mo, *vn = vel_n + CS + mo, *wn = vel_n + 2 * CS + mo;
  const double2 *Nun = nl_n + mo, *Nvn = nl_n + CS + mo, *Nwn = nl_n + 2 * CS + mo;
  const double2 *Nuj = nl_j + mo, *Nvj = nl_j + CS + mo, *Nwj = nl_j + 2 * CS + mo;

  stage_factors<KL, NU, RS>(AB, dpiv, a.Lk_ab + abase, a.Lk_piv + mo, Ny, row0, lane);

  // d_hat^n = i kx u + D1 v + i kz w  -> T[2]
  for (int y = lane; y < Ny; y += 32) T[y] = vn[y];
  __syncwarp();
  for (int y = lane; y < Ny; y += 32)
    T[2 * Ny + y] = cadd(cadd(cik(kx, un[y]), sband<S1>(T, d1j, d1w, y)), cik(kz, wn[y]));
  __syncwarp();
  // Stage 1: f_hat (wall rows zero)
  for (int y = lane; y < Ny; y += 32) {
    T[y] = Nvj[y];
    T[Ny + y] = Nvn[y];
  }
  __syncwarp();
  for (int y = lane; y < Ny; y += 32) {
    double2 fy = make_double2(0.0, 0.0);
    if (y > 0 && y < Ny - 1) {
      const double2 divNj = cadd(cadd(cik(kx, Nuj[y]), sband<S1>(T, d1j, d1w, y)),
                                 cik(kz, Nwj[y]));
      const double2 divNn = cadd(cadd(cik(kx, Nun[y]), sband<S1>(T + Ny, d1j, d1w, y)),
                                 cik(kz, Nwn[y]));
      const double2 dy = T[2 * Ny + y];
      const double2 Lkd = csub(sband<S2>(T + 2 * Ny, d2j, d2w, y), cscale(dy, k2));
      const double2 dd = make_double2(dy.x / dt, dy.y / dt);
      fy = cadd(cadd(cadd(dd, cscale(divNj, c)), cscale(divNn, omc)),
                cscale(Lkd, omc_nu));
    }
    f[y] = fy;
  }
  cp_async_wait_all();
  __syncwarp();
  finish_factors<KL>(AB, dpiv, RS, Ny, lane, a.status);
  __syncwarp();
  // Stage 2: p_P = Lk^-1 f_hat (real / imaginary columns on lanes 0, 1)
  if (lane < 2) {
    double* col = reinterpret_cast<double*>(f) + lane;
    forward_chain<KL, RS>(AB, dpiv, col, Ny);
    backward_chain<KL, NU, RS>(AB, col, Ny);
  }
  __syncwarp();
  stage_factors<KL, NU, RS>(AB, dpiv, a.Hk_ab + abase, a.Hk_piv + mo, Ny, row0, lane);
  // Stage 3: R = Hk^- u^n - grad p_P + c N_j + (1-c) N_n (wall rows zero)
  for (int y = lane; y < Ny; y += 32) {
    T[y] = un[y];
    T[Ny + y] = vn[y];
    T[2 * Ny + y] = wn[y];
  }
  __syncwarp();
  const double idt = 1.0 / dt;
  for (int y = lane; y < Ny; y += 32) {
    double2 ru = make_double2(0.0, 0.0), rv = ru, rw = ru;
    if (y > 0 && y < Ny - 1) {
      const double2 p = f[y];
      const double2 dxp = cik(kx, p);
      const double2 dyp = sband<S1>(f, d1j, d1w, y);
      const double2 dzp = cik(kz, p);
      const double2 u = T[y], v = T[Ny + y], w = T[2 * Ny + y];
      const double2 D2u = sband<S2>(T, d2j, d2w, y);
      const double2 D2v = sband<S2>(T + Ny, d2j, d2w, y);
      const double2 D2w = sband<S2>(T + 2 * Ny, d2j, d2w, y);
      const double2 hu = cadd(cscale(u, idt), cscale(csub(D2u, cscale(u, k2)), omc_nu));
      const double2 hv = cadd(cscale(v, idt), cscale(csub(D2v, cscale(v, k2)), omc_nu));
      const double2 hw = cadd(cscale(w, idt), cscale(csub(D2w, cscale(w, k2)), omc_nu));
      ru = cadd(cadd(csub(hu, dxp), cscale(Nuj[y], c)), cscale(Nun[y], omc));
      rv = cadd(cadd(csub(hv, dyp), cscale(Nvj[y], c)), cscale(Nvn[y], omc));
      rw = cadd(cadd(csub(hw, dzp), cscale(Nwj[y], c)), cscale(Nwn[y], omc));
    }
    R[y] = ru;
    R[Ny + y] = rv;
    R[2 * Ny + y] = rw;
  }
  cp_async_wait_all();
  __syncwarp();
  finish_factors<KL>(AB, dpiv, RS, Ny, lane, a.status);
  __syncwarp();
  // Helmholtz solves for u_arb, v_arb, w_arb (6 real columns, lanes 0..5)
  if (lane < 6) {
    double* col = reinterpret_cast<double*>(R + (lane >> 1) * Ny) + (lane & 1);
    forward_chain<KL, RS>(AB, dpiv, col, Ny);
    backward_chain<KL, NU, RS>(AB, col, Ny);
  }
  __syncwarp();
  // Stages 4-5: wall divergence and influence-matrix weights
  const double2* va = R + Ny;
  double2 dw0 = sband<S1>(va, d1j, d1w, 0);
  const double2 dw1 = sband<S1>(va, d1j, d1w, Ny - 1);
  if (k2zero) dw0 = make_double2(0.0, 0.0);
  const double* Mi = a.M_inv + (long long)m * 4;
  const double2 a1 = make_double2(-(Mi[0] * dw0.x + Mi[1] * dw1.x),
                                  -(Mi[0] * dw0.y + Mi[1] * dw1.y));
  const double2 a2 = make_double2(-(Mi[2] * dw0.x + Mi[3] * dw1.x),
                                  -(Mi[2] * dw0.y + Mi[3] * dw1.y));
  // Stage 6: assemble, store, correction norm
  const double km = (ix == 0) ? 1.0 : 2.0;
  const double* v1 = a.v1 + mo;
  const double* v2 = a.v2 + mo;
  const double* q1 = a.q1 + mo;
  const double* q2 = a.q2 + mo;
  double acc = 0.0;
  for (int y = lane; y < Ny; y += 32) {
    const double2 vnew = cadd(cadd(R[Ny + y], cscale(a1, v1[y])), cscale(a2, v2[y]));
    const double2 q = cadd(cscale(a1, q1[y]), cscale(a2, q2[y]));
    const double2 unew = csub(R[y], cik(kx, q));
    const double2 wnew = csub(R[2 * Ny + y], cik(kz, q));
    const double2 cu = csub(unew, vel_j[mo + y]);
    const double2 cv = csub(vnew, vel_j[CS + mo + y]);
    const double2 cw = csub(wnew, vel_j[2 * CS + mo + y]);
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

bool imm_v2_supported(int kl) { return kl == 2 || kl == 4 || kl == 6 || kl == 8; }

// Stored U rows: the nearest NU superdiagonals; NU = kl+1 when the rows
// above ab_row0 leave at most that many, else all 2 kl.
static int imm_nu(int kl, int row0) {
  const int nu = 2 * kl - row0;
  return nu <= kl + 1 ? kl + 1 : 2 * kl;
}

size_t imm_v2_smem(int Ny, int kl, int row0) {
  return imm_mode_smem(Ny, kl, imm_nu(kl, row0));
}

#define DNSB_IMM_CASE(KL_)                                                      \
  case KL_:                                                                     \
    if (nuv == KL_ + 1)                                                         \
      imm_mode_kernel<KL_, KL_ + 1><<<NM, 32, sm, st>>>(a, vel_n, vel_j, nl_n,  \
                                                        nl_j, vel_new, corr_out, \
                                                        partials);              \
    else                                                                        \
      imm_mode_kernel<KL_, 2 * KL_><<<NM, 32, sm, st>>>(a, vel_n, vel_j, nl_n,  \
                                                        nl_j, vel_new, corr_out, \
                                                        partials);              \
    break;

cudaError_t launch_imm_v2(const ImmArgs& a, const double2* vel_n,
                          const double2* vel_j, const double2* nl_n,
                          const double2* nl_j, double2* vel_new,
                          double2* corr_out, double* partials, cudaStream_t st) {
  const int NM = a.NZ1 * a.NKX;
  const int nuv = imm_nu(a.kl, a.ab_row0);
  const size_t sm = imm_mode_smem(a.Ny, a.kl, nuv);
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
