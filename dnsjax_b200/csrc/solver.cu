// Per-mode influence-matrix solve (plane Couette), banded LU substitution,
// periodic Helmholtz / corrector / projection kernels and deterministic
// FP64 reductions.
#include "solver.cuh"

namespace dnsb {

// ---------------------------------------------------------------------------
// Reductions: fixed grid, fixed per-thread order, tree in shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? red[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  return v;
}

__device__ __forceinline__ void finalize_body(const double* partials, int n, double* out,
                                              double scale, int do_sqrt) {
  // each thread adds its partials in index order; the loads of eight at a
  // time are issued together (the sum is the plain loop's, bit for bit)
  double s = 0.0;
  const int bd = blockDim.x;
  int i = threadIdx.x;
  for (; i + 7 * bd < n; i += 8 * bd) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = partials[i + k * bd];
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k];
  }
  for (; i < n; i += bd) s += partials[i];
  s = block_sum(s);
  if (threadIdx.x == 0) {
    s *= scale;
    out[0] = do_sqrt ? sqrt(s) : s;
  }
}

__global__ void finalize_kernel(const double* partials, int n, double* out,
                                double scale, int do_sqrt, const int* skip) {
  if (skip && *skip) return;
  finalize_body(partials, n, out, scale, do_sqrt);
}

cudaError_t launch_finalize(const double* partials, int n, double* out,
                            double scale, int do_sqrt, cudaStream_t st, const int* skip) {
  finalize_kernel<<<1, 1024, 0, st>>>(partials, n, out, scale, do_sqrt, skip);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Periodic pointwise kernels (monochromatic.py:320-355, 516-565).
// ---------------------------------------------------------------------------
// The pointwise bodies run as block vb of a grid of vgrid blocks (the
// kernels: blockIdx.x, gridDim.x; the work-list ensemble kernels: their own
// numbering, with the same vgrid, so sums are the same bit for bit).
__device__ __forceinline__ void periodic_predict_body(const PeriodicPointArgs& a,
                                                      const double2* __restrict__ state,
                                                      const double2* __restrict__ rhs,
                                                      double2* __restrict__ out, int vb,
                                                      int vgrid) {
  const long long n = 3LL * a.S;
  for (long long i = vb * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)vgrid * blockDim.x) {
    const int s = (int)(i % a.S);
    const double l1 = a.ldt_1[s], l2 = a.ildt_2[s];
    const double2 u = state[i], r = rhs[i];
    // (state * ldt_1 + rhs) * ildt_2
    out[i] = cscale(cadd(cscale(u, l1), r), l2);
  }
}

__global__ void periodic_predict_kernel(PeriodicPointArgs a,
                                        const double2* __restrict__ state,
                                        const double2* __restrict__ rhs,
                                        double2* __restrict__ out) {
  periodic_predict_body(a, state, rhs, out, blockIdx.x, gridDim.x);
}

cudaError_t launch_periodic_predict(const PeriodicPointArgs& a,
                                    const double2* state, const double2* rhs,
                                    double2* out, cudaStream_t st) {
  periodic_predict_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, state, rhs, out);
  return cudaGetLastError();
}

__device__ __forceinline__ void periodic_correct_body(const PeriodicPointArgs& a,
                                                      const double2* pred,
                                                      const double2* __restrict__ prev,
                                                      const double2* __restrict__ next,
                                                      double2* pred_out, double2* corr_out,
                                                      double* __restrict__ partials, int vb,
                                                      int vgrid) {
  const long long n = 3LL * a.S;
  double acc = 0.0;
  for (long long i = vb * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)vgrid * blockDim.x) {
    const int s = (int)(i % a.S);
    const double l2 = a.ildt_2[s];
    // c * (next - prev) * ildt_2
    const double2 corr = cscale(cscale(csub(next[i], prev[i]), a.c), l2);
    pred_out[i] = cadd(pred[i], corr);
    if (corr_out) corr_out[i] = corr;
    const double km = (s % a.NKX == 0 && a.kx0) ? 1.0 : 2.0;
    acc += km * (corr.x * corr.x + corr.y * corr.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0 && partials) partials[vb] = acc;
}

__global__ void periodic_correct_kernel(PeriodicPointArgs a,
                                        const double2* pred,
                                        const double2* __restrict__ prev,
                                        const double2* __restrict__ next,
                                        double2* pred_out, double2* corr_out,
                                        double* __restrict__ partials) {
  if (a.skip && *a.skip) return;
  periodic_correct_body(a, pred, prev, next, pred_out, corr_out, partials, blockIdx.x,
                        gridDim.x);
}

cudaError_t launch_periodic_correct(const PeriodicPointArgs& a,
                                    const double2* pred,
                                    const double2* rhs_prev,
                                    const double2* rhs_next, double2* pred_out,
                                    double2* corr_out, double* partials,
                                    cudaStream_t st) {
  periodic_correct_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(
      a, pred, rhs_prev, rhs_next, pred_out, corr_out, partials);
  return cudaGetLastError();
}

__global__ void periodic_norm2_kernel(PeriodicPointArgs a,
                                      const double2* __restrict__ v,
                                      double* __restrict__ partials) {
  const long long n = 3LL * a.S;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i % a.S);
    const double2 z = v[i];
    const double km = (s % a.NKX == 0 && a.kx0) ? 1.0 : 2.0;
    acc += km * (z.x * z.x + z.y * z.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

cudaError_t launch_periodic_norm2(const PeriodicPointArgs& a,
                                  const double2* v, double* partials,
                                  cudaStream_t st) {
  periodic_norm2_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, v, partials);
  return cudaGetLastError();
}

__global__ void periodic_stats_kernel(PeriodicPointArgs a,
                                      const double2* __restrict__ v,
                                      double* __restrict__ partials) {
  const long long n = 3LL * a.S;
  double e = 0.0, ens = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i % a.S);
    const double2 z = v[i];
    const double m2 = z.x * z.x + z.y * z.y;
    e += ((s % a.NKX == 0 && a.kx0) ? 1.0 : 2.0) * m2;
    ens += -a.lapl[s] * m2;
  }
  e = block_sum(e);
  __syncthreads();
  ens = block_sum(ens);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = e;
    partials[gridDim.x + blockIdx.x] = ens;
  }
}

cudaError_t launch_periodic_stats(const PeriodicPointArgs& a,
                                  const double2* v, double* partials,
                                  cudaStream_t st) {
  periodic_stats_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, v, partials);
  return cudaGetLastError();
}

// u - grad(inv_lapl div u), then (zero_mean) the mean mode set to zero.
__device__ __forceinline__ void periodic_cv_body(const PeriodicPointArgs& a, const double2* in,
                                                 double2* out, int divergence, int zero_mean,
                                                 int vb, int vgrid) {
  const int S = a.S;
  for (int s = vb * blockDim.x + threadIdx.x; s < S; s += vgrid * blockDim.x) {
    double2 u0 = in[s], u1 = in[S + s], u2 = in[2 * S + s];
    if (divergence) {
      const int ix = s % a.NKX;
      const int iz = (s / a.NKX) % a.NZ1;
      const int iy = s / (a.NKX * a.NZ1);
      const double kx = a.kx[ix], ky = a.ky[iy], kz = a.kz[iz];
      const double2 div = cadd(cadd(cik(kx, u0), cik(ky, u1)), cik(kz, u2));
      const double2 p = cscale(div, a.inv_lapl[s]);
      // state + (-grad p)
      const double2 g0 = cik(kx, p), g1 = cik(ky, p), g2 = cik(kz, p);
      u0 = cadd(u0, make_double2(-g0.x, -g0.y));
      u1 = cadd(u1, make_double2(-g1.x, -g1.y));
      u2 = cadd(u2, make_double2(-g2.x, -g2.y));
    }
    if (s == 0 && zero_mean && a.kx0) {
      u0 = u1 = u2 = make_double2(0.0, 0.0);
    }
    out[s] = u0;
    out[S + s] = u1;
    out[2 * S + s] = u2;
  }
}

__global__ void periodic_cv_kernel(PeriodicPointArgs a,
                                   const double2* in, double2* out,
                                   int divergence, int zero_mean) {
  if (a.skip && *a.skip) return;
  periodic_cv_body(a, in, out, divergence, zero_mean, blockIdx.x, gridDim.x);
}

cudaError_t launch_periodic_correct_velocity(const PeriodicPointArgs& a,
                                             const double2* in, double2* out,
                                             int divergence, cudaStream_t st) {
  periodic_cv_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, in, out, divergence, 1);
  return cudaGetLastError();
}

// The RHS projection NL - grad(inv_lapl div NL) (monochromatic.py:377-385),
// in place, the mean mode kept.
cudaError_t launch_periodic_project(const PeriodicPointArgs& a, double2* rhs,
                                   cudaStream_t st) {
  periodic_cv_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, rhs, rhs, 1, 0);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Work-list forms for ensembles (csrc/capi.cu, dnsb_ensemble_*): every
// member's kRedBlocks virtual blocks of the pointwise kernels in one launch,
// members whose `active` flag is 0 skipped.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool ens_skip(const int* active, int m) {
  return active && !active[m];
}

__global__ void __launch_bounds__(kRedThreads)
ens_point_kernel(const EnsPointItem* __restrict__ items, int n, const int* __restrict__ active,
                 int op, int divergence, int zero_mean) {
  const int total = n * kRedBlocks;
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    const int k = vb / kRedBlocks, b = vb % kRedBlocks;
    const EnsPointItem it = items[k];
    if (!ens_skip(active, it.member)) {
      if (op == 0)
        periodic_predict_body(it.a, it.in0, it.in1, it.out, b, kRedBlocks);
      else if (op == 1)
        periodic_correct_body(it.a, it.in0, it.in1, it.in2, it.out, nullptr, it.partials, b,
                              kRedBlocks);
      else
        periodic_cv_body(it.a, it.in0, it.out, divergence, zero_mean, b, kRedBlocks);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(1024)
ens_finalize_kernel(const EnsPointItem* __restrict__ items, const int* __restrict__ active,
                    double* err) {
  const EnsPointItem& it = items[blockIdx.x];
  if (ens_skip(active, it.member)) return;
  finalize_body(it.partials, kRedBlocks, err + it.member, 1.0, 1);
}

cudaError_t launch_ens_point(const EnsPointItem* items, int n, const int* active, int op,
                             int divergence, int zero_mean, int grid, cudaStream_t st) {
  ens_point_kernel<<<grid, kRedThreads, 0, st>>>(items, n, active, op, divergence, zero_mean);
  return cudaGetLastError();
}

cudaError_t launch_ens_finalize(const EnsPointItem* items, int n, const int* active,
                                double* err, cudaStream_t st) {
  ens_finalize_kernel<<<n, 1024, 0, st>>>(items, active, err);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Banded LU substitution for one real column (dgbtrs 'N', LAPACK ab
// packing: A[i][j] at ab[kl+ku+i-j][j]); cartesian.py:360-441.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void banded_solve_col(
    const double* __restrict__ ab, const int* __restrict__ piv, double* b,
    int bs, int Ny, int kl, int ku, int* status) {
  const int kuu = kl + ku;
  for (int j = 0; j < Ny - 1; ++j) {
    int p = piv[j];
    if (p < j || p > j + kl || p >= Ny) {
      if (status) atomicOr(status, 1);
      p = j;
    }
    const double bpj = b[p * bs];
    if (p != j) {
      b[p * bs] = b[j * bs];
      b[j * bs] = bpj;
    }
    const int lim = min(kl, Ny - 1 - j);
    for (int i = 1; i <= lim; ++i)
      b[(j + i) * bs] -= ab[(kuu + i) * Ny + j] * bpj;
  }
  for (int j = Ny - 1; j >= 0; --j) {
    const double xj = b[j * bs] / ab[kuu * Ny + j];
    b[j * bs] = xj;
    const int lim = min(kuu, j);
    for (int i = 1; i <= lim; ++i)
      b[(j - i) * bs] -= ab[(kuu - i) * Ny + j] * xj;
  }
}

__global__ void banded_solve_kernel(const double* __restrict__ ab,
                                    const int* __restrict__ ipiv, double* b,
                                    int nmodes, int ny, int kl, int ku,
                                    int ncols, int* status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nmodes * ncols) return;
  const int m = t / ncols, col = t % ncols;
  const int rows = 2 * kl + ku + 1;
  banded_solve_col(ab + (long long)m * rows * ny, ipiv + (long long)m * ny,
                   b + (long long)m * ny * ncols + col, ncols, ny, kl, ku,
                   status);
}

cudaError_t launch_banded_solve(const double* ab, const int* ipiv, double* b,
                                int nmodes, int ny, int kl, int ku,
                                int ncols, int* status, cudaStream_t st) {
  const int n = nmodes * ncols;
  banded_solve_kernel<<<(n + 127) / 128, 128, 0, st>>>(ab, ipiv, b, nmodes,
                                                      ny, kl, ku, ncols, status);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Plane Couette: six-stage Kleiser-Schumann IMM, one warp per (kz, kx)
// mode (plane_couette.py:376-504).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ double2 band_apply(const T* x, const int* j0,
                                              const double* w, int s, int y) {
  const int j = j0[y];
  const double* wy = w + (long long)y * s;
  double2 acc = make_double2(0.0, 0.0);
  for (int m = 0; m < s; ++m) {
    const double2 v = x[j + m];
    acc.x += wy[m] * v.x;
    acc.y += wy[m] * v.y;
  }
  return acc;
}

size_t imm_smem(int Ny) {
  return sizeof(double2) * (size_t)(5 * Ny) * kImmWarps;
}

__global__ void __launch_bounds__(32 * kImmWarps)
imm_kernel(ImmArgs a, const double2* __restrict__ vel_n,
           const double2* vel_j, const double2* __restrict__ nl_n,
           const double2* __restrict__ nl_j, double2* vel_new,
           double2* corr_out, double* __restrict__ partials) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int NKX = a.NKX, Ny = a.Ny;
  const int NM = a.NZ1 * NKX;
  const int m = blockIdx.x * kImmWarps + warp;
  if (m >= NM) return;  // whole warp leaves; only __syncwarp below
  double2* d = sm + (size_t)warp * 5 * Ny;
  double2* f = d + Ny;
  double2* R = f + Ny;  // [3][Ny]
  const int iz = m / NKX, ix = m % NKX;
  const double kx = a.kx[ix], kz = a.kz[iz];
  const double k2 = kx * kx + kz * kz;
  const bool k2zero = (k2 == 0.0);
  const double c = a.c, dt = a.dt, nu = a.nu;
  const double omc = 1.0 - c;
  const double omc_nu = omc * nu;
  const long long CS = (long long)NM * Ny;
  const long long mo = (long long)m * Ny;
  const double2 *un = vel_n + mo, *vn = vel_n + CS + mo, *wn = vel_n + 2 * CS + mo;
  const double2 *Nun = nl_n + mo, *Nvn = nl_n + CS + mo, *Nwn = nl_n + 2 * CS + mo;
  const double2 *Nuj = nl_j + mo, *Nvj = nl_j + CS + mo, *Nwj = nl_j + 2 * CS + mo;

  // d_hat^n = i kx u + D1 v + i kz w
  for (int y = lane; y < Ny; y += 32) {
    const double2 dyv = band_apply(vn, a.d1_j0, a.d1_w, a.s1, y);
    d[y] = cadd(cadd(cik(kx, un[y]), dyv), cik(kz, wn[y]));
  }
  __syncwarp();
  // Stage 1: f_hat (wall rows zero)
  for (int y = lane; y < Ny; y += 32) {
    double2 fy = make_double2(0.0, 0.0);
    if (y > 0 && y < Ny - 1) {
      const double2 divNj = cadd(cadd(cik(kx, Nuj[y]),
                                      band_apply(Nvj, a.d1_j0, a.d1_w, a.s1, y)),
                                 cik(kz, Nwj[y]));
      const double2 divNn = cadd(cadd(cik(kx, Nun[y]),
                                      band_apply(Nvn, a.d1_j0, a.d1_w, a.s1, y)),
                                 cik(kz, Nwn[y]));
      const double2 D2d = band_apply(d, a.d2_j0, a.d2_w, a.s2, y);
      const double2 Lkd = csub(D2d, cscale(d[y], k2));
      const double2 dd = make_double2(d[y].x / dt, d[y].y / dt);
      fy = cadd(cadd(cadd(dd, cscale(divNj, c)), cscale(divNn, omc)),
                cscale(Lkd, omc_nu));
    }
    f[y] = fy;
  }
  __syncwarp();
  // Stage 2: p_P = Lk^-1 f_hat (real and imaginary columns on lanes 0, 1)
  const int rows = 2 * a.kl + a.ku + 1;
  if (lane < 2) {
    banded_solve_col(a.Lk_ab + mo * rows, a.Lk_piv + mo,
                     reinterpret_cast<double*>(f) + lane, 2, Ny, a.kl, a.ku,
                     a.status);
  }
  __syncwarp();
  // Stage 3: R = Hk^- u^n - grad p_P + c N_j + (1-c) N_n (wall rows zero)
  for (int y = lane; y < Ny; y += 32) {
    double2 ru = make_double2(0.0, 0.0), rv = ru, rw = ru;
    if (y > 0 && y < Ny - 1) {
      const double2 p = f[y];
      const double2 dxp = cik(kx, p);
      const double2 dyp = band_apply(f, a.d1_j0, a.d1_w, a.s1, y);
      const double2 dzp = cik(kz, p);
      const double idt = 1.0 / dt;
      const double2 u = un[y], v = vn[y], w = wn[y];
      const double2 D2u = band_apply(un, a.d2_j0, a.d2_w, a.s2, y);
      const double2 D2v = band_apply(vn, a.d2_j0, a.d2_w, a.s2, y);
      const double2 D2w = band_apply(wn, a.d2_j0, a.d2_w, a.s2, y);
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
  __syncwarp();
  // Helmholtz solves for u_arb, v_arb, w_arb (6 real columns, lanes 0..5)
  if (lane < 6) {
    banded_solve_col(a.Hk_ab + mo * rows, a.Hk_piv + mo,
                     reinterpret_cast<double*>(R + (lane >> 1) * Ny) + (lane & 1),
                     2, Ny, a.kl, a.ku, a.status);
  }
  __syncwarp();
  // Stage 4-5: wall divergence and influence-matrix weights
  const double2* va = R + Ny;
  double2 dw0 = band_apply(va, a.d1_j0, a.d1_w, a.s1, 0);
  const double2 dw1 = band_apply(va, a.d1_j0, a.d1_w, a.s1, Ny - 1);
  if (k2zero) dw0 = make_double2(0.0, 0.0);
  const double* Mi = a.M_inv + (long long)m * 4;
  const double2 a1 = make_double2(-(Mi[0] * dw0.x + Mi[1] * dw1.x),
                                  -(Mi[0] * dw0.y + Mi[1] * dw1.y));
  const double2 a2 = make_double2(-(Mi[2] * dw0.x + Mi[3] * dw1.x),
                                  -(Mi[2] * dw0.y + Mi[3] * dw1.y));
  // Stage 6: assemble, store, correction norm
  const double km = (ix == 0 && a.kx0) ? 1.0 : 2.0;
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
  acc = warp_sum(acc);
  if (lane == 0 && partials) partials[m] = acc;
}

cudaError_t launch_imm(const ImmArgs& a, const double2* vel_n,
                       const double2* vel_j, const double2* nl_n,
                       const double2* nl_j, double2* vel_new,
                       double2* corr_out, double* partials, cudaStream_t st) {
  const int NM = a.NZ1 * a.NKX;
  const int grid = (NM + kImmWarps - 1) / kImmWarps;
  imm_kernel<<<grid, 32 * kImmWarps, imm_smem(a.Ny), st>>>(
      a, vel_n, vel_j, nl_n, nl_j, vel_new, corr_out, partials);
  return cudaGetLastError();
}

__global__ void couette_norm2_kernel(ImmArgs a, const double2* __restrict__ v,
                                     double* __restrict__ partials) {
  const int NM = a.NZ1 * a.NKX;
  const long long n = 3LL * NM * a.Ny;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % a.Ny);
    const int m = (int)((i / a.Ny) % NM);
    const double km = (m % a.NKX == 0 && a.kx0) ? 1.0 : 2.0;
    const double2 z = v[i];
    acc += a.simpson[y] * km * (z.x * z.x + z.y * z.y);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

cudaError_t launch_couette_norm2(const ImmArgs& a, const double2* v,
                                 double* partials, cudaStream_t st) {
  couette_norm2_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(a, v, partials);
  return cudaGetLastError();
}

cudaError_t set_solver_attributes(int max_smem) {
  return allow_dynamic_smem((const void*)imm_kernel, max_smem);
}

}  // namespace dnsb
