// Influence-matrix precompute for plane Couette on the GPU: for every
// (kz, kx) mode, the LAPACK-ab banded LU factors of L_k (Neumann pressure
// operator) and H_k (Dirichlet Helmholtz operator), the homogeneous
// solutions p1, p2, v1, v2, q1, q2 and the inverted 2x2 influence matrix.
//
// Follows src/dnsjax/geometries/cartesian.py:575-801 (precompute_imm, banded
// backend): build_Lk_neumann (:491-526), build_Hk_dirichlet (:529-572),
// _pack_banded (:291-320) and _banded_lu_numpy (:323-357, SciPy gbtrf).
//
//   factor   one thread per (operator, mode): the operator's band entries
//            packed as ab[kl+ku+i-j][j] = A[i][j] (the first kl rows zero),
//            then LAPACK's unblocked banded LU (dgbtf2, the code dgbtrf runs
//            when its block size exceeds kl) in place; pivots 0-based.
//   p1, p2   L_k^-1 e_0 and L_k^-1 e_{Ny-1} with the banded substitution.
//   v, q     H_k^-1 of (-D1 p1, -D1 p2, p1, p2), wall rows zeroed.
//   M_inv    M = [D1[0] . v1, D1[0] . v2; D1[Ny-1] . v1, D1[Ny-1] . v2],
//            inverted; [[0, 0], [0, 1 / M11]] for k^2 = 0.
//
// The operator entries are formed with the reference's operation order and
// single roundings (no contraction), so the matrices handed to the
// factorisation equal the reference's.  The reference solves for p, v, q
// with dense LU (numpy.linalg.solve); here they use the banded factors, so
// those vectors agree with the reference's to rounding, not bit for bit.
#include "solver.cuh"

namespace dnsb {

namespace {

__device__ __forceinline__ double op_entry(int op, const double* __restrict__ D1,
                                           const double* __restrict__ D2, int ny, int i, int j,
                                           double k2, double idt, double cn) {
  const double d = (i == j) ? 1.0 : 0.0;
  if (op == 0) {  // L_k = D2 - k2 I, Neumann rows (row 0 pinned when k2 = 0)
    if (i == 0) return (k2 == 0.0) ? d : D1[j];
    if (i == ny - 1) return D1[(long long)(ny - 1) * ny + j];
    return __dsub_rn(D2[(long long)i * ny + j], __dmul_rn(k2, d));
  }
  // H_k = (1/dt) I - (c nu) (D2 - k2 I), identity wall rows
  if (i == 0 || i == ny - 1) return d;
  const double lraw = __dsub_rn(D2[(long long)i * ny + j], __dmul_rn(k2, d));
  return __dsub_rn(__dmul_rn(idt, d), __dmul_rn(cn, lraw));
}

// Build and factor one operator of one mode.  info bit (2 << op) is set
// when a zero pivot is met (LAPACK's info > 0).
__global__ void imm_factor_kernel(const double* __restrict__ D1, const double* __restrict__ D2,
                                  const double* __restrict__ kx, const double* __restrict__ kz,
                                  int nkx, int nkz, int ny, int kl, int ku, double dt, double c,
                                  double nu, double* Lk_ab, int* Lk_piv, double* Hk_ab,
                                  int* Hk_piv, int* info) {
  const int nm = nkx * nkz;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nm) return;
  const int op = t / nm, m = t % nm;
  const int iz = m / nkx, ix = m % nkx;
  const double k2 = __dadd_rn(__dmul_rn(kx[ix], kx[ix]), __dmul_rn(kz[iz], kz[iz]));
  const double idt = __ddiv_rn(1.0, dt), cn = __dmul_rn(c, nu);
  const int rows = 2 * kl + ku + 1, kv = kl + ku;
  double* ab = (op ? Hk_ab : Lk_ab) + (long long)m * rows * ny;
  int* piv = (op ? Hk_piv : Lk_piv) + (long long)m * ny;
  auto AB = [&](int r, int j) -> double& { return ab[(long long)r * ny + j]; };
  // pack (cartesian.py:291-320)
  for (int r = 0; r < rows; ++r)
    for (int j = 0; j < ny; ++j) AB(r, j) = 0.0;
  for (int j = 0; j < ny; ++j) {
    const int lo = max(0, j - ku), hi = min(ny - 1, j + kl);
    for (int i = lo; i <= hi; ++i)
      AB(kv + i - j, j) = op_entry(op, D1, D2, ny, i, j, k2, idt, cn);
  }
  // dgbtf2: column j, pivot among rows j .. j+km, row interchange across
  // columns j .. ju, multipliers scaled by the pivot's reciprocal, rank-1
  // update of the trailing km x (ju - j) block.
  int ju = 0, bad = 0;
  for (int j = 0; j < ny; ++j) {
    const int km = min(kl, ny - 1 - j);
    int jp = 0;
    double amax = fabs(AB(kv, j));
    for (int s = 1; s <= km; ++s) {
      const double a = fabs(AB(kv + s, j));
      if (a > amax) {
        amax = a;
        jp = s;
      }
    }
    piv[j] = j + jp;
    if (AB(kv + jp, j) != 0.0) {
      ju = max(ju, min(j + ku + jp, ny - 1));
      if (jp != 0)
        for (int s = 0; s <= ju - j; ++s) {
          const double x = AB(kv + jp - s, j + s);
          AB(kv + jp - s, j + s) = AB(kv - s, j + s);
          AB(kv - s, j + s) = x;
        }
      if (km > 0) {
        const double r = __ddiv_rn(1.0, AB(kv, j));
        for (int s = 1; s <= km; ++s) AB(kv + s, j) = __dmul_rn(AB(kv + s, j), r);
        for (int q = 1; q <= ju - j; ++q) {
          const double y = AB(kv - q, j + q);
          if (y != 0.0)
            for (int s = 1; s <= km; ++s)
              AB(kv + s - q, j + q) = __fma_rn(-AB(kv + s, j), y, AB(kv + s - q, j + q));
        }
      }
    } else {
      bad = 1;
    }
  }
  if (bad) atomicOr(info, 2 << op);
}

// Right-hand sides e_0, e_{Ny-1} for p1, p2: b[m][y][2].
__global__ void imm_prhs_kernel(double* b, int nm, int ny) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nm * ny) return;
  const int y = (int)(t % ny);
  b[2 * t] = (y == 0) ? 1.0 : 0.0;
  b[2 * t + 1] = (y == ny - 1) ? 1.0 : 0.0;
}

// p1, p2 out; right-hand sides (-D1 p1, -D1 p2, p1, p2), wall rows zero,
// for the H_k solves: bv[m][y][4].
__global__ void imm_vrhs_kernel(const double* __restrict__ D1, const double* __restrict__ bp,
                                double* bv, double* p1, double* p2, int nm, int ny) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nm * ny) return;
  const int y = (int)(t % ny);
  const long long m = t / ny;
  const double* P = bp + m * ny * 2;
  const double* d = D1 + (long long)y * ny;
  double s1 = 0.0, s2 = 0.0;
  for (int j = 0; j < ny; ++j) {
    s1 += d[j] * P[2 * j];
    s2 += d[j] * P[2 * j + 1];
  }
  const double a = P[2 * y], b = P[2 * y + 1];
  p1[t] = a;
  p2[t] = b;
  const bool wall = (y == 0 || y == ny - 1);
  double* o = bv + 4 * t;
  o[0] = wall ? 0.0 : -s1;
  o[1] = wall ? 0.0 : -s2;
  o[2] = wall ? 0.0 : a;
  o[3] = wall ? 0.0 : b;
}

// v1, v2, q1, q2 out.
__global__ void imm_vout_kernel(const double* __restrict__ bv, double* v1, double* v2,
                                double* q1, double* q2, int nm, int ny) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nm * ny) return;
  const double* o = bv + 4 * t;
  v1[t] = o[0];
  v2[t] = o[1];
  q1[t] = o[2];
  q2[t] = o[3];
}

// Influence matrix of each mode and its inverse.
__global__ void imm_minv_kernel(const double* __restrict__ D1, const double* __restrict__ bv,
                                const double* __restrict__ kx, const double* __restrict__ kz,
                                int nkx, int nkz, int ny, double* M_inv) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nkx * nkz) return;
  const int iz = m / nkx, ix = m % nkx;
  const double k2 = __dadd_rn(__dmul_rn(kx[ix], kx[ix]), __dmul_rn(kz[iz], kz[iz]));
  const double* V = bv + (long long)m * ny * 4;
  const double* r0 = D1;
  const double* r1 = D1 + (long long)(ny - 1) * ny;
  double m00 = 0.0, m01 = 0.0, m10 = 0.0, m11 = 0.0;
  for (int j = 0; j < ny; ++j) {
    m00 += r0[j] * V[4 * j];
    m01 += r0[j] * V[4 * j + 1];
    m10 += r1[j] * V[4 * j];
    m11 += r1[j] * V[4 * j + 1];
  }
  double* o = M_inv + 4LL * m;
  if (k2 == 0.0) {
    o[0] = 0.0;
    o[1] = 0.0;
    o[2] = 0.0;
    o[3] = 1.0 / m11;
  } else {
    const double det = m00 * m11 - m01 * m10;
    o[0] = m11 / det;
    o[1] = -m01 / det;
    o[2] = -m10 / det;
    o[3] = m00 / det;
  }
}

}  // namespace

cudaError_t launch_imm_precompute(const ImmPrecomputeArgs& a, double* bp, double* bv,
                                  cudaStream_t st, int* launches) {
  const int nm = a.nkx * a.nkz;
  const long long nmy = (long long)nm * a.ny;
  const int tb = 128;
  const int gy = (int)((nmy + tb - 1) / tb);
  cudaError_t e;
  *launches = 0;
  imm_factor_kernel<<<(2 * nm + tb - 1) / tb, tb, 0, st>>>(
      a.D1, a.D2, a.kx, a.kz, a.nkx, a.nkz, a.ny, a.p, a.p, a.dt, a.c, a.nu, a.Lk_ab, a.Lk_piv,
      a.Hk_ab, a.Hk_piv, a.info);
  ++*launches;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  imm_prhs_kernel<<<gy, tb, 0, st>>>(bp, nm, a.ny);
  ++*launches;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_banded_solve(a.Lk_ab, a.Lk_piv, bp, nm, a.ny, a.p, a.p, 2, a.status, st)) !=
      cudaSuccess)
    return e;
  ++*launches;
  imm_vrhs_kernel<<<gy, tb, 0, st>>>(a.D1, bp, bv, a.p1, a.p2, nm, a.ny);
  ++*launches;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_banded_solve(a.Hk_ab, a.Hk_piv, bv, nm, a.ny, a.p, a.p, 4, a.status, st)) !=
      cudaSuccess)
    return e;
  ++*launches;
  imm_vout_kernel<<<gy, tb, 0, st>>>(bv, a.v1, a.v2, a.q1, a.q2, nm, a.ny);
  ++*launches;
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  imm_minv_kernel<<<(nm + tb - 1) / tb, tb, 0, st>>>(a.D1, bv, a.kx, a.kz, a.nkx, a.nkz, a.ny,
                                                     a.M_inv);
  ++*launches;
  return cudaGetLastError();
}

}  // namespace dnsb
