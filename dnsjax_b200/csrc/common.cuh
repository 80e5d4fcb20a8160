// Shared device code for libdnsb: complex helpers, the shared-memory
// Stockham FFT used by every axis pass, and launch/error plumbing.
//
// FFT conventions follow the reference solver (src/dnsjax/fft.py):
// norm="forward" -- the forward transform divides by the length, the
// inverse applies no factor -- and stored spectral axes omit the Nyquist
// mode.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#define DNSB_MAX_RADIX 8
#define DNSB_MAX_STAGES 12

namespace dnsb {

__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) {
  return make_double2(a.x, -a.y);
}
// i * k * z for real k, evaluated as numpy evaluates 1j * k * z:
// (0 + k i)(a + b i) = (-k b) + (k a) i.
__host__ __device__ __forceinline__ double2 cik(double k, double2 z) {
  return make_double2(-(k * z.y), k * z.x);
}
// i * z
__host__ __device__ __forceinline__ double2 ci(double2 z) {
  return make_double2(-z.y, z.x);
}

// Single-precision complex (the FP32 form of the Couette RHS passes).
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) {
  return make_float2(a.x * s, a.y * s);
}

// Complex type <-> real type and constructor.
template <typename C>
struct cplx;
template <>
struct cplx<double2> {
  using real = double;
  __host__ __device__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <>
struct cplx<float2> {
  using real = float;
  __host__ __device__ static float2 make(float x, float y) { return make_float2(x, y); }
};
template <typename C>
__host__ __device__ __forceinline__ C cmake(typename cplx<C>::real x, typename cplx<C>::real y) {
  return cplx<C>::make(x, y);
}
// FP32 complex whose register DFTs (dft2/3/4/8, dft_3p) carry compensated
// (two-sum) accumulation: the FP32 pass buffers and every other operation
// are those of float2 (same layout); see the compensated DFTs below.
struct __align__(8) cf2 : public float2 {
  cf2() = default;
  __host__ __device__ cf2(float2 v) : float2(v) {}
};
template <>
struct cplx<cf2> {
  using real = float;
  __host__ __device__ static cf2 make(float x, float y) { return cf2(make_float2(x, y)); }
};
// Element types of a pass kernel instantiated on T: double (FP64), float
// (FP32), fcomp (FP32 buffers, compensated butterflies).
struct fcomp {};
template <typename T>
struct pass_types {
  using C = double2;
  using R = double;
};
template <>
struct pass_types<float> {
  using C = float2;
  using R = float;
};
template <>
struct pass_types<fcomp> {
  using C = cf2;
  using R = float;
};

// Conversions between the two precisions.
__host__ __device__ __forceinline__ double2 to_c(double2 z, double2*) { return z; }
__host__ __device__ __forceinline__ float2 to_c(double2 z, float2*) {
  return make_float2((float)z.x, (float)z.y);
}
__host__ __device__ __forceinline__ double2 to_d(double2 z) { return z; }
__host__ __device__ __forceinline__ double2 to_d(float2 z) {
  return make_double2((double)z.x, (double)z.y);
}

// An FFT length L = product of radices (each 2, 3, 4 or 8), applied as
// Stockham auto-sort stages so the output is in natural order.
struct FFTPlan {
  int L;
  int nst;
  int radix[DNSB_MAX_STAGES];
};

// ---- small DFTs in registers; sign = -1 forward, +1 inverse ------------
// Generic over the complex type (double2, float2): the same operations in
// either precision.
template <typename C>
__device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename C>
__device__ __forceinline__ void dft3(C* v, int sign) {
  using R = typename cplx<C>::real;
  const R s3 = (R)0.86602540378443864676;  // sin(2 pi / 3)
  const R half = (R)0.5;
  C t1 = cadd(v[1], v[2]);
  C t2 = cmake<C>(v[0].x - half * t1.x, v[0].y - half * t1.y);
  C d = csub(v[1], v[2]);
  // i * sign * s3 * d
  C t3 = cmake<C>(-sign * s3 * d.y, sign * s3 * d.x);
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}

template <typename C>
__device__ __forceinline__ void dft4(C* v, int sign) {
  C a = cadd(v[0], v[2]);
  C b = csub(v[0], v[2]);
  C c = cadd(v[1], v[3]);
  C d = csub(v[1], v[3]);
  // i * sign * d
  C isd = cmake<C>(-sign * d.y, sign * d.x);
  v[0] = cadd(a, c);
  v[2] = csub(a, c);
  v[1] = cadd(b, isd);
  v[3] = csub(b, isd);
}

template <typename C>
__device__ __forceinline__ void dft8(C* v, int sign) {
  using R = typename cplx<C>::real;
  const R h = (R)0.70710678118654752440;  // sqrt(2)/2
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e, sign);
  dft4(o, sign);
  // twiddles w8^q = exp(sign * 2 pi i q / 8), q = 0..3
  C t1 = cmake<C>(h * (o[1].x - sign * o[1].y), h * (o[1].y + sign * o[1].x));
  C t2 = cmake<C>(-sign * o[2].y, sign * o[2].x);
  C t3 = cmake<C>(h * (-o[3].x - sign * o[3].y), h * (-o[3].y + sign * o[3].x));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], t1);
  v[5] = csub(e[1], t1);
  v[2] = cadd(e[2], t2);
  v[6] = csub(e[2], t2);
  v[3] = cadd(e[3], t3);
  v[7] = csub(e[3], t3);
}

// ---- compensated FP32 butterflies (the cf2 overloads) -----------------------
// Each FP32 value is carried as h + l: a sum or difference keeps its exact
// rounding error (Knuth's two-sum) in l, a product by a constant keeps the
// product's rounding error (from an FMA) and the constant's own FP32 rounding
// error; l is folded back (h + l, one rounding) when the DFT stores its
// outputs.  Only the register DFTs are compensated; the twiddle
// multiplications between stages and the pass buffers stay FP32.
struct ffv {
  float h, l;
};
__device__ __forceinline__ ffv ff_two_sum(float a, float b) {
  const float s = a + b;
  const float bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
__device__ __forceinline__ ffv ff_add(ffv a, ffv b) {
  ffv s = ff_two_sum(a.h, b.h);
  s.l += a.l + b.l;
  return s;
}
__device__ __forceinline__ ffv ff_sub(ffv a, ffv b) {
  ffv s = ff_two_sum(a.h, -b.h);
  s.l += a.l - b.l;
  return s;
}
// a (ch + cl): ch the FP32 constant, cl its rounding error
__device__ __forceinline__ ffv ff_mulc(ffv a, float ch, float cl) {
  const float p = a.h * ch;
  return {p, fmaf(a.h, ch, -p) + (a.h * cl + a.l * ch)};
}
struct cff {
  ffv x, y;
};
__device__ __forceinline__ cff cff_of(float2 v) { return {{v.x, 0.0f}, {v.y, 0.0f}}; }
__device__ __forceinline__ cf2 cff_fold(cff v) {
  return cf2(make_float2(v.x.h + v.x.l, v.y.h + v.y.l));
}
__device__ __forceinline__ cff cff_add(cff a, cff b) { return {ff_add(a.x, b.x), ff_add(a.y, b.y)}; }
__device__ __forceinline__ cff cff_sub(cff a, cff b) { return {ff_sub(a.x, b.x), ff_sub(a.y, b.y)}; }
__device__ __forceinline__ cff cff_scale(cff a, float ch, float cl) {
  return {ff_mulc(a.x, ch, cl), ff_mulc(a.y, ch, cl)};
}
// i * sign * a (exact)
__device__ __forceinline__ cff cff_isign(cff a, int sign) {
  const ffv nx = {-a.y.h, -a.y.l};
  return sign > 0 ? cff{nx, a.x} : cff{a.y, {-a.x.h, -a.x.l}};
}
// FP32 constant and its rounding error, evaluated in double at compile time.
struct fconst {
  float h, l;
};
__host__ __device__ constexpr fconst fsplit(double c) {
  return {(float)c, (float)(c - (double)(float)c)};
}
constexpr fconst kS3 = fsplit(0.86602540378443864676);  // sin(2 pi / 3)
constexpr fconst kH8 = fsplit(0.70710678118654752440);  // sqrt(2) / 2

__device__ __forceinline__ void cff_dft2(cff* v) {
  const cff a = v[0], b = v[1];
  v[0] = cff_add(a, b);
  v[1] = cff_sub(a, b);
}
__device__ __forceinline__ void cff_dft3(cff* v, int sign) {
  const cff t1 = cff_add(v[1], v[2]);
  const cff t2 = cff_sub(v[0], cff_scale(t1, 0.5f, 0.0f));
  const cff t3 = cff_scale(cff_isign(cff_sub(v[1], v[2]), sign), kS3.h, kS3.l);
  v[0] = cff_add(v[0], t1);
  v[1] = cff_add(t2, t3);
  v[2] = cff_sub(t2, t3);
}
__device__ __forceinline__ void cff_dft4(cff* v, int sign) {
  const cff a = cff_add(v[0], v[2]), b = cff_sub(v[0], v[2]);
  const cff c = cff_add(v[1], v[3]), d = cff_sub(v[1], v[3]);
  const cff isd = cff_isign(d, sign);
  v[0] = cff_add(a, c);
  v[2] = cff_sub(a, c);
  v[1] = cff_add(b, isd);
  v[3] = cff_sub(b, isd);
}
__device__ __forceinline__ void cff_dft8(cff* v, int sign) {
  cff e[4] = {v[0], v[2], v[4], v[6]};
  cff o[4] = {v[1], v[3], v[5], v[7]};
  cff_dft4(e, sign);
  cff_dft4(o, sign);
  // twiddles w8^q = exp(sign 2 pi i q / 8): (1 + sign i) h, sign i, (-1 + sign i) h
  const cff t1 = cff_scale(cff_add(o[1], cff_isign(o[1], sign)), kH8.h, kH8.l);
  const cff t2 = cff_isign(o[2], sign);
  const cff t3 = cff_scale(cff_sub(cff_isign(o[3], sign), o[3]), kH8.h, kH8.l);
  v[0] = cff_add(e[0], o[0]);
  v[4] = cff_sub(e[0], o[0]);
  v[1] = cff_add(e[1], t1);
  v[5] = cff_sub(e[1], t1);
  v[2] = cff_add(e[2], t2);
  v[6] = cff_sub(e[2], t2);
  v[3] = cff_add(e[3], t3);
  v[7] = cff_sub(e[3], t3);
}
template <int P>
__device__ __forceinline__ void cff_dft_small(cff* v, int sign) {
  if constexpr (P == 2) cff_dft2(v);
  else if constexpr (P == 3) cff_dft3(v, sign);
  else if constexpr (P == 4) cff_dft4(v, sign);
  else cff_dft8(v, sign);
}
template <int N>
__device__ __forceinline__ void cf2_dft(cf2* v, int sign) {
  cff w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) w[i] = cff_of(v[i]);
  cff_dft_small<N>(w, sign);
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = cff_fold(w[i]);
}
__device__ __forceinline__ void dft2(cf2* v) { cf2_dft<2>(v, 1); }
__device__ __forceinline__ void dft3(cf2* v, int sign) { cf2_dft<3>(v, sign); }
__device__ __forceinline__ void dft4(cf2* v, int sign) { cf2_dft<4>(v, sign); }
__device__ __forceinline__ void dft8(cf2* v, int sign) { cf2_dft<8>(v, sign); }

// One Stockham radix-R stage over C columns stored as buf[t * C + c].
template <int R>
__device__ __forceinline__ void fft_stage(const double2* __restrict__ in,
                                          double2* __restrict__ out, int L,
                                          int C, int Ns, int sign,
                                          const double2* __restrict__ tw) {
  const int nb = L / R;
  const int step = L / (Ns * R);
  const int total = nb * C;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int c = idx % C;
    const int j = idx / C;
    const int k = j % Ns;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[(j + r * nb) * C + c];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      double2 w = tw[r * k * step];
      if (sign > 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    if (R == 2) dft2(v);
    if (R == 3) dft3(v, sign);
    if (R == 4) dft4(v, sign);
    if (R == 8) dft8(v, sign);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[(base + r * Ns) * C + c] = v[r];
  }
}

// Transform C columns of length P.L held in a[t * C + c]; b is scratch of
// the same size.  tw[m] = exp(-2 pi i m / L).  Returns the buffer that
// holds the result.  Ends with __syncthreads().
__device__ inline double2* fft_columns(double2* a, double2* b,
                                       const FFTPlan& P, int C, int sign,
                                       const double2* tw) {
  int Ns = 1;
  double2* in = a;
  double2* out = b;
  for (int s = 0; s < P.nst; ++s) {
    const int R = P.radix[s];
    switch (R) {
      case 2: fft_stage<2>(in, out, P.L, C, Ns, sign, tw); break;
      case 3: fft_stage<3>(in, out, P.L, C, Ns, sign, tw); break;
      case 4: fft_stage<4>(in, out, P.L, C, Ns, sign, tw); break;
      default: fft_stage<8>(in, out, P.L, C, Ns, sign, tw); break;
    }
    __syncthreads();
    double2* t = in;
    in = out;
    out = t;
    Ns *= R;
  }
  return in;
}

// ---- compile-time plans -----------------------------------------------
// Same factorisation rule as make_plan (8s first unless the rest is 8, then
// 4s, 2s, 3s), evaluated at compile time so every stage's stride, twiddle
// step and trip count are constants.
__host__ __device__ constexpr int cplan_radix(int L, int s) {
  int n = L, k = 0;
  while (n % 8 == 0 && n != 8) { if (k == s) return 8; ++k; n /= 8; }
  while (n % 4 == 0 && n > 1) { if (k == s) return 4; ++k; n /= 4; }
  while (n % 2 == 0 && n > 1) { if (k == s) return 2; ++k; n /= 2; }
  while (n % 3 == 0 && n > 1) { if (k == s) return 3; ++k; n /= 3; }
  if (n == 8) { if (k == s) return 8; ++k; }
  return 0;
}
__host__ __device__ constexpr int cplan_nst(int L) {
  int s = 0;
  while (cplan_radix(L, s) != 0) ++s;
  return s;
}

// CT: the complex type of the columns and twiddles (double2, or float2).
template <int L, int R, int C, int NS, int SIGN, int NT, typename CT = double2>
__device__ __forceinline__ void fft_stage_t(const CT* __restrict__ in,
                                            CT* __restrict__ out,
                                            const CT* __restrict__ tw) {
  constexpr int NB = L / R;
  constexpr int STEP = L / (NS * R);
  constexpr int TOTAL = NB * C;
#pragma unroll 2
  for (int idx = threadIdx.x; idx < TOTAL; idx += NT) {
    const int c = idx % C;
    const int j = idx / C;
    const int k = j % NS;
    CT v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[(j + r * NB) * C + c];
    if (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        CT w = tw[r * k * STEP];
        if (SIGN > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    if (R == 2) dft2(v);
    if (R == 3) dft3(v, SIGN);
    if (R == 4) dft4(v, SIGN);
    if (R == 8) dft8(v, SIGN);
    const int base = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[(base + r * NS) * C + c] = v[r];
  }
}

template <int L, int C, int SIGN, int NT, int S = 0, int NS = 1, typename CT = double2>
__device__ __forceinline__ CT* fft_stages_t(CT* a, CT* b, const CT* tw) {
  if constexpr (S >= cplan_nst(L)) {
    return a;
  } else {
    constexpr int R = cplan_radix(L, S);
    fft_stage_t<L, R, C, NS, SIGN, NT, CT>(a, b, tw);
    __syncthreads();
    return fft_stages_t<L, C, SIGN, NT, S + 1, NS * R, CT>(b, a, tw);
  }
}

// Compile-time-planned version of fft_columns (blockDim.x must equal NT).
template <int L, int C, int SIGN, int NT, typename CT = double2>
__device__ __forceinline__ CT* fft_columns_t(CT* a, CT* b, const CT* tw) {
  return fft_stages_t<L, C, SIGN, NT, 0, 1, CT>(a, b, tw);
}

// Dispatch: ML > 0 uses the compile-time plan for length ML, ML == 0 the
// runtime plan (FP64 only).
template <int ML, int C, int NT, typename CT = double2>
__device__ __forceinline__ CT* fft_cols(CT* a, CT* b, const FFTPlan& P, int sign,
                                        const CT* tw) {
  if constexpr (ML > 0) {
    if (sign > 0) return fft_columns_t<ML, C, 1, NT, CT>(a, b, tw);
    return fft_columns_t<ML, C, -1, NT, CT>(a, b, tw);
  } else {
    static_assert(std::is_same<CT, double2>::value, "runtime-planned FFTs are FP64");
    return fft_columns(a, b, P, C, sign, tw);
  }
}

// ---- register DFTs of size N = 3P (P in {2, 3, 4, 8}) --------------------
// tw[m * TS] = exp(-2 pi i m / N) (a length-N*TS table); SIGN -1 forward,
// +1 inverse; natural-order output in v.
template <int P, typename C>
__device__ __forceinline__ void dft_small(C* v, int sign) {
  if constexpr (P == 2) dft2(v);
  else if constexpr (P == 3) dft3(v, sign);
  else if constexpr (P == 4) dft4(v, sign);
  else dft8(v, sign);
}

// Modular inverse of a mod m (a, m coprime), by search (compile time).
__host__ __device__ constexpr int inv_mod(int a, int m) {
  int r = 1;
  while ((a * r) % m != 1) ++r;
  return r;
}

template <int N, int SIGN, typename C>
__device__ __forceinline__ void dft_3p_ct(C* v, const C* __restrict__ tw, int TS);

// PFA: with 3 and P coprime, the prime-factor form (no twiddles); else the
// Cooley-Tukey form with the twiddle table.
template <int N, int SIGN, bool PFA>
__device__ __forceinline__ void dft_3p_comp(cf2* v, const cf2* __restrict__ tw, int TS);

template <int N, int SIGN, typename C, bool PFA = false>
__device__ __forceinline__ void dft_3p(C* v, const C* __restrict__ tw, int TS) {
  constexpr int P = N / 3;
  if constexpr (std::is_same<C, cf2>::value) {
    dft_3p_comp<N, SIGN, PFA>(v, tw, TS);
  } else if constexpr (PFA && P % 3 != 0) {
    // 3 and P coprime: prime-factor (Good-Thomas) DFT, no twiddles.  Input
    // n = (P n1 + 3 n2) mod N; P-point DFTs over n2, 3-point DFTs over n1;
    // output k = (P (P^-1 mod 3) k1 + 3 (3^-1 mod P) k2) mod N (Chinese
    // remainder map).
    constexpr int A = P * inv_mod(P % 3, 3), B = 3 * inv_mod(3 % P, P);
    (void)tw;
    (void)TS;
    C a[3][P];
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1)
#pragma unroll
      for (int n2 = 0; n2 < P; ++n2) a[n1][n2] = v[(P * n1 + 3 * n2) % N];
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) dft_small<P>(a[n1], SIGN);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) {
      C b[3] = {a[0][k2], a[1][k2], a[2][k2]};
      dft3(b, SIGN);
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) v[(A * k1 + B * k2) % N] = b[k1];
    }
  } else {
    dft_3p_ct<N, SIGN>(v, tw, TS);
  }
}

template <int N, int SIGN, typename C>
__device__ __forceinline__ void dft_3p_ct(C* v, const C* __restrict__ tw, int TS) {
  constexpr int P = N / 3;
  C a[3][P];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int p = 0; p < P; ++p) a[q][p] = v[3 * p + q];
#pragma unroll
  for (int q = 0; q < 3; ++q) dft_small<P>(a[q], SIGN);
#pragma unroll
  for (int q = 1; q < 3; ++q)
#pragma unroll
    for (int k1 = 1; k1 < P; ++k1) {
      C w = tw[(q * k1) * TS];
      if (SIGN > 0) w.y = -w.y;
      a[q][k1] = cmul(a[q][k1], w);
    }
#pragma unroll
  for (int k1 = 0; k1 < P; ++k1) {
    C b[3] = {a[0][k1], a[1][k1], a[2][k1]};
    dft3(b, SIGN);
#pragma unroll
    for (int k2 = 0; k2 < 3; ++k2) v[k1 + P * k2] = b[k2];
  }
}

// The compensated form of dft_3p: the P-point and 3-point DFTs (and, in the
// Cooley-Tukey form, the twiddle products between them) stay in h + l
// until the outputs are stored.
template <int N, int SIGN, bool PFA>
__device__ __forceinline__ void dft_3p_comp(cf2* v, const cf2* __restrict__ tw, int TS) {
  constexpr int P = N / 3;
  cff a[3][P];
  if constexpr (PFA && P % 3 != 0) {
    constexpr int A = P * inv_mod(P % 3, 3), B = 3 * inv_mod(3 % P, P);
    (void)tw;
    (void)TS;
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1)
#pragma unroll
      for (int n2 = 0; n2 < P; ++n2) a[n1][n2] = cff_of(v[(P * n1 + 3 * n2) % N]);
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) cff_dft_small<P>(a[n1], SIGN);
#pragma unroll
    for (int k2 = 0; k2 < P; ++k2) {
      cff b[3] = {a[0][k2], a[1][k2], a[2][k2]};
      cff_dft3(b, SIGN);
#pragma unroll
      for (int k1 = 0; k1 < 3; ++k1) v[(A * k1 + B * k2) % N] = cff_fold(b[k1]);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
      for (int p = 0; p < P; ++p) a[q][p] = cff_of(v[3 * p + q]);
#pragma unroll
    for (int q = 0; q < 3; ++q) cff_dft_small<P>(a[q], SIGN);
#pragma unroll
    for (int q = 1; q < 3; ++q)
#pragma unroll
      for (int k1 = 1; k1 < P; ++k1) {
        float2 w = tw[(q * k1) * TS];
        if (SIGN > 0) w.y = -w.y;
        // (x + i y)(wx + i wy) with each product's rounding error kept
        const cff z = a[q][k1];
        a[q][k1] = {ff_sub(ff_mulc(z.x, w.x, 0.0f), ff_mulc(z.y, w.y, 0.0f)),
                    ff_add(ff_mulc(z.x, w.y, 0.0f), ff_mulc(z.y, w.x, 0.0f))};
      }
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      cff b[3] = {a[0][k1], a[1][k1], a[2][k1]};
      cff_dft3(b, SIGN);
#pragma unroll
      for (int k2 = 0; k2 < 3; ++k2) v[k1 + P * k2] = cff_fold(b[k2]);
    }
  }
}

// Stored index -> padded FFT position for a Nyquist-free complex axis of
// n-1 stored modes placed in a length-M transform (zeropad_fft /
// truncate_fft index maps, src/dnsjax/fft.py:41-137).
__device__ __forceinline__ int stored_to_pos(int s, int nstored, int M) {
  const int n = nstored + 1;
  return (s < n / 2) ? s : s + M - n + 1;
}
// Padded position -> stored index, or -1 where the padded array is zero.
__device__ __forceinline__ int pos_to_stored(int t, int nstored, int M) {
  const int n = nstored + 1;
  if (t < n / 2) return t;
  if (t >= M - n / 2 + 1) return t - M + n - 1;
  return -1;
}

// Raise a kernel's dynamic shared-memory limit to what is left of max_smem
// after its static shared memory.
inline cudaError_t allow_dynamic_smem(const void* fn, int max_smem) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  const int dyn = max_smem - (int)fa.sharedSizeBytes;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              dyn > 0 ? dyn : 0);
}

// Copy a global twiddle table of length L into shared memory.
// Asynchronous global -> shared copies (cp.async): a thread issues all of
// its copies before waiting, so their latencies overlap.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
// One complex element, either precision.
__device__ __forceinline__ void cp_async_elem(double2* smem, const double2* gmem) {
  cp_async16(smem, gmem);
}
__device__ __forceinline__ void cp_async_elem(float2* smem, const float2* gmem) {
  cp_async8(smem, gmem);
}
// L2 eviction priority of global accesses: a policy from createpolicy,
// carried by .L2::cache_hint loads, stores and cp.async copies.  l2_keep:
// every line evict_last; l2_keep_half: evict_last on half of the lines
// (address-hashed), the rest unchanged; l2_drop: evict_first.
__device__ __forceinline__ unsigned long long l2_keep() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_keep_half() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.L2::evict_unchanged.b64 %0, 0.5;\n"
               : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_drop() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_l2(double2* g, double2 v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;\n" ::"l"(g), "d"(v.x),
               "d"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_l2(float2* g, float2 v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;\n" ::"l"(g), "f"(v.x),
               "f"(v.y), "l"(pol)
               : "memory");
}
__device__ __forceinline__ double2 ld_l2(const double2* g, unsigned long long pol) {
  double2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;\n"
               : "=d"(v.x), "=d"(v.y)
               : "l"(g), "l"(pol)
               : "memory");
  return v;
}
__device__ __forceinline__ float2 ld_l2(const float2* g, unsigned long long pol) {
  float2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;\n"
               : "=f"(v.x), "=f"(v.y)
               : "l"(g), "l"(pol)
               : "memory");
  return v;
}
__device__ __forceinline__ void cp_async16_l2(void* smem, const void* g, unsigned long long pol) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(s), "l"(g),
               "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async8_l2(void* smem, const void* g, unsigned long long pol) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;\n" ::"r"(s), "l"(g),
               "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_async_elem_l2(double2* smem, const double2* g,
                                                 unsigned long long pol) {
  cp_async16_l2(smem, g, pol);
}
__device__ __forceinline__ void cp_async_elem_l2(float2* smem, const float2* g,
                                                 unsigned long long pol) {
  cp_async8_l2(smem, g, pol);
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_1() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_2() {
  asm volatile("cp.async.wait_group 2;\n" ::: "memory");
}

template <typename C>
__device__ __forceinline__ void load_twiddles(C* s, const C* g, int L) {
  for (int i = threadIdx.x; i < L; i += blockDim.x) s[i] = g[i];
}

}  // namespace dnsb
