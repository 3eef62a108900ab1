// Shared device code of the nsrno_b200 library: complex arithmetic, the PML
// geometry, the h^2-scaled 5-point viscoacoustic Helmholtz stencil and a
// shared-memory mixed-radix FFT used by the shifted-Laplace preconditioner.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "nsrno_b200.h"

#define NSR_MAX_RADIX_STAGES 12
#define NSR_MAX_LINE 2048
// Largest prime radix of the transforms (direct DFT stages, see fft_stage_prime).
#define NSR_MAX_PRIME_RADIX 61
#define NSR_PI 3.14159265358979323846

// ---------------------------------------------------------------------------
// Complex helpers on float2 / double2.
// ---------------------------------------------------------------------------
template <typename T> struct CxT;
template <> struct CxT<float> { typedef float2 type; };
template <> struct CxT<double> { typedef double2 type; };

template <typename C> __host__ __device__ __forceinline__ C cx(decltype(C::x) re, decltype(C::x) im) {
  C z; z.x = re; z.y = im; return z;
}
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 conjc(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 conjc(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 divc(float2 a, float2 b) {
  float d = 1.0f / (b.x * b.x + b.y * b.y);
  return make_float2((a.x * b.x + a.y * b.y) * d, (a.y * b.x - a.x * b.y) * d);
}
__host__ __device__ __forceinline__ double2 divc(double2 a, double2 b) {
  double d = 1.0 / (b.x * b.x + b.y * b.y);
  return make_double2((a.x * b.x + a.y * b.y) * d, (a.y * b.x - a.x * b.y) * d);
}
__host__ __device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__host__ __device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
// conj(a) * b accumulated in double
__device__ __forceinline__ void dot_acc(double& re, double& im, float2 a, float2 b) {
  re += (double)a.x * b.x + (double)a.y * b.y;
  im += (double)a.x * b.y - (double)a.y * b.x;
}

// ---------------------------------------------------------------------------
// Geometry.  Index-space form of Solver._stretch (theranostic/wave.py:127-135):
// the fraction max((lower + w - x)/w, (x - upper + w)/w) with x = x0 + pos*h
// and w = n_pml*h becomes max(n_pml - pos, pos - (n-1-n_pml)) / n_pml.
// ---------------------------------------------------------------------------
struct Geo {
  int nz, nx, n_pml, face;
  double h, c0, rho0, strength, alpha_power, ap_half;
};

__host__ __device__ __forceinline__ Geo make_geo(const NsrGrid& g) {
  Geo o;
  o.nz = g.nz; o.nx = g.nx; o.n_pml = g.n_pml; o.face = g.face;
  o.h = g.h; o.c0 = g.c0; o.rho0 = g.rho0; o.strength = g.pml_strength;
  o.alpha_power = g.alpha_power; o.ap_half = g.aperture_half_width;
  return o;
}

template <typename T>
__device__ __forceinline__ T pml_profile(T pos, int n, int n_pml) {
  if (n_pml <= 0) return T(0);
  T f = fmax(T(n_pml) - pos, pos - T(n - 1 - n_pml)) / T(n_pml);
  f = fmin(fmax(f, T(0)), T(1));
  return f * f;
}

// Material buffer: float planes a, b, t ([3][n], used by the FP32 Krylov
// kernels) followed, at a 256-byte aligned offset, by the same planes in
// double ([3][n], used by the FP64 true residual, the FP64 apply and the
// gradient, so that those evaluate exactly the operator of the oracle).
__host__ __device__ inline size_t nsr_material_off64(long long n) {
  return ((size_t)(12 * n) + 255) & ~(size_t)255;
}
__host__ __device__ inline size_t nsr_material_size(long long n) { return nsr_material_off64(n) + 24 * (size_t)n; }

struct MatPlanes {
  const float *a32, *b32, *t32;
  const double *a64, *b64, *t64;
};

__host__ __device__ inline MatPlanes nsr_planes(const void* mat, long long n) {
  MatPlanes m;
  const float* f = (const float*)mat;
  const double* d = (const double*)((const char*)mat + nsr_material_off64(n));
  m.a32 = f; m.b32 = f + n; m.t32 = f + 2 * n;
  m.a64 = d; m.b64 = d + n; m.t64 = d + 2 * n;
  return m;
}

// Per-system scalars of one frequency.
struct SysScalars {
  double kh2;    // (k0 h)^2
  double sig;    // sigma_max / omega (stretch = 1 + i sig * profile)
  double fpow;   // (f / 1 MHz)^(y - 1)
  double k0;     // omega / c0
};

__host__ __device__ __forceinline__ SysScalars sys_scalars(const Geo& g, double f) {
  SysScalars s;
  double omega = 2.0 * NSR_PI * f;
  s.k0 = omega / g.c0;
  s.kh2 = (s.k0 * g.h) * (s.k0 * g.h);
  s.sig = g.n_pml > 0 ? g.strength * g.c0 / (g.n_pml * g.h) / omega : 0.0;
  s.fpow = pow(f / 1e6, g.alpha_power - 1.0);
  return s;
}

// h^2-scaled stencil at node (i, j).  `P` fetches the field at (i2, j2) and
// returns zero outside the grid (the reference's zero ghost,
// theranostic/wave.py:109-115); `A` fetches the inverse-density ratio a and
// returns 1 outside (zero ghost contrast).  Fluxes follow
// theranostic/wave.py:150-155,179: stretch * (a_i + a_j) / 2; the mass term is
// theranostic/wave.py:180 times the attenuation factor (1 + i e)^2.
template <typename T, bool ADJ, typename FP, typename FA>
__device__ __forceinline__ typename CxT<T>::type stencil(const Geo& g, const SysScalars& s, int i, int j,
                                                         T b_c, T t_c, FP P, FA A) {
  typedef typename CxT<T>::type C;
  const T sig = (T)s.sig;
  const T a_c = A(i, j);
  const C pc = P(i, j);
  // stretches at nodes and half nodes
  const C sx = cx<C>(T(1), sig * pml_profile<T>(T(j), g.nx, g.n_pml));
  const C sz = cx<C>(T(1), sig * pml_profile<T>(T(i), g.nz, g.n_pml));
  const C sxe = cx<C>(T(1), sig * pml_profile<T>(T(j) + T(0.5), g.nx, g.n_pml));
  const C sxw = cx<C>(T(1), sig * pml_profile<T>(T(j) - T(0.5), g.nx, g.n_pml));
  const C szs = cx<C>(T(1), sig * pml_profile<T>(T(i) + T(0.5), g.nz, g.n_pml));
  const C szn = cx<C>(T(1), sig * pml_profile<T>(T(i) - T(0.5), g.nz, g.n_pml));
  C fe = T(0.5) * (a_c + A(i, j + 1)) * divc(sz, sxe);
  C fw = T(0.5) * (a_c + A(i, j - 1)) * divc(sz, sxw);
  C fs = T(0.5) * (a_c + A(i + 1, j)) * divc(sx, szs);
  C fn = T(0.5) * (a_c + A(i - 1, j)) * divc(sx, szn);
  const T e = t_c * (T)s.fpow;
  C loss = cx<C>(T(1) - e * e, T(2) * e);
  C mass = ((T)s.kh2 * b_c) * ((sx * sz) * loss);
  if (ADJ) { fe = conjc(fe); fw = conjc(fw); fs = conjc(fs); fn = conjc(fn); mass = conjc(mass); }
  C y = mass * pc;
  y = y + fe * (P(i, j + 1) - pc);
  y = y + fw * (P(i, j - 1) - pc);
  y = y + fs * (P(i + 1, j) - pc);
  y = y + fn * (P(i - 1, j) - pc);
  return y;
}

// Plane-wave source line value at column j (SI line amplitude, no 1/h^2):
// taper(x) exp(-i k0 x sin(theta)), nsrno/wave_operator.py:114-115.
__device__ __forceinline__ double2 source_line(const Geo& g, double k0, double sin_theta, int j) {
  double x = (j - 0.5 * (g.nx - 1)) * g.h;
  if (fabs(x) > g.ap_half || g.ap_half <= 0.0) return make_double2(0.0, 0.0);
  double taper = 0.5 * (1.0 + cos(NSR_PI * x / g.ap_half));
  double sn, cs;
  sincos(-k0 * x * sin_theta, &sn, &cs);
  return make_double2(taper * cs, taper * sn);
}

// ---------------------------------------------------------------------------
// Mixed-radix FFT along lines held in shared memory.
//
// Forward transforms are decimation-in-frequency (natural order in,
// digit-reversed order out); inverse transforms are the exact stage-by-stage
// inverse (digit-reversed in, natural out, unnormalised).  The preconditioner
// multiplies in the digit-reversed domain, so no reordering pass is needed.
// ---------------------------------------------------------------------------
struct FftPlan {
  int n;
  int nst;
  int radix[NSR_MAX_RADIX_STAGES];
  const float2* tw;   // tw[k] = exp(-2 pi i k / n), k < n
  // Twiddles of the specialised transforms, stage by stage: for every stage
  // with m = L/R > 1 (L its length, R its radix), (R-1) m entries, entry
  // (k-1) m + j holding tw[j k n/L] for 1 <= k < R, j < m.  Butterflies j of
  // one warp read consecutive entries for each k.
  const float2* tws;
};

template <int R, bool INV>
__device__ __forceinline__ void small_dft(float2* x) {
  if (R == 2) {
    float2 a = x[0], b = x[1];
    x[0] = a + b; x[1] = a - b;
  } else if (R == 3) {
    const float h3 = 0.86602540378443864676f;
    float2 t1 = x[1] + x[2];
    float2 t2 = x[0] - 0.5f * t1;
    float2 d = x[1] - x[2];
    // forward: t3 = -i (sqrt3/2) d ; inverse: +i (sqrt3/2) d
    float2 t3 = INV ? make_float2(-h3 * d.y, h3 * d.x) : make_float2(h3 * d.y, -h3 * d.x);
    x[0] = x[0] + t1; x[1] = t2 + t3; x[2] = t2 - t3;
  } else if (R == 4) {
    float2 a = x[0] + x[2], b = x[0] - x[2], c = x[1] + x[3], e = x[1] - x[3];
    float2 d = INV ? make_float2(-e.y, e.x) : make_float2(e.y, -e.x);
    x[0] = a + c; x[2] = a - c; x[1] = b + d; x[3] = b - d;
  } else if (R == 16) {
    // 16 = 4 x 4: DFT4 over n1 for each n2, twiddle W16^(n2 k1), DFT4 over n2.
    const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, r2 = 0.70710678118654752440f;
    float2 y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      float2 t[4] = {x[n2], x[4 + n2], x[8 + n2], x[12 + n2]};
      small_dft<4, INV>(t);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = t[k1];
    }
    // W16^e for e = n2*k1 in {0..9}: exp(-+ 2 pi i e / 16)
    const float2 w[10] = {make_float2(1.f, 0.f), make_float2(c1, INV ? s1 : -s1), make_float2(r2, INV ? r2 : -r2),
                          make_float2(s1, INV ? c1 : -c1), make_float2(0.f, INV ? 1.f : -1.f),
                          make_float2(-s1, INV ? c1 : -c1), make_float2(-r2, INV ? r2 : -r2),
                          make_float2(-c1, INV ? s1 : -s1), make_float2(-1.f, 0.f),
                          make_float2(-c1, INV ? -s1 : s1)};
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
      for (int k1 = 1; k1 < 4; ++k1) y[n2][k1] = y[n2][k1] * w[n2 * k1];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      float2 t[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
      small_dft<4, INV>(t);
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) x[k1 + 4 * k2] = t[k2];
    }
  } else if (R == 8) {
    float2 ev[4] = {x[0], x[2], x[4], x[6]};
    float2 od[4] = {x[1], x[3], x[5], x[7]};
    small_dft<4, INV>(ev);
    small_dft<4, INV>(od);
    const float r2 = 0.70710678118654752440f;
    // W8^k = exp(-+ i pi k / 4)
    float2 w1 = INV ? make_float2(r2, r2) : make_float2(r2, -r2);
    float2 w2 = INV ? make_float2(0.f, 1.f) : make_float2(0.f, -1.f);
    float2 w3 = INV ? make_float2(-r2, r2) : make_float2(-r2, -r2);
    float2 o1 = w1 * od[1], o2 = w2 * od[2], o3 = w3 * od[3];
    x[0] = ev[0] + od[0]; x[4] = ev[0] - od[0];
    x[1] = ev[1] + o1;    x[5] = ev[1] - o1;
    x[2] = ev[2] + o2;    x[6] = ev[2] - o2;
    x[3] = ev[3] + o3;    x[7] = ev[3] - o3;
  }
}

// One DIF stage (forward) or its inverse over `nl` lines.
// Element k of line l lives at s[l*lstride + k*estride].  When `line_fast`
// the thread index runs over lines first (columns held side by side in
// shared memory), otherwise over butterflies of one line first (rows).
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(float2* s, int nl, int lstride, int estride, bool line_fast,
                                          const FftPlan& P, int L) {
  const int m = L / R;
  const int per_line = P.n / R;
  const int nb = nl * per_line;
  const int tstep = P.n / L;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    int l, bb;
    if (line_fast) { l = b % nl; bb = b / nl; } else { l = b / per_line; bb = b % per_line; }
    const int o = bb / m, j = bb - o * m;
    float2* base = s + l * lstride + (o * L + j) * estride;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = base[q * m * estride];
    if (!INV) {
      small_dft<R, false>(v);
#pragma unroll
      for (int k = 1; k < R; ++k) v[k] = v[k] * __ldg(&P.tw[j * k * tstep]);
    } else {
#pragma unroll
      for (int k = 1; k < R; ++k) v[k] = v[k] * conjc(__ldg(&P.tw[j * k * tstep]));
      small_dft<R, true>(v);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) base[q * m * estride] = v[q];
  }
}

// One DIF stage (forward) or its inverse for a prime radix R > 3, as a direct
// R-point DFT: y_k = sum_q v_q W_R^(q k), W_R^e = tw[e n / R].  The cost is
// R complex multiply-adds per point, which the sizes that need these stages
// (paddings such as 1056 = 2^5 3 11 and 1216 = 2^6 19) can afford.
template <bool INV>
__device__ __noinline__ void fft_stage_prime(float2* s, int nl, int lstride, int estride, bool line_fast,
                                             const FftPlan& P, int L, int R) {
  const int m = L / R;
  const int per_line = P.n / R;
  const int nb = nl * per_line;
  const int tstep = P.n / L;
  const int rstep = P.n / R;
  float2 v[NSR_MAX_PRIME_RADIX], y[NSR_MAX_PRIME_RADIX];
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    int l, bb;
    if (line_fast) { l = b % nl; bb = b / nl; } else { l = b / per_line; bb = b % per_line; }
    const int o = bb / m, j = bb - o * m;
    float2* base = s + l * lstride + (o * L + j) * estride;
    for (int q = 0; q < R; ++q) v[q] = base[q * m * estride];
    if (INV)
      for (int k = 1; k < R; ++k) v[k] = v[k] * conjc(__ldg(&P.tw[j * k * tstep]));
    for (int k = 0; k < R; ++k) {
      float2 acc = v[0];
      int e = 0;
      for (int q = 1; q < R; ++q) {
        e += k;
        if (e >= R) e -= R;
        const float2 w = __ldg(&P.tw[e * rstep]);
        acc = acc + v[q] * (INV ? conjc(w) : w);
      }
      y[k] = acc;
    }
    if (!INV)
      for (int k = 1; k < R; ++k) y[k] = y[k] * __ldg(&P.tw[j * k * tstep]);
    for (int q = 0; q < R; ++q) base[q * m * estride] = y[q];
  }
}

template <bool INV>
__device__ void fft_lines(float2* s, int nl, int lstride, int estride, bool line_fast, const FftPlan& P) {
  if (!INV) {
    int L = P.n;
    for (int st = 0; st < P.nst; ++st) {
      const int R = P.radix[st];
      switch (R) {
        case 2: fft_stage<2, false>(s, nl, lstride, estride, line_fast, P, L); break;
        case 3: fft_stage<3, false>(s, nl, lstride, estride, line_fast, P, L); break;
        case 4: fft_stage<4, false>(s, nl, lstride, estride, line_fast, P, L); break;
        case 8: fft_stage<8, false>(s, nl, lstride, estride, line_fast, P, L); break;
        case 16: fft_stage<16, false>(s, nl, lstride, estride, line_fast, P, L); break;
        default: fft_stage_prime<false>(s, nl, lstride, estride, line_fast, P, L, R); break;
      }
      __syncthreads();
      L /= R;
    }
  } else {
    // Lengths of the forward stages, replayed backwards.
    int Ls[NSR_MAX_RADIX_STAGES];
    int L = P.n;
    for (int st = 0; st < P.nst; ++st) { Ls[st] = L; L /= P.radix[st]; }
    for (int st = P.nst - 1; st >= 0; --st) {
      const int R = P.radix[st];
      switch (R) {
        case 2: fft_stage<2, true>(s, nl, lstride, estride, line_fast, P, Ls[st]); break;
        case 3: fft_stage<3, true>(s, nl, lstride, estride, line_fast, P, Ls[st]); break;
        case 4: fft_stage<4, true>(s, nl, lstride, estride, line_fast, P, Ls[st]); break;
        case 8: fft_stage<8, true>(s, nl, lstride, estride, line_fast, P, Ls[st]); break;
        case 16: fft_stage<16, true>(s, nl, lstride, estride, line_fast, P, Ls[st]); break;
        default: fft_stage_prime<true>(s, nl, lstride, estride, line_fast, P, Ls[st], R); break;
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Compile-time specialised line FFTs for the common sizes.  Same stage
// sequence (and therefore the same digit-reversed order) as the runtime plan.
// ---------------------------------------------------------------------------
struct RadixList {
  int nst;
  int r[NSR_MAX_RADIX_STAGES];
};

__host__ __device__ constexpr bool nsr_is_prime(int p) {
  if (p < 2) return false;
  for (int d = 2; d * d <= p; ++d)
    if (p % d == 0) return false;
  return true;
}

__host__ __device__ constexpr RadixList nsr_radix_list(int n) {
  // n = p1 p2 ... 2^a 3^b with primes 5 <= p <= NSR_MAX_PRIME_RADIX: one
  // direct-DFT stage per such prime first, then the radix-3 stages, then
  // 2^(a mod 4) (one radix-2, -4 or -8 stage), then radix-16 stages, so that
  // every size divisible by 16 ends with a radix-16 stage on contiguous
  // 16-element groups.  nst = 0 for sizes with a larger prime factor.
  RadixList L{0, {0}};
  int a = 0, b = 0, m = n;
  int k = 0;
  for (int p = 5; p <= NSR_MAX_PRIME_RADIX; p += 2) {
    if (!nsr_is_prime(p)) continue;
    while (m % p == 0 && k < NSR_MAX_RADIX_STAGES) { m /= p; L.r[k++] = p; }
  }
  while (m % 2 == 0) { m /= 2; ++a; }
  while (m % 3 == 0) { m /= 3; ++b; }
  if (m != 1 || n < 2) return RadixList{0, {0}};
  for (int i = 0; i < b && k < NSR_MAX_RADIX_STAGES; ++i) L.r[k++] = 3;
  const int rem = a % 4;
  if (rem > 0 && k < NSR_MAX_RADIX_STAGES) L.r[k++] = 1 << rem;
  for (int i = 0; i < a / 4 && k < NSR_MAX_RADIX_STAGES; ++i) L.r[k++] = 16;
  L.nst = k;
  return L;
}

__host__ __device__ constexpr int nsr_stage_len(int n, int stage) {
  RadixList L = nsr_radix_list(n);
  int len = n;
  for (int s = 0; s < stage; ++s) len /= L.r[s];
  return len;
}

// Offset (in float2) of the twiddle rows of the stage of length `len` in
// FftPlan::tws; with len = 0, the total number of entries.
__host__ __device__ constexpr int nsr_twiddle_offset(int n, int len) {
  RadixList L = nsr_radix_list(n);
  int l = n, off = 0;
  for (int s = 0; s < L.nst; ++s) {
    if (l == len) return off;
    const int m = l / L.r[s];
    if (m > 1) off += m * (L.r[s] - 1);
    l = m;
  }
  return off;
}

// One stage, everything but the number of lines known at compile time.
// Elements: s[l*LS + k*ES].  LF: thread index runs over lines first.
template <int N, int R, int L, bool INV, bool LF, int LS, int ES, bool PAD>
__device__ __forceinline__ void ct_stage(float2* s, int nl, const float2* __restrict__ tws) {
  constexpr int m = L / R, per_line = N / R;
  const float2* __restrict__ tst = tws + nsr_twiddle_offset(N, L);
  constexpr int U = R >= 16 ? 1 : 2;   // butterflies in flight per thread
  const int nb = nl * per_line;
  auto at = [](int k) { return PAD ? k + (k >> 4) : k; };
  for (int b0 = threadIdx.x; b0 < nb; b0 += U * blockDim.x) {
    float2 v[U][R];
    float2* base[U];
    int first[U], jj[U];
    bool ok[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int bq = b0 + u * blockDim.x;
      ok[u] = (u == 0) || bq < nb;
      const int b = ok[u] ? bq : b0;
      int l, bb;
      if (LF) { l = b % nl; bb = b / nl; } else { l = b / per_line; bb = b - l * per_line; }
      const int o = bb / m, j = bb - o * m;
      jj[u] = j;
      base[u] = s + l * LS;
      first[u] = o * L + j;
#pragma unroll
      for (int q = 0; q < R; ++q) v[u][q] = base[u][at(first[u] + q * m) * ES];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      // The stage with m == 1 (the last forward, first inverse) has unit
      // twiddles.  Otherwise entry k of butterfly j sits at (k-1) m + j.
      auto twiddle = [&](float2* x) {
        if constexpr (m > 1) {
          const float2* __restrict__ tj = tst + jj[u];
#pragma unroll
          for (int k = 1; k < R; ++k) {
            const float2 w = __ldg(tj + (k - 1) * m);
            x[k] = x[k] * (INV ? conjc(w) : w);
          }
        }
      };
      if (!INV) {
        small_dft<R, false>(v[u]);
        twiddle(v[u]);
      } else {
        twiddle(v[u]);
        small_dft<R, true>(v[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (ok[u]) {
#pragma unroll
        for (int q = 0; q < R; ++q) base[u][at(first[u] + q * m) * ES] = v[u][q];
      }
    }
  }
}

template <int N, int S, bool LF, int LS, int ES, bool PAD>
__device__ __forceinline__ void ct_forward(float2* s, int nl, const float2* __restrict__ tws) {
  constexpr RadixList RL = nsr_radix_list(N);
  if constexpr (S < RL.nst) {
    constexpr int R = RL.r[S];
    constexpr int L = nsr_stage_len(N, S);
    ct_stage<N, R, L, false, LF, LS, ES, PAD>(s, nl, tws);
    __syncthreads();
    ct_forward<N, S + 1, LF, LS, ES, PAD>(s, nl, tws);
  }
}

// Forward stages S .. STOP-1.
template <int N, int S, int STOP, bool LF, int LS, int ES, bool PAD>
__device__ __forceinline__ void ct_forward_upto(float2* s, int nl, const float2* __restrict__ tws) {
  if constexpr (S < STOP) {
    constexpr RadixList RL = nsr_radix_list(N);
    constexpr int R = RL.r[S];
    constexpr int L = nsr_stage_len(N, S);
    ct_stage<N, R, L, false, LF, LS, ES, PAD>(s, nl, tws);
    __syncthreads();
    ct_forward_upto<N, S + 1, STOP, LF, LS, ES, PAD>(s, nl, tws);
  }
}

template <int N, int S, bool LF, int LS, int ES, bool PAD>
__device__ __forceinline__ void ct_inverse(float2* s, int nl, const float2* __restrict__ tws) {
  constexpr RadixList RL = nsr_radix_list(N);
  if constexpr (S >= 0) {
    constexpr int R = RL.r[S];
    constexpr int L = nsr_stage_len(N, S);
    ct_stage<N, R, L, true, LF, LS, ES, PAD>(s, nl, tws);
    __syncthreads();
    ct_inverse<N, S - 1, LF, LS, ES, PAD>(s, nl, tws);
  }
}

template <int N, bool INV, bool LF, int LS, int ES, bool PAD>
__device__ __forceinline__ void ct_fft(float2* s, int nl, const float2* __restrict__ tws) {
  constexpr RadixList RL = nsr_radix_list(N);
  if (!INV) ct_forward<N, 0, LF, LS, ES, PAD>(s, nl, tws);
  else ct_inverse<N, RL.nst - 1, LF, LS, ES, PAD>(s, nl, tws);
}

// Row layout in shared memory: the specialised sizes insert one pad element
// after every 16 (element k of a row at k + k/16), which keeps every row FFT
// stage free of shared-memory bank conflicts.
__host__ __device__ inline bool nsr_row_padded(int n) {
  switch (n) {
    case 256: case 384: case 512: case 768: case 1024: case 1536: case 2048: return true;
    default: return false;
  }
}
__host__ __device__ inline int nsr_row_stride(int n) { return nsr_row_padded(n) ? n + (n >> 4) : n; }

// Rows: nl lines of length n, row stride nsr_row_stride(n) (padded for the
// specialised sizes, plain otherwise).
template <bool INV>
__device__ void fft_rows(float2* s, int nl, const FftPlan& P) {
  switch (P.n) {
    case 256: ct_fft<256, INV, false, 256 + 16, 1, true>(s, nl, P.tws); return;
    case 384: ct_fft<384, INV, false, 384 + 24, 1, true>(s, nl, P.tws); return;
    case 512: ct_fft<512, INV, false, 512 + 32, 1, true>(s, nl, P.tws); return;
    case 768: ct_fft<768, INV, false, 768 + 48, 1, true>(s, nl, P.tws); return;
    case 1024: ct_fft<1024, INV, false, 1024 + 64, 1, true>(s, nl, P.tws); return;
    case 1536: ct_fft<1536, INV, false, 1536 + 96, 1, true>(s, nl, P.tws); return;
    case 2048: ct_fft<2048, INV, false, 2048 + 128, 1, true>(s, nl, P.tws); return;
    default: fft_lines<INV>(s, nl, P.n, 1, false, P); return;
  }
}

// Columns: TC lines side by side (lstride 1, estride TC), unpadded.
template <bool INV, int TC>
__device__ void fft_cols(float2* s, const FftPlan& P) {
  switch (P.n) {
    case 256: ct_fft<256, INV, true, 1, TC, false>(s, TC, P.tws); return;
    case 384: ct_fft<384, INV, true, 1, TC, false>(s, TC, P.tws); return;
    case 512: ct_fft<512, INV, true, 1, TC, false>(s, TC, P.tws); return;
    case 768: ct_fft<768, INV, true, 1, TC, false>(s, TC, P.tws); return;
    case 1024: ct_fft<1024, INV, true, 1, TC, false>(s, TC, P.tws); return;
    case 1536: ct_fft<1536, INV, true, 1, TC, false>(s, TC, P.tws); return;
    case 2048: ct_fft<2048, INV, true, 1, TC, false>(s, TC, P.tws); return;
    default: fft_lines<INV>(s, TC, 1, TC, true, P); return;
  }
}

// Forward column FFT, a pointwise multiply in the digit-reversed domain and the
// inverse column FFT, with the last forward stage, the multiply and the first
// inverse stage done in registers in one shared-memory pass (that stage has
// m == 1: contiguous groups of R elements and unit twiddles).  `mul(l, k)`
// returns the factor of line l (column of the tile) at digit-reversed position k.
template <int N, int TC, typename MUL>
__device__ __forceinline__ void ct_cols_fused(float2* s, const float2* __restrict__ tws, MUL mul) {
  constexpr RadixList RL = nsr_radix_list(N);
  constexpr int LAST = RL.nst - 1;
  constexpr int R = RL.r[LAST];
  if constexpr (LAST > 0) ct_forward_upto<N, 0, LAST, true, 1, TC, false>(s, TC, tws);
  constexpr int per_line = N / R;
  const int nb = TC * per_line;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int l = b % TC, o = b / TC;
    float2* base = s + l + o * R * TC;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = base[q * TC];
    small_dft<R, false>(v);
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = v[q] * mul(l, o * R + q);
    small_dft<R, true>(v);
#pragma unroll
    for (int q = 0; q < R; ++q) base[q * TC] = v[q];
  }
  __syncthreads();
  if constexpr (LAST > 0) ct_inverse<N, LAST - 1, true, 1, TC, false>(s, TC, tws);
}

// Inverse stages S down to STOP (inclusive).
template <int N, int S, int STOP, bool LF, int LS, int ES, bool PAD>
__device__ __forceinline__ void ct_inverse_downto(float2* s, int nl, const float2* __restrict__ tws) {
  if constexpr (S >= STOP) {
    constexpr RadixList RL = nsr_radix_list(N);
    constexpr int R = RL.r[S];
    constexpr int L = nsr_stage_len(N, S);
    ct_stage<N, R, L, true, LF, LS, ES, PAD>(s, nl, tws);
    __syncthreads();
    ct_inverse_downto<N, S - 1, STOP, LF, LS, ES, PAD>(s, nl, tws);
  }
}

// The column pass of a TC-column tile of a field in global memory (row stride
// nx), with the first forward stage computed straight from the global loads
// and the last inverse stage written straight to global memory: the tile
// crosses shared memory two times fewer than load-transform-store.  Columns
// at or beyond `ncol` read as zero and are not written.  `mul(l, k)` as in
// ct_cols_fused.  Needs at least two stages (every specialised size has).
template <int N, int TC, typename MUL>
__device__ __forceinline__ void ct_cols_direct(float2* s, const float2* __restrict__ tws, float2* __restrict__ g,
                                               int nx, int ncol, MUL mul) {
  constexpr RadixList RL = nsr_radix_list(N);
  constexpr int LAST = RL.nst - 1;
  static_assert(LAST >= 1, "two stages at least");
  constexpr int R0 = RL.r[0];
  constexpr int M0 = N / R0;
  const float2* __restrict__ tw0 = tws + nsr_twiddle_offset(N, N);
  // stage 0 forward: global -> registers -> shared, U butterflies per thread
  // with their loads issued together (radix 2: 8 loads in flight, 3 and 4: 6-8)
  constexpr int U = R0 <= 2 ? 4 : (R0 <= 4 ? 2 : 1);
  const int nb0 = TC * M0;
  for (int b0 = threadIdx.x; b0 < nb0; b0 += U * blockDim.x) {
    float2 v[U][R0];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int b = b0 + u * blockDim.x;
      const int l = b % TC, j = b / TC;
      const bool live = b < nb0 && l < ncol;
#pragma unroll
      for (int q = 0; q < R0; ++q) v[u][q] = live ? g[(long long)(j + q * M0) * nx + l] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int b = b0 + u * blockDim.x;
      if (b < nb0) {
        const int l = b % TC, j = b / TC;
        small_dft<R0, false>(v[u]);
#pragma unroll
        for (int k = 1; k < R0; ++k) v[u][k] = v[u][k] * __ldg(tw0 + (k - 1) * M0 + j);
#pragma unroll
        for (int q = 0; q < R0; ++q) s[l + (j + q * M0) * TC] = v[u][q];
      }
    }
  }
  __syncthreads();
  if constexpr (LAST > 1) ct_forward_upto<N, 1, LAST, true, 1, TC, false>(s, TC, tws);
  // last forward stage, multiply, first inverse stage (unit twiddles, m == 1)
  constexpr int R = RL.r[LAST];
  constexpr int per_line = N / R;
  for (int b = threadIdx.x; b < TC * per_line; b += blockDim.x) {
    const int l = b % TC, o = b / TC;
    float2* base = s + l + o * R * TC;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = base[q * TC];
    small_dft<R, false>(v);
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = v[q] * mul(l, o * R + q);
    small_dft<R, true>(v);
#pragma unroll
    for (int q = 0; q < R; ++q) base[q * TC] = v[q];
  }
  __syncthreads();
  if constexpr (LAST > 1) ct_inverse_downto<N, LAST - 1, 1, true, 1, TC, false>(s, TC, tws);
  // stage 0 inverse: shared -> registers -> global
  for (int b = threadIdx.x; b < TC * M0; b += blockDim.x) {
    const int l = b % TC, j = b / TC;
    float2 v[R0];
#pragma unroll
    for (int q = 0; q < R0; ++q) v[q] = s[l + (j + q * M0) * TC];
#pragma unroll
    for (int k = 1; k < R0; ++k) v[k] = v[k] * conjc(__ldg(tw0 + (k - 1) * M0 + j));
    small_dft<R0, true>(v);
    if (l < ncol) {
#pragma unroll
      for (int q = 0; q < R0; ++q) g[(long long)(j + q * M0) * nx + l] = v[q];
    }
  }
}

// Column pass of a tile straight between global and shared memory for the
// specialised sizes; returns false for other sizes.
template <int TC, typename MUL>
__device__ __forceinline__ bool fft_cols_direct(float2* s, const FftPlan& P, float2* __restrict__ g, int nx,
                                                int ncol, MUL mul) {
  switch (P.n) {
    case 256: ct_cols_direct<256, TC>(s, P.tws, g, nx, ncol, mul); return true;
    case 384: ct_cols_direct<384, TC>(s, P.tws, g, nx, ncol, mul); return true;
    case 512: ct_cols_direct<512, TC>(s, P.tws, g, nx, ncol, mul); return true;
    case 768: ct_cols_direct<768, TC>(s, P.tws, g, nx, ncol, mul); return true;
    case 1024: ct_cols_direct<1024, TC>(s, P.tws, g, nx, ncol, mul); return true;
    case 1536: ct_cols_direct<1536, TC>(s, P.tws, g, nx, ncol, mul); return true;
    case 2048: ct_cols_direct<2048, TC>(s, P.tws, g, nx, ncol, mul); return true;
    default: return false;
  }
}

// Row transforms of the specialised sizes straight between global memory and
// padded shared-memory rows (element k of a row at k + k/16, row stride
// N + N/16).  The tile is nl rows of N points, contiguous in global memory
// (flat index k = row * N + column).  Every specialised size ends its forward
// transform with a radix-16 stage on contiguous groups of 16 with unit
// twiddles, which is the inverse transform's first stage: that stage goes
// straight between registers and global memory as eight 16-byte accesses per
// group.  The other end of the transform, stage 0 (radix R0, elements
// j + q N/R0 of a row), is coalesced across threads:
//  * forward: `in(std::integral_constant<int, R0>{}, k0, step, v)` fills v[q]
//    with the value to transform at flat index k0 + q step (q < R0), doing
//    whatever elementwise work produces it; stage 0 runs on those registers,
//    the middle stages in shared memory, the last stage writes `g`;
//  * inverse: the first stage reads `g`, the middle stages run in shared
//    memory, and `out(k, v)` receives each output of stage 0 (flat index k)
//    and stores it.
// Two shared-memory round trips fewer than load, transform, store.
template <int R>
struct RadixTag { static constexpr int value = R; };

template <int N, typename IN>
__device__ __forceinline__ void ct_rows_forward_direct(float2* s, int nl, const float2* __restrict__ tws,
                                                       float2* __restrict__ g, IN in) {
  constexpr RadixList RL = nsr_radix_list(N);
  constexpr int LAST = RL.nst - 1;
  static_assert(LAST >= 1 && RL.r[LAST] == 16, "specialised sizes end with a radix-16 stage");
  constexpr int LS = N + N / 16;
  constexpr int R0 = RL.r[0], M0 = N / R0;
  const float2* __restrict__ tw0 = tws + nsr_twiddle_offset(N, N);
  for (int b = threadIdx.x; b < nl * M0; b += blockDim.x) {
    const int l = b / M0, j = b - l * M0;
    float2 v[R0];
    in(RadixTag<R0>{}, l * N + j, M0, v);
    small_dft<R0, false>(v);
#pragma unroll
    for (int k = 1; k < R0; ++k) v[k] = v[k] * __ldg(tw0 + (k - 1) * M0 + j);
    float2* d = s + l * LS;
#pragma unroll
    for (int q = 0; q < R0; ++q) {
      const int e = j + q * M0;
      d[e + (e >> 4)] = v[q];
    }
  }
  __syncthreads();
  if constexpr (LAST > 1) ct_forward_upto<N, 1, LAST, false, LS, 1, true>(s, nl, tws);
  constexpr int G = N / 16;
  for (int b = threadIdx.x; b < nl * G; b += blockDim.x) {
    const int l = b / G, o = b - l * G;
    const float2* src = s + l * LS + o * 17;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = src[q];
    small_dft<16, false>(v);
    float4* dst = reinterpret_cast<float4*>(g + (long long)l * N + o * 16);
#pragma unroll
    for (int q = 0; q < 8; ++q) dst[q] = make_float4(v[2 * q].x, v[2 * q].y, v[2 * q + 1].x, v[2 * q + 1].y);
  }
}

template <int N, typename OUT>
__device__ __forceinline__ void ct_rows_inverse_direct(float2* s, int nl, const float2* __restrict__ tws,
                                                       const float2* g, OUT out) {
  constexpr RadixList RL = nsr_radix_list(N);
  constexpr int LAST = RL.nst - 1;
  static_assert(LAST >= 1 && RL.r[LAST] == 16, "specialised sizes end with a radix-16 stage");
  constexpr int LS = N + N / 16;
  constexpr int G = N / 16;
  for (int b = threadIdx.x; b < nl * G; b += blockDim.x) {
    const int l = b / G, o = b - l * G;
    const float4* src = reinterpret_cast<const float4*>(g + (long long)l * N + o * 16);
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 t = src[q];
      v[2 * q] = make_float2(t.x, t.y);
      v[2 * q + 1] = make_float2(t.z, t.w);
    }
    small_dft<16, true>(v);
    float2* d = s + l * LS + o * 17;
#pragma unroll
    for (int q = 0; q < 16; ++q) d[q] = v[q];
  }
  __syncthreads();
  if constexpr (LAST > 1) ct_inverse_downto<N, LAST - 1, 1, false, LS, 1, true>(s, nl, tws);
  constexpr int R0 = RL.r[0], M0 = N / R0;
  const float2* __restrict__ tw0 = tws + nsr_twiddle_offset(N, N);
  for (int b = threadIdx.x; b < nl * M0; b += blockDim.x) {
    const int l = b / M0, j = b - l * M0;
    const float2* src = s + l * LS;
    float2 v[R0];
#pragma unroll
    for (int q = 0; q < R0; ++q) {
      const int e = j + q * M0;
      v[q] = src[e + (e >> 4)];
    }
#pragma unroll
    for (int k = 1; k < R0; ++k) v[k] = v[k] * conjc(__ldg(tw0 + (k - 1) * M0 + j));
    small_dft<R0, true>(v);
#pragma unroll
    for (int q = 0; q < R0; ++q) out(l * N + j + q * M0, v[q]);
  }
}

// Dispatch of the direct row transforms over the specialised sizes; false for
// any other size (the caller then stages the tile itself).
template <typename IN>
__device__ __forceinline__ bool fft_rows_forward_direct(float2* s, int nl, const FftPlan& P, float2* __restrict__ g,
                                                        IN in) {
  switch (P.n) {
    case 256: ct_rows_forward_direct<256>(s, nl, P.tws, g, in); return true;
    case 384: ct_rows_forward_direct<384>(s, nl, P.tws, g, in); return true;
    case 512: ct_rows_forward_direct<512>(s, nl, P.tws, g, in); return true;
    case 768: ct_rows_forward_direct<768>(s, nl, P.tws, g, in); return true;
    case 1024: ct_rows_forward_direct<1024>(s, nl, P.tws, g, in); return true;
    case 1536: ct_rows_forward_direct<1536>(s, nl, P.tws, g, in); return true;
    case 2048: ct_rows_forward_direct<2048>(s, nl, P.tws, g, in); return true;
    default: return false;
  }
}

template <typename OUT>
__device__ __forceinline__ bool fft_rows_inverse_direct(float2* s, int nl, const FftPlan& P, const float2* g,
                                                        OUT out) {
  switch (P.n) {
    case 256: ct_rows_inverse_direct<256>(s, nl, P.tws, g, out); return true;
    case 384: ct_rows_inverse_direct<384>(s, nl, P.tws, g, out); return true;
    case 512: ct_rows_inverse_direct<512>(s, nl, P.tws, g, out); return true;
    case 768: ct_rows_inverse_direct<768>(s, nl, P.tws, g, out); return true;
    case 1024: ct_rows_inverse_direct<1024>(s, nl, P.tws, g, out); return true;
    case 1536: ct_rows_inverse_direct<1536>(s, nl, P.tws, g, out); return true;
    case 2048: ct_rows_inverse_direct<2048>(s, nl, P.tws, g, out); return true;
    default: return false;
  }
}

// Column pass with the fused middle stage for the specialised sizes; other
// sizes run the separate transforms and multiply.  Returns false for those
// other sizes, which the caller then handles itself.
template <int TC, typename MUL>
__device__ __forceinline__ bool fft_cols_fused(float2* s, const FftPlan& P, MUL mul) {
  switch (P.n) {
    case 256: ct_cols_fused<256, TC>(s, P.tws, mul); return true;
    case 384: ct_cols_fused<384, TC>(s, P.tws, mul); return true;
    case 512: ct_cols_fused<512, TC>(s, P.tws, mul); return true;
    case 768: ct_cols_fused<768, TC>(s, P.tws, mul); return true;
    case 1024: ct_cols_fused<1024, TC>(s, P.tws, mul); return true;
    case 1536: ct_cols_fused<1536, TC>(s, P.tws, mul); return true;
    case 2048: ct_cols_fused<2048, TC>(s, P.tws, mul); return true;
    default: return false;
  }
}

// Host-side radix plan of a line of n points, 8 <= n <= 2048, every prime
// factor at most NSR_MAX_PRIME_RADIX (the stages of nsr_radix_list).
__host__ __device__ inline bool nsr_make_radices(int n, int* radix, int* nst) {
  if (n < 8 || n > NSR_MAX_LINE) return false;
  const RadixList L = nsr_radix_list(n);
  if (L.nst == 0) return false;
  int prod = 1;
  for (int k = 0; k < L.nst; ++k) prod *= L.r[k];
  if (prod != n) return false;
  for (int k = 0; k < L.nst; ++k) radix[k] = L.r[k];
  *nst = L.nst;
  return true;
}

// Frequency index held at DIF output position p (mixed-radix digit reversal).
__host__ __device__ inline int nsr_digit_reverse(int p, int n, const int* radix, int nst) {
  int freq = 0, scale = 1, L = n;
  for (int st = 0; st < nst; ++st) {
    int m = L / radix[st];
    int k = p / m;
    p -= k * m;
    freq += k * scale;
    scale *= radix[st];
    L = m;
  }
  return freq;
}
