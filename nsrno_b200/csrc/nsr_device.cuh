// Device helpers shared by the Krylov solvers: block reductions and the
// 5-point stencil at an explicit neighbourhood.
#pragma once

#include "nsr_common.cuh"
#include "nsr_internal.cuh"

#define NSR_NPART 8

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-reduce NV doubles into red[0..NV) (valid in thread 0 afterwards).
template <int NV>
__device__ __forceinline__ void block_sum(double* vals, double* red) {
  __shared__ double wsum[32][NSR_NPART];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = warp_sum(vals[q]);
    if (lane == 0) wsum[wid][q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
    for (int q = 0; q < NV; ++q) {
      double s = 0.0;
      for (int w = 0; w < nw; ++w) s += wsum[w][q];
      red[q] = s;
    }
  }
}


// Stencil at an explicit 5-point neighbourhood.  Interior nodes (all six
// stretches equal to one) take the real-flux path.
template <bool ADJ>
__device__ __forceinline__ float2 stencil_pts(const Geo& g, const SysScalars& sc, int i, int j, float a_c, float a_e,
                                              float a_w, float a_s, float a_n, float b_c, float t_c, float2 pc,
                                              float2 pe, float2 pw, float2 ps, float2 pn) {
  const bool inner = i > g.n_pml && i < g.nz - 1 - g.n_pml && j > g.n_pml && j < g.nx - 1 - g.n_pml;
  if (inner) {
    const float e = t_c * (float)sc.fpow;
    const float mb = (float)sc.kh2 * b_c;
    const float2 mass = make_float2(mb * (1.0f - e * e), (ADJ ? -2.0f : 2.0f) * mb * e);
    float2 y = mass * pc;
    y = y + (0.5f * (a_c + a_e)) * (pe - pc);
    y = y + (0.5f * (a_c + a_w)) * (pw - pc);
    y = y + (0.5f * (a_c + a_s)) * (ps - pc);
    y = y + (0.5f * (a_c + a_n)) * (pn - pc);
    return y;
  }
  auto P = [&](int i2, int j2) -> float2 {
    if (i2 == i && j2 == j) return pc;
    if (i2 == i) return j2 > j ? pe : pw;
    return i2 > i ? ps : pn;
  };
  auto Aa = [&](int i2, int j2) -> float {
    if (i2 == i && j2 == j) return a_c;
    if (i2 == i) return j2 > j ? a_e : a_w;
    return i2 > i ? a_s : a_n;
  };
  return stencil<float, ADJ>(g, sc, i, j, b_c, t_c, P, Aa);
}


// The same stencil with every per-system scalar already in float (set up once
// per work item), so that no node pays a double-to-float conversion; the PML
// profile multiplies by 1/n_pml instead of dividing.
struct SysScalarsF {
  float kh2, sig, fpow, inv_npml;
  int lo, hi_z, hi_x;   // interior: lo < i < hi_z, lo < j < hi_x
};

__device__ __forceinline__ SysScalarsF sys_scalars_f(const Geo& g, const SysScalars& s) {
  SysScalarsF f;
  f.kh2 = (float)s.kh2;
  f.sig = (float)s.sig;
  f.fpow = (float)s.fpow;
  f.inv_npml = g.n_pml > 0 ? 1.0f / (float)g.n_pml : 0.0f;
  f.lo = g.n_pml;
  f.hi_z = g.nz - 1 - g.n_pml;
  f.hi_x = g.nx - 1 - g.n_pml;
  return f;
}

__device__ __forceinline__ float pml_profile_f(float pos, int n, int n_pml, float inv_npml) {
  float f = fmaxf((float)n_pml - pos, pos - (float)(n - 1 - n_pml)) * inv_npml;
  f = fminf(fmaxf(f, 0.0f), 1.0f);
  return f * f;
}

// `inside`: node (i, j) lies off the PML (sf.lo < i < sf.hi_z and
// sf.lo < j < sf.hi_x), tested by the caller once per row and column.
template <bool ADJ>
__device__ __forceinline__ float2 stencil_pts_f(const Geo& g, const SysScalarsF& sf, bool inside, int i, int j,
                                                float a_c, float a_e, float a_w, float a_s, float a_n, float b_c,
                                                float t_c, float2 pc, float2 pe, float2 pw, float2 ps, float2 pn) {
  const float e = t_c * sf.fpow;
  const float mb = sf.kh2 * b_c;
  float2 mass = make_float2(mb * (1.0f - e * e), (ADJ ? -2.0f : 2.0f) * mb * e);
  if (inside) {
    float2 y = mass * pc;
    y = y + (0.5f * (a_c + a_e)) * (pe - pc);
    y = y + (0.5f * (a_c + a_w)) * (pw - pc);
    y = y + (0.5f * (a_c + a_s)) * (ps - pc);
    y = y + (0.5f * (a_c + a_n)) * (pn - pc);
    return y;
  }
  // PML: stretches at the node and the four half nodes (theranostic/wave.py:127-155)
  const float fi = (float)i, fj = (float)j;
  const float2 sx = make_float2(1.0f, sf.sig * pml_profile_f(fj, g.nx, g.n_pml, sf.inv_npml));
  const float2 sz = make_float2(1.0f, sf.sig * pml_profile_f(fi, g.nz, g.n_pml, sf.inv_npml));
  const float2 sxe = make_float2(1.0f, sf.sig * pml_profile_f(fj + 0.5f, g.nx, g.n_pml, sf.inv_npml));
  const float2 sxw = make_float2(1.0f, sf.sig * pml_profile_f(fj - 0.5f, g.nx, g.n_pml, sf.inv_npml));
  const float2 szs = make_float2(1.0f, sf.sig * pml_profile_f(fi + 0.5f, g.nz, g.n_pml, sf.inv_npml));
  const float2 szn = make_float2(1.0f, sf.sig * pml_profile_f(fi - 0.5f, g.nz, g.n_pml, sf.inv_npml));
  float2 fe = (0.5f * (a_c + a_e)) * divc(sz, sxe);
  float2 fw = (0.5f * (a_c + a_w)) * divc(sz, sxw);
  float2 fs = (0.5f * (a_c + a_s)) * divc(sx, szs);
  float2 fn = (0.5f * (a_c + a_n)) * divc(sx, szn);
  // mass * (sx sz): (sx sz) is the stretched cell measure
  const float2 sxz = sx * sz;
  mass = mass * (ADJ ? conjc(sxz) : sxz);
  if (ADJ) { fe = conjc(fe); fw = conjc(fw); fs = conjc(fs); fn = conjc(fn); }
  float2 y = mass * pc;
  y = y + fe * (pe - pc);
  y = y + fw * (pw - pc);
  y = y + fs * (ps - pc);
  y = y + fn * (pn - pc);
  return y;
}

// Complex conj(a) * b accumulated in float (short partial sums of the FP64
// inner products).
__device__ __forceinline__ void dot_acc_f(float& re, float& im, float2 a, float2 b) {
  re = fmaf(a.x, b.x, fmaf(a.y, b.y, re));
  im = fmaf(a.x, b.y, fmaf(-a.y, b.x, im));
}

// ---------------------------------------------------------------------------
// Preconditioner passes shared by the Krylov solvers.
// ---------------------------------------------------------------------------
// Column pass on one field w: forward FFT along z, shifted-Laplace multiply in
// the digit-reversed domain, inverse FFT along z.  Columns [c0, c0+TC) in place.
// Learned spectral multiplier of the 5-point path (the conjugate map of
// nsrno/conditioned_wave.py:112-115): with q2 = 4 (s2z + s2x)/(k0 h)^2, the
// angular term 4 s2x / (4 (s2x + s2z) + h^2) and the basis
// (1, q2/(1+q2), angular, angular q2/(1+q2)),
//   m = exp(tanh(mod0)/2 - i tanh(mod1)/2) / (sym + (k0h)^2 (1 + i s)),
// s = clamp(exp(log_shift), 0.01, 1).  `lp` holds spectral[2][4], log_shift.
struct LearnedSpec {
  float sp[8];
  float shift;
};

__device__ __forceinline__ LearnedSpec load_learned_spec(const float* __restrict__ lp) {
  LearnedSpec L;
#pragma unroll
  for (int k = 0; k < 8; ++k) L.sp[k] = __ldg(&lp[k]);
  L.shift = fminf(fmaxf(expf(__ldg(&lp[8])), 0.01f), 1.0f);
  return L;
}

// tanh from the exponential, 1 - 2 / (e^{2x} + 1); exact at both saturations.
__device__ __forceinline__ float fast_tanh(float x) { return 1.0f - __fdividef(2.0f, __expf(2.0f * x) + 1.0f); }

// The column pass evaluates this once per Fourier point and system, so it uses
// the hardware exponential and sine/cosine (relative error near 1e-6 on these
// bounded arguments): the multiplier is still one fixed function of q, which
// is all the Krylov solvers require of a preconditioner.
__device__ __forceinline__ float2 learned_symbol(const LearnedSpec& L, float s2z, float s2x, float kh2, float h2) {
  const float s4 = 4.0f * (s2z + s2x);
  const float q2 = __fdividef(s4, kh2);
  const float rq = __fdividef(q2, 1.0f + q2);
  const float ang = __fdividef(4.0f * s2x, s4 + h2);
  const float mod0 = L.sp[0] + L.sp[1] * rq + (L.sp[2] + L.sp[3] * rq) * ang;
  const float mod1 = L.sp[4] + L.sp[5] * rq + (L.sp[6] + L.sp[7] * rq) * ang;
  const float mag = __expf(0.5f * fast_tanh(mod0));
  float sn, cs;
  __sincosf(0.5f * fast_tanh(mod1), &sn, &cs);
  // E / D with D = (kh2 - s4) + i kh2 shift
  const float dr = kh2 - s4, di = kh2 * L.shift;
  const float inv = __fdividef(mag, dr * dr + di * di);
  const float er = cs * inv, ei = -sn * inv;
  return make_float2(er * dr + ei * di, ei * dr - er * di);
}

// Column pass with an arbitrary multiplier: `mul(c, z)` is the factor of tile
// column c at digit-reversed z position, including the 1/n of the transform
// pair; columns at or beyond the grid edge are never multiplied.
template <int TC, typename MUL>
__device__ __forceinline__ void cols_pass_with(float2* sm, const Geo& g, const PrecTables& tab,
                                               float2* __restrict__ ws, int c0, MUL mul) {
  const int ncol = min(TC, g.nx - c0);
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    sm[k] = c < ncol ? ws[(long long)z * g.nx + c0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  auto m = [&](int c, int z) -> float2 { return c < ncol ? mul(c, z) : make_float2(0.f, 0.f); };
  if (!fft_cols_fused<TC>(sm, tab.pz, m)) {
    // Sizes without a specialised transform: separate passes.
    fft_cols<false, TC>(sm, tab.pz);
    for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
      const int z = k / TC, c = k - z * TC;
      sm[k] = sm[k] * m(c, z);
    }
    __syncthreads();
    fft_cols<true, TC>(sm, tab.pz);
  }
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    if (c < ncol) ws[(long long)z * g.nx + c0 + c] = sm[k];
  }
}

// The same pass with the first forward and the last inverse stage fused into
// the global load and store (the specialised sizes of nsr_row_padded only);
// STAGED selects cols_pass_with instead (every size: load, every stage in
// shared memory, store).
template <int TC, bool STAGED, typename MUL>
__device__ __forceinline__ void cols_pass_direct(float2* sm, const Geo& g, const PrecTables& tab,
                                                 float2* __restrict__ ws, int c0, MUL mul) {
  if constexpr (STAGED) {
    cols_pass_with<TC>(sm, g, tab, ws, c0, mul);
  } else {
    const int ncol = min(TC, g.nx - c0);
    auto m = [&](int c, int z) -> float2 { return c < ncol ? mul(c, z) : make_float2(0.f, 0.f); };
    fft_cols_direct<TC>(sm, tab.pz, ws + c0, g.nx, ncol, m);
  }
}

// Fixed shifted-Laplace multiplier 1 / (n (-4 (s2z + s2x) + (k0 h)^2 (1 + i shift))).
template <int TC>
__device__ __forceinline__ void cols_pass_fixed(float2* sm, const Geo& g, const PrecTables& tab,
                                                float2* __restrict__ ws, double freq, double shift, int adjoint,
                                                int c0) {
  const SysScalars s = sys_scalars(g, freq);
  const float inv_n = 1.0f / (float)((long long)g.nz * g.nx);
  const float2 shiftc = make_float2((float)s.kh2, (float)(s.kh2 * shift));
  cols_pass_with<TC>(sm, g, tab, ws, c0, [&](int c, int z) -> float2 {
    const float sym = -4.0f * (tab.s2z[z] + tab.s2x[c0 + c]);
    const float2 mul = divc(make_float2(inv_n, 0.f), make_float2(sym + shiftc.x, shiftc.y));
    return adjoint ? conjc(mul) : mul;
  });
}

// Learned multiplier times 1/n at digit-reversed position (z, x) of frequency
// `freq`: the value the batched solver's column pass reads from a system's
// multiplier plane.
__device__ __forceinline__ float2 learned_plane_value(const LearnedSpec& L, const Geo& g, const PrecTables& tab,
                                                      float kh2, int z, int x) {
  const float h2 = (float)(g.h * g.h);
  const float inv_n = 1.0f / (float)((long long)g.nz * g.nx);
  return inv_n * learned_symbol(L, tab.s2z[z], tab.s2x[x], kh2, h2);
}

// Column pass of either preconditioner, chosen at run time: the learned
// multiplier evaluated on the fly from `lp` (non-null), else the fixed one.
template <int TC>
__device__ __forceinline__ void cols_pass(float2* sm, const Geo& g, const PrecTables& tab, float2* __restrict__ ws,
                                          double freq, double shift, int adjoint, int c0,
                                          const float* __restrict__ lp = nullptr) {
  if (!lp) {
    cols_pass_fixed<TC>(sm, g, tab, ws, freq, shift, adjoint, c0);
    return;
  }
  // The spectral parameters go through shared memory so that the fused radix
  // stage keeps its registers for the butterfly.
  __shared__ LearnedSpec Ls;
  if (threadIdx.x == 0) Ls = load_learned_spec(lp);
  __syncthreads();
  const float kh2 = (float)sys_scalars(g, freq).kh2;
  cols_pass_with<TC>(sm, g, tab, ws, c0, [&](int c, int z) -> float2 {
    const float2 mul = learned_plane_value(Ls, g, tab, kh2, z, c0 + c);
    return adjoint ? conjc(mul) : mul;
  });
}

// Rows z0-1 .. z0+nb of w (zero outside the grid) into the padded row layout
// of shared memory, inverse row FFT.  Row rr of the band is sm[(rr+1)*rs].
__device__ __forceinline__ void band_inverse_rows(float2* sm, const Geo& g, const PrecTables& tab,
                                                  const float2* __restrict__ w, int z0, int nb) {
  const int nx = g.nx;
  const int rs = nsr_row_stride(nx);
  const bool pad = nsr_row_padded(nx);
  const int nl = nb + 2;
  for (int rr = 0; rr < nl; ++rr) {
    const int z = z0 - 1 + rr;
    const bool in = z >= 0 && z < g.nz;
#pragma unroll 4
    for (int j = threadIdx.x; j < nx; j += blockDim.x)
      sm[rr * rs + (pad ? j + (j >> 4) : j)] = in ? w[(long long)z * nx + j] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_rows<true>(sm, nl, tab.px);
}

// Stores `val` for element (l, c) of a row tile in the padded row layout.
__device__ __forceinline__ int row_slot(int l, int c, int rs, bool pad) { return l * rs + (pad ? c + (c >> 4) : c); }

// Diagonal gains of the learned preconditioner.  Plane 0 of a gain pair is the
// inner gain (applied before the FFTs), plane 1 the outer one (after them);
// the adjoint applies the conjugated outer gain first and the conjugated
// inner gain last (nsrno/dense_wave.py:163-164).
struct GainPair {
  const float2* pre;    // multiplies the field before the forward FFT (nullptr: none)
  const float2* post;   // multiplies it after the inverse FFT (nullptr: none)
  bool conj;
};

__device__ __forceinline__ GainPair gain_pair(const float2* gains, int gidx, long long n, int adjoint) {
  GainPair G;
  if (!gains) {
    G.pre = G.post = nullptr;
    G.conj = false;
    return G;
  }
  const float2* base = gains + 2LL * gidx * n;
  G.pre = adjoint ? base + n : base;
  G.post = adjoint ? base : base + n;
  G.conj = adjoint != 0;
  return G;
}

__device__ __forceinline__ float2 gain_mul(const float2* plane, long long idx, bool cj, float2 v) {
  float2 gv = __ldg(&plane[idx]);
  if (cj) gv.y = -gv.y;
  return gv * v;
}

// After band_inverse_rows: multiply band rows z0-1 .. z0+nb (those inside the
// grid) by the post gain.
__device__ __forceinline__ void band_post_gain(float2* sm, const Geo& g, const float2* __restrict__ post, bool cj,
                                               int z0, int nb) {
  if (!post) return;
  const int nx = g.nx;
  const int rs = nsr_row_stride(nx);
  const bool pad = nsr_row_padded(nx);
  __syncthreads();
  for (int rr = 0; rr < nb + 2; ++rr) {
    const int z = z0 - 1 + rr;
    if (z < 0 || z >= g.nz) continue;
    for (int j = threadIdx.x; j < nx; j += blockDim.x) {
      float2& v = sm[rr * rs + (pad ? j + (j >> 4) : j)];
      v = gain_mul(post, (long long)z * nx + j, cj, v);
    }
  }
  __syncthreads();
}
