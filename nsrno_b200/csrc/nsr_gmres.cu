// Restarted right-preconditioned GMRES(m) for a batch of 5-point Helmholtz
// systems -- the reference's `gmres` (nsrno/wave_solver.py:9-36), which
// `solve_frequency` uses and which is the fallback of `solve_system`
// (nsrno/dense_wave.py:212-220).
//
// The systems of a batch share the Arnoldi index j, so j is a launch argument
// and one restart cycle is a fixed sequence of launches captured once in a
// CUDA graph.  Per Arnoldi step (8 launches):
//   fwd   v_j = (j ? w / h_{j,j-1} : r / beta), forward row FFT of v_j
//   cols  column FFT, shifted-Laplace multiply, inverse column FFT
//   rinv  inverse row FFT in place: W = M^-1 v_j
//   inv   5-point stencil: w = A W
//   dot   h_i = <v_i, w> (i <= j), FP64 partials, last-CTA sum
//   axpy  w -= sum_i h_i v_i                (classical Gram-Schmidt, pass 1)
//   dot   h'_i = <v_i, w>                   (pass 2)
//   axpy  w -= sum_i h'_i v_i, ||w||^2; the last CTA applies the previous
//         Givens rotations to column j, forms the new one and the residual
//         estimate, all in FP64 on the device (no host least squares).
// At the end of a cycle: back substitution for y (FP64), u = V y fused with
// the forward row FFT, the column and inverse row passes, and an FP64 pass
// that applies x += M^-1 u and recomputes the true residual b - A x.
#include "nsr_internal.cuh"
#include "nsr_device.cuh"

#include <stdlib.h>
#include <string.h>

#define NSR_GMRES_MAX_M 64
#define NSR_GDOT_CELLS 8     // nodes per thread in the dot / axpy kernels

struct __align__(16) GSlot {
  int sys;        // system index, -1 when the slot is empty
  int done;       // finished (status written)
  int status;
  int iters;      // Arnoldi steps so far
  int used;       // Arnoldi steps of the current cycle
  int stop;       // the current cycle ends after step `used`
  int xpar;       // which x buffer holds the iterate
  int gidx;       // gain pair of the learned preconditioner
  double bnorm;   // ||b||
  double beta;    // ||r|| at the start of the cycle
  double resid;   // true relative residual at the start of the cycle
  double hlast;   // h_{j+1,j} of the last step (the norm that normalises v_{j+1})
  double freq, angle;
};

struct GArgs {
  Geo g;
  PrecTables tab;
  MatPlanes mat;
  int m;               // restart length
  int n_slots;
  int nb_band;         // CTAs of the band kernels per slot
  int nb_dot;          // CTAs of the dot/axpy kernels per slot
  int tz, rows, tc;
  double tol;
  double shift;
  int max_it;
  int adjoint;
  GSlot* slots;
  int* arrive;         // [n_slots]
  double* partials;    // [n_slots][max(nb_dot, nb_band)][2 (m+1)]
  double2* H;          // [n_slots][(m+1) m] column-major: H[j*(m+1) + i]
  double* cs;          // [n_slots][m]
  double2* sn;         // [n_slots][m]
  double2* gv;         // [n_slots][m+1]
  double2* hc;         // [n_slots][m+1]  coefficients of the current CGS pass
  double2* y;          // [n_slots][m]
  float2* V;           // [n_slots][m+1][n]
  float2* w;           // [n_slots][n]
  float2* W;           // [n_slots][n]   FFT work field
  float2* r;           // [n_slots][n]
  double2* x;          // [n_slots][2][n]
  const double* freq;
  const double* angle;
  const float2* rhs;
  const float2* x0;
  // Learned preconditioner (all null: the fixed shifted-Laplace one).
  const float* lp;
  const float2* gains;
  const int* gain_index;
};

__device__ __forceinline__ bool g_active(const GSlot& S, int j) {
  return S.sys >= 0 && !S.done && !S.stop && j >= S.used;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return a * b; }
__device__ __forceinline__ double cabs(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

// Per-CTA partials of NV doubles, arrival counter, last CTA returns true with
// the column sums in `tot` (shared, length NV).
template <int NVMAX>
__device__ bool g_reduce(const GArgs& A, int slot, const double* vals, int nv, double* tot) {
  __shared__ double wsum[32][2];
  __shared__ int am_last;
  double* part = A.partials + (long long)slot * max(A.nb_dot, A.nb_band) * 2 * (NSR_GMRES_MAX_M + 1);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int q = 0; q < nv; ++q) {
    double s = warp_sum(vals[q]);
    if (lane == 0) wsum[wid][q & 1] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int u = 0; u < nw; ++u) t += wsum[u][q & 1];
      part[blockIdx.x * 2 * (NSR_GMRES_MAX_M + 1) + q] = t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const int prev = atomicAdd(&A.arrive[slot], 1);
    am_last = (prev == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  for (int q = threadIdx.x; q < nv; q += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) s += __ldcg(&part[b * 2 * (NSR_GMRES_MAX_M + 1) + q]);
    tot[q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) A.arrive[slot] = 0;
  return true;
}

// ---------------------------------------------------------------------------
// fwd: v_j from r (j = 0) or w (j > 0), stored in V and transformed by rows.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) gk_fwd(GArgs A, int j) {
  extern __shared__ float2 sm[];
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  if (!g_active(S, j)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * A.rows;
  const int nr = min(A.rows, g.nz - z0);
  const long long off = (long long)z0 * g.nx;
  const float2* src = (j == 0 ? A.r : A.w) + slot * n + off;
  const float scale = (float)(1.0 / (j == 0 ? S.beta : S.hlast));   // both real and positive
  float2* vj = A.V + ((long long)slot * (A.m + 1) + j) * n + off;
  const int nx = g.nx, rs = nsr_row_stride(nx);
  const bool pad = nsr_row_padded(nx);
  const GainPair G = gain_pair(A.gains, S.gidx, n, A.adjoint);
  for (int l = 0; l < nr; ++l)
    for (int c = threadIdx.x; c < nx; c += blockDim.x) {
      const float2 v = scale * src[l * nx + c];
      vj[l * nx + c] = v;
      sm[row_slot(l, c, rs, pad)] = G.pre ? gain_mul(G.pre, off + l * nx + c, G.conj, v) : v;
    }
  __syncthreads();
  fft_rows<false>(sm, nr, A.tab.px);
  float2* Wp = A.W + slot * n + off;
  for (int l = 0; l < nr; ++l)
    for (int c = threadIdx.x; c < nx; c += blockDim.x) Wp[l * nx + c] = sm[row_slot(l, c, rs, pad)];
}

// cols for slots active at step j (j < 0: slots that run a cycle-end update)
template <int TC>
__global__ void __launch_bounds__(512) gk_cols(GArgs A, int j) {
  extern __shared__ float2 sm[];
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  const bool on = j >= 0 ? g_active(S, j) : (S.sys >= 0 && !S.done && S.used > 0);
  if (!on) return;
  const long long n = (long long)A.g.nz * A.g.nx;
  cols_pass<TC>(sm, A.g, A.tab, A.W + slot * n, S.freq, A.shift, A.adjoint, blockIdx.x * TC, A.lp);
}

// rinv: inverse row FFT of W in place, times the outer gain (W becomes M^-1 v_j,
// or M^-1 u at the end of a cycle when j < 0).
__global__ void __launch_bounds__(256, 4) gk_rinv(GArgs A, int j) {
  extern __shared__ float2 sm[];
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  const bool on = j >= 0 ? g_active(S, j) : (S.sys >= 0 && !S.done && S.used > 0);
  if (!on) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * A.rows;
  const int nr = min(A.rows, g.nz - z0);
  const long long off = (long long)z0 * g.nx;
  float2* __restrict__ Wp = A.W + slot * n + off;
  const int nx = g.nx, rs = nsr_row_stride(nx);
  const bool pad = nsr_row_padded(nx);
  for (int l = 0; l < nr; ++l)
    for (int c = threadIdx.x; c < nx; c += blockDim.x) sm[row_slot(l, c, rs, pad)] = Wp[l * nx + c];
  __syncthreads();
  fft_rows<true>(sm, nr, A.tab.px);
  __syncthreads();
  const GainPair G = gain_pair(A.gains, S.gidx, n, A.adjoint);
  for (int l = 0; l < nr; ++l)
    for (int c = threadIdx.x; c < nx; c += blockDim.x) {
      const float2 v = sm[row_slot(l, c, rs, pad)];
      Wp[l * nx + c] = G.post ? gain_mul(G.post, off + l * nx + c, G.conj, v) : v;
    }
}

// inv: w = A z with z = M^-1 v_j in W.  One thread per column of a
// NSR_GST_TZ x NSR_GST_TX tile walks down its rows with the north/centre/south
// values of z and a in registers.
#define NSR_GST_TZ 32
#define NSR_GST_TX 256
template <bool ADJ>
__global__ void __launch_bounds__(256, 4) gk_inv(GArgs A, int j) {
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  if (!g_active(S, j)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int nx = g.nx;
  const int nbx = (nx + NSR_GST_TX - 1) / NSR_GST_TX;
  const int rb = blockIdx.x / nbx, cb = blockIdx.x - rb * nbx;
  const int z0 = rb * NSR_GST_TZ;
  const int z1 = min(z0 + NSR_GST_TZ, g.nz);
  const int jj = cb * NSR_GST_TX + threadIdx.x;
  if (jj >= nx) return;
  const SysScalars sc = sys_scalars(g, S.freq);
  const float* __restrict__ ca = A.mat.a32;
  const float2* __restrict__ z = A.W + slot * n;
  float2* __restrict__ w = A.w + slot * n;
  const float2 zero = make_float2(0.f, 0.f);
  const bool has_e = jj + 1 < nx, has_w = jj > 0;
  long long idx = (long long)z0 * nx + jj;
  float2 zu = z0 > 0 ? z[idx - nx] : zero;
  float2 zc = z[idx];
  float a_n = z0 > 0 ? __ldg(&ca[idx - nx]) : 1.0f;
  float a_c = __ldg(&ca[idx]);
  for (int i = z0; i < z1; ++i, idx += nx) {
    const bool has_s = i + 1 < g.nz;
    const float2 zd = has_s ? z[idx + nx] : zero;
    const float a_s = has_s ? __ldg(&ca[idx + nx]) : 1.0f;
    const float2 ze = has_e ? z[idx + 1] : zero;
    const float2 zw = has_w ? z[idx - 1] : zero;
    const float a_e = has_e ? __ldg(&ca[idx + 1]) : 1.0f;
    const float a_w = has_w ? __ldg(&ca[idx - 1]) : 1.0f;
    w[idx] = stencil_pts<ADJ>(g, sc, i, jj, a_c, a_e, a_w, a_s, a_n, __ldg(&A.mat.b32[idx]), __ldg(&A.mat.t32[idx]),
                              zc, ze, zw, zd, zu);
    zu = zc;
    zc = zd;
    a_n = a_c;
    a_c = a_s;
  }
}

// dot: hc_i = <v_i, w> for i <= j (FP64), into hc (pass 1 overwrites, pass 2 too)
__global__ void __launch_bounds__(256) gk_dot(GArgs A, int j) {
  __shared__ double tot[2 * (NSR_GMRES_MAX_M + 1)];
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  if (!g_active(S, j)) return;
  const long long n = (long long)A.g.nz * A.g.nx;
  const long long base = (long long)blockIdx.x * blockDim.x * NSR_GDOT_CELLS;
  const float2* w = A.w + slot * n;
  float2 wl[NSR_GDOT_CELLS];
#pragma unroll
  for (int c = 0; c < NSR_GDOT_CELLS; ++c) {
    const long long k = base + (long long)c * blockDim.x + threadIdx.x;
    wl[c] = k < n ? w[k] : make_float2(0.f, 0.f);
  }
  double vals[2 * (NSR_GMRES_MAX_M + 1)];
  for (int i = 0; i <= j; ++i) {
    const float2* v = A.V + ((long long)slot * (A.m + 1) + i) * n;
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int c = 0; c < NSR_GDOT_CELLS; ++c) {
      const long long k = base + (long long)c * blockDim.x + threadIdx.x;
      if (k < n) dot_acc(re, im, v[k], wl[c]);
    }
    vals[2 * i] = re;
    vals[2 * i + 1] = im;
  }
  if (g_reduce<2 * (NSR_GMRES_MAX_M + 1)>(A, slot, vals, 2 * (j + 1), tot)) {
    for (int i = threadIdx.x; i <= j; i += blockDim.x)
      A.hc[(long long)slot * (A.m + 1) + i] = make_double2(tot[2 * i], tot[2 * i + 1]);
  }
}

// axpy: w -= sum_i hc_i v_i.  Pass 1 adds hc into H; pass 2 adds hc into H,
// takes ||w||, applies the Givens rotations and decides whether the cycle stops.
__global__ void __launch_bounds__(256) gk_axpy(GArgs A, int j, int pass) {
  __shared__ double tot[2];
  __shared__ float2 coef[NSR_GMRES_MAX_M + 1];
  const int slot = blockIdx.y;
  GSlot& S = A.slots[slot];
  if (!g_active(S, j)) return;
  const long long n = (long long)A.g.nz * A.g.nx;
  const int m = A.m;
  const double2* hc = A.hc + (long long)slot * (m + 1);
  for (int i = threadIdx.x; i <= j; i += blockDim.x) coef[i] = to_f(hc[i]);
  __syncthreads();
  const long long base = (long long)blockIdx.x * blockDim.x * NSR_GDOT_CELLS;
  float2* w = A.w + slot * n;
  double nrm = 0.0;
#pragma unroll
  for (int c = 0; c < NSR_GDOT_CELLS; ++c) {
    const long long k = base + (long long)c * blockDim.x + threadIdx.x;
    if (k >= n) continue;
    float2 acc = w[k];
    for (int i = 0; i <= j; ++i) acc = acc - coef[i] * A.V[((long long)slot * (m + 1) + i) * n + k];
    w[k] = acc;
    nrm += (double)acc.x * acc.x + (double)acc.y * acc.y;
  }
  double vals[1] = {nrm};
  // Pass 1 needs no reduction: the coefficients go into H by the first CTA.
  if (pass == 1) {
    if (blockIdx.x == 0)
      for (int i = threadIdx.x; i <= j; i += blockDim.x)
        A.H[(long long)slot * (m + 1) * m + j * (m + 1) + i] = hc[i];
    return;
  }
  if (!g_reduce<2>(A, slot, vals, 1, tot)) return;
  if (threadIdx.x != 0) return;
  double2* Hc = A.H + (long long)slot * (m + 1) * m + j * (m + 1);   // column j
  for (int i = 0; i <= j; ++i) Hc[i] = Hc[i] + hc[i];
  const double hnext = sqrt(tot[0]);
  Hc[j + 1] = make_double2(hnext, 0.0);
  S.hlast = hnext;
  double* cs = A.cs + (long long)slot * m;
  double2* sn = A.sn + (long long)slot * m;
  double2* gv = A.gv + (long long)slot * (m + 1);
  // previous rotations on column j
  for (int i = 0; i < j; ++i) {
    const double2 a = Hc[i], b = Hc[i + 1];
    Hc[i] = cs[i] * a + cmul(sn[i], b);
    Hc[i + 1] = cs[i] * b - cmul(conjc(sn[i]), a);
  }
  // new rotation zeroing Hc[j+1]
  const double2 a = Hc[j];
  const double b = hnext;
  const double aa = cabs(a);
  const double nu = sqrt(aa * aa + b * b);
  double c;
  double2 s;
  if (aa == 0.0) {
    c = 0.0;
    s = make_double2(1.0, 0.0);
    Hc[j] = make_double2(b, 0.0);
  } else {
    const double2 ph = make_double2(a.x / aa, a.y / aa);
    c = aa / nu;
    s = make_double2(ph.x * b / nu, ph.y * b / nu);
    Hc[j] = make_double2(ph.x * nu, ph.y * nu);
  }
  Hc[j + 1] = make_double2(0.0, 0.0);
  cs[j] = c;
  sn[j] = s;
  const double2 gj = gv[j];
  gv[j] = c * gj;
  gv[j + 1] = make_double2(0.0, 0.0) - cmul(conjc(s), gj);
  S.used = j + 1;
  S.iters += 1;
  const double est = cabs(gv[j + 1]) / S.bnorm;
  // Stop the cycle on convergence of the estimate, on a happy breakdown
  // (nsrno/wave_solver.py:31-32), at the restart length or at the budget.
  if (est < 0.5 * A.tol || !(hnext > 1e-12 * S.beta) || j + 1 == m || S.iters >= A.max_it || !isfinite(est))
    S.stop = 1;
}

// Back substitution R y = g for the slots that ran a cycle.
__global__ void gk_solve(GArgs A) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= A.n_slots) return;
  GSlot& S = A.slots[slot];
  if (S.sys < 0 || S.done || S.used == 0) return;
  const int m = A.m, u = S.used;
  const double2* H = A.H + (long long)slot * (m + 1) * m;
  const double2* gv = A.gv + (long long)slot * (m + 1);
  double2* y = A.y + (long long)slot * m;
  for (int i = u - 1; i >= 0; --i) {
    double2 acc = gv[i];
    for (int k = i + 1; k < u; ++k) acc = acc - cmul(H[k * (m + 1) + i], y[k]);
    y[i] = divc(acc, H[i * (m + 1) + i]);
  }
}

// u = V y, forward row FFT into W.
__global__ void __launch_bounds__(256) gk_comb(GArgs A) {
  extern __shared__ float2 sm[];
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  if (S.sys < 0 || S.done || S.used == 0) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int m = A.m, u = S.used;
  __shared__ float2 yc[NSR_GMRES_MAX_M];
  for (int i = threadIdx.x; i < u; i += blockDim.x) yc[i] = to_f(A.y[(long long)slot * m + i]);
  __syncthreads();
  const int z0 = blockIdx.x * A.rows;
  const int nr = min(A.rows, g.nz - z0);
  const long long off = (long long)z0 * g.nx;
  const int nx = g.nx, rs = nsr_row_stride(nx);
  const bool pad = nsr_row_padded(nx);
  const GainPair G = gain_pair(A.gains, S.gidx, n, A.adjoint);
  for (int l = 0; l < nr; ++l)
    for (int c = threadIdx.x; c < nx; c += blockDim.x) {
      float2 acc = make_float2(0.f, 0.f);
      for (int i = 0; i < u; ++i) acc = acc + yc[i] * A.V[((long long)slot * (m + 1) + i) * n + off + l * nx + c];
      sm[row_slot(l, c, rs, pad)] = G.pre ? gain_mul(G.pre, off + l * nx + c, G.conj, acc) : acc;
    }
  __syncthreads();
  fft_rows<false>(sm, nr, A.tab.px);
  float2* Wp = A.W + slot * n + off;
  for (int l = 0; l < nr; ++l)
    for (int c = threadIdx.x; c < nx; c += blockDim.x) Wp[l * nx + c] = sm[row_slot(l, c, rs, pad)];
}

// FP64 true residual.  init = 1: x = x0 (or 0); init = 0: x += M^-1 V y.
template <bool ADJ>
__global__ void __launch_bounds__(256) gk_res(GArgs A, int init) {
  const int slot = blockIdx.y;
  GSlot& S = A.slots[slot];
  if (S.sys < 0 || S.done) return;
  if (!init && S.used == 0) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * A.tz;
  const int nb = min(A.tz, g.nz - z0);
  const int nx = g.nx;
  const float2* zW = A.W + slot * n;   // M^-1 u after the rinv pass
  const SysScalars sc = sys_scalars(g, S.freq);
  const double2* xo = A.x + (2LL * slot + S.xpar) * n;
  double2* xn = A.x + (2LL * slot + (S.xpar ^ 1)) * n;
  const float2* x0 = (init && A.x0) ? A.x0 + (long long)S.sys * n : nullptr;
  auto P = [&](int i2, int j2) -> double2 {
    if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= nx) return make_double2(0.0, 0.0);
    const long long id = (long long)i2 * nx + j2;
    if (init) return x0 ? to_d(x0[id]) : make_double2(0.0, 0.0);
    return xo[id] + to_d(zW[id]);
  };
  auto Aa = [&](int i2, int j2) -> double {
    if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= nx) return 1.0;
    return __ldg(&A.mat.a64[(long long)i2 * nx + j2]);
  };
  const double h2 = g.h * g.h;
  const float2* rhs = A.rhs ? A.rhs + (long long)S.sys * n : nullptr;
  const double st = sin(S.angle);
  float2* r = A.r + slot * n;
  double acc[2] = {0.0, 0.0};
  for (int k = threadIdx.x; k < nb * nx; k += blockDim.x) {
    const int i = z0 + k / nx, jj = k % nx;
    const long long idx = (long long)i * nx + jj;
    double2 b;
    if (rhs) {
      b = h2 * to_d(rhs[idx]);
    } else if (i == g.face) {
      const double2 l = source_line(g, sc.k0, st, jj);
      b = make_double2(-l.x, -l.y);
    } else {
      b = make_double2(0.0, 0.0);
    }
    const double2 ax = stencil<double, ADJ>(g, sc, i, jj, __ldg(&A.mat.b64[idx]), __ldg(&A.mat.t64[idx]), P, Aa);
    const double2 res = b - ax;
    xn[idx] = P(i, jj);
    const float2 rf = to_f(res);
    r[idx] = rf;
    acc[0] += res.x * res.x + res.y * res.y;
    acc[1] += b.x * b.x + b.y * b.y;
  }
  __shared__ double red[NSR_NPART];
  double vals[NSR_NPART] = {acc[0], acc[1], 0, 0, 0, 0, 0, 0};
  block_sum<NSR_NPART>(vals, red);
  double* part = A.partials + (long long)slot * max(A.nb_dot, A.nb_band) * 2 * (NSR_GMRES_MAX_M + 1);
  __shared__ int am_last;
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2 * (NSR_GMRES_MAX_M + 1)] = red[0];
    part[blockIdx.x * 2 * (NSR_GMRES_MAX_M + 1) + 1] = red[1];
    __threadfence();
    am_last = atomicAdd(&A.arrive[slot], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double rr = 0.0, bb = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) {
      rr += __ldcg(&part[b * 2 * (NSR_GMRES_MAX_M + 1)]);
      bb += __ldcg(&part[b * 2 * (NSR_GMRES_MAX_M + 1) + 1]);
    }
    A.arrive[slot] = 0;
    S.xpar ^= 1;
    if (init) S.bnorm = sqrt(bb);
    const double rn = sqrt(rr);
    const double rel = S.bnorm > 0.0 ? rn / S.bnorm : 0.0;
    S.resid = rel;
    S.used = 0;
    S.stop = 0;
    S.beta = rn;
    if (!(S.bnorm > 0.0)) {
      S.done = 1;
      S.status = isfinite(S.bnorm) ? NSR_CONVERGED : NSR_NONFINITE;
      S.resid = 0.0;
    } else if (!isfinite(rel)) {
      S.done = 1;
      S.status = NSR_NONFINITE;
    } else if (rel < A.tol) {
      S.done = 1;
      S.status = NSR_CONVERGED;
    } else if (S.iters >= A.max_it) {
      S.done = 1;
      S.status = NSR_ITERATION_BUDGET;
    } else {
      double2* gv = A.gv + (long long)slot * (A.m + 1);
      gv[0] = make_double2(rn, 0.0);
    }
    __threadfence();
  }
}

// Outputs of one batch: IQ, residual, iterations, status, fields.
__global__ void gk_emit(GArgs A, double2* iq, const int* rx, int n_rx, double* residual, int* iterations,
                        int* status, void* fields, int fields_fp64) {
  const int slot = blockIdx.y;
  const GSlot& S = A.slots[slot];
  if (S.sys < 0) return;
  const long long n = (long long)A.g.nz * A.g.nx;
  const double2* x = A.x + (2LL * slot + S.xpar) * n;
  const bool zero = !(S.bnorm > 0.0);
  if (blockIdx.x == 0) {
    for (int k = threadIdx.x; k < n_rx; k += blockDim.x) {
      const int idx = rx[k];
      const bool ok = idx >= 0 && (long long)idx < n;
      iq[(long long)S.sys * n_rx + k] = !ok ? make_double2(NAN, NAN) : (zero ? make_double2(0.0, 0.0) : x[idx]);
    }
    if (threadIdx.x == 0) {
      residual[S.sys] = S.resid;
      iterations[S.sys] = S.iters;
      status[S.sys] = S.done ? S.status : NSR_ITERATION_BUDGET;
    }
  }
  if (fields) {
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
      const double2 v = zero ? make_double2(0.0, 0.0) : x[k];
      if (fields_fp64) ((double2*)fields)[(long long)S.sys * n + k] = v;
      else ((float2*)fields)[(long long)S.sys * n + k] = to_f(v);
    }
  }
}

__global__ void gk_load(GArgs A, int first, int count, const double* freq, const double* angle) {
  const int slot = blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= A.n_slots) return;
  GSlot S;
  memset(&S, 0, sizeof(S));
  if (slot < count) {
    S.sys = first + slot;
    S.gidx = A.gain_index ? A.gain_index[first + slot] : first + slot;
    S.freq = freq[first + slot];
    S.angle = angle ? angle[first + slot] : 0.0;
  } else {
    S.sys = -1;
    S.done = 1;
  }
  A.slots[slot] = S;
  A.arrive[slot] = 0;
}

__global__ void gk_count(GArgs A, int* remaining) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < A.n_slots; s += blockDim.x)
    if (A.slots[s].sys >= 0 && !A.slots[s].done) atomicAdd(&cnt, 1);
  __syncthreads();
  if (threadIdx.x == 0) *remaining = cnt;
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct GLayout {
  size_t tables, slots, arrive, count, partials, H, cs, sn, gv, hc, y, V, w, W, r, x, total;
  int nb_band, nb_dot, tz;
};

static int g_band_rows(const NsrGrid* g) {
  int budget = g->nx <= 1024 ? 8192 : 16384;
  int tz = budget / g->nx - 2;
  if (tz < 1) tz = 1;
  if (tz > g->nz) tz = g->nz;
  return tz;
}

static GLayout g_layout(const NsrGrid* g, int n_slots, int m) {
  GLayout L;
  const size_t n = (size_t)g->nz * g->nx;
  L.tz = g_band_rows(g);
  L.nb_band = (g->nz + L.tz - 1) / L.tz;
  L.nb_dot = (int)((n + 256 * NSR_GDOT_CELLS - 1) / (256 * NSR_GDOT_CELLS));
  const int nbm = L.nb_band > L.nb_dot ? L.nb_band : L.nb_dot;
  size_t off = 0;
  L.tables = off; off += nsr_align(nsr_prec_table_bytes(g));
  L.slots = off; off += nsr_align(sizeof(GSlot) * n_slots);
  L.arrive = off; off += nsr_align(sizeof(int) * n_slots);
  L.count = off; off += nsr_align(sizeof(int));
  L.partials = off; off += nsr_align(sizeof(double) * (size_t)n_slots * nbm * 2 * (NSR_GMRES_MAX_M + 1));
  L.H = off; off += nsr_align(sizeof(double2) * (size_t)n_slots * (m + 1) * m);
  L.cs = off; off += nsr_align(sizeof(double) * (size_t)n_slots * m);
  L.sn = off; off += nsr_align(sizeof(double2) * (size_t)n_slots * m);
  L.gv = off; off += nsr_align(sizeof(double2) * (size_t)n_slots * (m + 1));
  L.hc = off; off += nsr_align(sizeof(double2) * (size_t)n_slots * (m + 1));
  L.y = off; off += nsr_align(sizeof(double2) * (size_t)n_slots * m);
  L.V = off; off += nsr_align(sizeof(float2) * n * (m + 1) * n_slots);
  L.w = off; off += nsr_align(sizeof(float2) * n * n_slots);
  L.W = off; off += nsr_align(sizeof(float2) * n * n_slots);
  L.r = off; off += nsr_align(sizeof(float2) * n * n_slots);
  L.x = off; off += nsr_align(sizeof(double2) * n * 2 * n_slots);
  L.total = off;
  return L;
}

extern "C" size_t nsr_gmres_workspace_size(const NsrGrid* grid, int32_t n_slots, int32_t restart) {
  if (nsr_check_grid(grid, true) || n_slots <= 0 || n_slots > 65535 || restart < 1 || restart > NSR_GMRES_MAX_M)
    return 0;
  return g_layout(grid, n_slots, restart).total;
}

extern "C" int nsr_gmres_batched(const NsrGrid* grid, const void* material, const double* freq_hz,
                                 const double* angle_rad, int32_t n_systems, const float* rhs, const float* x0,
                                 const int32_t* rx_index, int32_t n_rx, const NsrGmresParams* params,
                                 void* workspace, size_t workspace_bytes, double* iq, double* residual,
                                 int32_t* iterations, int32_t* status, void* fields, void* stream) {
  int err = nsr_check_grid(grid, true);
  if (err) return err;
  if (!params || !material || n_systems < 0 || n_rx < 0) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;   // an empty batch touches no buffer
  if (!freq_hz || (n_rx > 0 && (!rx_index || !iq))) return NSR_ERR_ARGUMENT;
  if (!rhs && !angle_rad) return NSR_ERR_ARGUMENT;
  if (!residual || !iterations || !status || !workspace) return NSR_ERR_ARGUMENT;
  const int m = params->restart, n_slots = params->n_slots;
  if (m < 1 || m > NSR_GMRES_MAX_M || n_slots <= 0 || n_slots > 65535 || !(params->tolerance > 0) ||
      params->max_iterations <= 0 || !(params->shift >= 0))
    return NSR_ERR_ARGUMENT;
  if (params->learned && !params->learned->params) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  const GLayout L = g_layout(grid, n_slots, m);
  if (workspace_bytes < L.total) return NSR_ERR_WORKSPACE;
  const size_t n = (size_t)grid->nz * grid->nx;
  cudaStream_t caller = (cudaStream_t)stream;
  cudaStream_t st = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int remaining_host = 0;
  cudaError_t ce;
#define NSR_TRY(x) do { ce = (x); if (ce != cudaSuccess) { err = (int)ce; goto cleanup; } } while (0)
  {
    NSR_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    NSR_TRY(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    NSR_TRY(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
    NSR_TRY(cudaEventRecord(ev_in, caller));
    NSR_TRY(cudaStreamWaitEvent(st, ev_in, 0));
    err = nsr_check_learned(params->learned, n_systems, st);
    if (err) goto cleanup;
    char* ws = (char*)workspace;
    GArgs A;
    memset(&A, 0, sizeof(A));
    A.g = make_geo(*grid);
    err = nsr_prec_setup(grid, &A.tab, ws + L.tables, st);
    if (err) goto cleanup;
    A.mat = nsr_planes(material, (long long)n);
    A.m = m;
    A.n_slots = n_slots;
    A.nb_band = L.nb_band;
    A.nb_dot = L.nb_dot;
    A.tz = L.tz;
    A.rows = nsr_rows_per_cta(grid);
    A.tc = nsr_cols_tc(grid);
    A.tol = params->tolerance;
    A.shift = params->shift;
    A.max_it = params->max_iterations;
    A.adjoint = params->adjoint ? 1 : 0;
    A.slots = (GSlot*)(ws + L.slots);
    A.arrive = (int*)(ws + L.arrive);
    int* remaining = (int*)(ws + L.count);
    A.partials = (double*)(ws + L.partials);
    A.H = (double2*)(ws + L.H);
    A.cs = (double*)(ws + L.cs);
    A.sn = (double2*)(ws + L.sn);
    A.gv = (double2*)(ws + L.gv);
    A.hc = (double2*)(ws + L.hc);
    A.y = (double2*)(ws + L.y);
    A.V = (float2*)(ws + L.V);
    A.w = (float2*)(ws + L.w);
    A.W = (float2*)(ws + L.W);
    A.r = (float2*)(ws + L.r);
    A.x = (double2*)(ws + L.x);
    A.freq = freq_hz;
    A.angle = rhs ? nullptr : angle_rad;
    A.rhs = (const float2*)rhs;
    A.x0 = (const float2*)x0;
    if (params->learned) {
      A.lp = params->learned->params;
      A.gains = (const float2*)params->learned->gains;
      A.gain_index = params->learned->gain_index;
    }

    const int rs = nsr_row_stride(grid->nx);
    const size_t fwd_smem = sizeof(float2) * A.rows * rs;
    const size_t col_smem = nsr_cols_smem(grid);
    const int nb_st = ((grid->nz + NSR_GST_TZ - 1) / NSR_GST_TZ) * ((grid->nx + NSR_GST_TX - 1) / NSR_GST_TX);
    NSR_TRY(cudaFuncSetAttribute(gk_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem));
    NSR_TRY(cudaFuncSetAttribute(gk_comb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem));
    NSR_TRY(cudaFuncSetAttribute(gk_cols<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem));
    NSR_TRY(cudaFuncSetAttribute(gk_cols<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem));
    NSR_TRY(cudaFuncSetAttribute(gk_rinv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem));

    const dim3 g_rows((grid->nz + A.rows - 1) / A.rows, n_slots);
    const dim3 g_col((grid->nx + A.tc - 1) / A.tc, n_slots);
    const dim3 g_band(L.nb_band, n_slots);
    const dim3 g_st(nb_st, n_slots);
    const dim3 g_dot(L.nb_dot, n_slots);
    auto cols = [&](int j) {
      if (A.tc == 16) gk_cols<16><<<g_col, 512, col_smem, st>>>(A, j);
      else gk_cols<8><<<g_col, 512, col_smem, st>>>(A, j);
    };
    auto res = [&](int init) {
      if (A.adjoint) gk_res<true><<<g_band, 256, 0, st>>>(A, init);
      else gk_res<false><<<g_band, 256, 0, st>>>(A, init);
    };

    // One restart cycle.
    NSR_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int j = 0; j < m; ++j) {
      gk_fwd<<<g_rows, 256, fwd_smem, st>>>(A, j);
      cols(j);
      gk_rinv<<<g_rows, 256, fwd_smem, st>>>(A, j);
      if (A.adjoint) gk_inv<true><<<g_st, 256, 0, st>>>(A, j);
      else gk_inv<false><<<g_st, 256, 0, st>>>(A, j);
      gk_dot<<<g_dot, 256, 0, st>>>(A, j);
      gk_axpy<<<g_dot, 256, 0, st>>>(A, j, 1);
      gk_dot<<<g_dot, 256, 0, st>>>(A, j);
      gk_axpy<<<g_dot, 256, 0, st>>>(A, j, 2);
    }
    gk_solve<<<(n_slots + 127) / 128, 128, 0, st>>>(A);
    gk_comb<<<g_rows, 256, fwd_smem, st>>>(A);
    cols(-1);
    gk_rinv<<<g_rows, 256, fwd_smem, st>>>(A, -1);
    res(0);
    gk_count<<<1, 256, 0, st>>>(A, remaining);
    ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) { err = (int)ce; goto cleanup; }
    NSR_TRY(cudaGraphInstantiate(&exec, graph, 0));

    const int max_cycles = (params->max_iterations + m - 1) / m + 1;
    for (int first = 0; first < n_systems; first += n_slots) {
      const int count = (n_systems - first) < n_slots ? (n_systems - first) : n_slots;
      gk_load<<<(n_slots + 127) / 128, 128, 0, st>>>(A, first, count, freq_hz, A.angle);
      NSR_TRY(cudaGetLastError());
      res(1);
      NSR_TRY(cudaGetLastError());
      for (int cyc = 0; cyc < max_cycles; ++cyc) {
        NSR_TRY(cudaGraphLaunch(exec, st));
        NSR_TRY(cudaMemcpyAsync(&remaining_host, remaining, sizeof(int), cudaMemcpyDeviceToHost, st));
        NSR_TRY(cudaStreamSynchronize(st));
        if (remaining_host == 0) break;
      }
      dim3 g_emit(fields ? 148 : 1, n_slots);
      gk_emit<<<g_emit, 256, 0, st>>>(A, (double2*)iq, rx_index, n_rx, residual, iterations, status, fields,
                                      params->fields_fp64);
      NSR_TRY(cudaGetLastError());
    }
    NSR_TRY(cudaEventRecord(ev_out, st));
    NSR_TRY(cudaStreamWaitEvent(caller, ev_out, 0));
  }
cleanup:
  if (st) cudaStreamSynchronize(st);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (ev_in) cudaEventDestroy(ev_in);
  if (ev_out) cudaEventDestroy(ev_out);
  if (st) cudaStreamDestroy(st);
#undef NSR_TRY
  return err;
}
