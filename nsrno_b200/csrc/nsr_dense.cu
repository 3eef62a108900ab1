// The dense path's operator (nsrno/conditioned_wave.py:52-80, projected as in
// nsrno/dense_wave.py:66-68) and its analytic adjoint (nsrno/dense_wave.py:70-82),
// evaluated as a direct radius-4 staggered stencil instead of 11 FFTs.
//
// The reference evaluates the 8th-order staggered derivative D (forward, at
// n + 1/2) and its negative adjoint (divergence) by FFT on a padded grid.  The
// field is masked to the native region and the padding is at least 8 nodes
// wide, so the periodic FFT evaluation equals the direct stencil with zero
// values outside the grid:
//   (D p)[n]     = (1/dx) sum_k a_k (p[n+1+k] - p[n-k])
//   (-D^H f)[n]  = (1/dx) sum_k a_k (f[n+k]   - f[n-1-k])
// with a = (1225/1024, -245/3072, 49/5120, -5/7168).
// Pass 1 writes the staggered fluxes, pass 2 takes their divergence.
#include "nsr_internal.cuh"

#include <string.h>

__constant__ double c_dense_a[4] = {1225.0 / 1024.0, -245.0 / 3072.0, 49.0 / 5120.0, -5.0 / 7168.0};

struct DenseCoef {
  // planes [H][W]
  const double* ax;
  const double* az;
  const double2* mass;
  // profiles along x [W] and z [H]
  const double2 *svx, *gvx, *lx, *rx;
  const double2 *svz, *gvz, *lz, *rz;
};

struct DenseGeo {
  int H, W, pz, px, h, w;
  double dx;
  double2 scal;   // (D - 1) / (D k0^2)
};

__host__ __device__ inline size_t dense_coef_doubles(int H, int W) { return (size_t)H * W * 4 + 8 * (size_t)W + 8 * (size_t)H; }

__host__ __device__ inline DenseCoef dense_unpack(const double* c, int H, int W) {
  DenseCoef d;
  const size_t n = (size_t)H * W;
  d.ax = c;
  d.az = c + n;
  d.mass = (const double2*)(c + 2 * n);
  const double2* px = (const double2*)(c + 4 * n);
  d.svx = px; d.gvx = px + W; d.lx = px + 2 * W; d.rx = px + 3 * W;
  const double2* pz = px + 4 * W;
  d.svz = pz; d.gvz = pz + H; d.lz = pz + 2 * H; d.rz = pz + 3 * H;
  return d;
}

template <typename T> struct DC;
template <> struct DC<float> { typedef float2 C; static __device__ C from(double2 a) { return make_float2((float)a.x, (float)a.y); } };
template <> struct DC<double> { typedef double2 C; static __device__ C from(double2 a) { return a; } };

__device__ __forceinline__ bool dense_inside(const DenseGeo& g, int i, int j) {
  return i >= g.pz && i < g.pz + g.h && j >= g.px && j < g.px + g.w;
}

// Pass 1.  Forward: X = ax svx D_x(mask p), gX = gvx X, and the same along z.
// Adjoint: w = conj(scal) mask p, flux_x = conj(ax svx) (-D_x(conj(lx) w) - conj(gvx) D_x(conj(rx) w)).
template <typename T, bool ADJ>
__global__ void k_dense_flux(DenseGeo g, const double* __restrict__ coef, const typename DC<T>::C* __restrict__ p,
                             typename DC<T>::C* __restrict__ tmp, int nf) {
  typedef typename DC<T>::C C;
  const DenseCoef dc = dense_unpack(coef, g.H, g.W);
  const long long n = (long long)g.H * g.W;
  const int f = blockIdx.y;
  const C* pf = p + f * n;
  C* t = tmp + f * 4 * n;
  const C zero = cx<C>(T(0), T(0));
  const T inv_dx = (T)(1.0 / g.dx);
  const C wscal = DC<T>::from(conjc(g.scal));
  auto PM = [&](int i2, int j2) -> C {
    if (i2 < 0 || i2 >= g.H || j2 < 0 || j2 >= g.W || !dense_inside(g, i2, j2)) return zero;
    return pf[(long long)i2 * g.W + j2];
  };
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.W), j = (int)(k - (long long)i * g.W);
    if (!ADJ) {
      C gx = zero, gz = zero;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T a = (T)c_dense_a[q];
        gx = gx + a * (PM(i, j + 1 + q) - PM(i, j - q));
        gz = gz + a * (PM(i + 1 + q, j) - PM(i - q, j));
      }
      const C X = (inv_dx * (T)dc.ax[k]) * (DC<T>::from(dc.svx[j]) * gx);
      const C Z = (inv_dx * (T)dc.az[k]) * (DC<T>::from(dc.svz[i]) * gz);
      t[k] = X;
      t[n + k] = DC<T>::from(dc.gvx[j]) * X;
      t[2 * n + k] = Z;
      t[3 * n + k] = DC<T>::from(dc.gvz[i]) * Z;
    } else {
      // along x the left/right factors depend on the column of each node
      C fl = zero, fr = zero, zl = zero, zr = zero;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T a = (T)c_dense_a[q];
        const int je = j + 1 + q, jw = j - q;
        const C we = PM(i, je), ww = PM(i, jw);
        const C le = je < g.W ? conjc(DC<T>::from(dc.lx[je])) * we : zero;
        const C lw = jw >= 0 ? conjc(DC<T>::from(dc.lx[jw])) * ww : zero;
        const C re = je < g.W ? conjc(DC<T>::from(dc.rx[je])) * we : zero;
        const C rw = jw >= 0 ? conjc(DC<T>::from(dc.rx[jw])) * ww : zero;
        fl = fl + a * (le - lw);
        fr = fr + a * (re - rw);
        const int is = i + 1 + q, in = i - q;
        const C ws = PM(is, j), wn = PM(in, j);
        const C ls = is < g.H ? conjc(DC<T>::from(dc.lz[is])) * ws : zero;
        const C ln = in >= 0 ? conjc(DC<T>::from(dc.lz[in])) * wn : zero;
        const C rs = is < g.H ? conjc(DC<T>::from(dc.rz[is])) * ws : zero;
        const C rn = in >= 0 ? conjc(DC<T>::from(dc.rz[in])) * wn : zero;
        zl = zl + a * (ls - ln);
        zr = zr + a * (rs - rn);
      }
      // w = conj(scal) mask p was left out of the sums: apply it once here
      const C fx = (T(-1) * inv_dx) * (wscal * (fl + conjc(DC<T>::from(dc.gvx[j])) * fr));
      const C fz = (T(-1) * inv_dx) * (wscal * (zl + conjc(DC<T>::from(dc.gvz[i])) * zr));
      t[k] = conjc(DC<T>::from(dc.svx[j]) * cx<C>((T)dc.ax[k], T(0))) * fx;
      t[2 * n + k] = conjc(DC<T>::from(dc.svz[i]) * cx<C>((T)dc.az[k], T(0))) * fz;
    }
  }
}

// Pass 2.  Forward: y = mask (scal (lx divX + rx div gX + lz divZ + rz div gZ) + mass p) + (1 - mask) p.
// Adjoint: y = mask (D^H flux_x + D^H flux_z + conj(mass) p) + (1 - mask) p.
template <typename T, bool ADJ>
__global__ void k_dense_div(DenseGeo g, const double* __restrict__ coef, const typename DC<T>::C* __restrict__ p,
                            const typename DC<T>::C* __restrict__ tmp, typename DC<T>::C* __restrict__ y, int nf) {
  typedef typename DC<T>::C C;
  const DenseCoef dc = dense_unpack(coef, g.H, g.W);
  const long long n = (long long)g.H * g.W;
  const int f = blockIdx.y;
  const C* pf = p + f * n;
  const C* t = tmp + f * 4 * n;
  C* yf = y + f * n;
  const C zero = cx<C>(T(0), T(0));
  const T inv_dx = (T)(1.0 / g.dx);
  auto F = [&](int plane, int i2, int j2) -> C {
    if (i2 < 0 || i2 >= g.H || j2 < 0 || j2 >= g.W) return zero;
    return t[plane * n + (long long)i2 * g.W + j2];
  };
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.W), j = (int)(k - (long long)i * g.W);
    const C pk = pf[k];
    if (!dense_inside(g, i, j)) { yf[k] = pk; continue; }
    if (!ADJ) {
      C dX = zero, dgX = zero, dZ = zero, dgZ = zero;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T a = (T)c_dense_a[q];
        dX = dX + a * (F(0, i, j + q) - F(0, i, j - 1 - q));
        dgX = dgX + a * (F(1, i, j + q) - F(1, i, j - 1 - q));
        dZ = dZ + a * (F(2, i + q, j) - F(2, i - 1 - q, j));
        dgZ = dgZ + a * (F(3, i + q, j) - F(3, i - 1 - q, j));
      }
      const C part = DC<T>::from(dc.lx[j]) * dX + DC<T>::from(dc.rx[j]) * dgX +
                     DC<T>::from(dc.lz[i]) * dZ + DC<T>::from(dc.rz[i]) * dgZ;
      yf[k] = DC<T>::from(g.scal) * (inv_dx * part) + DC<T>::from(dc.mass[k]) * pk;
    } else {
      C dX = zero, dZ = zero;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const T a = (T)c_dense_a[q];
        dX = dX + a * (F(0, i, j + q) - F(0, i, j - 1 - q));
        dZ = dZ + a * (F(2, i + q, j) - F(2, i - 1 - q, j));
      }
      // D^H f = -(-D^H f)
      yf[k] = (T(-1) * inv_dx) * (dX + dZ) + conjc(DC<T>::from(dc.mass[k])) * pk;
    }
  }
}

extern "C" size_t nsr_dense_coef_bytes(const NsrDenseGrid* g) {
  if (!g || g->H <= 0 || g->W <= 0) return 0;
  return sizeof(double) * dense_coef_doubles(g->H, g->W);
}

extern "C" size_t nsr_dense_workspace_size(const NsrDenseGrid* g, int32_t n_fields, int32_t precision) {
  if (!g || g->H <= 0 || g->W <= 0 || n_fields < 0 || (precision != 0 && precision != 1)) return 0;
  return (size_t)4 * g->H * g->W * n_fields * (precision ? 16 : 8);
}

extern "C" int nsr_dense_apply(const NsrDenseGrid* grid, const double* coef, double scal_re, double scal_im,
                               int32_t n_fields, int32_t adjoint, int32_t precision, const void* x, void* y,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (!grid || !coef || !x || !y || n_fields < 0 || n_fields > 65535) return NSR_ERR_ARGUMENT;
  if (grid->H < 3 || grid->W < 3 || grid->h < 1 || grid->w < 1 || grid->pz < 0 || grid->px < 0 ||
      grid->pz + grid->h > grid->H || grid->px + grid->w > grid->W || !(grid->dx > 0))
    return NSR_ERR_ARGUMENT;
  if (precision != 0 && precision != 1) return NSR_ERR_ARGUMENT;
  if (n_fields == 0) return 0;
  if (!workspace || workspace_bytes < nsr_dense_workspace_size(grid, n_fields, precision)) return NSR_ERR_WORKSPACE;
  DenseGeo g;
  g.H = grid->H; g.W = grid->W; g.pz = grid->pz; g.px = grid->px; g.h = grid->h; g.w = grid->w; g.dx = grid->dx;
  g.scal = make_double2(scal_re, scal_im);
  const long long n = (long long)g.H * g.W;
  int bx = (int)((n + 255) / 256);
  if (bx > 4096) bx = 4096;
  const dim3 gr(bx, n_fields);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == 0) {
    float2* t = (float2*)workspace;
    if (adjoint) {
      k_dense_flux<float, true><<<gr, 256, 0, st>>>(g, coef, (const float2*)x, t, n_fields);
      k_dense_div<float, true><<<gr, 256, 0, st>>>(g, coef, (const float2*)x, t, (float2*)y, n_fields);
    } else {
      k_dense_flux<float, false><<<gr, 256, 0, st>>>(g, coef, (const float2*)x, t, n_fields);
      k_dense_div<float, false><<<gr, 256, 0, st>>>(g, coef, (const float2*)x, t, (float2*)y, n_fields);
    }
  } else {
    double2* t = (double2*)workspace;
    if (adjoint) {
      k_dense_flux<double, true><<<gr, 256, 0, st>>>(g, coef, (const double2*)x, t, n_fields);
      k_dense_div<double, true><<<gr, 256, 0, st>>>(g, coef, (const double2*)x, t, (double2*)y, n_fields);
    } else {
      k_dense_flux<double, false><<<gr, 256, 0, st>>>(g, coef, (const double2*)x, t, n_fields);
      k_dense_div<double, false><<<gr, 256, 0, st>>>(g, coef, (const double2*)x, t, (double2*)y, n_fields);
    }
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// ---------------------------------------------------------------------------
// Implicit gradient of the dense operator: cotangents of its coefficient
// planes for the bilinear form
//   L = -Re sum_f sum_n conj(lam_f[n]) mask[n] (A(m) (mask u_f))[n]
// that ImplicitChannels.backward differentiates (nsrno/dense_wave.py:250-255).
// A depends on the medium only through ax, az (the face coefficients) and the
// mass term, and L is linear in each, so
//   dL/dax[k]   = -Re sum_f svx[j] gx_f[k] Qx_f[k],   gx = D_x(mask u) / dx,
//   Qx = Div^T(mu lx) + gvx Div^T(mu rx),   mu = conj(lam) mask scal,
//   (Div^T v)[k] = (1/dx) sum_q a_q (v[k-q] - v[k+1+q]),
// likewise along z, and with w = conj(lam) mask u:
//   dL/dRe(mass) = -Re w,  dL/dIm(mass) = Im w.
// One thread per node sums the fields in order (deterministic).
// ---------------------------------------------------------------------------
__global__ void k_dense_grad(DenseGeo g, const double* __restrict__ coef, const double2* __restrict__ u,
                             const double2* __restrict__ lam, int nf, double* __restrict__ g_ax,
                             double* __restrict__ g_az, double* __restrict__ g_mass) {
  const DenseCoef dc = dense_unpack(coef, g.H, g.W);
  const long long n = (long long)g.H * g.W;
  const double inv_dx = 1.0 / g.dx;
  const double2 zero = make_double2(0.0, 0.0);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.W), j = (int)(k - (long long)i * g.W);
    double sax = 0.0, saz = 0.0, smr = 0.0, smi = 0.0;
    for (int f = 0; f < nf; ++f) {
      const double2* uf = u + (long long)f * n;
      const double2* lf = lam + (long long)f * n;
      // masked field and mu = conj(lam) mask scal at (i2, j2); zero outside the grid
      auto U = [&](int i2, int j2) -> double2 {
        if (i2 < 0 || i2 >= g.H || j2 < 0 || j2 >= g.W || !dense_inside(g, i2, j2)) return zero;
        return uf[(long long)i2 * g.W + j2];
      };
      auto MU = [&](int i2, int j2) -> double2 {
        if (i2 < 0 || i2 >= g.H || j2 < 0 || j2 >= g.W || !dense_inside(g, i2, j2)) return zero;
        return conjc(lf[(long long)i2 * g.W + j2]) * g.scal;
      };
      double2 gx = zero, gz = zero, qxl = zero, qxr = zero, qzl = zero, qzr = zero;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double a = c_dense_a[q];
        gx = gx + a * (U(i, j + 1 + q) - U(i, j - q));
        gz = gz + a * (U(i + 1 + q, j) - U(i - q, j));
        const int jw = j - q, je = j + 1 + q, in_ = i - q, is = i + 1 + q;
        const double2 mw = MU(i, jw), me = MU(i, je), mn = MU(in_, j), ms = MU(is, j);
        const double2 lxw = jw >= 0 ? dc.lx[jw] : zero, lxe = je < g.W ? dc.lx[je] : zero;
        const double2 rxw = jw >= 0 ? dc.rx[jw] : zero, rxe = je < g.W ? dc.rx[je] : zero;
        const double2 lzn = in_ >= 0 ? dc.lz[in_] : zero, lzs = is < g.H ? dc.lz[is] : zero;
        const double2 rzn = in_ >= 0 ? dc.rz[in_] : zero, rzs = is < g.H ? dc.rz[is] : zero;
        qxl = qxl + a * (mw * lxw - me * lxe);
        qxr = qxr + a * (mw * rxw - me * rxe);
        qzl = qzl + a * (mn * lzn - ms * lzs);
        qzr = qzr + a * (mn * rzn - ms * rzs);
      }
      const double2 Qx = inv_dx * (qxl + dc.gvx[j] * qxr);
      const double2 Qz = inv_dx * (qzl + dc.gvz[i] * qzr);
      sax -= (dc.svx[j] * (inv_dx * gx) * Qx).x;
      saz -= (dc.svz[i] * (inv_dx * gz) * Qz).x;
      if (dense_inside(g, i, j)) {
        const double2 w = conjc(lf[k]) * uf[k];
        smr -= w.x;
        smi += w.y;
      }
    }
    g_ax[k] = sax;
    g_az[k] = saz;
    g_mass[k] = smr;
    g_mass[n + k] = smi;
  }
}

extern "C" int nsr_dense_grad(const NsrDenseGrid* grid, const double* coef, double scal_re, double scal_im,
                              int32_t n_fields, const double* u, const double* lam, double* g_ax, double* g_az,
                              double* g_mass, void* stream) {
  if (!grid || !coef || !u || !lam || !g_ax || !g_az || !g_mass || n_fields < 0 || n_fields > 65535)
    return NSR_ERR_ARGUMENT;
  if (grid->H < 3 || grid->W < 3 || grid->h < 1 || grid->w < 1 || grid->pz < 0 || grid->px < 0 ||
      grid->pz + grid->h > grid->H || grid->px + grid->w > grid->W || !(grid->dx > 0))
    return NSR_ERR_ARGUMENT;
  DenseGeo g;
  g.H = grid->H; g.W = grid->W; g.pz = grid->pz; g.px = grid->px; g.h = grid->h; g.w = grid->w; g.dx = grid->dx;
  g.scal = make_double2(scal_re, scal_im);
  const long long n = (long long)g.H * g.W;
  int bx = (int)((n + 255) / 256);
  if (bx > 4096) bx = 4096;
  k_dense_grad<<<bx, 256, 0, (cudaStream_t)stream>>>(g, coef, (const double2*)u, (const double2*)lam, n_fields,
                                                     g_ax, g_az, g_mass);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// ---------------------------------------------------------------------------
// Fixed preconditioner of the dense path (nsrno/conditioned_wave.py:90-92,
// nsrno/dense_wave.py:194-196):
//   M r = mask * IFFT((1 + lap/k0^2 - i shift)^-1 FFT(r)),
// lap = -(|Dx|^2 + |Dz|^2) with the 8th-order staggered symbols
// |D(q)|^2 = (2 sum_k a_k sin((k + 1/2) q))^2 / dx^2 (conditioned_wave.py:24-27).
// The transforms are the solver's row and column FFTs (sizes 8..2048 whose
// prime factors are at most 61, e.g. the 1056 x 1216 padding of the reference).
// ---------------------------------------------------------------------------
__global__ void k_dense_symbol(int n, FftPlan plan, float* d2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int f = nsr_digit_reverse(k, n, plan.radix, plan.nst);
    const double q = 2.0 * NSR_PI * f / n;
    double s = 0.0;
    for (int j = 0; j < 4; ++j) s += c_dense_a[j] * sin((j + 0.5) * q);
    d2[k] = (float)(4.0 * s * s);   // |D|^2 dx^2
  }
}

template <int TC>
__global__ void __launch_bounds__(512) k_dense_cols(int nz, int nx, PrecTables t, const float* __restrict__ d2z,
                                                    const float* __restrict__ d2x, float2* __restrict__ w,
                                                    float inv_k0dx2, float shift, int adjoint) {
  extern __shared__ float2 sm[];
  const long long n = (long long)nz * nx;
  float2* ws = w + blockIdx.y * n;
  const int c0 = blockIdx.x * TC;
  const int ncol = min(TC, nx - c0);
  for (int k = threadIdx.x; k < nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    sm[k] = c < ncol ? ws[(long long)z * nx + c0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_cols<false, TC>(sm, t.pz);
  const float inv_n = 1.0f / (float)n;
  for (int k = threadIdx.x; k < nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    if (c < ncol) {
      const float re = 1.0f - (d2z[z] + d2x[c0 + c]) * inv_k0dx2;
      float2 mul = divc(make_float2(inv_n, 0.f), make_float2(re, -shift));
      if (adjoint) mul = conjc(mul);
      sm[k] = sm[k] * mul;
    }
  }
  __syncthreads();
  fft_cols<true, TC>(sm, t.pz);
  for (int k = threadIdx.x; k < nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    if (c < ncol) ws[(long long)z * nx + c0 + c] = sm[k];
  }
}

__global__ void k_dense_rows(int nz, int nx, int pz, int px, int h, int w, PrecTables t,
                             const float2* __restrict__ x, float2* __restrict__ y, int rows, int inverse) {
  extern __shared__ float2 sm[];
  const long long n = (long long)nz * nx;
  const int z0 = blockIdx.x * rows;
  const int nr = min(rows, nz - z0);
  const float2* xs = x + blockIdx.y * n + (long long)z0 * nx;
  const int rs = nsr_row_stride(nx);
  const bool pad = nsr_row_padded(nx);
  for (int k = threadIdx.x; k < nr * nx; k += blockDim.x) {
    const int l = k / nx, c = k - l * nx;
    sm[l * rs + (pad ? c + (c >> 4) : c)] = xs[k];
  }
  __syncthreads();
  if (inverse) fft_rows<true>(sm, nr, t.px);
  else fft_rows<false>(sm, nr, t.px);
  __syncthreads();
  float2* ys = y + blockIdx.y * n + (long long)z0 * nx;
  for (int k = threadIdx.x; k < nr * nx; k += blockDim.x) {
    const int l = k / nx, c = k - l * nx;
    const int i = z0 + l;
    const bool in = !inverse || (i >= pz && i < pz + h && c >= px && c < px + w);
    ys[k] = in ? sm[l * rs + (pad ? c + (c >> 4) : c)] : make_float2(0.f, 0.f);
  }
}

static NsrGrid dense_fft_grid(const NsrDenseGrid* g) {
  NsrGrid q;
  memset(&q, 0, sizeof(q));
  q.nz = g->H;
  q.nx = g->W;
  q.h = g->dx;
  q.c0 = 1540.0;      // only the transform sizes of this grid are used
  q.rho0 = 1000.0;
  return q;
}

extern "C" size_t nsr_dense_precondition_workspace_size(const NsrDenseGrid* g, int32_t n_fields) {
  if (!g || n_fields <= 0 || n_fields > 65535) return 0;
  NsrGrid q = dense_fft_grid(g);
  if (nsr_check_grid(&q, true)) return 0;
  return nsr_align(nsr_prec_table_bytes(&q)) + nsr_align(sizeof(float) * (g->H + g->W)) +
         nsr_align(sizeof(float2) * (size_t)g->H * g->W * n_fields);
}

extern "C" int nsr_dense_precondition(const NsrDenseGrid* grid, double k0dx2, double shift, int32_t n_fields,
                                      int32_t adjoint, const float* x, float* y, void* workspace,
                                      size_t workspace_bytes, void* stream) {
  if (!grid || !x || !y || !workspace || n_fields < 0 || n_fields > 65535 || !(k0dx2 > 0) || !(shift >= 0))
    return NSR_ERR_ARGUMENT;
  if (grid->pz < 0 || grid->px < 0 || grid->pz + grid->h > grid->H || grid->px + grid->w > grid->W)
    return NSR_ERR_ARGUMENT;
  if (n_fields == 0) return 0;
  const size_t need = nsr_dense_precondition_workspace_size(grid, n_fields);
  if (need == 0) return NSR_ERR_UNSUPPORTED_SIZE;
  if (workspace_bytes < need) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  NsrGrid q = dense_fft_grid(grid);
  char* ws = (char*)workspace;
  PrecTables t;
  int err = nsr_prec_setup(&q, &t, ws, st);
  if (err) return err;
  float* d2x = (float*)(ws + nsr_align(nsr_prec_table_bytes(&q)));
  float* d2z = d2x + grid->W;
  float2* w = (float2*)(ws + nsr_align(nsr_prec_table_bytes(&q)) + nsr_align(sizeof(float) * (grid->H + grid->W)));
  k_dense_symbol<<<(grid->W + 255) / 256, 256, 0, st>>>(grid->W, t.px, d2x);
  k_dense_symbol<<<(grid->H + 255) / 256, 256, 0, st>>>(grid->H, t.pz, d2z);
  const int rows = nsr_rows_per_cta(&q);
  const size_t row_smem = sizeof(float2) * (size_t)rows * nsr_row_stride(grid->W);
  const dim3 gr((grid->H + rows - 1) / rows, n_fields);
  k_dense_rows<<<gr, 256, row_smem, st>>>(grid->H, grid->W, grid->pz, grid->px, grid->h, grid->w, t,
                                          (const float2*)x, w, rows, 0);
  const int tc = nsr_cols_tc(&q);
  const dim3 gc((grid->W + tc - 1) / tc, n_fields);
  const size_t csm = nsr_cols_smem(&q);
  const float inv = (float)(1.0 / k0dx2);
  if (tc == 16) {
    cudaFuncSetAttribute(k_dense_cols<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    k_dense_cols<16><<<gc, 512, csm, st>>>(grid->H, grid->W, t, d2z, d2x, w, inv, (float)shift, adjoint);
  } else {
    cudaFuncSetAttribute(k_dense_cols<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    k_dense_cols<8><<<gc, 512, csm, st>>>(grid->H, grid->W, t, d2z, d2x, w, inv, (float)shift, adjoint);
  }
  k_dense_rows<<<gr, 256, row_smem, st>>>(grid->H, grid->W, grid->pz, grid->px, grid->h, grid->w, t, w,
                                          (float2*)y, rows, 1);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}
