// Stand-alone operators of the nsrno_b200 C ABI: material planes, the 5-point
// operator apply, the FFT shifted-Laplace preconditioner, plane-wave
// right-hand sides and the adjoint-state material gradient.
#include "nsr_common.cuh"
#include "nsr_internal.cuh"

#include <string.h>

// ---------------------------------------------------------------------------
// Error strings and argument checks.
// ---------------------------------------------------------------------------
extern "C" int nsr_version(void) { return 100; }

extern "C" const char* nsr_error_string(int code) {
  switch (code) {
    case 0: return "ok";
    case NSR_ERR_ARGUMENT: return "nsrno_b200: invalid argument";
    case NSR_ERR_UNSUPPORTED_SIZE: return "nsrno_b200: nz and nx must be between 8 and 2048 with no prime factor above 61";
    case NSR_ERR_WORKSPACE: return "nsrno_b200: workspace too small";
    case NSR_ERR_INTERNAL: return "nsrno_b200: solver queue did not drain";
    case NSR_ERR_CAPACITY: return "nsrno_b200: request exceeds the fixed capacity";
    case NSR_ERR_TIMEOUT: return "nsrno_b200: a kernel timed out waiting for its shared-memory copies";
    default: break;
  }
  if (code > 0 && code < 1000) return cudaGetErrorString((cudaError_t)code);
  return "nsrno_b200: unknown error";
}

int nsr_check_grid(const NsrGrid* g, bool need_fft) {
  if (!g) return NSR_ERR_ARGUMENT;
  if (g->nz < 3 || g->nx < 3 || g->n_pml < 0 || 2 * g->n_pml >= g->nz || 2 * g->n_pml >= g->nx) return NSR_ERR_ARGUMENT;
  if (!(g->h > 0) || !(g->c0 > 0) || !(g->rho0 > 0) || !(g->pml_strength >= 0)) return NSR_ERR_ARGUMENT;
  if (g->face < 0 || g->face >= g->nz) return NSR_ERR_ARGUMENT;
  if ((long long)g->nz * g->nx > (1LL << 30)) return NSR_ERR_ARGUMENT;
  if (need_fft) {
    int r[NSR_MAX_RADIX_STAGES], k;
    if (!nsr_make_radices(g->nz, r, &k) || !nsr_make_radices(g->nx, r, &k)) return NSR_ERR_UNSUPPORTED_SIZE;
  }
  return 0;
}

static inline int last_error() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// ---------------------------------------------------------------------------
// Material planes.
// ---------------------------------------------------------------------------
__global__ void k_setup_material(Geo g, const float* __restrict__ c, const float* __restrict__ rho,
                                 const float* __restrict__ alpha, void* __restrict__ mat, long long n) {
  const double neper = 100.0 * 2.302585092994045684 / 20.0;  // dB/cm -> Np/m
  float* f = (float*)mat;
  double* d = (double*)((char*)mat + nsr_material_off64(n));
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double cc = c[k], rr = rho[k], al = alpha[k];
    const double a = g.rho0 / rr;
    const double b = g.rho0 * g.c0 * g.c0 / (rr * cc * cc);
    const double t = al * neper * cc / (2.0 * NSR_PI * 1e6);
    d[k] = a; d[n + k] = b; d[2 * n + k] = t;
    f[k] = (float)a; f[n + k] = (float)b; f[2 * n + k] = (float)t;
  }
}

extern "C" size_t nsr_material_bytes(const NsrGrid* grid) {
  if (nsr_check_grid(grid, false)) return 0;
  return nsr_material_size((long long)grid->nz * grid->nx);
}

extern "C" int nsr_setup_material(const NsrGrid* grid, const float* c, const float* rho,
                                  const float* alpha_db, void* material, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!c || !rho || !alpha_db || !material) return NSR_ERR_ARGUMENT;
  long long n = (long long)grid->nz * grid->nx;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_setup_material<<<blocks, 256, 0, (cudaStream_t)stream>>>(make_geo(*grid), c, rho, alpha_db, material, n);
  return last_error();
}

// ---------------------------------------------------------------------------
// Operator apply (one thread per node; used for checks and true residuals).
// ---------------------------------------------------------------------------
template <typename T> struct PlaneOf;
template <> struct PlaneOf<float> {
  static __device__ __forceinline__ const float* a(const MatPlanes& m) { return m.a32; }
  static __device__ __forceinline__ const float* b(const MatPlanes& m) { return m.b32; }
  static __device__ __forceinline__ const float* t(const MatPlanes& m) { return m.t32; }
};
template <> struct PlaneOf<double> {
  static __device__ __forceinline__ const double* a(const MatPlanes& m) { return m.a64; }
  static __device__ __forceinline__ const double* b(const MatPlanes& m) { return m.b64; }
  static __device__ __forceinline__ const double* t(const MatPlanes& m) { return m.t64; }
};

// FP32 fields use the float planes, FP64 fields the double planes.
template <typename T, bool ADJ>
__global__ void k_apply(Geo g, const void* __restrict__ mat, const double* __restrict__ freq,
                        const typename CxT<T>::type* __restrict__ x, typename CxT<T>::type* __restrict__ y) {
  typedef typename CxT<T>::type C;
  const long long n = (long long)g.nz * g.nx;
  const int sysi = blockIdx.y;
  const SysScalars s = sys_scalars(g, freq[sysi]);
  const C* xs = x + sysi * n;
  const MatPlanes mp = nsr_planes(mat, n);
  const T* ca = PlaneOf<T>::a(mp);
  const T* cb = PlaneOf<T>::b(mp);
  const T* ct = PlaneOf<T>::t(mp);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.nx), j = (int)(k - (long long)i * g.nx);
    auto P = [&](int i2, int j2) -> C {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return cx<C>(T(0), T(0));
      return xs[(long long)i2 * g.nx + j2];
    };
    auto A = [&](int i2, int j2) -> T {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return T(1);
      return (T)ca[(long long)i2 * g.nx + j2];
    };
    y[sysi * n + k] = stencil<T, ADJ>(g, s, i, j, cb[k], ct[k], P, A);
  }
}

extern "C" int nsr_apply(const NsrGrid* grid, const void* coef, const double* freq_hz,
                         int32_t n_systems, int32_t adjoint, int32_t precision,
                         const void* x, void* y, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!coef || !freq_hz || !x || !y || n_systems < 0 || n_systems > 65535) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  long long n = (long long)grid->nz * grid->nx;
  int bx = (int)((n + 255) / 256);
  if (bx > 4096) bx = 4096;
  dim3 gridd(bx, n_systems);
  cudaStream_t st = (cudaStream_t)stream;
  Geo g = make_geo(*grid);
  if (precision == 0) {
    if (adjoint) k_apply<float, true><<<gridd, 256, 0, st>>>(g, coef, freq_hz, (const float2*)x, (float2*)y);
    else k_apply<float, false><<<gridd, 256, 0, st>>>(g, coef, freq_hz, (const float2*)x, (float2*)y);
  } else if (precision == 1) {
    if (adjoint) k_apply<double, true><<<gridd, 256, 0, st>>>(g, coef, freq_hz, (const double2*)x, (double2*)y);
    else k_apply<double, false><<<gridd, 256, 0, st>>>(g, coef, freq_hz, (const double2*)x, (double2*)y);
  } else {
    return NSR_ERR_ARGUMENT;
  }
  return last_error();
}

// ---------------------------------------------------------------------------
// Preconditioner tables and passes (shared with the solver).
// ---------------------------------------------------------------------------
__global__ void k_fft_tables(int n, FftPlan plan, float2* tw, float* s2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double sn, cs;
    sincospi(-2.0 * k / n, &sn, &cs);
    tw[k] = make_float2((float)cs, (float)sn);
    int f = nsr_digit_reverse(k, n, plan.radix, plan.nst);
    double sp = sinpi((double)f / n);
    s2[k] = (float)(sp * sp);
  }
}

// Per-stage twiddle rows of the specialised transforms (layout: FftPlan::tws),
// with the same rounding of the same angles as k_fft_tables.
__global__ void k_fft_stage_twiddles(int n, FftPlan plan, float2* tws, int total) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    int l = n, off = 0;
    for (int st = 0; st < plan.nst; ++st) {
      const int r = plan.radix[st], m = l / r;
      if (m > 1) {
        if (e < off + m * (r - 1)) {
          const int k = (e - off) / m + 1, j = (e - off) % m;
          double sn, cs;
          sincospi(-2.0 * (j * k * (n / l)) / n, &sn, &cs);
          tws[e] = make_float2((float)cs, (float)sn);
          break;
        }
        off += m * (r - 1);
      }
      l = m;
    }
  }
}

int nsr_prec_setup(const NsrGrid* g, PrecTables* t, void* table_mem, cudaStream_t st) {
  char* p = (char*)table_mem;
  t->px.n = g->nx;
  t->pz.n = g->nz;
  if (!nsr_make_radices(g->nx, t->px.radix, &t->px.nst)) return NSR_ERR_UNSUPPORTED_SIZE;
  if (!nsr_make_radices(g->nz, t->pz.radix, &t->pz.nst)) return NSR_ERR_UNSUPPORTED_SIZE;
  float2* twx = (float2*)p; p += nsr_align(sizeof(float2) * g->nx);
  float2* twz = (float2*)p; p += nsr_align(sizeof(float2) * g->nz);
  float* s2x = (float*)p; p += nsr_align(sizeof(float) * g->nx);
  float* s2z = (float*)p; p += nsr_align(sizeof(float) * g->nz);
  const int nwx = nsr_twiddle_offset(g->nx, 0), nwz = nsr_twiddle_offset(g->nz, 0);
  float2* twsx = (float2*)p; p += nsr_align(sizeof(float2) * nwx);
  float2* twsz = (float2*)p; p += nsr_align(sizeof(float2) * nwz);
  t->px.tw = twx; t->pz.tw = twz; t->s2x = s2x; t->s2z = s2z;
  t->px.tws = twsx; t->pz.tws = twsz;
  k_fft_tables<<<(g->nx + 255) / 256, 256, 0, st>>>(g->nx, t->px, twx, s2x);
  k_fft_tables<<<(g->nz + 255) / 256, 256, 0, st>>>(g->nz, t->pz, twz, s2z);
  if (nwx > 0) k_fft_stage_twiddles<<<(nwx + 255) / 256, 256, 0, st>>>(g->nx, t->px, twsx, nwx);
  if (nwz > 0) k_fft_stage_twiddles<<<(nwz + 255) / 256, 256, 0, st>>>(g->nz, t->pz, twsz, nwz);
  return last_error();
}

size_t nsr_prec_table_bytes(const NsrGrid* g) {
  return nsr_align(sizeof(float2) * g->nx) + nsr_align(sizeof(float2) * g->nz) +
         nsr_align(sizeof(float) * g->nx) + nsr_align(sizeof(float) * g->nz) +
         nsr_align(sizeof(float2) * nsr_twiddle_offset(g->nx, 0)) +
         nsr_align(sizeof(float2) * nsr_twiddle_offset(g->nz, 0));
}

// Column pass: forward DIF along z, multiply by the shifted-Laplace symbol in
// the digit-reversed domain, inverse along z.  In place on w.
template <int TC>
__global__ void __launch_bounds__(512) k_prec_cols(Geo g, PrecTables t, const double* __restrict__ freq,
                                                   float2* __restrict__ w, double shift, int adjoint) {
  extern __shared__ float2 sm[];
  const int sysi = blockIdx.y;
  const long long n = (long long)g.nz * g.nx;
  float2* ws = w + sysi * n;
  const int c0 = blockIdx.x * TC;
  const int ncol = min(TC, g.nx - c0);
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    sm[k] = c < ncol ? ws[(long long)z * g.nx + c0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_cols<false, TC>(sm, t.pz);
  const SysScalars s = sys_scalars(g, freq[sysi]);
  const float kh2 = (float)s.kh2;
  const float inv_n = 1.0f / (float)n;
  const float2 shiftc = make_float2(kh2, (float)(s.kh2 * shift));
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    if (c < ncol) {
      const float sym = -4.0f * (t.s2z[z] + t.s2x[c0 + c]);
      float2 mul = divc(make_float2(inv_n, 0.f), make_float2(sym + shiftc.x, shiftc.y));
      if (adjoint) mul = conjc(mul);
      sm[k] = sm[k] * mul;
    }
  }
  __syncthreads();
  fft_cols<true, TC>(sm, t.pz);
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    if (c < ncol) ws[(long long)z * g.nx + c0 + c] = sm[k];
  }
}

int nsr_cols_tc(const NsrGrid* g) { return g->nz <= 1024 ? 16 : 8; }
int nsr_cols_threads() { return 512; }
size_t nsr_cols_smem(const NsrGrid* g) { return sizeof(float2) * (size_t)g->nz * nsr_cols_tc(g); }

// Stand-alone row passes of nsr_precondition.
__global__ void __launch_bounds__(256) k_prec_rows_fwd(Geo g, PrecTables t, const float2* __restrict__ x,
                                                       float2* __restrict__ w, int rows) {
  extern __shared__ float2 sm[];
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * rows;
  const int nr = min(rows, g.nz - z0);
  const float2* xs = x + blockIdx.y * n + (long long)z0 * g.nx;
  const int rs = nsr_row_stride(g.nx);
  const bool pad = nsr_row_padded(g.nx);
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    sm[l * rs + (pad ? c + (c >> 4) : c)] = xs[k];
  }
  __syncthreads();
  fft_rows<false>(sm, nr, t.px);
  float2* ws = w + blockIdx.y * n + (long long)z0 * g.nx;
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    ws[k] = sm[l * rs + (pad ? c + (c >> 4) : c)];
  }
}

__global__ void __launch_bounds__(256) k_prec_rows_inv(Geo g, PrecTables t, const float2* __restrict__ w,
                                                       float2* __restrict__ y, int rows) {
  extern __shared__ float2 sm[];
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * rows;
  const int nr = min(rows, g.nz - z0);
  const float2* ws = w + blockIdx.y * n + (long long)z0 * g.nx;
  const int rs = nsr_row_stride(g.nx);
  const bool pad = nsr_row_padded(g.nx);
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    sm[l * rs + (pad ? c + (c >> 4) : c)] = ws[k];
  }
  __syncthreads();
  fft_rows<true>(sm, nr, t.px);
  float2* ys = y + blockIdx.y * n + (long long)z0 * g.nx;
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    ys[k] = sm[l * rs + (pad ? c + (c >> 4) : c)];
  }
}

extern "C" size_t nsr_precondition_workspace_size(const NsrGrid* grid, int32_t n_systems) {
  if (nsr_check_grid(grid, true) || n_systems < 0) return 0;
  return nsr_prec_table_bytes(grid) + nsr_align(sizeof(float2) * (size_t)grid->nz * grid->nx * n_systems);
}

extern "C" int nsr_precondition(const NsrGrid* grid, const double* freq_hz, int32_t n_systems,
                                double shift, int32_t adjoint, const float* x, float* y,
                                void* workspace, size_t workspace_bytes, void* stream) {
  int err = nsr_check_grid(grid, true);
  if (err) return err;
  if (!freq_hz || !x || !y || !workspace || n_systems < 0 || n_systems > 65535) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  if (workspace_bytes < nsr_precondition_workspace_size(grid, n_systems)) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  PrecTables t;
  err = nsr_prec_setup(grid, &t, workspace, st);
  if (err) return err;
  float2* w = (float2*)((char*)workspace + nsr_prec_table_bytes(grid));
  Geo g = make_geo(*grid);
  const int rows = nsr_rows_per_cta(grid);
  const size_t row_smem = sizeof(float2) * (size_t)rows * nsr_row_stride(grid->nx);
  dim3 gr((grid->nz + rows - 1) / rows, n_systems);
  k_prec_rows_fwd<<<gr, 256, row_smem, st>>>(g, t, (const float2*)x, w, rows);
  const int tc = nsr_cols_tc(grid);
  dim3 gc((grid->nx + tc - 1) / tc, n_systems);
  size_t csm = nsr_cols_smem(grid);
  if (tc == 16) {
    cudaFuncSetAttribute(k_prec_cols<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    k_prec_cols<16><<<gc, 512, csm, st>>>(g, t, freq_hz, w, shift, adjoint);
  } else {
    cudaFuncSetAttribute(k_prec_cols<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    k_prec_cols<8><<<gc, 512, csm, st>>>(g, t, freq_hz, w, shift, adjoint);
  }
  k_prec_rows_inv<<<gr, 256, row_smem, st>>>(g, t, w, (float2*)y, rows);
  return last_error();
}

int nsr_rows_per_cta(const NsrGrid* g) {
  // Keep row tiles near 32 KB of shared memory.
  int rows = (int)(4096 / g->nx);
  if (rows < 1) rows = 1;
  if (rows > 8) rows = 8;
  return rows;
}

// ---------------------------------------------------------------------------
// Plane-wave right-hand side (SI units, c128).
// ---------------------------------------------------------------------------
__global__ void k_plane_wave_rhs(Geo g, const double* __restrict__ freq, const double* __restrict__ angle,
                                 double2* __restrict__ b) {
  const long long n = (long long)g.nz * g.nx;
  const int sysi = blockIdx.y;
  const SysScalars s = sys_scalars(g, freq[sysi]);
  const double st = sin(angle[sysi]);
  const double inv_h2 = 1.0 / (g.h * g.h);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.nx), j = (int)(k - (long long)i * g.nx);
    double2 v = make_double2(0.0, 0.0);
    if (i == g.face) {
      double2 l = source_line(g, s.k0, st, j);
      v = make_double2(-l.x * inv_h2, -l.y * inv_h2);
    }
    b[sysi * n + k] = v;
  }
}

extern "C" int nsr_plane_wave_rhs(const NsrGrid* grid, const double* freq_hz, const double* angle_rad,
                                  int32_t n_systems, void* b, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!freq_hz || !angle_rad || !b || n_systems < 0 || n_systems > 65535) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  long long n = (long long)grid->nz * grid->nx;
  int bx = (int)((n + 255) / 256);
  if (bx > 4096) bx = 4096;
  k_plane_wave_rhs<<<dim3(bx, n_systems), 256, 0, (cudaStream_t)stream>>>(make_geo(*grid), freq_hz, angle_rad,
                                                                           (double2*)b);
  return last_error();
}

// ---------------------------------------------------------------------------
// Material gradient: -Re(lambda^H dA/dm u) for m = log c, log rho.
// d mass / d log c  = -2 k0^2 sx sz b (1 + i e)
// d mass / d log rho = -mass
// each edge e=(i,j): d(lam^H A u)/d log rho_i = a_i w_e conj(lam_j - lam_i)(u_j - u_i),
// w_e = stretch_e / (2 h^2).
// ---------------------------------------------------------------------------
template <typename CT>
__global__ void k_grad(Geo g, const void* __restrict__ mat, const double* __restrict__ freq, int ns,
                       const CT* __restrict__ u, const CT* __restrict__ lam,
                       double* __restrict__ gc, double* __restrict__ gr) {
  const long long n = (long long)g.nz * g.nx;
  const double inv_h2 = 1.0 / (g.h * g.h);
  const MatPlanes mp = nsr_planes(mat, n);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.nx), j = (int)(k - (long long)i * g.nx);
    const double a_c = mp.a64[k], b_c = mp.b64[k], t_c = mp.t64[k];
    double acc_c = 0.0, acc_r = 0.0;
    for (int sidx = 0; sidx < ns; ++sidx) {
      const SysScalars s = sys_scalars(g, freq[sidx]);
      const CT* us = u + sidx * n;
      const CT* ls = lam + sidx * n;
      auto U = [&](int i2, int j2) -> double2 {
        if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return make_double2(0.0, 0.0);
        const CT q = us[(long long)i2 * g.nx + j2];
        return make_double2((double)q.x, (double)q.y);
      };
      auto L = [&](int i2, int j2) -> double2 {
        if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return make_double2(0.0, 0.0);
        const CT q = ls[(long long)i2 * g.nx + j2];
        return make_double2((double)q.x, (double)q.y);
      };
      const double2 uc = U(i, j), lc = L(i, j);
      const double2 lu = conjc(lc) * uc;
      const double sig = s.sig;
      const double2 sx = make_double2(1.0, sig * pml_profile<double>((double)j, g.nx, g.n_pml));
      const double2 sz = make_double2(1.0, sig * pml_profile<double>((double)i, g.nz, g.n_pml));
      const double e = t_c * s.fpow;
      const double2 onepie = make_double2(1.0, e);
      const double2 cell = (s.kh2 * b_c) * (sx * sz);          // h^2 k0^2 sx sz b
      const double2 dm_c = (-2.0) * (cell * onepie);
      const double2 dm_r = (-1.0) * (cell * (onepie * onepie));
      double2 edge = make_double2(0.0, 0.0);
      const int di[4] = {0, 0, 1, -1}, dj[4] = {1, -1, 0, 0};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double2 st;
        if (q < 2) {
          double2 sh = make_double2(1.0, sig * pml_profile<double>(j + 0.5 * dj[q], g.nx, g.n_pml));
          st = divc(sz, sh);
        } else {
          double2 sh = make_double2(1.0, sig * pml_profile<double>(i + 0.5 * di[q], g.nz, g.n_pml));
          st = divc(sx, sh);
        }
        const double2 du = U(i + di[q], j + dj[q]) - uc;
        const double2 dl = conjc(L(i + di[q], j + dj[q]) - lc);
        edge = edge + (0.5 * st) * (dl * du);
      }
      acc_c += -(lu * dm_c).x;
      acc_r += -(lu * dm_r).x - a_c * edge.x;
    }
    gc[k] += acc_c * inv_h2;
    gr[k] += acc_r * inv_h2;
  }
}

extern "C" int nsr_grad_accum(const NsrGrid* grid, const void* coef, const double* freq_hz,
                              int32_t n_systems, int32_t precision, const void* u, const void* lam,
                              double* g_logc, double* g_logrho, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!coef || !freq_hz || !u || !lam || !g_logc || !g_logrho || n_systems < 0) return NSR_ERR_ARGUMENT;
  if (precision != 0 && precision != 1) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  long long n = (long long)grid->nz * grid->nx;
  int bx = (int)((n + 255) / 256);
  if (bx > 148 * 16) bx = 148 * 16;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == 0)
    k_grad<float2><<<bx, 256, 0, st>>>(make_geo(*grid), coef, freq_hz, n_systems, (const float2*)u,
                                        (const float2*)lam, g_logc, g_logrho);
  else
    k_grad<double2><<<bx, 256, 0, st>>>(make_geo(*grid), coef, freq_hz, n_systems, (const double2*)u,
                                         (const double2*)lam, g_logc, g_logrho);
  return last_error();
}

// ---------------------------------------------------------------------------
// Tangent right-hand side -dA[dm] u (the Born perturbation of
// theranostic/wave.py:280-329 for a direction dm = (dlog c, dlog rho)).
// The flux part is the stencil evaluated with a' = -a dlogrho and zero ghost
// contrast (the fluxes are linear in a); the mass part is
// -2 k0^2 sx sz b (1+ie) dlogc - k0^2 sx sz b (1+ie)^2 dlogrho.  Output in SI
// units, the units of the solver's right-hand side.
// ---------------------------------------------------------------------------
template <typename CT>
__global__ void k_tangent(Geo g, const void* __restrict__ mat, const double* __restrict__ freq,
                          const CT* __restrict__ u, const double* __restrict__ dlogc,
                          const double* __restrict__ dlogrho, CT* __restrict__ rhs) {
  const long long n = (long long)g.nz * g.nx;
  const int sidx = blockIdx.y;
  const SysScalars s = sys_scalars(g, freq[sidx]);
  const MatPlanes mp = nsr_planes(mat, n);
  const CT* us = u + sidx * n;
  const double inv_h2 = 1.0 / (g.h * g.h);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.nx), j = (int)(k - (long long)i * g.nx);
    auto U = [&](int i2, int j2) -> double2 {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return make_double2(0.0, 0.0);
      const CT q = us[(long long)i2 * g.nx + j2];
      return make_double2((double)q.x, (double)q.y);
    };
    auto DA = [&](int i2, int j2) -> double {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return 0.0;
      const long long id = (long long)i2 * g.nx + j2;
      return -mp.a64[id] * dlogrho[id];
    };
    const double2 flux = stencil<double, false>(g, s, i, j, 0.0, mp.t64[k], U, DA);
    const double sig = s.sig;
    const double2 sx = make_double2(1.0, sig * pml_profile<double>((double)j, g.nx, g.n_pml));
    const double2 sz = make_double2(1.0, sig * pml_profile<double>((double)i, g.nz, g.n_pml));
    const double2 onepie = make_double2(1.0, mp.t64[k] * s.fpow);
    const double2 cell = (s.kh2 * mp.b64[k]) * (sx * sz);
    const double2 dmass = (-2.0 * dlogc[k]) * (cell * onepie) + (-dlogrho[k]) * (cell * (onepie * onepie));
    const double2 d = flux + dmass * U(i, j);
    const double2 r = (-inv_h2) * d;
    CT o;
    o.x = r.x;
    o.y = r.y;
    rhs[sidx * n + k] = o;
  }
}

extern "C" int nsr_tangent_rhs(const NsrGrid* grid, const void* coef, const double* freq_hz, int32_t n_systems,
                               int32_t precision, const void* u, const double* dlogc, const double* dlogrho,
                               void* rhs, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!coef || !freq_hz || !u || !dlogc || !dlogrho || !rhs || n_systems < 0 || n_systems > 65535)
    return NSR_ERR_ARGUMENT;
  if (precision != 0 && precision != 1) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  long long n = (long long)grid->nz * grid->nx;
  int bx = (int)((n + 255) / 256);
  if (bx > 148 * 8) bx = 148 * 8;
  dim3 gd(bx, n_systems);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == 0)
    k_tangent<float2><<<gd, 256, 0, st>>>(make_geo(*grid), coef, freq_hz, (const float2*)u, dlogc, dlogrho,
                                          (float2*)rhs);
  else
    k_tangent<double2><<<gd, 256, 0, st>>>(make_geo(*grid), coef, freq_hz, (const double2*)u, dlogc, dlogrho,
                                           (double2*)rhs);
  return last_error();
}

// ---------------------------------------------------------------------------
// Band-limited RF traces from receiver spectra (predict_band_rf,
// nsrno/wave_operator.py:169-180): the inverse real DFT with 'forward'
// normalisation of a spectrum that is zero except on the given positive bins,
//   x[t] = sum_b 2 Re(S[b] exp(2 pi i k_b t / n)),   0 < k_b < n/2.
// The phase k_b t is reduced modulo n in integers, so every term is exact to
// double rounding whatever the trace length.
// ---------------------------------------------------------------------------
__global__ void k_band_rf(int n_ch, int n_bins, int n, const double2* __restrict__ spec,
                          const int* __restrict__ bins, double* __restrict__ out) {
  const int ch = blockIdx.y;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < n_bins; ++b) {
      const long long m = ((long long)bins[b] * t) % n;
      double sn, cs;
      sincospi(2.0 * (double)m / (double)n, &sn, &cs);
      const double2 s = spec[(long long)ch * n_bins + b];
      acc += 2.0 * (s.x * cs - s.y * sn);
    }
    out[(long long)ch * n + t] = acc;
  }
}

extern "C" int nsr_band_rf(int32_t n_channels, int32_t n_bins, int32_t n_samples, const double* spectrum,
                           const int32_t* bins, double* rf, void* stream) {
  if (n_channels < 0 || n_bins < 0 || n_samples <= 0 || n_channels > 65535 || !rf ||
      (n_bins > 0 && (!spectrum || !bins)))
    return NSR_ERR_ARGUMENT;
  if (n_channels == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_bins == 0) {
    cudaError_t e = cudaMemsetAsync(rf, 0, sizeof(double) * (size_t)n_channels * n_samples, st);
    return e == cudaSuccess ? 0 : (int)e;
  }
  const int bx = (n_samples + 255) / 256;
  k_band_rf<<<dim3(bx, n_channels), 256, 0, st>>>(n_channels, n_bins, n_samples, (const double2*)spectrum, bins, rf);
  return last_error();
}

// ---------------------------------------------------------------------------
// FP64 true relative residual ||b - A x|| / ||b|| of n_systems fields
// (the acceptance check of nsrno/dense_wave.py:146-147,221-225 and
// theranostic/wave.py:320-323).  b is the given SI right-hand side or, when
// rhs is null, the plane-wave source of (freq, angle).  Per-CTA partials are
// summed in CTA order by a second kernel, so the result is deterministic.
// ---------------------------------------------------------------------------
#define NSR_TR_BLOCKS 256
__global__ void __launch_bounds__(256) k_true_residual(Geo g, const void* __restrict__ mat,
                                                       const double* __restrict__ freq,
                                                       const double* __restrict__ angle,
                                                       const double2* __restrict__ x, const double2* __restrict__ rhs,
                                                       int adjoint, double* __restrict__ partials) {
  const long long n = (long long)g.nz * g.nx;
  const int sidx = blockIdx.y;
  const SysScalars s = sys_scalars(g, freq[sidx]);
  const MatPlanes mp = nsr_planes(mat, n);
  const double2* xs = x + sidx * n;
  const double st = angle ? sin(angle[sidx]) : 0.0;
  const double h2 = g.h * g.h;
  double rr = 0.0, bb = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / g.nx), j = (int)(k - (long long)i * g.nx);
    auto P = [&](int i2, int j2) -> double2 {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return make_double2(0.0, 0.0);
      return xs[(long long)i2 * g.nx + j2];
    };
    auto Aa = [&](int i2, int j2) -> double {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= g.nx) return 1.0;
      return mp.a64[(long long)i2 * g.nx + j2];
    };
    double2 b;
    if (rhs) {
      b = h2 * rhs[sidx * n + k];
    } else if (i == g.face) {
      const double2 l = source_line(g, s.k0, st, j);
      b = make_double2(-l.x, -l.y);
    } else {
      b = make_double2(0.0, 0.0);
    }
    const double2 ax = adjoint ? stencil<double, true>(g, s, i, j, mp.b64[k], mp.t64[k], P, Aa)
                               : stencil<double, false>(g, s, i, j, mp.b64[k], mp.t64[k], P, Aa);
    const double2 r = b - ax;
    rr += r.x * r.x + r.y * r.y;
    bb += b.x * b.x + b.y * b.y;
  }
  __shared__ double wr[8], wb[8];
  for (int o = 16; o > 0; o >>= 1) {
    rr += __shfl_xor_sync(0xffffffffu, rr, o);
    bb += __shfl_xor_sync(0xffffffffu, bb, o);
  }
  if ((threadIdx.x & 31) == 0) { wr[threadIdx.x >> 5] = rr; wb[threadIdx.x >> 5] = bb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tr = 0.0, tb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tr += wr[w]; tb += wb[w]; }
    partials[((long long)sidx * gridDim.x + blockIdx.x) * 2] = tr;
    partials[((long long)sidx * gridDim.x + blockIdx.x) * 2 + 1] = tb;
  }
}

__global__ void k_true_residual_sum(int n_systems, int nb, const double* __restrict__ partials,
                                    double* __restrict__ residual) {
  const int sidx = blockIdx.x * blockDim.x + threadIdx.x;
  if (sidx >= n_systems) return;
  double rr = 0.0, bb = 0.0;
  for (int b = 0; b < nb; ++b) {
    rr += partials[((long long)sidx * nb + b) * 2];
    bb += partials[((long long)sidx * nb + b) * 2 + 1];
  }
  residual[sidx] = bb > 0.0 ? sqrt(rr / bb) : sqrt(rr);
}

extern "C" size_t nsr_true_residual_workspace_size(const NsrGrid* grid, int32_t n_systems) {
  if (nsr_check_grid(grid, false) || n_systems <= 0 || n_systems > 65535) return 0;
  return nsr_align(sizeof(double) * 2 * NSR_TR_BLOCKS * (size_t)n_systems);
}

extern "C" int nsr_true_residual(const NsrGrid* grid, const void* coef, const double* freq_hz,
                                 const double* angle_rad, int32_t n_systems, int32_t adjoint, const double* x,
                                 const double* rhs, double* residual, void* workspace, size_t workspace_bytes,
                                 void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!coef || !freq_hz || !x || !residual || !workspace || n_systems < 0 || n_systems > 65535) return NSR_ERR_ARGUMENT;
  if (!rhs && !angle_rad) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  if (workspace_bytes < nsr_true_residual_workspace_size(grid, n_systems)) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  double* partials = (double*)workspace;
  k_true_residual<<<dim3(NSR_TR_BLOCKS, n_systems), 256, 0, st>>>(make_geo(*grid), coef, freq_hz,
                                                                   rhs ? nullptr : angle_rad, (const double2*)x,
                                                                   (const double2*)rhs, adjoint ? 1 : 0, partials);
  k_true_residual_sum<<<(n_systems + 127) / 128, 128, 0, st>>>(n_systems, NSR_TR_BLOCKS, partials, residual);
  return last_error();
}
