// Converged solve of the dense path's operator on the device: restarted,
// right-preconditioned GMRES(m) with two classical Gram-Schmidt passes, all
// fields of a frequency (the angles) treated as one vector as the reference's
// solver does (nsrno/wave_solver.py:9-36 used by solve_system,
// nsrno/dense_wave.py:212-220).
//
// Precision: Krylov vectors are complex64; every inner product, norm, the
// Hessenberg matrix, the Givens rotations and the small triangular solve are
// FP64 on the device; the iterate x is complex128 and each cycle restarts from
// the FP64 true residual b - A x of the complex128 operator -- the mixed FP32
// inverse / FP64 residual refinement of nsrno/dense_wave.py:168-191 folded
// into the restart.
//
// Per Arnoldi step j the host enqueues (no synchronisation):
//   z_j = M v_j                 nsr_dense_precondition (fixed shifted Laplacian)
//   w   = A z_j                 nsr_dense_apply (complex64)
//   h   = V_{0..j}^H w          k_dg_dots     (FP64 partials, last CTA sums)
//   w  -= V h                   k_dg_update
//   h' = V^H w ; w -= V h'      k_dg_dots, k_dg_update (+ ||w||^2, Givens)
//   v_{j+1} = w / ||w||         k_dg_next
// and per cycle the FP64 residual, the back substitution and x += Z y.  The
// host reads one small state record per cycle to decide whether to go on.
#include "nsr_internal.cuh"
#include "nsr_device.cuh"

#include <stdlib.h>
#include <string.h>

#define NSR_DG_MAX_M 64
#define NSR_DG_THREADS 256
#define NSR_DG_GROUP 8   // basis vectors per accumulation pass of k_dg_dots

struct DgState {
  int done;        // 1: converged / budget / non-finite, status is final
  int status;      // NSR_* status
  int used;        // Arnoldi steps of the current cycle
  int stop;        // happy breakdown: the cycle ends after `used` steps
  int steps;       // Arnoldi steps so far
  int cycles;      // cycles started
  int pad0, pad1;
  double bnorm;    // ||b||
  double beta;     // ||r|| at the start of the cycle
  double rel;      // true relative residual at the start of the last cycle
};

struct DgArgs {
  long long n;         // complex entries of the whole vector (fields x H x W)
  int m;
  int nb;              // CTAs of the vector kernels
  DgState* st;
  int* arrive;
  double* part;        // [nb][2 (m + 1)]
  double2* H;          // [(m + 1) m], column j at H[j (m + 1) + i]
  double* cs;          // [m]
  double2* sn;         // [m]
  double2* gv;         // [m + 1]
  double2* hc;         // [m + 1] coefficients of the current Gram-Schmidt pass
  double2* y;          // [m]
  float2* V;           // [m + 1][n]
  float2* Z;           // [m][n]
  float2* w;           // [n]
  const double2* b;    // [n]
  double2* x;          // [n]
  const double2* ax;   // [n]  A x of the current iterate
  double tol;
  int max_cycles;
};

// Block sum of `v` over NSR_DG_THREADS threads; thread 0 gets the total.
__device__ __forceinline__ double dg_block_sum(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < NSR_DG_THREADS / 32; ++k) t += red[k];
  return t;
}

// Publishes this CTA's `nv` partials and returns true in the last CTA to
// arrive, after summing every CTA's partials in CTA order into tot[0..nv).
__device__ bool dg_arrive(const DgArgs& A, const double* mine, int nv, double* tot) {
  __shared__ int last;
  __shared__ double red[NSR_DG_THREADS / 32];
  if (threadIdx.x == 0) {
    for (int q = 0; q < nv; ++q) A.part[(long long)blockIdx.x * 2 * (A.m + 1) + q] = mine[q];
    __threadfence();
    last = atomicAdd(A.arrive, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int q = 0; q < nv; ++q) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += NSR_DG_THREADS)
      s += __ldcg(&A.part[(long long)b * 2 * (A.m + 1) + q]);
    s = dg_block_sum(s, red);
    if (threadIdx.x == 0) tot[q] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *A.arrive = 0;
  return true;
}

// ||b||^2 (once per solve).
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_bnorm(DgArgs A) {
  __shared__ double red[NSR_DG_THREADS / 32];
  __shared__ double mine[1], tot[1];
  double s = 0.0;
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    const double2 v = A.b[e];
    s += v.x * v.x + v.y * v.y;
  }
  s = dg_block_sum(s, red);
  if (threadIdx.x == 0) mine[0] = s;
  if (dg_arrive(A, mine, 1, tot) && threadIdx.x == 0) {
    DgState& S = *A.st;
    S.bnorm = sqrt(tot[0]);
    S.done = 0;
    S.status = NSR_NOT_RUN;
    S.steps = 0;
    S.cycles = 0;
  }
}

// r = b - A x (FP64), v_0 = r in complex64, ||r||^2; the last CTA decides
// whether the solve has converged and sets up the cycle.
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_residual(DgArgs A) {
  __shared__ double red[NSR_DG_THREADS / 32];
  __shared__ double mine[1], tot[1];
  if (A.st->done) return;
  double s = 0.0;
  float2* v0 = A.V;
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    const double2 r = A.b[e] - A.ax[e];
    s += r.x * r.x + r.y * r.y;
    v0[e] = to_f(r);
  }
  s = dg_block_sum(s, red);
  if (threadIdx.x == 0) mine[0] = s;
  if (dg_arrive(A, mine, 1, tot) && threadIdx.x == 0) {
    DgState& S = *A.st;
    const double beta = sqrt(tot[0]);
    const double rel = S.bnorm > 0.0 ? beta / S.bnorm : 0.0;
    S.rel = rel;
    S.beta = beta;
    S.used = 0;
    S.stop = 0;
    if (!isfinite(rel)) {
      S.done = 1;
      S.status = NSR_NONFINITE;
    } else if (rel < A.tol || !(S.bnorm > 0.0)) {
      S.done = 1;
      S.status = NSR_CONVERGED;
    } else if (S.cycles >= A.max_cycles) {
      S.done = 1;
      S.status = NSR_ITERATION_BUDGET;
    } else {
      S.cycles += 1;
      for (int i = 0; i <= A.m; ++i) A.gv[i] = make_double2(0.0, 0.0);
      A.gv[0] = make_double2(beta, 0.0);
    }
  }
}

// v_0 /= beta (the division of the reference's basis[0] = r / beta).
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_scale0(DgArgs A) {
  const DgState& S = *A.st;
  if (S.done) return;
  const float inv = (float)(1.0 / S.beta);
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    const float2 v = A.V[e];
    A.V[e] = make_float2(v.x * inv, v.y * inv);
  }
}

__device__ __forceinline__ bool dg_skip(const DgState& S) { return S.done || S.stop; }

// hc[i] = <v_i, w> for i <= j, also added to column j of the Hessenberg matrix
// (the two Gram-Schmidt passes sum into it).
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_dots(DgArgs A, int j) {
  __shared__ double red[NSR_DG_THREADS / 32];
  __shared__ double mine[2 * (NSR_DG_MAX_M + 1)], tot[2 * (NSR_DG_MAX_M + 1)];
  if (dg_skip(*A.st)) return;
  const int nv = j + 1;
  for (int i0 = 0; i0 < nv; i0 += NSR_DG_GROUP) {
    const int cnt = min(NSR_DG_GROUP, nv - i0);
    double re[NSR_DG_GROUP], im[NSR_DG_GROUP];
#pragma unroll
    for (int k = 0; k < NSR_DG_GROUP; ++k) re[k] = im[k] = 0.0;
    for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
         e += (long long)gridDim.x * NSR_DG_THREADS) {
      const float2 wv = A.w[e];
#pragma unroll
      for (int k = 0; k < NSR_DG_GROUP; ++k)
        if (k < cnt) dot_acc(re[k], im[k], A.V[(long long)(i0 + k) * A.n + e], wv);
    }
#pragma unroll
    for (int k = 0; k < NSR_DG_GROUP; ++k) {
      if (k < cnt) {
        const double sr = dg_block_sum(re[k], red);
        const double si = dg_block_sum(im[k], red);
        if (threadIdx.x == 0) { mine[2 * (i0 + k)] = sr; mine[2 * (i0 + k) + 1] = si; }
      }
    }
  }
  __syncthreads();
  if (dg_arrive(A, mine, 2 * nv, tot)) {
    for (int i = threadIdx.x; i < nv; i += NSR_DG_THREADS) {
      const double2 h = make_double2(tot[2 * i], tot[2 * i + 1]);
      A.hc[i] = h;
      A.H[(long long)j * (A.m + 1) + i] = A.H[(long long)j * (A.m + 1) + i] + h;
    }
  }
}

// w -= sum_i hc[i] v_i.  With `last`, also ||w||^2; the last CTA then
// completes column j of the Hessenberg matrix, applies the earlier Givens
// rotations, forms the new one and detects a happy breakdown.
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_update(DgArgs A, int j, int last) {
  __shared__ double red[NSR_DG_THREADS / 32];
  __shared__ double mine[1], tot[1];
  __shared__ double2 h[NSR_DG_MAX_M + 1];
  if (dg_skip(*A.st)) return;
  const int nv = j + 1;
  for (int i = threadIdx.x; i < nv; i += NSR_DG_THREADS) h[i] = A.hc[i];
  __syncthreads();
  double s = 0.0;
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    float2 wv = A.w[e];
    double2 acc = make_double2(wv.x, wv.y);
    for (int i = 0; i < nv; ++i) {
      const float2 v = A.V[(long long)i * A.n + e];
      const double2 hi = h[i];
      acc.x -= hi.x * v.x - hi.y * v.y;
      acc.y -= hi.x * v.y + hi.y * v.x;
    }
    wv = to_f(acc);
    A.w[e] = wv;
    if (last) s += (double)wv.x * wv.x + (double)wv.y * wv.y;
  }
  if (!last) return;
  s = dg_block_sum(s, red);
  if (threadIdx.x == 0) mine[0] = s;
  if (dg_arrive(A, mine, 1, tot) && threadIdx.x == 0) {
    DgState& S = *A.st;
    const int m1 = A.m + 1;
    double2* col = A.H + (long long)j * m1;
    const double hn = sqrt(tot[0]);
    col[j + 1] = make_double2(hn, 0.0);
    S.steps += 1;
    S.used = j + 1;
    // Givens rotations G_i = [[c, s], [-conj(s), c]] (c real) applied to rows i, i+1.
    for (int i = 0; i < j; ++i) {
      const double2 a = col[i], b = col[i + 1];
      col[i] = A.cs[i] * a + A.sn[i] * b;
      col[i + 1] = A.cs[i] * b - conjc(A.sn[i]) * a;
    }
    const double2 a = col[j];
    const double an = sqrt(a.x * a.x + a.y * a.y);
    const double den = sqrt(an * an + hn * hn);
    double c;
    double2 sgn;
    if (den == 0.0) {
      c = 1.0; sgn = make_double2(0.0, 0.0);
    } else if (an == 0.0) {
      c = 0.0; sgn = make_double2(1.0, 0.0);
    } else {
      c = an / den;
      const double2 ph = make_double2(a.x / an, a.y / an);
      sgn = (hn / den) * ph;   // s = (a / |a|) hn / den
    }
    A.cs[j] = c;
    A.sn[j] = sgn;
    col[j] = c * a + hn * sgn;   // = (a / |a|) den
    col[j + 1] = make_double2(0.0, 0.0);
    const double2 g = A.gv[j];
    A.gv[j] = c * g;
    A.gv[j + 1] = make_double2(0.0, 0.0) - conjc(sgn) * g;
    if (!isfinite(hn)) {
      S.done = 1;
      S.status = NSR_NONFINITE;
    } else if (hn < 1e-12) {
      S.stop = 1;   // happy breakdown (nsrno/wave_solver.py:29-31)
    }
    S.beta = hn;   // normaliser of v_{j+1}
  }
}

// v_{j+1} = w / ||w|| (skipped after a happy breakdown).
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_next(DgArgs A, int j) {
  const DgState& S = *A.st;
  if (dg_skip(S)) return;
  const float inv = (float)(1.0 / S.beta);
  float2* v = A.V + (long long)(j + 1) * A.n;
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    const float2 wv = A.w[e];
    v[e] = make_float2(wv.x * inv, wv.y * inv);
  }
}

// y = R^-1 g over the steps of the cycle (FP64, one thread).
__global__ void k_dg_solve(DgArgs A) {
  const DgState& S = *A.st;
  if (S.done || threadIdx.x != 0) return;
  const int k = S.used;
  const int m1 = A.m + 1;
  for (int i = k - 1; i >= 0; --i) {
    double2 s = A.gv[i];
    for (int l = i + 1; l < k; ++l) s = s - A.H[(long long)l * m1 + i] * A.y[l];
    A.y[i] = divc(s, A.H[(long long)i * m1 + i]);
  }
  // a fresh Hessenberg matrix for the next cycle
  for (int e = 0; e < m1 * A.m; ++e) A.H[e] = make_double2(0.0, 0.0);
}

// x += sum_j y_j z_j (FP64).
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_xupdate(DgArgs A) {
  __shared__ double2 y[NSR_DG_MAX_M];
  const DgState& S = *A.st;
  if (S.done) return;
  const int k = S.used;
  for (int i = threadIdx.x; i < k; i += NSR_DG_THREADS) y[i] = A.y[i];
  __syncthreads();
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < A.n;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    double2 acc = A.x[e];
    for (int i = 0; i < k; ++i) acc = acc + y[i] * to_d(A.Z[(long long)i * A.n + e]);
    A.x[e] = acc;
  }
}

// Per-field relative residual ||b_f - A x_f|| / ||b_f|| (the reference's
// max_angle_residual, nsrno/dense_wave.py:221-223); grid (chunks, fields).
__global__ void __launch_bounds__(NSR_DG_THREADS) k_dg_field_residual(const double2* __restrict__ b,
                                                                      const double2* __restrict__ ax, long long nf,
                                                                      double* __restrict__ part, int* arrive,
                                                                      double* __restrict__ out) {
  __shared__ double red[NSR_DG_THREADS / 32];
  __shared__ int last;
  const int f = blockIdx.y;
  double rr = 0.0, bb = 0.0;
  for (long long e = blockIdx.x * (long long)NSR_DG_THREADS + threadIdx.x; e < nf;
       e += (long long)gridDim.x * NSR_DG_THREADS) {
    const double2 bv = b[f * nf + e];
    const double2 r = bv - ax[f * nf + e];
    rr += r.x * r.x + r.y * r.y;
    bb += bv.x * bv.x + bv.y * bv.y;
  }
  rr = dg_block_sum(rr, red);
  bb = dg_block_sum(bb, red);
  double* p = part + 2LL * gridDim.x * f;
  if (threadIdx.x == 0) {
    p[2 * blockIdx.x] = rr;
    p[2 * blockIdx.x + 1] = bb;
    __threadfence();
    last = atomicAdd(&arrive[f], 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double sr = 0.0, sb = 0.0;
  for (int k = 0; k < (int)gridDim.x; ++k) {
    sr += __ldcg(&p[2 * k]);
    sb += __ldcg(&p[2 * k + 1]);
  }
  out[f] = sb > 0.0 ? sqrt(sr / sb) : sqrt(sr);
  arrive[f] = 0;
}

__global__ void k_dg_zero_ints(int* p, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) p[k] = 0;
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct DgLayout {
  size_t state, arrive, part, small, V, Z, w, ax, apply_ws, prec_ws, total;
  int nb;
};

static int dg_blocks() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return 4 * sms;
}

static DgLayout dg_layout(const NsrDenseGrid* g, int n_fields, int m, int nb) {
  DgLayout L;
  const size_t n = (size_t)g->H * g->W * n_fields;
  size_t off = 0;
  L.nb = nb;
  L.state = off; off += nsr_align(sizeof(DgState));
  L.arrive = off; off += nsr_align(sizeof(int) * (1 + (size_t)n_fields));
  L.part = off; off += nsr_align(sizeof(double) * 2 * (size_t)(m + 1) * (nb > n_fields * 64 ? nb : n_fields * 64));
  L.small = off; off += nsr_align(sizeof(double2) * ((size_t)(m + 1) * m + 4 * (m + 1)) + sizeof(double) * m);
  L.V = off; off += nsr_align(sizeof(float2) * n * (m + 1));
  L.Z = off; off += nsr_align(sizeof(float2) * n * m);
  L.w = off; off += nsr_align(sizeof(float2) * n);
  L.ax = off; off += nsr_align(sizeof(double2) * n);
  L.apply_ws = off; off += nsr_align(nsr_dense_workspace_size(g, n_fields, 1));
  L.prec_ws = off; off += nsr_align(nsr_dense_precondition_workspace_size(g, n_fields));
  L.total = off;
  return L;
}

extern "C" size_t nsr_dense_solve_workspace_size(const NsrDenseGrid* grid, int32_t n_fields, int32_t restart) {
  if (!grid || n_fields <= 0 || n_fields > 65535 || restart < 1 || restart > NSR_DG_MAX_M) return 0;
  if (nsr_dense_precondition_workspace_size(grid, n_fields) == 0) return 0;
  return dg_layout(grid, n_fields, restart, dg_blocks()).total;
}

extern "C" int nsr_dense_solve(const NsrDenseGrid* grid, const double* coef, const NsrDenseSolveParams* p,
                               int32_t n_fields, const double* rhs, double* x, double* field_residual,
                               NsrDenseSolveInfo* info, void* workspace, size_t workspace_bytes, void* stream) {
  if (!grid || !coef || !p || !rhs || !x || !workspace || n_fields <= 0 || n_fields > 65535) return NSR_ERR_ARGUMENT;
  const int m = p->restart;
  if (m < 1 || m > NSR_DG_MAX_M || p->max_cycles < 1 || !(p->tolerance > 0) || !(p->k0dx2 > 0) || !(p->shift >= 0))
    return NSR_ERR_ARGUMENT;
  if (nsr_dense_precondition_workspace_size(grid, n_fields) == 0) return NSR_ERR_UNSUPPORTED_SIZE;
  const int nb = dg_blocks();
  const DgLayout L = dg_layout(grid, n_fields, m, nb);
  if (workspace_bytes < L.total) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  const long long nf = (long long)grid->H * grid->W;
  DgArgs A;
  memset(&A, 0, sizeof(A));
  A.n = nf * n_fields;
  A.m = m;
  A.nb = nb;
  A.st = (DgState*)(ws + L.state);
  A.arrive = (int*)(ws + L.arrive);
  A.part = (double*)(ws + L.part);
  double2* small = (double2*)(ws + L.small);
  A.H = small;
  A.sn = A.H + (size_t)(m + 1) * m;
  A.gv = A.sn + (m + 1);
  A.hc = A.gv + (m + 1);
  A.y = A.hc + (m + 1);
  A.cs = (double*)(A.y + (m + 1));
  A.V = (float2*)(ws + L.V);
  A.Z = (float2*)(ws + L.Z);
  A.w = (float2*)(ws + L.w);
  A.b = (const double2*)rhs;
  A.x = (double2*)x;
  A.ax = (const double2*)(ws + L.ax);
  A.tol = p->tolerance;
  A.max_cycles = p->max_cycles;
  void* apply_ws = ws + L.apply_ws;
  const size_t apply_bytes = nsr_dense_workspace_size(grid, n_fields, 1);
  void* prec_ws = ws + L.prec_ws;
  const size_t prec_bytes = nsr_dense_precondition_workspace_size(grid, n_fields);
  const int adj = p->adjoint ? 1 : 0;
  int err = 0;
  // Pinned host record of the solve state, one per host thread, kept for the
  // life of the thread (read once per restart cycle).
  static thread_local DgState* host = nullptr;
  if (!host && cudaHostAlloc((void**)&host, sizeof(DgState), cudaHostAllocDefault) != cudaSuccess) {
    host = nullptr;
    return cudaErrorMemoryAllocation;
  }
#define DG_TRY(expr) do { int e_ = (int)(expr); if (e_) { err = e_; goto done; } } while (0)
  k_dg_zero_ints<<<1, 256, 0, st>>>(A.arrive, 1 + n_fields);
  DG_TRY(cudaMemsetAsync(A.H, 0, sizeof(double2) * (size_t)(m + 1) * m, st));
  k_dg_bnorm<<<nb, NSR_DG_THREADS, 0, st>>>(A);
  DG_TRY(cudaGetLastError());
  for (;;) {
    DG_TRY(nsr_dense_apply(grid, coef, p->scal_re, p->scal_im, n_fields, adj, 1, x, (void*)A.ax, apply_ws,
                           apply_bytes, stream));
    k_dg_residual<<<nb, NSR_DG_THREADS, 0, st>>>(A);
    DG_TRY(cudaGetLastError());
    DG_TRY(cudaMemcpyAsync(host, A.st, sizeof(DgState), cudaMemcpyDeviceToHost, st));
    DG_TRY(cudaStreamSynchronize(st));
    if (host->done) break;
    k_dg_scale0<<<nb, NSR_DG_THREADS, 0, st>>>(A);
    for (int j = 0; j < m; ++j) {
      DG_TRY(nsr_dense_precondition(grid, p->k0dx2, p->shift, n_fields, adj, (const float*)(A.V + j * A.n),
                                    (float*)(A.Z + j * A.n), prec_ws, prec_bytes, stream));
      DG_TRY(nsr_dense_apply(grid, coef, p->scal_re, p->scal_im, n_fields, adj, 0, A.Z + j * A.n, A.w, apply_ws,
                             apply_bytes, stream));
      k_dg_dots<<<nb, NSR_DG_THREADS, 0, st>>>(A, j);
      k_dg_update<<<nb, NSR_DG_THREADS, 0, st>>>(A, j, 0);
      k_dg_dots<<<nb, NSR_DG_THREADS, 0, st>>>(A, j);
      k_dg_update<<<nb, NSR_DG_THREADS, 0, st>>>(A, j, 1);
      k_dg_next<<<nb, NSR_DG_THREADS, 0, st>>>(A, j);
      DG_TRY(cudaGetLastError());
    }
    k_dg_solve<<<1, 32, 0, st>>>(A);
    k_dg_xupdate<<<nb, NSR_DG_THREADS, 0, st>>>(A);
    DG_TRY(cudaGetLastError());
  }
  if (field_residual) {
    dim3 gr(nb / n_fields > 8 ? nb / n_fields : 8, n_fields);
    k_dg_field_residual<<<gr, NSR_DG_THREADS, 0, st>>>(A.b, A.ax, nf, A.part, A.arrive + 1, field_residual);
    DG_TRY(cudaGetLastError());
  }
  if (info) {
    info->status = host->status;
    info->steps = host->steps;
    info->cycles = host->cycles;
    info->reserved = 0;
    info->residual = host->rel;
  }
done:
#undef DG_TRY
  return err;
}
