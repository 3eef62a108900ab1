// Learned preconditioner of the 5-point path: inference and training kernels.
//
// The network is the reference's LearnedPreconditioner
// (nsrno/conditioned_wave.py:94-117): an 8x average-pooled five-channel
// context, three 3x3 convolutions 5->16->16->4 with tanh between, bilinear
// upsampling, bounded complex inner/outer gains and a spectrally modulated
// shifted-Laplace multiplier, applied as
//     M r = outer * IFFT(m * FFT(inner * r))
// (learned_apply, nsrno/dense_wave.py:150-165).  On the 5-point grid the map is
// the complex conjugate of the reference's (exp(-i omega t) convention) in the
// units of the h^2-scaled operator.
//
// Sizes: the network runs on (nz/8) x (nx/8) pixels -- 12,288 at 768 x 1024 --
// with 3,636 weights, about 90 MFLOP per frequency.  It is set up once per
// frequency and is bound by launch latency, not by the tensor cores or HBM, so
// the convolutions are CUDA-core loops with the weights staged in shared
// memory.  Two precisions share the kernels: FP32, and BF16 (weights rounded
// to bfloat16, activations stored as bfloat16, every product accumulated in
// FP32; the master weights and their gradients stay FP32).  What matters for the solve is that the gains are stored once
// per frequency as two complex64 planes (16 B per node) that the Krylov kernels
// read next to the vectors they already stream.
//
// Training kernels give the exact gradient of any real loss with respect to
// all 3,645 parameters, given the cotangents of the gains (per node) and of the
// spectral multiplier (per Fourier point, formed here from two transformed
// fields):
//   nsr_learned_map_backward      gain cotangents -> d(maps) at low resolution
//                                 (chain through tanh/exp, transposed bilinear)
//   nsr_learned_network_backward  d(maps) -> d(conv weights, biases)
//   nsr_learned_spectral_backward d(spectral[2][4], log_shift)
//   nsr_learned_adam              clipped Adam step (the reference's optimiser,
//                                 nsrno/train_dense_wave.py:37,76)
#include "nsr_internal.cuh"
#include "nsr_device.cuh"

#include <cuda_bf16.h>
#include <stdlib.h>
#include <string.h>

// Flat parameter layout (the reference module's state_dict order).
#define LP_SPEC 0
#define LP_LOGSHIFT 8
#define LP_W1 9
#define LP_B1 (LP_W1 + 16 * 5 * 9)
#define LP_W2 (LP_B1 + 16)
#define LP_B2 (LP_W2 + 16 * 16 * 9)
#define LP_W3 (LP_B2 + 16)
#define LP_B3 (LP_W3 + 4 * 16 * 9)
#define LP_NPARAM (LP_B3 + 4)
static_assert(LP_NPARAM == NSR_LEARNED_PARAMS, "parameter count");

// Low-resolution state planes of one frequency.
#define LP_POOL 0      // 5 pooled context channels
#define LP_A1 5        // tanh(conv1), 16
#define LP_A2 21       // tanh(conv2), 16
#define LP_MAPS 37     // conv3, 4
#define LP_PLANES 41

namespace {

// Activation storage of the network: float, or bfloat16 (the BF16 network:
// weights rounded to bfloat16 and activations stored in bfloat16, every
// product accumulated in float).
__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void stv(float* p, float v) { *p = v; }
__device__ __forceinline__ void stv(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
template <typename T> __device__ __forceinline__ float wround(float w);
template <> __device__ __forceinline__ float wround<float>(float w) { return w; }
template <> __device__ __forceinline__ float wround<__nv_bfloat16>(float w) {
  return __bfloat162float(__float2bfloat16_rn(w));
}

inline int lp_h(const NsrGrid* g) { return g->nz / 8; }
inline int lp_w(const NsrGrid* g) { return g->nx / 8; }

inline int last_error() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : (int)e;
}

// Bilinear source of output index `dst` (F.interpolate, align_corners=False).
struct Lerp {
  int i0, i1;
  float l1;
};
__device__ __forceinline__ Lerp lerp_of(int dst, int n_in, int n_out) {
  const float scale = (float)n_in / (float)n_out;
  const float src = fmaxf(((float)dst + 0.5f) * scale - 0.5f, 0.0f);
  Lerp L;
  L.i0 = min((int)src, n_in - 1);
  L.i1 = min(L.i0 + 1, n_in - 1);
  L.l1 = src - (float)L.i0;
  return L;
}
__device__ __forceinline__ float lerp_weight(const Lerp& L, int p) {
  return (L.i0 == p ? 1.0f - L.l1 : 0.0f) + (L.i1 == p ? L.l1 : 0.0f);
}

template <typename T>
__device__ __forceinline__ void node_maps(const T* __restrict__ maps, int hw, int w8, const Lerp& lz,
                                          const Lerp& lx, float m[4]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const T* M = maps + c * hw;
    const float top = (1.0f - lx.l1) * ld(M + lz.i0 * w8 + lx.i0) + lx.l1 * ld(M + lz.i0 * w8 + lx.i1);
    const float bot = (1.0f - lx.l1) * ld(M + lz.i1 * w8 + lx.i0) + lx.l1 * ld(M + lz.i1 * w8 + lx.i1);
    m[c] = (1.0f - lz.l1) * top + lz.l1 * bot;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Set-up: context and pooling, convolutions, gains.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_lp_pool(int nz, int nx, int h8, int w8, const float* __restrict__ c, const float* __restrict__ rho,
                          const float* __restrict__ alpha, const double* __restrict__ freq, int n_freq,
                          T* __restrict__ state) {
  const int hw = h8 * w8;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= hw) return;
  const int py = p / w8, px = p - py * w8;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int dy = 0; dy < 8; ++dy)
    for (int dx = 0; dx < 8; ++dx) {
      const long long k = (long long)(8 * py + dy) * nx + 8 * px + dx;
      s0 += log((double)c[k] / 1540.0) / 0.06;
      s1 += log((double)rho[k] / 1000.0) / 0.08;
      s2 += log1p((double)alpha[k]);
    }
  for (int f = 0; f < n_freq; ++f) {
    T* sp = state + (long long)f * LP_PLANES * hw + LP_POOL * hw;
    stv(sp + p, (float)(s0 / 64.0));
    stv(sp + hw + p, (float)(s1 / 64.0));
    stv(sp + 2 * hw + p, (float)(s2 / 64.0));
    stv(sp + 3 * hw + p, (float)(freq[f] / 6e6 - 1.0));
    stv(sp + 4 * hw + p, 1.0f);
  }
}

// 3x3 cross-correlation, zero padding 1, one thread per pixel and all COUT outputs.
template <typename T, int CIN, int COUT, bool TANH>
__global__ void __launch_bounds__(128) k_lp_conv(int h8, int w8, const float* __restrict__ wt,
                                                 const float* __restrict__ bias, T* __restrict__ state,
                                                 int in_plane, int out_plane) {
  __shared__ float sw[COUT * CIN * 9];
  __shared__ float sb[COUT];
  for (int k = threadIdx.x; k < COUT * CIN * 9; k += blockDim.x) sw[k] = wround<T>(wt[k]);
  for (int k = threadIdx.x; k < COUT; k += blockDim.x) sb[k] = wround<T>(bias[k]);
  __syncthreads();
  const int hw = h8 * w8;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= hw) return;
  const T* in = state + (long long)blockIdx.y * LP_PLANES * hw + in_plane * hw;
  T* out = state + (long long)blockIdx.y * LP_PLANES * hw + out_plane * hw;
  const int y = p / w8, x = p - y * w8;
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = sb[co];
  for (int ci = 0; ci < CIN; ++ci)
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      const int yy = y + ky - 1;
      if (yy < 0 || yy >= h8) continue;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int xx = x + kx - 1;
        if (xx < 0 || xx >= w8) continue;
        const float v = ld(in + ci * hw + yy * w8 + xx);
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] += sw[((co * CIN + ci) * 3 + ky) * 3 + kx] * v;
      }
    }
#pragma unroll
  for (int co = 0; co < COUT; ++co) stv(out + co * hw + p, TANH ? tanhf(acc[co]) : acc[co]);
}

// inner = (1 + tanh(m0)/2) exp(-i tanh(m1)/2), outer likewise from m2, m3.
template <typename T>
__global__ void k_lp_gains(int nz, int nx, int h8, int w8, const T* __restrict__ state,
                           float2* __restrict__ gains) {
  const long long n = (long long)nz * nx;
  const int hw = h8 * w8;
  const int f = blockIdx.y;
  const T* maps = state + (long long)f * LP_PLANES * hw + LP_MAPS * hw;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / nx), j = (int)(k - (long long)i * nx);
    float m[4];
    node_maps(maps, hw, w8, lerp_of(i, h8, nz), lerp_of(j, w8, nx), m);
    float s1, c1, s3, c3;
    sincosf(0.5f * tanhf(m[1]), &s1, &c1);
    sincosf(0.5f * tanhf(m[3]), &s3, &c3);
    const float g0 = 1.0f + 0.5f * tanhf(m[0]);
    const float g2 = 1.0f + 0.5f * tanhf(m[2]);
    gains[(2LL * f) * n + k] = make_float2(g0 * c1, -g0 * s1);
    gains[(2LL * f + 1) * n + k] = make_float2(g2 * c3, -g2 * s3);
  }
}

extern "C" size_t nsr_learned_state_bytes(const NsrGrid* grid, int32_t n_freq) {
  if (nsr_check_grid(grid, false) || n_freq <= 0) return 0;
  return nsr_align(sizeof(float) * (size_t)LP_PLANES * lp_h(grid) * lp_w(grid) * n_freq);
}

template <typename T>
static void learned_setup_t(const NsrGrid* grid, const float* c, const float* rho, const float* alpha,
                            const double* freq_hz, int n_freq, const float* params, T* state, void* gains,
                            cudaStream_t st) {
  const int h8 = lp_h(grid), w8 = lp_w(grid), hw = h8 * w8;
  const int pb = (hw + 127) / 128;
  k_lp_pool<T><<<pb, 128, 0, st>>>(grid->nz, grid->nx, h8, w8, c, rho, alpha, freq_hz, n_freq, state);
  const dim3 gconv(pb, n_freq);
  k_lp_conv<T, 5, 16, true><<<gconv, 128, 0, st>>>(h8, w8, params + LP_W1, params + LP_B1, state, LP_POOL, LP_A1);
  k_lp_conv<T, 16, 16, true><<<gconv, 128, 0, st>>>(h8, w8, params + LP_W2, params + LP_B2, state, LP_A1, LP_A2);
  k_lp_conv<T, 16, 4, false><<<gconv, 128, 0, st>>>(h8, w8, params + LP_W3, params + LP_B3, state, LP_A2, LP_MAPS);
  if (gains) {
    const long long n = (long long)grid->nz * grid->nx;
    int bx = (int)((n + 255) / 256);
    if (bx > 1184) bx = 1184;
    k_lp_gains<T><<<dim3(bx, n_freq), 256, 0, st>>>(grid->nz, grid->nx, h8, w8, state, (float2*)gains);
  }
}

extern "C" int nsr_learned_setup_ex(const NsrGrid* grid, const float* c, const float* rho, const float* alpha,
                                    const double* freq_hz, int32_t n_freq, const float* params, int32_t precision,
                                    void* state, void* gains, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!c || !rho || !alpha || !freq_hz || !params || !state || n_freq < 0 || n_freq > 65535) return NSR_ERR_ARGUMENT;
  if (precision != NSR_LEARNED_FP32 && precision != NSR_LEARNED_BF16) return NSR_ERR_ARGUMENT;
  if (n_freq == 0) return 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == NSR_LEARNED_BF16)
    learned_setup_t(grid, c, rho, alpha, freq_hz, n_freq, params, (__nv_bfloat16*)state, gains, st);
  else
    learned_setup_t(grid, c, rho, alpha, freq_hz, n_freq, params, (float*)state, gains, st);
  return last_error();
}

extern "C" int nsr_learned_setup(const NsrGrid* grid, const float* c, const float* rho, const float* alpha,
                                 const double* freq_hz, int32_t n_freq, const float* params, void* state,
                                 void* gains, void* stream) {
  return nsr_learned_setup_ex(grid, c, rho, alpha, freq_hz, n_freq, params, NSR_LEARNED_FP32, state, gains, stream);
}

// ---------------------------------------------------------------------------
// Gain-index validation shared by every entry point that reads gains.
// ---------------------------------------------------------------------------
int nsr_check_learned(const NsrLearned* L, int n_systems, cudaStream_t st) {
  if (!L) return 0;
  if (!L->params) return NSR_ERR_ARGUMENT;
  if (!L->gains) return 0;
  if (L->n_gain <= 0) return NSR_ERR_ARGUMENT;
  if (!L->gain_index) return n_systems <= L->n_gain ? 0 : NSR_ERR_ARGUMENT;
  if (n_systems <= 0) return 0;
  int32_t* host = (int32_t*)malloc(sizeof(int32_t) * (size_t)n_systems);
  if (!host) return (int)cudaErrorMemoryAllocation;
  cudaError_t ce = cudaMemcpyAsync(host, L->gain_index, sizeof(int32_t) * (size_t)n_systems, cudaMemcpyDeviceToHost, st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  int err = ce == cudaSuccess ? 0 : (int)ce;
  for (int s = 0; !err && s < n_systems; ++s)
    if (host[s] < 0 || host[s] >= L->n_gain) err = NSR_ERR_ARGUMENT;
  free(host);
  return err;
}

// ---------------------------------------------------------------------------
// Learned apply: rows (pre gain) -> columns (learned multiplier) -> rows (post gain).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lp_gidx(const int* gain_index, int s) { return gain_index ? gain_index[s] : s; }

__global__ void __launch_bounds__(256) k_lp_rows_fwd(Geo g, PrecTables t, const float2* __restrict__ x,
                                                     float2* __restrict__ w, int rows, const float2* gains,
                                                     const int* gain_index, int adjoint) {
  extern __shared__ float2 sm[];
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * rows;
  const int nr = min(rows, g.nz - z0);
  const long long off = (long long)z0 * g.nx;
  const float2* xs = x + blockIdx.y * n + off;
  const GainPair G = gain_pair(gains, gains ? lp_gidx(gain_index, blockIdx.y) : 0, n, adjoint);
  const int rs = nsr_row_stride(g.nx);
  const bool pad = nsr_row_padded(g.nx);
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    const float2 v = xs[k];
    sm[l * rs + (pad ? c + (c >> 4) : c)] = G.pre ? gain_mul(G.pre, off + k, G.conj, v) : v;
  }
  __syncthreads();
  fft_rows<false>(sm, nr, t.px);
  float2* ws = w + blockIdx.y * n + off;
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    ws[k] = sm[l * rs + (pad ? c + (c >> 4) : c)];
  }
}

template <int TC>
__global__ void __launch_bounds__(512) k_lp_cols(Geo g, PrecTables t, const double* __restrict__ freq,
                                                 float2* __restrict__ w, const float* __restrict__ lp, int adjoint) {
  extern __shared__ float2 sm[];
  const long long n = (long long)g.nz * g.nx;
  cols_pass<TC>(sm, g, t, w + blockIdx.y * n, freq[blockIdx.y], 0.0, adjoint, blockIdx.x * TC, lp);
}

__global__ void __launch_bounds__(256) k_lp_rows_inv(Geo g, PrecTables t, const float2* __restrict__ w,
                                                     float2* __restrict__ y, int rows, const float2* gains,
                                                     const int* gain_index, int adjoint) {
  extern __shared__ float2 sm[];
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.x * rows;
  const int nr = min(rows, g.nz - z0);
  const long long off = (long long)z0 * g.nx;
  const float2* ws = w + blockIdx.y * n + off;
  const GainPair G = gain_pair(gains, gains ? lp_gidx(gain_index, blockIdx.y) : 0, n, adjoint);
  const int rs = nsr_row_stride(g.nx);
  const bool pad = nsr_row_padded(g.nx);
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    sm[l * rs + (pad ? c + (c >> 4) : c)] = ws[k];
  }
  __syncthreads();
  fft_rows<true>(sm, nr, t.px);
  __syncthreads();
  float2* ys = y + blockIdx.y * n + off;
  for (int k = threadIdx.x; k < nr * g.nx; k += blockDim.x) {
    const int l = k / g.nx, c = k - l * g.nx;
    const float2 v = sm[l * rs + (pad ? c + (c >> 4) : c)];
    ys[k] = G.post ? gain_mul(G.post, off + k, G.conj, v) : v;
  }
}

extern "C" int nsr_learned_precondition(const NsrGrid* grid, const NsrLearned* learned, const double* freq_hz,
                                        int32_t n_systems, int32_t adjoint, const float* x, float* y,
                                        void* workspace, size_t workspace_bytes, void* stream) {
  int err = nsr_check_grid(grid, true);
  if (err) return err;
  if (!learned || !learned->params || !freq_hz || !x || !y || !workspace || n_systems < 0 || n_systems > 65535)
    return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  if (workspace_bytes < nsr_precondition_workspace_size(grid, n_systems)) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  err = nsr_check_learned(learned, n_systems, st);
  if (err) return err;
  PrecTables t;
  err = nsr_prec_setup(grid, &t, workspace, st);
  if (err) return err;
  float2* w = (float2*)((char*)workspace + nsr_prec_table_bytes(grid));
  Geo g = make_geo(*grid);
  const int rows = nsr_rows_per_cta(grid);
  const size_t row_smem = sizeof(float2) * (size_t)rows * nsr_row_stride(grid->nx);
  const dim3 gr((grid->nz + rows - 1) / rows, n_systems);
  const float2* gains = (const float2*)learned->gains;
  k_lp_rows_fwd<<<gr, 256, row_smem, st>>>(g, t, (const float2*)x, w, rows, gains, learned->gain_index, adjoint);
  const int tc = nsr_cols_tc(grid);
  const dim3 gc((grid->nx + tc - 1) / tc, n_systems);
  const size_t csm = nsr_cols_smem(grid);
  if (tc == 16) {
    cudaFuncSetAttribute(k_lp_cols<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    k_lp_cols<16><<<gc, 512, csm, st>>>(g, t, freq_hz, w, learned->params, adjoint);
  } else {
    cudaFuncSetAttribute(k_lp_cols<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csm);
    k_lp_cols<8><<<gc, 512, csm, st>>>(g, t, freq_hz, w, learned->params, adjoint);
  }
  k_lp_rows_inv<<<gr, 256, row_smem, st>>>(g, t, w, (float2*)y, rows, gains, learned->gain_index, adjoint);
  return last_error();
}

// ---------------------------------------------------------------------------
// Training: gain cotangents -> low-resolution map cotangents.
// ---------------------------------------------------------------------------
// d m0 = (1 - t0^2) Re(conj(Gi) e^{-i phi1}), d m1 = (1 - t1^2) Im(conj(Gi) inner),
// likewise m2, m3 with the outer gain; Gi = dL/d conj(inner) (the cotangent
// convention dL = 2 Re sum conj(G) d(gain)).
template <typename T>
__global__ void k_lp_dmaps(int nz, int nx, int h8, int w8, const T* __restrict__ state,
                           const float2* __restrict__ g_inner, const float2* __restrict__ g_outer,
                           float* __restrict__ dm) {
  const long long n = (long long)nz * nx;
  const int hw = h8 * w8;
  const int f = blockIdx.y;
  const T* maps = state + (long long)f * LP_PLANES * hw + LP_MAPS * hw;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k / nx), j = (int)(k - (long long)i * nx);
    float m[4];
    node_maps(maps, hw, w8, lerp_of(i, h8, nz), lerp_of(j, w8, nx), m);
    const float t0 = tanhf(m[0]), t1 = tanhf(m[1]), t2 = tanhf(m[2]), t3 = tanhf(m[3]);
    float s1, c1, s3, c3;
    sincosf(0.5f * t1, &s1, &c1);
    sincosf(0.5f * t3, &s3, &c3);
    const float2 gi = g_inner[(long long)f * n + k], go = g_outer[(long long)f * n + k];
    const float2 e1 = make_float2(c1, -s1), e3 = make_float2(c3, -s3);
    const float g0 = 1.0f + 0.5f * t0, g2 = 1.0f + 0.5f * t2;
    // conj(G) * e
    const float re1 = gi.x * e1.x + gi.y * e1.y, im1 = gi.x * e1.y - gi.y * e1.x;
    const float re3 = go.x * e3.x + go.y * e3.y, im3 = go.x * e3.y - go.y * e3.x;
    float* out = dm + (long long)f * 4 * n;
    out[k] = (1.0f - t0 * t0) * re1;
    out[n + k] = (1.0f - t1 * t1) * g0 * im1;
    out[2 * n + k] = (1.0f - t2 * t2) * re3;
    out[3 * n + k] = (1.0f - t3 * t3) * g2 * im3;
  }
}

// Transposed bilinear upsampling, one thread per (frequency, channel, pixel),
// gathering the nodes whose interpolation touches the pixel (deterministic).
__global__ void k_lp_upsample_adjoint(int nz, int nx, int h8, int w8, const float* __restrict__ dm,
                                      float* __restrict__ d_maps) {
  const int hw = h8 * w8;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 4 * hw) return;
  const int f = blockIdx.y;
  const int c = q / hw, p = q - c * hw;
  const int py = p / w8, px = p - py * w8;
  const long long n = (long long)nz * nx;
  const float sz = (float)h8 / (float)nz, sx = (float)w8 / (float)nx;
  const int zlo = max(0, (int)floorf(((float)py - 0.5f) / sz - 0.5f) - 2);
  const int zhi = py == h8 - 1 ? nz - 1 : min(nz - 1, (int)ceilf(((float)py + 1.5f) / sz - 0.5f) + 2);
  const int xlo = max(0, (int)floorf(((float)px - 0.5f) / sx - 0.5f) - 2);
  const int xhi = px == w8 - 1 ? nx - 1 : min(nx - 1, (int)ceilf(((float)px + 1.5f) / sx - 0.5f) + 2);
  const float* src = dm + ((long long)f * 4 + c) * n;
  double acc = 0.0;
  for (int i = zlo; i <= zhi; ++i) {
    const float wz = lerp_weight(lerp_of(i, h8, nz), py);
    if (wz == 0.0f) continue;
    double row = 0.0;
    for (int j = xlo; j <= xhi; ++j) {
      const float wx = lerp_weight(lerp_of(j, w8, nx), px);
      if (wx != 0.0f) row += (double)wx * src[(long long)i * nx + j];
    }
    acc += (double)wz * row;
  }
  d_maps[(long long)f * 4 * hw + q] = (float)acc;
}

extern "C" size_t nsr_learned_backward_workspace_size(const NsrGrid* grid, int32_t n_freq) {
  if (nsr_check_grid(grid, false) || n_freq <= 0) return 0;
  const size_t n = (size_t)grid->nz * grid->nx;
  const size_t hw = (size_t)lp_h(grid) * lp_w(grid);
  const size_t a = 4 * n, b = 32 * hw;
  return nsr_align(sizeof(float) * (a > b ? a : b) * n_freq);
}

extern "C" int nsr_learned_map_backward_ex(const NsrGrid* grid, const void* state, int32_t precision, int32_t n_freq,
                                           const float* g_inner, const float* g_outer, float* d_maps,
                                           void* workspace, size_t workspace_bytes, void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!state || !g_inner || !g_outer || !d_maps || !workspace || n_freq < 0 || n_freq > 65535) return NSR_ERR_ARGUMENT;
  if (precision != NSR_LEARNED_FP32 && precision != NSR_LEARNED_BF16) return NSR_ERR_ARGUMENT;
  if (n_freq == 0) return 0;
  if (workspace_bytes < nsr_learned_backward_workspace_size(grid, n_freq)) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int h8 = lp_h(grid), w8 = lp_w(grid), hw = h8 * w8;
  const long long n = (long long)grid->nz * grid->nx;
  int bx = (int)((n + 255) / 256);
  if (bx > 1184) bx = 1184;
  float* dm = (float*)workspace;
  if (precision == NSR_LEARNED_BF16)
    k_lp_dmaps<__nv_bfloat16><<<dim3(bx, n_freq), 256, 0, st>>>(grid->nz, grid->nx, h8, w8,
                                                                (const __nv_bfloat16*)state, (const float2*)g_inner,
                                                                (const float2*)g_outer, dm);
  else
    k_lp_dmaps<float><<<dim3(bx, n_freq), 256, 0, st>>>(grid->nz, grid->nx, h8, w8, (const float*)state,
                                                        (const float2*)g_inner, (const float2*)g_outer, dm);
  k_lp_upsample_adjoint<<<dim3((4 * hw + 127) / 128, n_freq), 128, 0, st>>>(grid->nz, grid->nx, h8, w8, dm, d_maps);
  return last_error();
}

extern "C" int nsr_learned_map_backward(const NsrGrid* grid, const void* state, int32_t n_freq, const float* g_inner,
                                        const float* g_outer, float* d_maps, void* workspace,
                                        size_t workspace_bytes, void* stream) {
  return nsr_learned_map_backward_ex(grid, state, NSR_LEARNED_FP32, n_freq, g_inner, g_outer, d_maps, workspace,
                                     workspace_bytes, stream);
}

// ---------------------------------------------------------------------------
// Training: backward through the three convolutions.
// ---------------------------------------------------------------------------
// d_in[ci] = (sum_co sum_k W[co][ci][k] dz[co][p - k]) * (1 - a[ci]^2)
template <typename T, int CIN, int COUT>
__global__ void __launch_bounds__(128) k_lp_conv_bwd_data(int h8, int w8, const float* __restrict__ wt,
                                                          const float* __restrict__ dz, int dz_stride,
                                                          const T* __restrict__ state, int act_plane,
                                                          float* __restrict__ din, int din_stride) {
  __shared__ float sw[COUT * CIN * 9];
  for (int k = threadIdx.x; k < COUT * CIN * 9; k += blockDim.x) sw[k] = wround<T>(wt[k]);
  __syncthreads();
  const int hw = h8 * w8;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= hw) return;
  const int f = blockIdx.y;
  const int y = p / w8, x = p - y * w8;
  const float* g = dz + (long long)f * dz_stride;
  const T* act = state + (long long)f * LP_PLANES * hw + act_plane * hw;
  float acc[CIN];
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.0f;
  for (int co = 0; co < COUT; ++co)
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      const int yy = y - ky + 1;
      if (yy < 0 || yy >= h8) continue;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int xx = x - kx + 1;
        if (xx < 0 || xx >= w8) continue;
        const float v = g[co * hw + yy * w8 + xx];
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) acc[ci] += sw[((co * CIN + ci) * 3 + ky) * 3 + kx] * v;
      }
    }
  float* out = din + (long long)f * din_stride;
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) {
    const float a = ld(act + ci * hw + p);
    out[ci * hw + p] = acc[ci] * (1.0f - a * a);
  }
}

// dW[co][ci][k] += sum_{f,p} dz[co][p] in[ci][p + k];  db[co] += sum dz[co][p].
// One CTA per (co, ci); a fixed-order block reduction keeps it deterministic.
template <typename T, int CIN, int COUT>
__global__ void __launch_bounds__(256) k_lp_conv_bwd_weight(int h8, int w8, int n_freq, const float* __restrict__ dz,
                                                            int dz_stride, const T* __restrict__ state,
                                                            int in_plane, float* __restrict__ dw,
                                                            float* __restrict__ db) {
  const int co = blockIdx.x / CIN, ci = blockIdx.x - co * CIN;
  const int hw = h8 * w8;
  double acc[10];
#pragma unroll
  for (int q = 0; q < 10; ++q) acc[q] = 0.0;
  for (int f = 0; f < n_freq; ++f) {
    const float* g = dz + (long long)f * dz_stride + co * hw;
    const T* in = state + (long long)f * LP_PLANES * hw + (in_plane + ci) * hw;
    for (int p = threadIdx.x; p < hw; p += blockDim.x) {
      const int y = p / w8, x = p - y * w8;
      const float gv = g[p];
      acc[9] += gv;
#pragma unroll
      for (int ky = 0; ky < 3; ++ky) {
        const int yy = y + ky - 1;
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const int xx = x + kx - 1;
          if (yy >= 0 && yy < h8 && xx >= 0 && xx < w8) acc[ky * 3 + kx] += (double)gv * ld(in + yy * w8 + xx);
        }
      }
    }
  }
  __shared__ double wsum[8][10];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 10; ++q) {
    const double s = warp_sum(acc[q]);
    if (lane == 0) wsum[wid][q] = s;
  }
  __syncthreads();
  if (threadIdx.x < 10) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wsum[w][threadIdx.x];
    if (threadIdx.x < 9) dw[(co * CIN + ci) * 9 + threadIdx.x] += (float)s;
    else if (ci == 0) db[co] += (float)s;
  }
}

template <typename T>
static void network_backward_t(int h8, int w8, int n_freq, const float* params, const T* S, const float* d_maps,
                               float* d_params, float* dz2, float* dz1, cudaStream_t st) {
  const int hw = h8 * w8;
  const dim3 gp((hw + 127) / 128, n_freq);
  // layer 3 (no activation): dz3 = d_maps
  k_lp_conv_bwd_weight<T, 16, 4><<<64, 256, 0, st>>>(h8, w8, n_freq, d_maps, 4 * hw, S, LP_A2, d_params + LP_W3,
                                                      d_params + LP_B3);
  k_lp_conv_bwd_data<T, 16, 4><<<gp, 128, 0, st>>>(h8, w8, params + LP_W3, d_maps, 4 * hw, S, LP_A2, dz2, 16 * hw);
  k_lp_conv_bwd_weight<T, 16, 16><<<256, 256, 0, st>>>(h8, w8, n_freq, dz2, 16 * hw, S, LP_A1, d_params + LP_W2,
                                                        d_params + LP_B2);
  k_lp_conv_bwd_data<T, 16, 16><<<gp, 128, 0, st>>>(h8, w8, params + LP_W2, dz2, 16 * hw, S, LP_A1, dz1, 16 * hw);
  k_lp_conv_bwd_weight<T, 5, 16><<<80, 256, 0, st>>>(h8, w8, n_freq, dz1, 16 * hw, S, LP_POOL, d_params + LP_W1,
                                                      d_params + LP_B1);
}

extern "C" int nsr_learned_network_backward_ex(const NsrGrid* grid, const float* params, const void* state,
                                               int32_t precision, int32_t n_freq, const float* d_maps,
                                               float* d_params, void* workspace, size_t workspace_bytes,
                                               void* stream) {
  int err = nsr_check_grid(grid, false);
  if (err) return err;
  if (!params || !state || !d_maps || !d_params || !workspace || n_freq < 0 || n_freq > 65535) return NSR_ERR_ARGUMENT;
  if (precision != NSR_LEARNED_FP32 && precision != NSR_LEARNED_BF16) return NSR_ERR_ARGUMENT;
  if (n_freq == 0) return 0;
  if (workspace_bytes < nsr_learned_backward_workspace_size(grid, n_freq)) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  const int h8 = lp_h(grid), w8 = lp_w(grid), hw = h8 * w8;
  float* dz2 = (float*)workspace;              // [f][16][hw]
  float* dz1 = dz2 + (size_t)16 * hw * n_freq; // [f][16][hw]
  if (precision == NSR_LEARNED_BF16)
    network_backward_t(h8, w8, n_freq, params, (const __nv_bfloat16*)state, d_maps, d_params, dz2, dz1, st);
  else
    network_backward_t(h8, w8, n_freq, params, (const float*)state, d_maps, d_params, dz2, dz1, st);
  return last_error();
}

extern "C" int nsr_learned_network_backward(const NsrGrid* grid, const float* params, const void* state,
                                            int32_t n_freq, const float* d_maps, float* d_params, void* workspace,
                                            size_t workspace_bytes, void* stream) {
  return nsr_learned_network_backward_ex(grid, params, state, NSR_LEARNED_FP32, n_freq, d_maps, d_params, workspace,
                                         workspace_bytes, stream);
}

// ---------------------------------------------------------------------------
// Training: spectral parameters.
// ---------------------------------------------------------------------------
// For z = outer * F^-1(m * F(u)), u = inner * r and Y = conj(outer) * dL/d conj(z),
//   dL/dtheta = 2 Re sum_q (1/N) conj(Y^(q)) u^(q) dm(q)/dtheta
// with ^ the unnormalised DFT.  P = conj(Y^) u^ m / N gives
//   dL/dmod0 = Re(P) (1 - t0^2),  dL/dmod1 = Im(P) (1 - t1^2),
//   dL/ds    = 2 Re(P (-i (k0h)^2) / D),
// and mod_c = sum_k spectral[c][k] basis_k, s = clamp(exp(log_shift), .01, 1).
template <int TC>
__global__ void __launch_bounds__(512) k_lp_spec_grad(Geo g, PrecTables t, const double* __restrict__ freq,
                                                      const float2* __restrict__ xr, const float2* __restrict__ yr,
                                                      const float* __restrict__ lp, double* __restrict__ partials) {
  extern __shared__ float2 sm[];
  float2* sa = sm;
  float2* sb = sm + g.nz * TC;
  const long long n = (long long)g.nz * g.nx;
  const int c0 = blockIdx.x * TC;
  const int ncol = min(TC, g.nx - c0);
  const float2* xs = xr + blockIdx.y * n;
  const float2* ys = yr + blockIdx.y * n;
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    sa[k] = c < ncol ? xs[(long long)z * g.nx + c0 + c] : make_float2(0.f, 0.f);
    sb[k] = c < ncol ? ys[(long long)z * g.nx + c0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_cols<false, TC>(sa, t.pz);
  __syncthreads();
  fft_cols<false, TC>(sb, t.pz);
  __syncthreads();
  const SysScalars s = sys_scalars(g, freq[blockIdx.y]);
  const float kh2 = (float)s.kh2;
  const float h2 = (float)(g.h * g.h);
  const LearnedSpec L = load_learned_spec(lp);
  const float inv_n = 1.0f / (float)n;
  double acc[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) acc[q] = 0.0;
  for (int k = threadIdx.x; k < g.nz * TC; k += blockDim.x) {
    const int z = k / TC, c = k - z * TC;
    if (c >= ncol) continue;
    const float s2z = t.s2z[z], s2x = t.s2x[c0 + c];
    const float q2 = 4.0f * (s2z + s2x) / kh2;
    const float rq = q2 / (1.0f + q2);
    const float ang = 4.0f * s2x / (4.0f * (s2x + s2z) + h2);
    const float basis[4] = {1.0f, rq, ang, ang * rq};
    const float mod0 = L.sp[0] + L.sp[1] * rq + L.sp[2] * ang + L.sp[3] * ang * rq;
    const float mod1 = L.sp[4] + L.sp[5] * rq + L.sp[6] * ang + L.sp[7] * ang * rq;
    const float t0 = tanhf(mod0), t1 = tanhf(mod1);
    const float mag = expf(0.5f * t0);
    float sn, cs;
    sincosf(0.5f * t1, &sn, &cs);
    const float sym = -4.0f * (s2z + s2x);
    const float2 D = make_float2(sym + kh2, kh2 * L.shift);
    const float2 m = divc(make_float2(mag * cs, -mag * sn), D);
    const float2 a = sa[k], b = sb[k];
    const float2 cb_a = make_float2(b.x * a.x + b.y * a.y, b.x * a.y - b.y * a.x);   // conj(b) a
    const float2 P = inv_n * (cb_a * m);
    const float dmod0 = P.x * (1.0f - t0 * t0);
    const float dmod1 = P.y * (1.0f - t1 * t1);
    const float2 dsd = divc(make_float2(0.f, -kh2), D);   // -i kh2 / D
    const float ds = 2.0f * (P.x * dsd.x - P.y * dsd.y);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      acc[q] += (double)dmod0 * basis[q];
      acc[4 + q] += (double)dmod1 * basis[q];
    }
    acc[8] += ds;
  }
  __shared__ double wsum[16][9];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) wsum[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += wsum[w][threadIdx.x];
    partials[((long long)blockIdx.y * gridDim.x + blockIdx.x) * 9 + threadIdx.x] = v;
  }
}

// Sum the per-CTA partials in order and add them to d_params[0..8].
__global__ void k_lp_spec_sum(int count, const double* __restrict__ partials, const float* __restrict__ lp,
                              float* __restrict__ d_params) {
  const int q = threadIdx.x;
  if (q >= 9) return;
  double v = 0.0;
  for (int b = 0; b < count; ++b) v += partials[(long long)b * 9 + q];
  if (q == 8) {
    const float e = expf(lp[8]);
    v = (e > 0.01f && e < 1.0f) ? v * e : 0.0;   // d s / d log_shift, zero where clamped
  }
  d_params[q] += (float)v;
}

static int spec_tc(const NsrGrid* g) { return g->nz <= 768 ? 16 : 8; }

extern "C" size_t nsr_learned_spectral_workspace_size(const NsrGrid* grid, int32_t n_systems) {
  if (nsr_check_grid(grid, true) || n_systems <= 0 || n_systems > 65535) return 0;
  const int tc = spec_tc(grid);
  if (sizeof(float2) * 2 * (size_t)grid->nz * tc > 227 * 1024) return 0;
  const size_t n = (size_t)grid->nz * grid->nx;
  const size_t nb = (size_t)(grid->nx + tc - 1) / tc;
  return nsr_align(nsr_prec_table_bytes(grid)) + 2 * nsr_align(sizeof(float2) * n * n_systems) +
         nsr_align(sizeof(double) * 9 * nb * n_systems);
}

extern "C" int nsr_learned_spectral_backward(const NsrGrid* grid, const float* params, const double* freq_hz,
                                             int32_t n_systems, const float* x, const float* y, float* d_params,
                                             void* workspace, size_t workspace_bytes, void* stream) {
  int err = nsr_check_grid(grid, true);
  if (err) return err;
  if (!params || !freq_hz || !x || !y || !d_params || !workspace || n_systems < 0 || n_systems > 65535)
    return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  const size_t need = nsr_learned_spectral_workspace_size(grid, n_systems);
  if (need == 0) return NSR_ERR_UNSUPPORTED_SIZE;
  if (workspace_bytes < need) return NSR_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)workspace;
  PrecTables t;
  err = nsr_prec_setup(grid, &t, ws, st);
  if (err) return err;
  const size_t n = (size_t)grid->nz * grid->nx;
  float2* xr = (float2*)(ws + nsr_align(nsr_prec_table_bytes(grid)));
  float2* yr = (float2*)((char*)xr + nsr_align(sizeof(float2) * n * n_systems));
  double* partials = (double*)((char*)yr + nsr_align(sizeof(float2) * n * n_systems));
  Geo g = make_geo(*grid);
  const int rows = nsr_rows_per_cta(grid);
  const size_t row_smem = sizeof(float2) * (size_t)rows * nsr_row_stride(grid->nx);
  const dim3 gr((grid->nz + rows - 1) / rows, n_systems);
  k_lp_rows_fwd<<<gr, 256, row_smem, st>>>(g, t, (const float2*)x, xr, rows, nullptr, nullptr, 0);
  k_lp_rows_fwd<<<gr, 256, row_smem, st>>>(g, t, (const float2*)y, yr, rows, nullptr, nullptr, 0);
  const int tc = spec_tc(grid);
  const int nb = (grid->nx + tc - 1) / tc;
  const size_t smem = sizeof(float2) * 2 * (size_t)grid->nz * tc;
  const dim3 gc(nb, n_systems);
  if (tc == 16) {
    cudaFuncSetAttribute(k_lp_spec_grad<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lp_spec_grad<16><<<gc, 512, smem, st>>>(g, t, freq_hz, xr, yr, params, partials);
  } else {
    cudaFuncSetAttribute(k_lp_spec_grad<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_lp_spec_grad<8><<<gc, 512, smem, st>>>(g, t, freq_hz, xr, yr, params, partials);
  }
  k_lp_spec_sum<<<1, 32, 0, st>>>(nb * n_systems, partials, params, d_params);
  return last_error();
}

// ---------------------------------------------------------------------------
// Training: clipped Adam step (torch.optim.Adam semantics with
// clip_grad_norm_, as nsrno/train_dense_wave.py:37,72-76 uses them).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_lp_adam(float* __restrict__ p, const float* __restrict__ grad,
                                                  float* __restrict__ m, float* __restrict__ v, int n, int step,
                                                  float lr, float b1, float b2, float eps, float clip,
                                                  float* __restrict__ norm_out) {
  __shared__ double wsum[32];
  __shared__ float scale;
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc += (double)grad[k] * grad[k];
  const double s = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += wsum[w];
    const float norm = (float)sqrt(tot);
    float sc = 1.0f;
    if (clip > 0.0f) {
      const float coef = clip / (norm + 1e-6f);
      sc = coef < 1.0f ? coef : 1.0f;
    }
    scale = sc;
    if (norm_out) *norm_out = norm;
  }
  __syncthreads();
  const float bc1 = 1.0f - powf(b1, (float)step);
  const float bc2 = 1.0f - powf(b2, (float)step);
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const float gk = grad[k] * scale;
    const float mk = b1 * m[k] + (1.0f - b1) * gk;
    const float vk = b2 * v[k] + (1.0f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= (lr / bc1) * mk / (sqrtf(vk) / sqrtf(bc2) + eps);
  }
}

extern "C" int nsr_learned_adam(float* params, const float* grad, float* m, float* v, int32_t n, int32_t step,
                                double lr, double beta1, double beta2, double eps, double clip_norm,
                                float* grad_norm, void* stream) {
  if (!params || !grad || !m || !v || n <= 0 || step <= 0 || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) ||
      !(beta2 >= 0 && beta2 < 1) || !(eps > 0))
    return NSR_ERR_ARGUMENT;
  k_lp_adam<<<1, 1024, 0, (cudaStream_t)stream>>>(params, grad, m, v, n, step, (float)lr, (float)beta1, (float)beta2,
                                                   (float)eps, (float)clip_norm, grad_norm);
  return last_error();
}
