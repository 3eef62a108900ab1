// Batched right-preconditioned BiCGSTAB for the 5-point Helmholtz systems of a
// record.  Design:
//   * n_slots systems are resident; a device-side queue refills a slot when
//     its system finishes (converged, budget, breakdown, divergence).
//   * One BiCGSTAB iteration = two halves; each half is four launches:
//       fwd  : elementwise Krylov update fused with the forward row FFT,
//       cols : column FFT, shifted-Laplace multiply, inverse column FFT,
//       rinv : inverse row FFT in place (z = M^-1 of the half's vector),
//       inv  : 5-point stencil on z (register sliding window down a column
//              strip) fused with the FP64 inner products of that half;
//     the second half adds `res`, the FP64 true residual of the slots that
//     replace their residual, start or emit.
//     The last CTA of a slot (arrival counter, no waiting) sums the per-CTA
//     partials in a fixed order and advances that slot's scalar recurrence,
//     so no host synchronisation happens inside the loop.
//   * The update of x is deferred: y accumulates alpha p + omega s and
//     x += M^-1 y is applied at every true-residual replacement, where
//     r = b - A x is recomputed in FP64 from an FP64 x.
//   * The host captures `graph_iterations` iterations in a CUDA graph and
//     relaunches it, polling a completion counter.
// Algorithmic reference: bicgstab, nsrno/dense_wave.py:118-148 (right
// preconditioned, shared-angle inner products, true residual every 40
// iterations, breakdown/divergence reasons) and the fixed preconditioner of
// nsrno/dense_wave.py:194-196.
#include "nsr_internal.cuh"
#include "nsr_device.cuh"
#include "nsr_tma.cuh"

#include <stdio.h>
#include <stdlib.h>
#include <type_traits>
#include <string.h>

enum { MODE_EMPTY = 0, MODE_INIT = 1, MODE_ITER_A = 2, MODE_ITER_B = 3, MODE_RES = 4, MODE_EMIT = 5 };

#define NSR_LAUNCHES_PER_IT 9
#define NSR_MAX_GROUPS 4        // slot groups on parallel graph branches
#define NSR_ST_TZ 32      // rows of one stencil CTA
#define NSR_ST_TX 512     // columns of one stencil CTA (two per thread; even nx)
#define NSR_ST_TX1 256    // columns of one stencil CTA of k_inv1 (one per thread; odd nx)

struct __align__(16) SlotState {
  int sys, mode, iters, final_reason;
  int xpar, zero_rhs, restart, force_restart;
  int breakdowns;   // consecutive restarts forced by a breakdown
  int x0_off;       // the initial field was rejected: start from zero
  int gidx;         // gain pair of the learned preconditioner
  int pad_b2;
  unsigned long long t_start;   // global timer (ns) when the system started
  double bnorm2, rnorm2, resid, r0norm2;
  double freq, angle;
  float kh2f, sigf, fpowf, pad_f;   // per-system stencil scalars in float (set when the slot starts)
  double2 rho, alpha, omega, beta;
  // s = r + c_sv v ; r_new = s + c_rt t ; y += c_yp p + c_ys s ; p_new = r_new + c_pp p + c_pv v
  double2 c_sv, c_rt, c_yp, c_ys, c_pp, c_pv;
};

struct SolveBufs {
  SlotState* slots;
  int* arrive;        // [n_slots]
  int* queue;         // next system to start
  int* done;          // systems finished
  int* warm;          // [2]: initial fields accepted, rejected
  int* error;         // set by a kernel that gave up waiting on its copy ring
  double* partials;   // [n_slots][nb_inv][NSR_NPART]
  float2 *r, *rh, *p, *v, *t, *y, *w;   // [n_slots][n]
  float2* sym;        // [n_slots][n] learned multiplier of the slot's system (learned solves only)
  double2* x;         // [n_slots][2][n]
};

struct SolveArgs {
  Geo g;
  PrecTables tab;
  SolveBufs B;
  MatPlanes mat;
  const double* freq;
  const double* angle;
  const float2* rhs;
  const float2* x0;
  const int* rx;
  int n_rx;
  int n_systems;
  int rows;      // rows per fwd CTA
  int tc;        // columns per cols CTA
  int tz;        // band rows per inv CTA
  int nb_inv;    // inv CTAs per slot
  double tol2;
  double shift;
  double restart2;   // squared restart factor
  double warm_gate2; // squared acceptance bound of an initial field's relative residual (0: none)
  int max_it;
  int replace_every;
  int adjoint;
  unsigned long long time_limit_ns;   // per-system wall-clock limit (0: none)
  double2* iq;
  double* residual;
  int* iterations;
  int* status;
  void* fields;     // float2 or double2 [S][n]
  int fields_fp64;
  // Learned preconditioner (all null: the fixed shifted-Laplace one).
  const float* lp;        // parameters (spectral multiplier)
  const float2* gains;    // [n_gain][2][n]
  const int* gain_index;  // [n_systems] (null: system s uses pair s)
  int slot0;              // first slot of the launch's slot group
};

// Which slots a launch serves.  The first half of an iteration runs only the
// ITER_A work; the second half runs ITER_B and every FP64 residual, start and
// emit pass.  A mode written by a finalize therefore never becomes active in
// the half that wrote it.
__device__ __forceinline__ bool fwd_active(int mode, int half) {
  return half == 0 ? mode == MODE_ITER_A
                   : (mode == MODE_ITER_B || mode == MODE_RES || mode == MODE_INIT || mode == MODE_EMIT);
}
__device__ __forceinline__ bool cols_active(int mode, int half) {
  return half == 0 ? mode == MODE_ITER_A : (mode == MODE_ITER_B || mode == MODE_RES);
}

__device__ __forceinline__ float2 f2(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ bool finite2(double2 a) { return isfinite(a.x) && isfinite(a.y); }
__device__ __forceinline__ double abs2(double2 a) { return a.x * a.x + a.y * a.y; }

// The staged row pass of k_fwd: the updated tile is written to padded shared
// rows, transformed there and copied to w.
__device__ __forceinline__ void fwd_staged(const SolveArgs& A, const SlotState& S, const GainPair& G, float2* sm,
                                           int mode, int nr, long long off, long long goff, int cnt, float2 sv,
                                           float2 rt, float2 yp, float2 ys, float2 pp, float2 pv) {
  const Geo& g = A.g;
  float2 *r = A.B.r + off, *p = A.B.p + off, *v = A.B.v + off, *t = A.B.t + off, *y = A.B.y + off;
  // The tile's rows are contiguous in HBM, so one flat index k = l*nx + c runs
  // over them.  The padded row layout puts (l, c) at l*(nx + nx/16) + c + c/16,
  // which equals k + k/16 because every padded width is a multiple of 16.
  const bool pad = nsr_row_padded(g.nx);
  float2* __restrict__ rr_ = r;
  float2* __restrict__ pp_ = p;
  float2* __restrict__ yy_ = y;
  const float2* __restrict__ vv_ = v;
  const float2* __restrict__ tt_ = t;
  if (mode == MODE_ITER_A) {
    const bool restart = S.restart != 0;
    float2* __restrict__ rh = A.B.rh + off;
#pragma unroll 4
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      const float2 rk = rr_[k], vk = vv_[k], tk = tt_[k], pk = pp_[k], yk = yy_[k];
      const float2 s1 = rk + sv * vk;
      const float2 rn = s1 + rt * tk;
      const float2 yn = yk + yp * pk + ys * s1;
      const float2 pn = rn + pp * pk + pv * vk;
      rr_[k] = rn; pp_[k] = pn; yy_[k] = yn;
      if (restart) rh[k] = rn;
      sm[pad ? k + (k >> 4) : k] = G.pre ? gain_mul(G.pre, goff + k, G.conj, pn) : pn;
    }
  } else if (mode == MODE_ITER_B) {
#pragma unroll 8
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      const float2 s1 = rr_[k] + sv * vv_[k];
      sm[pad ? k + (k >> 4) : k] = G.pre ? gain_mul(G.pre, goff + k, G.conj, s1) : s1;
    }
  } else {  // MODE_RES: apply the pending update to y, transform y, clear it
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
      const float2 s1 = rr_[k] + sv * vv_[k];
      const float2 yn = yy_[k] + yp * pp_[k] + ys * s1;
      sm[pad ? k + (k >> 4) : k] = G.pre ? gain_mul(G.pre, goff + k, G.conj, yn) : yn;
      yy_[k] = make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  fft_rows<false>(sm, nr, A.tab.px);
  float2* __restrict__ w = A.B.w + off;
#pragma unroll 8
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) w[k] = sm[pad ? k + (k >> 4) : k];
}

// ---------------------------------------------------------------------------
// fwd: elementwise update + forward row FFT into w.  DIRECT (row widths
// 256 ... 2048 of the form 2^a 3^b): the update runs inside the transform's
// first stage and its last stage writes w straight from registers
// (ct_rows_forward_direct); otherwise the updated tile is staged in shared
// memory first.
// ---------------------------------------------------------------------------
template <bool DIRECT>
__global__ void __launch_bounds__(256, 4) k_fwd(SolveArgs A, int half) {
  extern __shared__ float2 sm[];
  const int slot = A.slot0 + blockIdx.x;
  const SlotState& S = A.B.slots[slot];
  const int mode = S.mode;
  if (!fwd_active(mode, half)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.y * A.rows;
  const int nr = min(A.rows, g.nz - z0);
  const long long off = slot * n + (long long)z0 * g.nx;
  const int cnt = nr * g.nx;
  float2 *r = A.B.r + off, *p = A.B.p + off, *v = A.B.v + off, *t = A.B.t + off, *y = A.B.y + off;
  if (mode == MODE_INIT) {
    const float2 z = make_float2(0.f, 0.f);
    for (int k = threadIdx.x; k < cnt; k += blockDim.x) { p[k] = z; v[k] = z; t[k] = z; y[k] = z; }
    if (A.lp) {
      // The learned Fourier multiplier depends on the system's frequency only:
      // evaluate it once per system, in the digit-reversed (z, x) order of the
      // transformed field, for k_cols to read.
      const LearnedSpec L = load_learned_spec(A.lp);
      const float kh2 = (float)sys_scalars(g, S.freq).kh2;
      float2* __restrict__ sym = A.B.sym + off;
      for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
        const int l = k / g.nx;
        sym[k] = learned_plane_value(L, g, A.tab, kh2, z0 + l, k - l * g.nx);
      }
    }
    return;
  }
  if (mode == MODE_EMIT) {
    if (A.fields && S.sys >= 0) {
      const double2* x = A.B.x + (2LL * slot + S.xpar) * n + (long long)z0 * g.nx;
      if (A.fields_fp64) {
        double2* f = (double2*)A.fields + (long long)S.sys * n + (long long)z0 * g.nx;
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) f[k] = S.zero_rhs ? make_double2(0.0, 0.0) : x[k];
      } else {
        float2* f = (float2*)A.fields + (long long)S.sys * n + (long long)z0 * g.nx;
        for (int k = threadIdx.x; k < cnt; k += blockDim.x) f[k] = S.zero_rhs ? make_float2(0.f, 0.f) : f2(x[k]);
      }
    }
    return;
  }
  const float2 sv = f2(S.c_sv), rt = f2(S.c_rt), yp = f2(S.c_yp), ys = f2(S.c_ys), pp = f2(S.c_pp), pv = f2(S.c_pv);
  const GainPair G = gain_pair(A.gains, S.gidx, n, A.adjoint);
  const long long goff = (long long)z0 * g.nx;   // node index of this tile's first element
  float2* __restrict__ rr_ = r;
  float2* __restrict__ pp_ = p;
  float2* __restrict__ yy_ = y;
  const float2* __restrict__ vv_ = v;
  const float2* __restrict__ tt_ = t;
  if constexpr (DIRECT) {
    const bool restart = S.restart != 0;
    float2* __restrict__ rh = A.B.rh + off;
    // Values of one stage-0 butterfly: elements k0 + q*step, q < R.  The
    // loads of up to four elements are issued together (two for the radix-8
    // and radix-16 first stages, whose results already hold 16-32 registers).
    auto in = [&](auto tag, int k0, int step, float2* out) {
      constexpr int R = decltype(tag)::value;
      constexpr int CH = R <= 4 ? R : 2;
      if (mode == MODE_ITER_A) {
#pragma unroll
        for (int c = 0; c < R; c += CH) {
          float2 rk[CH], vk[CH], tk[CH], pk[CH], yk[CH];
#pragma unroll
          for (int q = 0; q < CH; ++q) {
            const int k = k0 + (c + q) * step;
            rk[q] = rr_[k]; vk[q] = vv_[k]; tk[q] = tt_[k]; pk[q] = pp_[k]; yk[q] = yy_[k];
          }
#pragma unroll
          for (int q = 0; q < CH; ++q) {
            const int k = k0 + (c + q) * step;
            const float2 s1 = rk[q] + sv * vk[q];
            const float2 rn = s1 + rt * tk[q];
            const float2 yn = yk[q] + yp * pk[q] + ys * s1;
            const float2 pn = rn + pp * pk[q] + pv * vk[q];
            rr_[k] = rn; pp_[k] = pn; yy_[k] = yn;
            if (restart) rh[k] = rn;
            out[c + q] = pn;
          }
        }
      } else if (mode == MODE_ITER_B) {
        float2 rk[R], vk[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int k = k0 + q * step;
          rk[q] = rr_[k]; vk[q] = vv_[k];
        }
#pragma unroll
        for (int q = 0; q < R; ++q) out[q] = rk[q] + sv * vk[q];
      } else {  // MODE_RES: apply the pending update to y, transform y, clear it
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int k = k0 + q * step;
          const float2 s1 = rr_[k] + sv * vv_[k];
          out[q] = yy_[k] + yp * pp_[k] + ys * s1;
          yy_[k] = make_float2(0.f, 0.f);
        }
      }
      if (G.pre) {
#pragma unroll
        for (int q = 0; q < R; ++q) out[q] = gain_mul(G.pre, goff + k0 + q * step, G.conj, out[q]);
      }
    };
    fft_rows_forward_direct(sm, nr, A.tab.px, A.B.w + off, in);
  } else {
    fwd_staged(A, S, G, sm, mode, nr, off, goff, cnt, sv, rt, yp, ys, pp, pv);
  }
}

// ---------------------------------------------------------------------------
// cols: column FFT, preconditioner multiply, inverse column FFT (in place).
// ---------------------------------------------------------------------------
template <int TC, bool LEARNED, bool STAGED>
__global__ void __launch_bounds__(512, 2) k_cols(SolveArgs A, int half) {
  extern __shared__ float2 sm[];
  const int slot = A.slot0 + blockIdx.x;
  const int mode = A.B.slots[slot].mode;
  if (!cols_active(mode, half)) return;
  const long long n = (long long)A.g.nz * A.g.nx;
  const int c0 = blockIdx.y * TC;
  const Geo& g = A.g;
  const int adjoint = A.adjoint;
  if (LEARNED) {
    const float2* __restrict__ symp = A.B.sym + slot * n;
    cols_pass_direct<TC, STAGED>(sm, g, A.tab, A.B.w + slot * n, c0, [&](int c, int z) -> float2 {
      const float2 mul = symp[(long long)z * g.nx + c0 + c];
      return adjoint ? conjc(mul) : mul;
    });
  } else {
    const SysScalars s = sys_scalars(g, A.B.slots[slot].freq);
    const float inv_n = 1.0f / (float)n;
    const float2 shiftc = make_float2((float)s.kh2, (float)(s.kh2 * A.shift));
    const PrecTables& tab = A.tab;
    cols_pass_direct<TC, STAGED>(sm, g, tab, A.B.w + slot * n, c0, [&](int c, int z) -> float2 {
      const float sym = -4.0f * (tab.s2z[z] + tab.s2x[c0 + c]);
      const float2 mul = divc(make_float2(inv_n, 0.f), make_float2(sym + shiftc.x, shiftc.y));
      return adjoint ? conjc(mul) : mul;
    });
  }
}

// ---------------------------------------------------------------------------
// rinv: inverse row FFT in place on w, times the outer gain of the learned
// preconditioner; afterwards w holds z = M^-1 (input of the half).  DIRECT:
// the transform's first stage reads w and its last stage writes it, with the
// gain, straight from registers (ct_rows_inverse_direct).
// ---------------------------------------------------------------------------
template <bool DIRECT>
__global__ void __launch_bounds__(256, 4) k_rinv(SolveArgs A, int half) {
  extern __shared__ float2 sm[];
  const int slot = A.slot0 + blockIdx.x;
  const SlotState& S = A.B.slots[slot];
  if (!cols_active(S.mode, half)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int z0 = blockIdx.y * A.rows;
  const int nr = min(A.rows, g.nz - z0);
  const long long goff = (long long)z0 * g.nx;
  float2* w = A.B.w + slot * n + goff;
  const GainPair G = gain_pair(A.gains, S.gidx, n, A.adjoint);
  if constexpr (DIRECT) {
    fft_rows_inverse_direct(sm, nr, A.tab.px, w, [&](int k, float2 v) {
      w[k] = G.post ? gain_mul(G.post, goff + k, G.conj, v) : v;
    });
    return;
  }
  const bool pad = nsr_row_padded(g.nx);   // flat index k + k/16, as in k_fwd
  const int cnt = nr * g.nx;
#pragma unroll 8
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) sm[pad ? k + (k >> 4) : k] = w[k];
  __syncthreads();
  fft_rows<true>(sm, nr, A.tab.px);
  __syncthreads();
#pragma unroll 8
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
    const float2 v = sm[pad ? k + (k >> 4) : k];
    w[k] = G.post ? gain_mul(G.post, goff + k, G.conj, v) : v;
  }
}

__device__ __forceinline__ void set_float_scalars(const Geo& g, SlotState& S) {
  const SysScalars sc = sys_scalars(g, S.freq);
  S.kh2f = (float)sc.kh2;
  S.sigf = (float)sc.sig;
  S.fpowf = (float)sc.fpow;
}

__device__ void pop_next(const SolveArgs& A, SlotState& S) {
  const int nxt = atomicAdd(A.B.queue, 1);
  if (nxt < A.n_systems) {
    S.sys = nxt;
    S.mode = MODE_INIT;
    S.x0_off = 0;
    S.gidx = A.gain_index ? A.gain_index[nxt] : nxt;
    S.freq = A.freq[nxt];
    S.angle = A.angle ? A.angle[nxt] : 0.0;
    set_float_scalars(A.g, S);
  } else {
    S.sys = -1;
    S.mode = MODE_EMPTY;
  }
}

__device__ void finish_system(const SolveArgs& A, SlotState& S, int reason, double rel) {
  const long long n = (long long)A.g.nz * A.g.nx;
  const int slot = (int)(&S - A.B.slots);
  const double2* x = A.B.x + (2LL * slot + S.xpar) * n;
  for (int k = 0; k < A.n_rx; ++k) {
    const int idx = A.rx[k];
    const bool ok = idx >= 0 && (long long)idx < n;   // out-of-range receivers read as NaN
    A.iq[(long long)S.sys * A.n_rx + k] = !ok ? make_double2(NAN, NAN)
                                         : (S.zero_rhs ? make_double2(0.0, 0.0) : __ldcg(&x[idx]));
  }
  A.residual[S.sys] = rel;
  A.iterations[S.sys] = S.iters;
  A.status[S.sys] = reason;
  if (A.fields) {
    // counted as done once the emit pass has written its field
    S.mode = MODE_EMIT;
    return;
  }
  __threadfence();
  atomicAdd(A.B.done, 1);
  pop_next(A, S);
}

// Scalar recurrence of one slot, run by thread 0 of the slot's last CTA.
__device__ void finalize(const SolveArgs& A, SlotState& S, int mode, const double* sum) {
  const double tol2 = A.tol2;
  if (mode == MODE_EMIT) {
    __threadfence();
    atomicAdd(A.B.done, 1);
    pop_next(A, S);
    return;
  }
  if (mode == MODE_INIT) {
    S.bnorm2 = sum[0];
    S.rnorm2 = sum[1];
    S.xpar ^= 1;
    S.iters = 0;
    S.final_reason = -1;
    S.zero_rhs = 0;
    if (!(S.bnorm2 > 0.0)) {
      S.zero_rhs = isfinite(S.bnorm2) ? 1 : 0;
      finish_system(A, S, isfinite(S.bnorm2) ? NSR_CONVERGED : NSR_NONFINITE, 0.0);
      return;
    }
    const double rel2 = S.rnorm2 / S.bnorm2;
    const bool used_x0 = A.x0 != nullptr && !S.x0_off;
    if (used_x0 && A.warm_gate2 > 0.0 && !(rel2 <= A.warm_gate2)) {
      // The initial field is worse than the gate: discard it and start from zero.
      S.x0_off = 1;
      S.xpar ^= 1;
      atomicAdd(&A.B.warm[1], 1);
      S.mode = MODE_INIT;
      return;
    }
    if (used_x0) atomicAdd(&A.B.warm[0], 1);
    if (!isfinite(rel2)) { finish_system(A, S, NSR_NONFINITE, rel2); return; }
    if (rel2 < tol2) { finish_system(A, S, NSR_CONVERGED, sqrt(rel2)); return; }
    S.t_start = global_ns();
    S.rho = make_double2(S.rnorm2, 0.0);
    S.r0norm2 = S.rnorm2;
    S.restart = 0;
    S.force_restart = 0;
    S.breakdowns = 0;
    S.alpha = S.omega = S.beta = make_double2(0.0, 0.0);
    const double2 z = make_double2(0.0, 0.0);
    S.c_sv = S.c_rt = S.c_yp = S.c_ys = S.c_pp = S.c_pv = z;
    S.mode = MODE_ITER_A;
    return;
  }
  if (mode == MODE_ITER_A) {
    const double2 sigma = make_double2(sum[0], sum[1]);
    const double z2 = abs2(sigma);
    S.restart = 0;
    if (!finite2(sigma) || !(z2 > 1e-60 * S.bnorm2 * S.bnorm2)) {
      // Lanczos breakdown: restart from the true residual (twice in a row: give up)
      if (S.breakdowns >= 2 || !finite2(sigma)) S.final_reason = finite2(sigma) ? NSR_BREAKDOWN : NSR_NONFINITE;
      S.force_restart = 1;
      S.breakdowns += 1;
      S.c_sv = S.c_yp = S.c_ys = make_double2(0.0, 0.0);
      S.omega = make_double2(0.0, 0.0);
      S.mode = MODE_RES;
      return;
    }
    S.alpha = divc(S.rho, sigma);
    S.c_sv = make_double2(-S.alpha.x, -S.alpha.y);
    S.mode = MODE_ITER_B;
    return;
  }
  if (mode == MODE_ITER_B) {
    const double2 ts = make_double2(sum[0], sum[1]);
    const double tt = sum[2], ss = sum[3];
    const double2 rt = make_double2(sum[4], sum[5]);
    const double2 rs = make_double2(sum[6], sum[7]);
    S.iters += 1;
    const double2 z = make_double2(0.0, 0.0);
    if (ss < tol2 * S.bnorm2) {   // early exit on s (nsrno/dense_wave.py:138-139)
      S.omega = z;
      S.c_yp = S.alpha; S.c_ys = z; S.c_sv = make_double2(-S.alpha.x, -S.alpha.y); S.c_rt = z;
      S.mode = MODE_RES;
      return;
    }
    if (!(tt > 0.0) || !isfinite(tt) || !finite2(ts)) {
      S.final_reason = isfinite(tt) ? NSR_BREAKDOWN : NSR_NONFINITE;
      S.omega = z;
      S.c_yp = S.alpha; S.c_ys = z; S.c_sv = make_double2(-S.alpha.x, -S.alpha.y);
      S.mode = MODE_RES;
      return;
    }
    const double2 omega = make_double2(ts.x / tt, ts.y / tt);
    const double2 rho_new = rs - omega * rt;
    double rn2 = ss - abs2(ts) / tt;
    S.rnorm2 = rn2 > 0.0 ? rn2 : 0.0;
    S.omega = omega;
    S.c_sv = make_double2(-S.alpha.x, -S.alpha.y);
    S.c_rt = make_double2(-omega.x, -omega.y);
    S.c_yp = S.alpha;
    S.c_ys = omega;
    const bool omega_ok = abs2(omega) > 1e-60;
    const bool rho_ok = finite2(rho_new) && abs2(rho_new) > 1e-60 * S.bnorm2 * S.bnorm2;
    if (omega_ok && rho_ok) {
      S.beta = divc(rho_new, S.rho) * divc(S.alpha, omega);
      S.rho = rho_new;
      S.c_pp = S.beta;
      S.c_pv = make_double2(0.0, 0.0) - S.beta * omega;
      S.breakdowns = 0;
    } else {
      // rho or omega vanished: restart from the true residual (three in a row: give up)
      if (S.breakdowns >= 2) S.final_reason = NSR_BREAKDOWN;
      S.force_restart = 1;
      S.breakdowns += 1;
    }
    if (A.time_limit_ns && S.final_reason < 0 && global_ns() - S.t_start > A.time_limit_ns)
      S.final_reason = NSR_TIMEOUT;   // stops after the FP64 true residual of the current iterate
    if (S.force_restart || S.final_reason >= 0 || S.rnorm2 < tol2 * S.bnorm2 || S.iters >= A.max_it ||
        (A.replace_every > 0 && S.iters % A.replace_every == 0)) {
      if (S.iters >= A.max_it && S.final_reason < 0) S.final_reason = NSR_ITERATION_BUDGET;
      S.mode = MODE_RES;
    } else {
      S.mode = MODE_ITER_A;
    }
    return;
  }
  if (mode == MODE_RES) {
    const double rr = sum[0];
    const double2 rhr = make_double2(sum[1], sum[2]);
    S.xpar ^= 1;
    const double rel2 = rr / S.bnorm2;
    const double rel = sqrt(rel2);
    S.resid = rel;
    if (!isfinite(rel2)) { finish_system(A, S, NSR_NONFINITE, rel); return; }
    if (rel2 < tol2) { finish_system(A, S, NSR_CONVERGED, rel); return; }
    if (S.final_reason >= 0) { finish_system(A, S, S.final_reason, rel); return; }
    if (rel > 1e5) { finish_system(A, S, NSR_DIVERGED, rel); return; }
    if (S.iters >= A.max_it) { finish_system(A, S, NSR_ITERATION_BUDGET, rel); return; }
    const double2 z = make_double2(0.0, 0.0);
    S.c_sv = S.c_rt = S.c_yp = S.c_ys = z;
    // Restart (fresh shadow vector rhat = r, written by the next fwd pass; p = r)
    // after a forced restart, after the true residual fell by restart_factor
    // since the last restart, or when it grew since then: the FP32 recurrence
    // has lost its bi-orthogonality and would otherwise run away (one system
    // in 24,000 of the training media diverged without this).
    if (S.force_restart || rr > S.r0norm2 || (A.restart2 > 0.0 && rr < A.restart2 * S.r0norm2)) {
      S.restart = 1;
      S.force_restart = 0;
      S.r0norm2 = rr;
      S.rho = make_double2(rr, 0.0);
      S.rnorm2 = rr;
      S.c_pp = S.c_pv = z;
      S.mode = MODE_ITER_A;
      return;
    }
    if (abs2(S.omega) > 1e-60 && abs2(S.rho) > 0.0) {
      // Replace the recursive residual by the true one and rescale beta.
      S.beta = S.beta * divc(rhr, S.rho);
      S.c_pp = S.beta;
      S.c_pv = z - S.beta * S.omega;
    } else {
      // The s-based exit was premature: restart the recurrence from r.
      S.c_pp = S.c_pv = z;
    }
    S.rho = rhr;
    S.rnorm2 = rr;
    S.mode = MODE_ITER_A;
    return;
  }
}

// ---------------------------------------------------------------------------
// Per-CTA partials, arrival, and the last CTA's finalize (no waiting).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reduce_and_finalize(const SolveArgs& A, SlotState& S, int slot, int mode,
                                                    double* acc) {
  __shared__ double red[NSR_NPART];
  __shared__ double tot[NSR_NPART];
  __shared__ int am_last;
  block_sum<NSR_NPART>(acc, red);
  double* part = A.B.partials + (long long)slot * A.nb_inv * NSR_NPART;
  if (threadIdx.x == 0) {
    for (int q = 0; q < NSR_NPART; ++q) part[blockIdx.x * NSR_NPART + q] = red[q];
    __threadfence();
    const int prev = atomicAdd(&A.B.arrive[slot], 1);
    am_last = (prev == (int)gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  // Deterministic sum over CTAs: thread q sums column q in CTA order.
  if (threadIdx.x < NSR_NPART) {
    double sacc = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) sacc += __ldcg(&part[b * NSR_NPART + threadIdx.x]);
    tot[threadIdx.x] = sacc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    A.B.arrive[slot] = 0;
    finalize(A, S, mode, tot);
    __threadfence();
  }
}

// ---------------------------------------------------------------------------
// inv: stencil on z = M^-1 (input) + inner products of the Krylov halves.
// One thread owns two adjacent columns of a NSR_ST_TZ x NSR_ST_TX tile and
// walks down its rows with the north/centre/south values of z and a in
// registers; every field is read as 16-byte pairs.  The east/west
// neighbours come from the adjacent threads by warp shuffles (global loads
// at the warp edges).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float4 pack2(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }

template <bool ADJ>
__global__ void __launch_bounds__(256, 4) k_inv(SolveArgs A, int half) {
  const int slot = A.slot0 + blockIdx.y;
  SlotState& S = A.B.slots[slot];
  const int mode = S.mode;
  if (mode != (half == 0 ? MODE_ITER_A : MODE_ITER_B)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int nx = g.nx;
  const int nbx = (nx + NSR_ST_TX - 1) / NSR_ST_TX;
  const int rb = blockIdx.x / nbx, cb = blockIdx.x - rb * nbx;
  const int z0 = rb * NSR_ST_TZ;
  const int z1 = min(z0 + NSR_ST_TZ, g.nz);
  const int j = cb * NSR_ST_TX + 2 * threadIdx.x;   // first of the thread's two columns
  const bool own = j < nx;                          // nx is even here: both columns exist
  const int lane = threadIdx.x & 31;
  const long long soff = slot * n;
  double acc[NSR_NPART];
#pragma unroll
  for (int q = 0; q < NSR_NPART; ++q) acc[q] = 0.0;
  // Every thread of a warp takes part in the shuffles; threads past the last
  // column carry zeros and store nothing.
  {
    const SysScalars sc = sys_scalars(g, S.freq);
    const float* __restrict__ ca = A.mat.a32;
    const float* __restrict__ cb_ = A.mat.b32;
    const float* __restrict__ ct = A.mat.t32;
    const float2* __restrict__ z = A.B.w + soff;
    const float2* __restrict__ rh = A.B.rh + soff;
    const float2* __restrict__ r = A.B.r + soff;
    const float2* __restrict__ v = A.B.v + soff;
    float2* __restrict__ out = (half == 0 ? A.B.v : A.B.t) + soff;
    const float2 sv = f2(S.c_sv);
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    const float2 zero = make_float2(0.f, 0.f);
    const int jc = own ? j : 0;
    const bool edge_w = lane == 0, edge_e = lane == 31 || j + 2 >= nx;
    long long idx = (long long)z0 * nx + jc;
    float4 zu = (own && z0 > 0) ? *reinterpret_cast<const float4*>(z + idx - nx) : zero4;
    float4 zc = own ? *reinterpret_cast<const float4*>(z + idx) : zero4;
    float2 an = (own && z0 > 0) ? __ldg(reinterpret_cast<const float2*>(ca + idx - nx)) : make_float2(1.f, 1.f);
    float2 ac = own ? __ldg(reinterpret_cast<const float2*>(ca + idx)) : make_float2(1.f, 1.f);
    for (int i = z0; i < z1; ++i, idx += nx) {
      const bool has_s = i + 1 < g.nz;
      const float4 zd = (own && has_s) ? *reinterpret_cast<const float4*>(z + idx + nx) : zero4;
      const float2 as = (own && has_s) ? __ldg(reinterpret_cast<const float2*>(ca + idx + nx)) : make_float2(1.f, 1.f);
      // west neighbour of column j, east neighbour of column j+1
      float2 zw = make_float2(__shfl_up_sync(0xffffffffu, zc.z, 1), __shfl_up_sync(0xffffffffu, zc.w, 1));
      float aw = __shfl_up_sync(0xffffffffu, ac.y, 1);
      float2 ze = make_float2(__shfl_down_sync(0xffffffffu, zc.x, 1), __shfl_down_sync(0xffffffffu, zc.y, 1));
      float ae = __shfl_down_sync(0xffffffffu, ac.x, 1);
      if (own && edge_w) {
        zw = j > 0 ? z[idx - 1] : zero;
        aw = j > 0 ? __ldg(&ca[idx - 1]) : 1.0f;
      }
      if (own && edge_e) {
        ze = j + 2 < nx ? z[idx + 2] : zero;
        ae = j + 2 < nx ? __ldg(&ca[idx + 2]) : 1.0f;
      }
      if (own) {
        const float2 bb = __ldg(reinterpret_cast<const float2*>(cb_ + idx));
        const float2 tt = __ldg(reinterpret_cast<const float2*>(ct + idx));
        const float2 c0 = lo2(zc), c1 = hi2(zc);
        const float2 av0 = stencil_pts<ADJ>(g, sc, i, j, ac.x, ac.y, aw, as.x, an.x, bb.x, tt.x, c0, c1, zw, lo2(zd),
                                            lo2(zu));
        const float2 av1 = stencil_pts<ADJ>(g, sc, i, j + 1, ac.y, ae, ac.x, as.y, an.y, bb.y, tt.y, c1, ze, c0,
                                            hi2(zd), hi2(zu));
        *reinterpret_cast<float4*>(out + idx) = pack2(av0, av1);
        const float4 rk = *reinterpret_cast<const float4*>(rh + idx);
        if (half == 0) {
          dot_acc(acc[0], acc[1], lo2(rk), av0);       // <rhat, v>
          dot_acc(acc[0], acc[1], hi2(rk), av1);
        } else {
          const float4 rr = *reinterpret_cast<const float4*>(r + idx);
          const float4 vv = *reinterpret_cast<const float4*>(v + idx);
          const float2 s0 = lo2(rr) + sv * lo2(vv), s1 = hi2(rr) + sv * hi2(vv);
          dot_acc(acc[0], acc[1], av0, s0);            // <t, s>
          dot_acc(acc[0], acc[1], av1, s1);
          acc[2] += (double)av0.x * av0.x + (double)av0.y * av0.y + (double)av1.x * av1.x + (double)av1.y * av1.y;
          acc[3] += (double)s0.x * s0.x + (double)s0.y * s0.y + (double)s1.x * s1.x + (double)s1.y * s1.y;
          dot_acc(acc[4], acc[5], lo2(rk), av0);       // <rhat, t>
          dot_acc(acc[4], acc[5], hi2(rk), av1);
          dot_acc(acc[6], acc[7], lo2(rk), s0);        // <rhat, s>
          dot_acc(acc[6], acc[7], hi2(rk), s1);
        }
      }
      zu = zc;
      zc = zd;
      an = ac;
      ac = as;
    }
  }
  reduce_and_finalize(A, S, slot, mode, acc);
}

// ---------------------------------------------------------------------------
// stn: the stencil of k_inv on rows staged through shared memory by bulk
// (TMA) copies, for widths that are a multiple of 4.
//
// A persistent CTA walks work items (slot, band of tz rows, strip of W
// columns).  One producer thread streams the rows of its items into a ring of
// D row buffers with cp.async.bulk, completing on a `full` mbarrier per ring
// entry; W/2 consumer threads (two columns each) compute row i from the
// buffers of rows i-1, i, i+1 and release the buffer of row i-1 on an `empty`
// mbarrier.  Every row buffer holds z (with two halo columns each side) and
// a (four each side), and for the band's own rows b, t, rhat and, in the
// second half, r and v: a row step moves about 22 B per column, and D-3 row
// steps are in flight per CTA while the consumers compute.  Nothing but the
// copies themselves touches HBM on the read side, so the loads overlap the
// stencil and FP64 dot products completely.
// ---------------------------------------------------------------------------
// One row of the ring.  The first half (H = 0) needs no r and v, so its rows
// are two fifths smaller and the same ring bytes hold more of them.
template <int W, int H>
struct StnLayout {
  static constexpr int OZ = 0;                    // float2 z[W + 4], column c0 - 2 + e
  static constexpr int ORH = OZ + (W + 4) * 8;    // float2 rhat[W]
  static constexpr int OR = ORH + W * 8;          // float2 r[W] (second half)
  static constexpr int OV = OR + (H ? W * 8 : 0);   // float2 v[W] (second half)
  static constexpr int OA = OV + (H ? W * 8 : 0);   // float a[W + 8], column c0 - 4 + e
  static constexpr int SLOT = OA + (W + 8) * 4;
  static_assert(ORH % 16 == 0 && OA % 16 == 0 && SLOT % 16 == 0, "alignment");
};

#define NSR_STN_WAIT_NS 2000000000ull   // a ring wait longer than 2 s is an error
#define NSR_STN_FLUSH 8                  // rows per float partial sum of the inner products

// Items of one launch and their decoding.  Item i is band-strip i / ns of
// slot i % ns: the slots run fastest, so the CTAs in flight at any time work
// on the same few bands of every slot, and the medium's coefficient rows
// (read by every slot) come from L2 after the first slot's copy.
struct StnItems {
  int tz, nbands, nstrips, per_slot, n_items;
};

template <int W>
__host__ __device__ inline StnItems stn_items(int nz, int nx, int tz, int ns) {
  StnItems it;
  it.tz = tz;
  it.nbands = (nz + tz - 1) / tz;
  it.nstrips = (nx + W - 1) / W;
  it.per_slot = it.nbands * it.nstrips;
  it.n_items = ns * it.per_slot;
  return it;
}

// Resident CTAs per SM that the shared-memory ring of a k_stn shape allows
// (at most 4): its register budget follows from it.
// Inner products of a half: <rhat, v> (first); <t, s>, <t, t>, <s, s>,
// <rhat, t>, <rhat, s> (second), as (re, im) pairs where complex.
__host__ __device__ constexpr int stn_parts(int H) { return H ? NSR_NPART : 2; }

// Ring depth of the first half for a second-half depth D: the same ring bytes.
template <int W>
__host__ __device__ constexpr int stn_depth0(int D) {
  return (D * StnLayout<W, 1>::SLOT) / StnLayout<W, 0>::SLOT;
}

template <int W, int D, int CPT, int H>
__host__ __device__ constexpr int stn_min_blocks() {
  // ring, barriers and block sums (2 KB), FP64 accumulators of the consumers
  constexpr int by_smem = (227 * 1024) / (D * StnLayout<W, H>::SLOT + 2048 + 8 * stn_parts(H) * (W / CPT));
  constexpr int cap = (W / CPT + 32) > 256 ? 2 : 4;
  return by_smem < 1 ? 1 : (by_smem > cap ? cap : by_smem);
}

template <int W, int D, int CPT, bool ADJ, int H>
__global__ void __launch_bounds__(W / CPT + 32, (stn_min_blocks<W, D, CPT, H>()))
    k_stn(SolveArgs A, int /*half: H*/, StnItems it, int ns) {
  typedef StnLayout<W, H> Ly;
  constexpr int half = H;
  constexpr int NP = stn_parts(H);
  constexpr int NC = W / CPT;   // consumer threads, CPT adjacent columns each
  constexpr int FLUSH = NSR_STN_FLUSH * 2 / CPT;   // rows per float partial sum
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ __align__(8) uint64_t full[D], empty[D];
  __shared__ int abort_word;
  volatile int& abort_flag = abort_word;
  __shared__ double wsum[NC / 32][NSR_NPART];
  __shared__ double tot[NSR_NPART];
  // Each consumer's FP64 accumulators live in shared memory (column tid): in
  // registers they pushed the 96-register budget of four CTAs per SM into
  // spills inside the row loop.
  __shared__ double accs[NP][NC];
  __shared__ int am_last;
  const Geo& g = A.g;
  const int nz = g.nz, nx = g.nx;
  const long long n = (long long)nz * nx;
  const int want = half == 0 ? MODE_ITER_A : MODE_ITER_B;
  if (threadIdx.x == 0) {
    for (int k = 0; k < D; ++k) {
      mbar_init(&full[k], 1);
      mbar_init(&empty[k], NC / 32);
    }
    abort_word = 0;
    mbar_init_fence();
  }
  __syncthreads();

  if (threadIdx.x >= NC) {
    // ---------------- producer ----------------
    if (threadIdx.x != NC) return;
    uint32_t q = 0;   // row step counter (ring entry q % D, phase q / D)
    for (int item = blockIdx.x; item < it.n_items && !abort_flag; item += gridDim.x) {
      const int rem = item / ns, sl = item - rem * ns;
      const int band = rem / it.nstrips, strip = rem - band * it.nstrips;
      const int slot = A.slot0 + sl;
      if (A.B.slots[slot].mode != want) continue;
      const int z0 = band * it.tz, z1 = min(z0 + it.tz, nz);
      const int c0 = strip * W;
      const long long soff = slot * n;
      const float2* zsrc = A.B.w + soff;
      const float2* rhsrc = A.B.rh + soff;
      const float2* rsrc = A.B.r + soff;
      const float2* vsrc = A.B.v + soff;
      const int zlo = max(c0 - 2, 0), zhi = min(c0 + W + 2, nx);
      const int alo = max(c0 - 4, 0), ahi = min(c0 + W + 4, nx);
      const int phi = min(c0 + W, nx);
      for (int row = z0 - 1; row <= z1; ++row, ++q) {
        const int e = q % D;
        if (q >= D && !mbar_wait(&empty[e], ((q / D) & 1) ^ 1, &abort_word, NSR_STN_WAIT_NS)) {
          abort_flag = 1;
          break;
        }
        unsigned char* buf = ring + (size_t)e * Ly::SLOT;
        const bool in = row >= 0 && row < nz;
        const bool own = row >= z0 && row < z1;
        uint32_t bytes = 0;
        if (in) bytes += (zhi - zlo) * 8 + (ahi - alo) * 4;
        if (own) bytes += (phi - c0) * 8 + (half ? 2 * (phi - c0) * 8 : 0);
        mbar_arrive_expect_tx(&full[e], bytes);
        if (in) {
          const long long ro = (long long)row * nx;
          bulk_load(buf + Ly::OZ + (zlo - (c0 - 2)) * 8, zsrc + ro + zlo, (zhi - zlo) * 8, &full[e]);
          bulk_load(buf + Ly::OA + (alo - (c0 - 4)) * 4, A.mat.a32 + ro + alo, (ahi - alo) * 4, &full[e]);
          if (own) {
            const uint32_t cb = (phi - c0) * 8;
            bulk_load(buf + Ly::ORH, rhsrc + ro + c0, cb, &full[e]);
            if (half) {
              bulk_load(buf + Ly::OR, rsrc + ro + c0, cb, &full[e]);
              bulk_load(buf + Ly::OV, vsrc + ro + c0, cb, &full[e]);
            }
          }
        }
      }
    }
    if (abort_flag) {
      atomicExch(A.B.error, 1);
      // Let the copies already issued land before the block's shared memory goes away.
      for (uint32_t k = (q > (uint32_t)D ? q - D : 0); k < q; ++k)
        mbar_wait(&full[k % D], (k / D) & 1, nullptr, NSR_STN_WAIT_NS);
    }
    return;
  }

  // ---------------- consumers ----------------
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  uint32_t q = 0;
  for (int item = blockIdx.x; item < it.n_items; item += gridDim.x) {
    const int rem = item / ns, sl = item - rem * ns;
    const int band = rem / it.nstrips, strip = rem - band * it.nstrips;
    const int slot = A.slot0 + sl;
    SlotState& S = A.B.slots[slot];
    if (S.mode != want) continue;
    const int z0 = band * it.tz, z1 = min(z0 + it.tz, nz);
    const int nrows = z1 - z0;
    const int c0 = strip * W;
    const int j = c0 + CPT * tid;
    const bool own = j < nx;
    const bool has_w = j > 0, has_e = j + CPT < nx;
    const long long soff = slot * n;
    float2* __restrict__ out = (half == 0 ? A.B.v : A.B.t) + soff;
    SysScalarsF sf;
    sf.kh2 = S.kh2f;
    sf.sig = S.sigf;
    sf.fpow = S.fpowf;
    sf.inv_npml = g.n_pml > 0 ? 1.0f / (float)g.n_pml : 0.0f;
    sf.lo = g.n_pml;
    sf.hi_z = nz - 1 - g.n_pml;
    sf.hi_x = nx - 1 - g.n_pml;
    const float2 sv = f2(S.c_sv);
    // Inner products: float partial sums over NSR_STN_FLUSH rows (2 NSR_STN_FLUSH
    // products per thread), accumulated in FP64.
    float accf[NSR_NPART];
#pragma unroll
    for (int k = 0; k < NSR_NPART; ++k) {
      if (k < NP) accs[k][tid] = 0.0;
      accf[k] = 0.0f;
    }
    const uint32_t q0 = q;   // step of row z0 - 1
    bool ok = !abort_flag;
    // rows z0 - 1 and z0
    for (uint32_t s = q0; s < q0 + 2 && ok; ++s) ok = mbar_wait(&full[s % D], (s / D) & 1, &abort_word, NSR_STN_WAIT_NS);
    // Ring entries of rows i - 1, i, i + 1 (advanced incrementally) and the
    // column's z and a of rows i - 1 and i, carried from row to row so that
    // each row reads only its south neighbours from the ring.
    int eN = q0 % D, eC = (eN + 1 == D) ? 0 : eN + 1;
    const int ez = (CPT * tid + 2) * 8, ea = (CPT * tid + 4) * 4;
    typedef typename std::conditional<CPT == 2, float4, float2>::type ZT;
    typedef typename std::conditional<CPT == 2, float2, float>::type AT;
    auto zload = [&](int e) -> ZT { return *reinterpret_cast<const ZT*>(ring + (size_t)e * Ly::SLOT + Ly::OZ + ez); };
    auto aload = [&](int e) -> AT { return *reinterpret_cast<const AT*>(ring + (size_t)e * Ly::SLOT + Ly::OA + ea); };
    ZT zN = ZT{}, zC = ZT{};
    AT aN, aC = AT{};
    if constexpr (CPT == 2) aN = make_float2(1.f, 1.f); else aN = 1.0f;   // no density contrast outside
    if (ok) {
      if (z0 > 0) { zN = zload(eN); aN = aload(eN); }
      zC = zload(eC); aC = aload(eC);
    }
    // The centre-only coefficients b and t are shared by every slot of the
    // launch and come from L2 (the CTAs in flight work on the same rows):
    // read directly, one row ahead, instead of through the ring.
    const float* __restrict__ bpl = A.mat.b32;
    const float* __restrict__ tpl = A.mat.t32;
    auto bt = [&](const float* __restrict__ pl, int row) -> AT {
      return own ? __ldg(reinterpret_cast<const AT*>(pl + (long long)row * nx + j)) : AT{};
    };
    AT bNext = bt(bpl, z0), tNext = bt(tpl, z0);
    // Interior test (no PML stretch) per column, once per item; per row below.
    const bool col_in0 = j > sf.lo && j < sf.hi_x, col_in1 = j + CPT - 1 > sf.lo && j + CPT - 1 < sf.hi_x;
    for (int k = 0; k < nrows; ++k) {
      const int i = z0 + k;
      const bool row_in = i > sf.lo && i < sf.hi_z;
      const AT bRow = bNext, tRow = tNext;
      if (k + 1 < nrows) { bNext = bt(bpl, i + 1); tNext = bt(tpl, i + 1); }
      const uint32_t sS = q0 + k + 2;
      const int eS = (eC + 1 == D) ? 0 : eC + 1;
      if (ok) ok = mbar_wait(&full[eS], (sS / D) & 1, &abort_word, NSR_STN_WAIT_NS);
      if (!ok) abort_flag = 1;
      ZT zS = ZT{};
      AT aS;
      if constexpr (CPT == 2) aS = make_float2(1.f, 1.f); else aS = 1.0f;
      if (ok && i + 1 < nz) { zS = zload(eS); aS = aload(eS); }
      if (ok && own) {
        const unsigned char* bC = ring + (size_t)eC * Ly::SLOT;
        const float2 zero = make_float2(0.f, 0.f);
        if constexpr (CPT == 2) {
          const float4 zc = zC, zn = zN, zs = zS;
          const float2 zw = has_w ? *reinterpret_cast<const float2*>(bC + Ly::OZ + ez - 8) : zero;
          const float2 ze = has_e ? *reinterpret_cast<const float2*>(bC + Ly::OZ + ez + 16) : zero;
          const float2 ac = aC, an = aN, as = aS;
          const float aw = has_w ? *reinterpret_cast<const float*>(bC + Ly::OA + ea - 4) : 1.0f;
          const float ae = has_e ? *reinterpret_cast<const float*>(bC + Ly::OA + ea + 8) : 1.0f;
          const float2 bb = bRow, tt = tRow;
          const float4 rk = *reinterpret_cast<const float4*>(bC + Ly::ORH + 16 * tid);
          const float2 c0v = lo2(zc), c1v = hi2(zc);
          const float2 av0 = stencil_pts_f<ADJ>(g, sf, row_in && col_in0, i, j, ac.x, ac.y, aw, as.x, an.x, bb.x,
                                                tt.x, c0v, c1v, zw, lo2(zs), lo2(zn));
          const float2 av1 = stencil_pts_f<ADJ>(g, sf, row_in && col_in1, i, j + 1, ac.y, ae, ac.x, as.y, an.y, bb.y,
                                                tt.y, c1v, ze, c0v, hi2(zs), hi2(zn));
          *reinterpret_cast<float4*>(out + (long long)i * nx + j) = pack2(av0, av1);
          if (half == 0) {
            dot_acc_f(accf[0], accf[1], lo2(rk), av0);       // <rhat, v>
            dot_acc_f(accf[0], accf[1], hi2(rk), av1);
          } else {
            const float4 rr = *reinterpret_cast<const float4*>(bC + Ly::OR + 16 * tid);
            const float4 vv = *reinterpret_cast<const float4*>(bC + Ly::OV + 16 * tid);
            const float2 s0 = lo2(rr) + sv * lo2(vv), s1 = hi2(rr) + sv * hi2(vv);
            dot_acc_f(accf[0], accf[1], av0, s0);            // <t, s>
            dot_acc_f(accf[0], accf[1], av1, s1);
            accf[2] = fmaf(av0.x, av0.x, fmaf(av0.y, av0.y, fmaf(av1.x, av1.x, fmaf(av1.y, av1.y, accf[2]))));
            accf[3] = fmaf(s0.x, s0.x, fmaf(s0.y, s0.y, fmaf(s1.x, s1.x, fmaf(s1.y, s1.y, accf[3]))));
            dot_acc_f(accf[4], accf[5], lo2(rk), av0);       // <rhat, t>
            dot_acc_f(accf[4], accf[5], hi2(rk), av1);
            dot_acc_f(accf[6], accf[7], lo2(rk), s0);        // <rhat, s>
            dot_acc_f(accf[6], accf[7], hi2(rk), s1);
          }
        } else {
          const float2 zc = zC, zn = zN, zs = zS;
          const float2 zw = has_w ? *reinterpret_cast<const float2*>(bC + Ly::OZ + ez - 8) : zero;
          const float2 ze = has_e ? *reinterpret_cast<const float2*>(bC + Ly::OZ + ez + 8) : zero;
          const float ac = aC, an = aN, as = aS;
          const float aw = has_w ? *reinterpret_cast<const float*>(bC + Ly::OA + ea - 4) : 1.0f;
          const float ae = has_e ? *reinterpret_cast<const float*>(bC + Ly::OA + ea + 4) : 1.0f;
          const float bb = bRow, tt = tRow;
          const float2 rk = *reinterpret_cast<const float2*>(bC + Ly::ORH + 8 * tid);
          const float2 av = stencil_pts_f<ADJ>(g, sf, row_in && col_in0, i, j, ac, ae, aw, as, an, bb, tt, zc, ze, zw,
                                               zs, zn);
          out[(long long)i * nx + j] = av;
          if (half == 0) {
            dot_acc_f(accf[0], accf[1], rk, av);       // <rhat, v>
          } else {
            const float2 rr = *reinterpret_cast<const float2*>(bC + Ly::OR + 8 * tid);
            const float2 vv = *reinterpret_cast<const float2*>(bC + Ly::OV + 8 * tid);
            const float2 s0 = rr + sv * vv;
            dot_acc_f(accf[0], accf[1], av, s0);       // <t, s>
            accf[2] = fmaf(av.x, av.x, fmaf(av.y, av.y, accf[2]));
            accf[3] = fmaf(s0.x, s0.x, fmaf(s0.y, s0.y, accf[3]));
            dot_acc_f(accf[4], accf[5], rk, av);       // <rhat, t>
            dot_acc_f(accf[6], accf[7], rk, s0);       // <rhat, s>
          }
        }
      }
      zN = zC; zC = zS; aN = aC; aC = aS;
      if ((k + 1) % FLUSH == 0 || k + 1 == nrows) {
#pragma unroll
        for (int qq = 0; qq < NSR_NPART; ++qq) {
          if (qq < NP) accs[qq][tid] += (double)accf[qq];
          accf[qq] = 0.0f;
        }
      }
      // The buffer of row i - 1 goes back to the producer one row after its
      // last use as centre.  Its values were loaded into registers during row
      // i - 1, but a release right after those loads can overtake them: the
      // arrival does not wait for shared-memory loads still in flight, and
      // the producer's next bulk copy into the buffer then races them (seen
      // as nondeterministic inner products with two slot groups).
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[eN]);
      eN = eC;
      eC = eS;
    }
    // rows z1 - 1 and z1
    __syncwarp();
    if (lane == 0) {
      mbar_arrive(&empty[eN]);
      mbar_arrive(&empty[eC]);
    }
    q = q0 + nrows + 2;

    // Block sum of the partials (consumer threads only), then the arrival.
#pragma unroll
    for (int k = 0; k < NSR_NPART; ++k) {
      const double s = k < NP ? warp_sum(accs[k][tid]) : 0.0;
      if (lane == 0) wsum[wid][k] = s;
    }
    named_sync(1, NC);
    double* part = A.B.partials + (long long)slot * A.nb_inv * NSR_NPART;
    if (tid == 0) {
      for (int k = 0; k < NSR_NPART; ++k) {
        double s = 0.0;
        for (int w2 = 0; w2 < NC / 32; ++w2) s += wsum[w2][k];
        part[rem * NSR_NPART + k] = s;
      }
      __threadfence();
      const int prev = atomicAdd(&A.B.arrive[slot], 1);
      am_last = (prev == it.per_slot - 1);
    }
    named_sync(1, NC);
    if (am_last) {
      __threadfence();
      if (tid < NSR_NPART) {
        double sacc = 0.0;
        for (int b = 0; b < it.per_slot; ++b) sacc += __ldcg(&part[b * NSR_NPART + tid]);
        tot[tid] = sacc;
      }
      named_sync(1, NC);
      if (tid == 0) {
        A.B.arrive[slot] = 0;
        finalize(A, S, want, tot);
        __threadfence();
      }
    }
    named_sync(1, NC);   // wsum, tot and am_last are reused by the next item
  }
  if (tid == 0 && abort_flag) atomicExch(A.B.error, 1);
}

// ---------------------------------------------------------------------------
// inv: stencil on z = M^-1 (input) + inner products of the Krylov halves.
// k_inv1 (grids of odd width, whose rows are not 16-byte aligned): one thread
// per column of a NSR_ST_TZ x NSR_ST_TX1 tile walks down its rows
// with the north/centre/south values of z and a in registers; east/west
// neighbours are the adjacent threads' loads (L1 hits).
// ---------------------------------------------------------------------------
template <bool ADJ>
__global__ void __launch_bounds__(256, 4) k_inv1(SolveArgs A, int half) {
  const int slot = A.slot0 + blockIdx.y;
  SlotState& S = A.B.slots[slot];
  const int mode = S.mode;
  if (mode != (half == 0 ? MODE_ITER_A : MODE_ITER_B)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int nx = g.nx;
  const int nbx = (nx + NSR_ST_TX1 - 1) / NSR_ST_TX1;
  const int rb = blockIdx.x / nbx, cb = blockIdx.x - rb * nbx;
  const int z0 = rb * NSR_ST_TZ;
  const int z1 = min(z0 + NSR_ST_TZ, g.nz);
  const int j = cb * NSR_ST_TX1 + threadIdx.x;
  const long long soff = slot * n;
  double acc[NSR_NPART];
#pragma unroll
  for (int q = 0; q < NSR_NPART; ++q) acc[q] = 0.0;
  if (j < nx) {
    const SysScalars sc = sys_scalars(g, S.freq);
    const float* __restrict__ ca = A.mat.a32;
    const float* __restrict__ cb_ = A.mat.b32;
    const float* __restrict__ ct = A.mat.t32;
    const float2* __restrict__ z = A.B.w + soff;
    const float2* __restrict__ rh = A.B.rh + soff;
    const float2* __restrict__ r = A.B.r + soff;
    const float2* __restrict__ v = A.B.v + soff;
    float2* __restrict__ out = (half == 0 ? A.B.v : A.B.t) + soff;
    const float2 sv = f2(S.c_sv);
    const float2 zero = make_float2(0.f, 0.f);
    const bool has_e = j + 1 < nx, has_w = j > 0;
    long long idx = (long long)z0 * nx + j;
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
      const float2 av = stencil_pts<ADJ>(g, sc, i, j, a_c, a_e, a_w, a_s, a_n, __ldg(&cb_[idx]), __ldg(&ct[idx]),
                                         zc, ze, zw, zd, zu);
      out[idx] = av;
      const float2 rk = rh[idx];
      if (half == 0) {
        dot_acc(acc[0], acc[1], rk, av);       // <rhat, v>
      } else {
        const float2 s1 = r[idx] + sv * v[idx];
        dot_acc(acc[0], acc[1], av, s1);       // <t, s>
        acc[2] += (double)av.x * av.x + (double)av.y * av.y;
        acc[3] += (double)s1.x * s1.x + (double)s1.y * s1.y;
        dot_acc(acc[4], acc[5], rk, av);       // <rhat, t>
        dot_acc(acc[6], acc[7], rk, s1);       // <rhat, s>
      }
      zu = zc;
      zc = zd;
      a_n = a_c;
      a_c = a_s;
    }
  }
  reduce_and_finalize(A, S, slot, mode, acc);
}

// ---------------------------------------------------------------------------
// res: FP64 true residual r = b - A x of a replacement (x += M^-1 y) or of a
// new system (x = x0); emit passes only arrive and hand the slot on.
// ---------------------------------------------------------------------------
template <bool ADJ>
__global__ void __launch_bounds__(256) k_res(SolveArgs A) {
  const int slot = A.slot0 + blockIdx.y;
  SlotState& S = A.B.slots[slot];
  const int mode = S.mode;
  if (!(mode == MODE_RES || mode == MODE_INIT || mode == MODE_EMIT)) return;
  const Geo& g = A.g;
  const long long n = (long long)g.nz * g.nx;
  const int tz = A.tz;
  const int z0 = blockIdx.x * tz;
  const int nb = min(tz, g.nz - z0);
  const int nx = g.nx;
  const SysScalars sc = sys_scalars(g, S.freq);
  const double* ca = A.mat.a64;
  const double* cb = A.mat.b64;
  const double* ct = A.mat.t64;
  auto Aa64 = [&](int i2, int j2) -> double {
    if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= nx) return 1.0;
    return __ldg(&ca[(long long)i2 * nx + j2]);
  };
  double acc[NSR_NPART];
#pragma unroll
  for (int q = 0; q < NSR_NPART; ++q) acc[q] = 0.0;
  const long long soff = slot * n;
  if (mode == MODE_RES || mode == MODE_INIT) {
    const float2* zw = A.B.w + soff;   // z = M^-1 y after the rinv pass
    const double2* xo = A.B.x + (2LL * slot + S.xpar) * n;
    double2* xn = A.B.x + (2LL * slot + (S.xpar ^ 1)) * n;
    const float2* x0 = (A.x0 && S.sys >= 0 && !S.x0_off) ? A.x0 + (long long)S.sys * n : nullptr;
    auto P = [&](int i2, int j2) -> double2 {
      if (i2 < 0 || i2 >= g.nz || j2 < 0 || j2 >= nx) return make_double2(0.0, 0.0);
      const long long id = (long long)i2 * nx + j2;
      if (mode == MODE_INIT) return x0 ? to_d(x0[id]) : make_double2(0.0, 0.0);
      return xo[id] + to_d(zw[id]);
    };
    const double h2 = g.h * g.h;
    const float2* rhs = A.rhs ? A.rhs + (long long)S.sys * n : nullptr;
    const double st = sin(S.angle);
    float2* r = A.B.r + soff;
    float2* rh = A.B.rh + soff;
    for (int k = threadIdx.x; k < nb * nx; k += blockDim.x) {
      const int i = z0 + k / nx, j = k % nx;
      const long long idx = (long long)i * nx + j;
      double2 b;
      if (rhs) {
        b = h2 * to_d(rhs[idx]);
      } else if (i == g.face) {
        double2 l = source_line(g, sc.k0, st, j);
        b = make_double2(-l.x, -l.y);
      } else {
        b = make_double2(0.0, 0.0);
      }
      const double2 ax = stencil<double, ADJ>(g, sc, i, j, __ldg(&cb[idx]), __ldg(&ct[idx]), P, Aa64);
      const double2 res = b - ax;
      xn[idx] = P(i, j);
      const float2 rf = to_f(res);
      r[idx] = rf;
      if (mode == MODE_INIT) {
        rh[idx] = rf;
        acc[0] += b.x * b.x + b.y * b.y;
        acc[1] += (double)rf.x * rf.x + (double)rf.y * rf.y;
      } else {
        acc[0] += (double)rf.x * rf.x + (double)rf.y * rf.y;
        dot_acc(acc[1], acc[2], rh[idx], rf);
      }
    }
  }
  reduce_and_finalize(A, S, slot, mode, acc);
}


__global__ void k_solve_init(SolveArgs A, int n_slots) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int s = tid; s < A.n_systems; s += gridDim.x * blockDim.x) {
    A.status[s] = NSR_NOT_RUN;
    A.iterations[s] = 0;
    A.residual[s] = NAN;
  }
  for (int s = tid; s < n_slots; s += gridDim.x * blockDim.x) {
    SlotState st;
    memset(&st, 0, sizeof(st));
    st.final_reason = -1;
    if (s < A.n_systems) {
      st.sys = s;
      st.mode = MODE_INIT;
      st.gidx = A.gain_index ? A.gain_index[s] : s;
      st.freq = A.freq[s];
      st.angle = A.angle ? A.angle[s] : 0.0;
      set_float_scalars(A.g, st);
    } else {
      st.sys = -1;
      st.mode = MODE_EMPTY;
    }
    A.B.slots[s] = st;
    A.B.arrive[s] = 0;
  }
  if (tid == 0) {
    *A.B.queue = min(A.n_systems, n_slots);
    *A.B.done = 0;
    A.B.warm[0] = 0;
    A.B.warm[1] = 0;
    *A.B.error = 0;
    *reinterpret_cast<unsigned long long*>(A.B.queue + 6) = 0ull;   // device-loop rounds
  }
}

// Last node of the device-side solve loop (the body of a conditional WHILE
// graph node): ends the loop once every system has finished, a kernel has
// reported an error, or the round budget (an upper bound on the rounds a full
// queue can need) is spent.
__global__ void k_loop_control(SolveArgs A, cudaGraphConditionalHandle loop, long long max_rounds) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long* rounds = reinterpret_cast<unsigned long long*>(A.B.queue + 6);
  const unsigned long long r = *rounds + 1;
  *rounds = r;
  const int done = *(volatile int*)A.B.done;
  const int error = *(volatile int*)A.B.error;
  if (done >= A.n_systems || error || r >= (unsigned long long)max_rounds) cudaGraphSetConditional(loop, 0);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
// Stencil CTAs per slot: two columns per thread on even widths (16-byte
// aligned rows), one column per thread otherwise.
static int stencil_ctas(const NsrGrid* g) {
  const int tx = (g->nx % 2 == 0) ? NSR_ST_TX : NSR_ST_TX1;
  return ((g->nz + NSR_ST_TZ - 1) / NSR_ST_TZ) * ((g->nx + tx - 1) / tx);
}

// Ring-staged stencil (k_stn): widths that are a multiple of 4 keep every
// bulk copy 16-byte aligned.
static bool stn_ok(const NsrGrid* g) { return g->nx % 4 == 0 && g->nx >= 8; }
#define NSR_STN_MIN_ROWS 4

// Stencil partials per slot of the finest allowed k_stn decomposition.
static int stn_items_max(const NsrGrid* g) {
  return ((g->nz + NSR_STN_MIN_ROWS - 1) / NSR_STN_MIN_ROWS) * ((g->nx + 255) / 256);
}

typedef void (*StnKernel)(SolveArgs, int, StnItems, int);

// Stencil kernel of one half for the shape (w, d, cpt): d is the second
// half's ring depth; the first half runs stn_depth0(d) of its smaller rows.
static StnKernel stn_kernel(int w, int d, int cpt, bool adj, int half) {
#define NSR_STN_CASE(W_, D_, C_)                                                                          \
  if (w == W_ && d == D_ && cpt == C_) {                                                                  \
    if (half) return adj ? k_stn<W_, D_, C_, true, 1> : k_stn<W_, D_, C_, false, 1>;                      \
    return adj ? k_stn<W_, stn_depth0<W_>(D_), C_, true, 0> : k_stn<W_, stn_depth0<W_>(D_), C_, false, 0>; \
  }
  NSR_STN_CASE(256, 4, 2) NSR_STN_CASE(256, 5, 2) NSR_STN_CASE(256, 6, 2) NSR_STN_CASE(512, 4, 2)
  NSR_STN_CASE(256, 4, 1)
#undef NSR_STN_CASE
  return nullptr;
}

static size_t stn_smem(int w, int d, int half) {
  if (w == 512) return half ? (size_t)d * StnLayout<512, 1>::SLOT : (size_t)stn_depth0<512>(d) * StnLayout<512, 0>::SLOT;
  return half ? (size_t)d * StnLayout<256, 1>::SLOT : (size_t)stn_depth0<256>(d) * StnLayout<256, 0>::SLOT;
}

// Launch shapes of one call: NsrTiles with zero fields replaced by defaults.
struct TileChoice {
  int sw, sd, sr, sctas, tc, rows, groups, scpt, cols_staged, rows_staged;
};

static int resolve_tiles(const NsrGrid* g, const NsrTiles* t, int n_slots, TileChoice* c) {
  c->sw = 256; c->sd = 4; c->sr = 64; c->sctas = 0; c->scpt = 2; c->cols_staged = 0; c->rows_staged = 0;
  c->tc = nsr_cols_tc(g);
  c->rows = nsr_rows_per_cta(g);
  c->groups = n_slots >= 8 ? 2 : 1;
  if (t) {
    if (t->stencil_width) c->sw = t->stencil_width;
    if (t->stencil_depth) c->sd = t->stencil_depth;
    if (t->stencil_rows) c->sr = t->stencil_rows;
    if (t->stencil_ctas) c->sctas = t->stencil_ctas;
    if (t->cols_width) c->tc = t->cols_width;
    if (t->row_tile) c->rows = t->row_tile;
    if (t->slot_groups) c->groups = t->slot_groups;
    if (t->stencil_cols) c->scpt = t->stencil_cols;
    c->cols_staged = t->cols_staged != 0;
    c->rows_staged = t->rows_staged != 0;
  }
  if (!stn_kernel(c->sw, c->sd, c->scpt, false, 1)) return NSR_ERR_ARGUMENT;
  if (c->sr < NSR_STN_MIN_ROWS || c->sr > 64 || c->sctas < 0 || c->sctas > 8) return NSR_ERR_ARGUMENT;
  if (!(c->tc == 8 || c->tc == 16) || (size_t)g->nz * c->tc * sizeof(float2) > 200 * 1024) return NSR_ERR_ARGUMENT;
  if (c->rows < 1 || c->rows > 8 || sizeof(float2) * (size_t)c->rows * nsr_row_stride(g->nx) > 200 * 1024)
    return NSR_ERR_ARGUMENT;
  if (c->groups < 1 || c->groups > NSR_MAX_GROUPS) return NSR_ERR_ARGUMENT;
  if (c->groups > n_slots) c->groups = n_slots;
  return 0;
}

static int band_rows(const NsrGrid* g) {
  int budget = g->nx <= 1024 ? 8192 : 16384;
  int tz = budget / g->nx - 2;
  if (tz < 1) tz = 1;
  if (tz > g->nz) tz = g->nz;
  return tz;
}

struct Layout {
  size_t tables, slots, arrive, queue, partials, vec, x, total;
  int nb_inv;
};

static Layout layout(const NsrGrid* g, int n_slots) {
  Layout L;
  const size_t n = (size_t)g->nz * g->nx;
  const int tz = band_rows(g);
  const int nb_res = (g->nz + tz - 1) / tz;
  int nb_st = stencil_ctas(g);
  if (stn_ok(g) && stn_items_max(g) > nb_st) nb_st = stn_items_max(g);
  L.nb_inv = nb_res > nb_st ? nb_res : nb_st;
  size_t off = 0;
  L.tables = off; off += nsr_align(nsr_prec_table_bytes(g));
  L.slots = off; off += nsr_align(sizeof(SlotState) * n_slots);
  L.arrive = off; off += nsr_align(sizeof(int) * n_slots);
  L.queue = off; off += nsr_align(sizeof(int) * 8);
  L.partials = off; off += nsr_align(sizeof(double) * NSR_NPART * (size_t)L.nb_inv * n_slots);
  L.vec = off; off += 8 * nsr_align(sizeof(float2) * n * n_slots);
  L.x = off; off += nsr_align(sizeof(double2) * n * 2 * n_slots);
  L.total = off;
  return L;
}

extern "C" size_t nsr_solve_workspace_size(const NsrGrid* grid, int32_t n_slots) {
  if (nsr_check_grid(grid, true) || n_slots <= 0 || n_slots > 65535) return 0;
  return layout(grid, n_slots).total;
}

// Pinned host word the solve loop polls; one per host thread, so that solves
// issued from different threads (e.g. one per device) do not share it.
static int* pinned_counter() {
  static thread_local int* p = nullptr;
  if (!p) {
    if (cudaHostAlloc((void**)&p, 8 * sizeof(int), cudaHostAllocDefault) != cudaSuccess) p = nullptr;
  }
  return p;
}

static int solve_impl(const NsrGrid* grid, const void* coef, const double* freq_hz, const double* angle_rad,
                      int32_t n_systems, const float* rhs, const float* x0, const int32_t* rx_index, int32_t n_rx,
                      const NsrSolveParams* params, void* workspace, size_t workspace_bytes, double* iq,
                      double* residual, int32_t* iterations, int32_t* status, void* fields, NsrSolveStats* stats,
                      void* stream, bool blocking) {
  int err = nsr_check_grid(grid, true);
  if (err) return err;
  if (!params || !coef || n_systems < 0 || n_rx < 0) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;   // an empty batch touches no buffer
  if (!freq_hz || (n_rx > 0 && !rx_index)) return NSR_ERR_ARGUMENT;
  if (!rhs && !angle_rad) return NSR_ERR_ARGUMENT;
  if (!iq && n_rx > 0) return NSR_ERR_ARGUMENT;
  if (!residual || !iterations || !status || !workspace) return NSR_ERR_ARGUMENT;
  const int n_slots = params->n_slots;
  if (n_slots <= 0 || n_slots > 65535 || params->max_iterations <= 0 || !(params->tolerance > 0) ||
      !(params->shift >= 0) || params->replace_every < 0 || !(params->restart_factor >= 0) ||
      params->restart_factor >= 1.0) return NSR_ERR_ARGUMENT;
  if (params->learned && !params->learned->params) return NSR_ERR_ARGUMENT;
  if (!(params->time_limit_s >= 0.0)) return NSR_ERR_ARGUMENT;
  TileChoice T;
  err = resolve_tiles(grid, params->tiles, n_slots, &T);
  if (err) return err;
  const Layout L = layout(grid, n_slots);
  if (workspace_bytes < L.total) return NSR_ERR_WORKSPACE;
  const size_t n = (size_t)grid->nz * grid->nx;
  cudaStream_t caller = (cudaStream_t)stream;

  // st runs slot group 0; sg[g] the other groups, forked from st and joined back
  cudaStream_t st = nullptr, sg[NSR_MAX_GROUPS] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[NSR_MAX_GROUPS] = {};
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_poll[2] = {nullptr, nullptr};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev_loop[2] = {nullptr, nullptr};
  cudaEvent_t* ev_prof = nullptr;
  int n_prof_events = 0;
  long long launches = 0;
  int graph_launches = 0;
  if (stats) memset(stats, 0, sizeof(*stats));
  if (!blocking && params->profile_iterations > 0) return NSR_ERR_ARGUMENT;   // event timings need the host
  int* host = blocking ? pinned_counter() : nullptr;
  if (blocking && !host) return (int)cudaErrorMemoryAllocation;
  cudaGraph_t loop_graph = nullptr;
  cudaError_t ce;
#define NSR_TRY(x) do { ce = (x); if (ce != cudaSuccess) { err = (int)ce; goto cleanup; } } while (0)
  {
    NSR_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (int g = 1; g < NSR_MAX_GROUPS; ++g) {
      NSR_TRY(cudaStreamCreateWithFlags(&sg[g], cudaStreamNonBlocking));
      NSR_TRY(cudaEventCreateWithFlags(&ev_join[g], cudaEventDisableTiming));
    }
    NSR_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    NSR_TRY(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    NSR_TRY(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
    NSR_TRY(cudaEventCreateWithFlags(&ev_poll[0], cudaEventDisableTiming));
    NSR_TRY(cudaEventCreateWithFlags(&ev_poll[1], cudaEventDisableTiming));
    NSR_TRY(cudaEventRecord(ev_in, caller));
    NSR_TRY(cudaStreamWaitEvent(st, ev_in, 0));
    err = nsr_check_learned(params->learned, n_systems, st);
    if (err) goto cleanup;

    char* ws = (char*)workspace;
    SolveArgs A;
    memset(&A, 0, sizeof(A));
    A.g = make_geo(*grid);
    err = nsr_prec_setup(grid, &A.tab, ws + L.tables, st);
    if (err) goto cleanup;
    A.B.slots = (SlotState*)(ws + L.slots);
    A.B.arrive = (int*)(ws + L.arrive);
    A.B.queue = (int*)(ws + L.queue);
    A.B.done = A.B.queue + 1;
    A.B.warm = A.B.queue + 2;
    A.B.error = A.B.queue + 4;
    A.B.partials = (double*)(ws + L.partials);
    const size_t vb = nsr_align(sizeof(float2) * n * n_slots);
    float2** vecs[8] = {&A.B.r, &A.B.rh, &A.B.p, &A.B.v, &A.B.t, &A.B.y, &A.B.w, &A.B.sym};
    for (int q = 0; q < 8; ++q) *vecs[q] = (float2*)(ws + L.vec + q * vb);
    A.B.x = (double2*)(ws + L.x);
    A.mat = nsr_planes(coef, (long long)grid->nz * grid->nx);
    A.freq = freq_hz;
    A.angle = rhs ? nullptr : angle_rad;
    A.rhs = (const float2*)rhs;
    A.x0 = (const float2*)x0;
    A.rx = rx_index;
    A.n_rx = n_rx;
    A.n_systems = n_systems;
    A.rows = T.rows;
    A.tc = T.tc;
    A.tz = band_rows(grid);
    A.nb_inv = L.nb_inv;
    A.tol2 = params->tolerance * params->tolerance;
    A.restart2 = params->restart_factor * params->restart_factor;
    A.warm_gate2 = params->warm_gate > 0.0 ? params->warm_gate * params->warm_gate : 0.0;
    A.shift = params->shift;
    A.max_it = params->max_iterations;
    A.replace_every = params->replace_every;
    A.adjoint = params->adjoint;
    A.time_limit_ns = params->time_limit_s > 0.0 ? (unsigned long long)(params->time_limit_s * 1e9) : 0ull;
    A.iq = (double2*)iq;
    A.residual = residual;
    A.iterations = iterations;
    A.status = status;
    A.fields = fields;
    A.fields_fp64 = params->fields_fp64 ? 1 : 0;
    if (params->learned) {
      A.lp = params->learned->params;
      A.gains = (const float2*)params->learned->gains;
      A.gain_index = params->learned->gain_index;
    }

    const size_t fwd_smem = sizeof(float2) * A.rows * nsr_row_stride(grid->nx);
    const size_t col_smem = nsr_cols_smem(grid);
    const int nb_res = (grid->nz + A.tz - 1) / A.tz;
    const int nb_st = stencil_ctas(grid);
    const bool pairs = grid->nx % 2 == 0;
    const bool use_stn = stn_ok(grid);
    const StnKernel stn_fn[2] = {stn_kernel(T.sw, T.sd, T.scpt, A.adjoint != 0, 0),
                                 stn_kernel(T.sw, T.sd, T.scpt, A.adjoint != 0, 1)};
    const int stn_threads = T.sw / T.scpt + 32;
    const size_t stn_sm[2] = {stn_smem(T.sw, T.sd, 0), stn_smem(T.sw, T.sd, 1)};
    int stn_per_sm[2] = {T.sctas, T.sctas};
    int n_sms = 1;
    {
      int dev = 0;
      NSR_TRY(cudaGetDevice(&dev));
      NSR_TRY(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    if (use_stn) {
      for (int h = 0; h < 2; ++h) {
        NSR_TRY(cudaFuncSetAttribute((const void*)stn_fn[h], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)stn_sm[h]));
        if (stn_per_sm[h] <= 0) {
          NSR_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&stn_per_sm[h], (const void*)stn_fn[h], stn_threads,
                                                                stn_sm[h]));
          if (stn_per_sm[h] < 1) { err = NSR_ERR_ARGUMENT; goto cleanup; }
        }
      }
    }
    // row kernels: direct (specialised widths) or staged through shared memory
    const bool direct_rows = nsr_row_padded(grid->nx) && !T.rows_staged;
    typedef void (*RowKernel)(SolveArgs, int);
    const RowKernel fwd_fn = direct_rows ? k_fwd<true> : k_fwd<false>;
    const RowKernel rinv_fn = direct_rows ? k_rinv<true> : k_rinv<false>;
    NSR_TRY(cudaFuncSetAttribute((const void*)fwd_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem));
    // column kernel: transform tile width, learned or fixed multiplier, direct
    // (specialised sizes) or staged through shared memory
    typedef void (*ColsKernel)(SolveArgs, int);
    const bool generic_cols = !nsr_row_padded(grid->nz) || T.cols_staged;
    ColsKernel cols_fn = nullptr;
#define NSR_COLS_PICK(TC_, L_) \
    if (A.tc == TC_ && (A.lp != nullptr) == L_) cols_fn = generic_cols ? k_cols<TC_, L_, true> : k_cols<TC_, L_, false>;
    NSR_COLS_PICK(16, false) NSR_COLS_PICK(8, false) NSR_COLS_PICK(16, true) NSR_COLS_PICK(8, true)
#undef NSR_COLS_PICK
    if (!cols_fn) { err = NSR_ERR_ARGUMENT; goto cleanup; }
    NSR_TRY(cudaFuncSetAttribute((const void*)cols_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)col_smem));
    NSR_TRY(cudaFuncSetAttribute((const void*)rinv_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem));

    k_solve_init<<<64, 256, 0, st>>>(A, n_slots);
    NSR_TRY(cudaGetLastError());
    launches = 3;  // two table kernels and the slot initialisation

    // The slots run as independent groups on branches of the captured graph,
    // so that one group's kernels fill the tail waves of the others'.
    const int n_groups = T.groups;
    int g_first[NSR_MAX_GROUPS] = {}, g_count[NSR_MAX_GROUPS] = {};
    for (int g = 0, first = 0; g < n_groups; ++g) {
      g_first[g] = first;
      g_count[g] = n_slots / n_groups + (g < n_slots % n_groups ? 1 : 0);
      first += g_count[g];
    }
    const int K = params->graph_iterations > 0 ? params->graph_iterations : 16;
    // One iteration = 9 launches: fwd, cols, rinv, inv of the first half, then
    // fwd, cols, rinv, res, inv of the second half.
    const int seq_half[NSR_LAUNCHES_PER_IT] = {0, 0, 0, 0, 1, 1, 1, 1, 1};
    const int seq_kind[NSR_LAUNCHES_PER_IT] = {0, 1, 4, 3, 0, 1, 4, 2, 3};
    auto launch = [&](int q, int grp, cudaStream_t sq) {
      const int half = seq_half[q], which = seq_kind[q];
      SolveArgs Ag = A;
      Ag.slot0 = g_first[grp];
      const int ns = g_count[grp];
      // Slots run fastest: the CTAs of one tile of every slot run together, so a
      // gain plane that several slots share (systems of one frequency) is read
      // once from HBM and then from L2.
      const dim3 g_fwd(ns, (grid->nz + A.rows - 1) / A.rows);
      const dim3 g_col(ns, (grid->nx + A.tc - 1) / A.tc);
      const dim3 g_inv(nb_st, ns);
      const dim3 g_res(nb_res, ns);
      if (which == 0) {
        int hv = half;
        void* args[] = {&Ag, &hv};
        cudaLaunchKernel((const void*)fwd_fn, g_fwd, dim3(256), args, fwd_smem, sq);
      } else if (which == 1) {
        int hv = half;
        void* args[] = {&Ag, &hv};
        cudaLaunchKernel((const void*)cols_fn, g_col, dim3(512), args, col_smem, sq);
      } else if (which == 2) {
        if (A.adjoint) k_res<true><<<g_res, 256, 0, sq>>>(Ag);
        else k_res<false><<<g_res, 256, 0, sq>>>(Ag);
      } else if (which == 3 && use_stn) {
        StnItems si;
        si.tz = T.sr;
        si.nbands = (grid->nz + T.sr - 1) / T.sr;
        si.nstrips = (grid->nx + T.sw - 1) / T.sw;
        si.per_slot = si.nbands * si.nstrips;
        si.n_items = ns * si.per_slot;
        int hv = half, nsv = ns;
        const int gx = si.n_items < stn_per_sm[half] * n_sms ? si.n_items : stn_per_sm[half] * n_sms;
        void* args[] = {&Ag, &hv, &si, &nsv};
        cudaLaunchKernel((const void*)stn_fn[half], dim3(gx), dim3(stn_threads), args, stn_sm[half], sq);
      } else if (which == 3) {
        if (pairs) {
          if (A.adjoint) k_inv<true><<<g_inv, 256, 0, sq>>>(Ag, half);
          else k_inv<false><<<g_inv, 256, 0, sq>>>(Ag, half);
        } else {
          if (A.adjoint) k_inv1<true><<<g_inv, 256, 0, sq>>>(Ag, half);
          else k_inv1<false><<<g_inv, 256, 0, sq>>>(Ag, half);
        }
      } else {
        int hv = half;
        void* args[] = {&Ag, &hv};
        cudaLaunchKernel((const void*)rinv_fn, g_fwd, dim3(256), args, fwd_smem, sq);
      }
    };

    NSR_TRY(cudaEventCreate(&ev_loop[0]));
    NSR_TRY(cudaEventCreate(&ev_loop[1]));
    NSR_TRY(cudaEventRecord(ev_loop[0], st));
    // Profiled iterations: launched one by one with an event between kernels.
    int P = params->profile_iterations;
    if (P < 0) P = 0;
    if (P > 256) P = 256;
    if (P > 0) {
      n_prof_events = NSR_LAUNCHES_PER_IT * P + 1;
      ev_prof = (cudaEvent_t*)calloc(n_prof_events, sizeof(cudaEvent_t));
      if (!ev_prof) { err = (int)cudaErrorMemoryAllocation; goto cleanup; }
      for (int e = 0; e < n_prof_events; ++e) NSR_TRY(cudaEventCreate(&ev_prof[e]));
      NSR_TRY(cudaEventRecord(ev_prof[0], st));
      // Both slot groups of a kernel between two events, running side by side
      // as in the captured iterations: the durations cover every resident system.
      for (int it = 0; it < P; ++it)
        for (int q = 0; q < NSR_LAUNCHES_PER_IT; ++q) {
          const int e = it * NSR_LAUNCHES_PER_IT + q;
          for (int g = 1; g < n_groups; ++g) NSR_TRY(cudaStreamWaitEvent(sg[g], ev_prof[e], 0));
          launch(q, 0, st);
          for (int g = 1; g < n_groups; ++g) {
            launch(q, g, sg[g]);
            NSR_TRY(cudaEventRecord(ev_join[g], sg[g]));
            NSR_TRY(cudaStreamWaitEvent(st, ev_join[g], 0));
          }
          NSR_TRY(cudaGetLastError());
          NSR_TRY(cudaEventRecord(ev_prof[e + 1], st));
        }
      launches += (long long)NSR_LAUNCHES_PER_IT * P * n_groups;
    }

    // Each system needs at most max_it iterations plus its replacement,
    // init and emit half-iterations; bound the number of graph rounds.
    const long long per_sys = (long long)params->max_iterations * 2 + 16;
    const long long waves = (n_systems + n_slots - 1) / n_slots + 1;
    const long long max_launch = waves * ((per_sys + K - 1) / K) + 4;
    // The K iterations of one round, captured from both slot-group streams.
    auto capture_round = [&]() -> cudaError_t {
      cudaError_t e = cudaSuccess;
      if (n_groups > 1 && (e = cudaEventRecord(ev_fork, st)) != cudaSuccess) return e;
      for (int g = 1; g < n_groups; ++g)
        if ((e = cudaStreamWaitEvent(sg[g], ev_fork, 0)) != cudaSuccess) return e;
      for (int it = 0; it < K; ++it)
        for (int q = 0; q < NSR_LAUNCHES_PER_IT; ++q)
          for (int g = 0; g < n_groups; ++g) launch(q, g, g ? sg[g] : st);
      for (int g = 1; g < n_groups; ++g) {
        if ((e = cudaEventRecord(ev_join[g], sg[g])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(st, ev_join[g], 0)) != cudaSuccess) return e;
      }
      return cudaGetLastError();
    };

    if (!blocking) {
      // Device-side loop: a conditional WHILE node whose body is one round
      // followed by k_loop_control, so the whole solve is one graph launch
      // on the stream and the host returns at once.
      cudaGraphConditionalHandle handle;
      NSR_TRY(cudaGraphCreate(&loop_graph, 0));
      NSR_TRY(cudaGraphConditionalHandleCreate(&handle, loop_graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
      cp.conditional.handle = handle;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t while_node;
      NSR_TRY(cudaGraphAddNode(&while_node, loop_graph, nullptr, 0, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      NSR_TRY(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
      ce = capture_round();
      if (ce == cudaSuccess) {
        k_loop_control<<<1, 32, 0, st>>>(A, handle, max_launch);
        ce = cudaGetLastError();
      }
      cudaGraph_t captured = nullptr;
      const cudaError_t ce2 = cudaStreamEndCapture(st, &captured);
      if (ce == cudaSuccess) ce = ce2;
      if (ce != cudaSuccess) { err = (int)ce; goto cleanup; }
      NSR_TRY(cudaGraphInstantiate(&exec, loop_graph, 0));
      NSR_TRY(cudaGraphLaunch(exec, st));
      graph_launches = 1;   // the rounds it runs are in the progress record
      if (stats) {
        stats->launches = launches;
        stats->graph_launches = graph_launches;
      }
      NSR_TRY(cudaEventRecord(ev_out, st));
      NSR_TRY(cudaStreamWaitEvent(caller, ev_out, 0));
      goto cleanup;
    }

    NSR_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    ce = capture_round();
    {
      const cudaError_t ce2 = cudaStreamEndCapture(st, &graph);
      if (ce == cudaSuccess) ce = ce2;
    }
    if (ce != cudaSuccess) { err = (int)ce; goto cleanup; }
    NSR_TRY(cudaGraphInstantiate(&exec, graph, 0));

    long long launched = 0;
    bool drained = false, failed = false;
    int pending = -1;
    while (launched < max_launch) {
      NSR_TRY(cudaGraphLaunch(exec, st));
      ++graph_launches;
      launches += (long long)NSR_LAUNCHES_PER_IT * K * n_groups;
      const int slot_i = (int)(launched & 1);
      // done, warm[2], error
      NSR_TRY(cudaMemcpyAsync(&host[4 * slot_i], A.B.done, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
      NSR_TRY(cudaEventRecord(ev_poll[slot_i], st));
      ++launched;
      if (pending >= 0) {
        NSR_TRY(cudaEventSynchronize(ev_poll[pending]));
        if (host[4 * pending + 3]) { failed = true; break; }
        if (host[4 * pending] >= n_systems) { drained = true; break; }
      }
      pending = slot_i;
    }
    if (!drained && !failed && pending >= 0) {
      NSR_TRY(cudaEventSynchronize(ev_poll[pending]));
      failed = host[4 * pending + 3] != 0;
      drained = host[4 * pending] >= n_systems;
    }
    NSR_TRY(cudaEventRecord(ev_loop[1], st));
    NSR_TRY(cudaStreamSynchronize(st));
    if (failed) err = NSR_ERR_TIMEOUT;
    else if (!drained) err = NSR_ERR_INTERNAL;
    if (stats) {
      int warm_host[2] = {0, 0};
      NSR_TRY(cudaMemcpyAsync(warm_host, A.B.warm, sizeof(warm_host), cudaMemcpyDeviceToHost, st));
      NSR_TRY(cudaStreamSynchronize(st));
      stats->warm_accepted = warm_host[0];
      stats->warm_rejected = warm_host[1];
      float ms = 0.f;
      NSR_TRY(cudaEventElapsedTime(&ms, ev_loop[0], ev_loop[1]));
      stats->loop_ms = ms;
      stats->launches = launches;
      stats->graph_launches = graph_launches;
      // Skip the first two profiled iterations (slot initialisation).
      for (int it = (P > 2 ? 2 : 0); it < P; ++it)
        for (int k = 0; k < NSR_LAUNCHES_PER_IT; ++k) {
          float d = 0.f;
          NSR_TRY(cudaEventElapsedTime(&d, ev_prof[it * NSR_LAUNCHES_PER_IT + k],
                                       ev_prof[it * NSR_LAUNCHES_PER_IT + k + 1]));
          stats->kernel_ms[k] += d;
          stats->kernel_timed[k] += 1;
        }
      for (int k = 0; k < NSR_LAUNCHES_PER_IT; ++k)
        if (stats->kernel_timed[k]) stats->kernel_ms[k] /= stats->kernel_timed[k];
    }
    NSR_TRY(cudaEventRecord(ev_out, st));
    NSR_TRY(cudaStreamWaitEvent(caller, ev_out, 0));
  }
cleanup:
  // A non-blocking call that enqueued its loop leaves the work in flight:
  // graph, streams and events are then released by CUDA once it completes.
  if (blocking || err) {
    if (st) cudaStreamSynchronize(st);
    for (int g = 1; g < NSR_MAX_GROUPS; ++g)
      if (sg[g]) cudaStreamSynchronize(sg[g]);
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (loop_graph) cudaGraphDestroy(loop_graph);
  if (ev_in) cudaEventDestroy(ev_in);
  if (ev_out) cudaEventDestroy(ev_out);
  if (ev_poll[0]) cudaEventDestroy(ev_poll[0]);
  if (ev_poll[1]) cudaEventDestroy(ev_poll[1]);
  if (ev_loop[0]) cudaEventDestroy(ev_loop[0]);
  if (ev_loop[1]) cudaEventDestroy(ev_loop[1]);
  if (ev_prof) {
    for (int e = 0; e < n_prof_events; ++e)
      if (ev_prof[e]) cudaEventDestroy(ev_prof[e]);
    free(ev_prof);
  }
  if (st) cudaStreamDestroy(st);
  for (int g = 1; g < NSR_MAX_GROUPS; ++g) {
    if (sg[g]) cudaStreamDestroy(sg[g]);
    if (ev_join[g]) cudaEventDestroy(ev_join[g]);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
#undef NSR_TRY
  return err;
}

extern "C" int nsr_solve_batched(const NsrGrid* grid, const void* coef, const double* freq_hz,
                                 const double* angle_rad, int32_t n_systems, const float* rhs, const float* x0,
                                 const int32_t* rx_index, int32_t n_rx, const NsrSolveParams* params,
                                 void* workspace, size_t workspace_bytes, double* iq, double* residual,
                                 int32_t* iterations, int32_t* status, void* fields, NsrSolveStats* stats,
                                 void* stream) {
  return solve_impl(grid, coef, freq_hz, angle_rad, n_systems, rhs, x0, rx_index, n_rx, params, workspace,
                    workspace_bytes, iq, residual, iterations, status, fields, stats, stream, false);
}

extern "C" int nsr_solve_batched_sync(const NsrGrid* grid, const void* coef, const double* freq_hz,
                                      const double* angle_rad, int32_t n_systems, const float* rhs,
                                      const float* x0, const int32_t* rx_index, int32_t n_rx,
                                      const NsrSolveParams* params, void* workspace, size_t workspace_bytes,
                                      double* iq, double* residual, int32_t* iterations, int32_t* status,
                                      void* fields, NsrSolveStats* stats, void* stream) {
  return solve_impl(grid, coef, freq_hz, angle_rad, n_systems, rhs, x0, rx_index, n_rx, params, workspace,
                    workspace_bytes, iq, residual, iterations, status, fields, stats, stream, true);
}

extern "C" size_t nsr_solve_progress_offset(const NsrGrid* grid, int32_t n_slots) {
  if (nsr_check_grid(grid, true) || n_slots <= 0 || n_slots > 65535) return 0;
  return layout(grid, n_slots).queue;
}

extern "C" int nsr_solve_progress(const NsrGrid* grid, int32_t n_slots, const void* workspace, int32_t* done,
                                  int64_t* rounds, int32_t* error, void* stream) {
  if (nsr_check_grid(grid, true) || n_slots <= 0 || n_slots > 65535 || !workspace) return NSR_ERR_ARGUMENT;
  const Layout L = layout(grid, n_slots);
  int words[8];
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t ce = cudaMemcpyAsync(words, (const char*)workspace + L.queue, sizeof(words), cudaMemcpyDeviceToHost,
                                   st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
  if (ce != cudaSuccess) return (int)ce;
  unsigned long long r;
  memcpy(&r, &words[6], sizeof(r));
  if (done) *done = words[1];
  if (rounds) *rounds = (int64_t)r;
  if (error) *error = words[4];
  return 0;
}
