// Allocation-free variant of nsr_precondition.
//
// Some callers cannot allocate device memory at the point where they need the
// preconditioner: code that runs while another framework is capturing a CUDA
// graph (an allocation there breaks or invalidates the capture), pipelines
// with hard latency budgets (cudaMalloc can synchronise the whole device), and
// plug-ins whose host application owns every device allocation.  For them the
// scratch space of the preconditioner (FFT tables and the transformed fields)
// lives in a fixed file-scope device array instead of a caller workspace.
#include "nsr_internal.cuh"

#include <cuda.h>
#include <mutex>

// 16 MiB: tables plus two 1024 x 768 complex64 fields, or 32 fields of 256 x 256.
#define NSR_STATIC_SCRATCH_BYTES ((size_t)16 << 20)
#define NSR_STATIC_MAX_CONTEXTS 64

// Reserved on each device where this module is loaded (with CUDA's lazy module
// loading, at the first use of nsr_precondition_noalloc on that device) and
// held until the context is destroyed or the process exits.
static __device__ __align__(256) unsigned char g_prec_scratch[NSR_STATIC_SCRATCH_BYTES];

namespace {
typedef CUresult (CUDAAPI* CtxCurrentFn)(CUcontext*);
typedef CUresult (CUDAAPI* CtxIdFn)(CUcontext, unsigned long long*);

std::mutex g_scratch_mutex;
CtxCurrentFn g_ctx_current = nullptr;
CtxIdFn g_ctx_id = nullptr;
bool g_entry_points_tried = false;
// (context id, device address of g_prec_scratch in that context)
unsigned long long g_cache_id[NSR_STATIC_MAX_CONTEXTS] = {0};
void* g_cache_addr[NSR_STATIC_MAX_CONTEXTS] = {nullptr};
int g_cache_next = 0;

// Unique id of the context current on this thread (never reused within the
// process, so a context created after cudaDeviceReset gets a new one); 0 when
// no context is current or the driver cannot say.
unsigned long long current_context_id() {
  if (!g_entry_points_tried) {
    g_entry_points_tried = true;
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &fn, 4000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_current = (CtxCurrentFn)fn;
    fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &fn, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_id = (CtxIdFn)fn;
  }
  if (!g_ctx_current || !g_ctx_id) return 0;
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  unsigned long long id = 0;
  if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_prec_scratch in the current context.  In host code the
// symbol name is only a host-side handle, so the address is looked up with
// the device current (cudaGetSymbolAddress) and cached per CUDA context: the
// module, and with it the array, can sit at another address in another
// context of the same device or after cudaDeviceReset.
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return (int)ce;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  unsigned long long id = current_context_id();
  if (id != 0) {
    for (int k = 0; k < NSR_STATIC_MAX_CONTEXTS; ++k)
      if (g_cache_id[k] == id) { *out = g_cache_addr[k]; return 0; }
  }
  void* p = nullptr;
  ce = cudaGetSymbolAddress(&p, g_prec_scratch);   // makes the device's primary context current if none is
  if (ce != cudaSuccess) return (int)ce;
  if (id == 0) id = current_context_id();
  if (id != 0) {
    g_cache_id[g_cache_next] = id;
    g_cache_addr[g_cache_next] = p;
    g_cache_next = (g_cache_next + 1) % NSR_STATIC_MAX_CONTEXTS;
  }
  *out = p;
  return 0;
}
}  // namespace

extern "C" int nsr_precondition_noalloc(const NsrGrid* grid, const double* freq_hz, int32_t n_systems,
                                        double shift, int32_t adjoint, const float* x, float* y, void* stream) {
  int err = nsr_check_grid(grid, true);
  if (err) return err;
  if (!freq_hz || !x || !y || n_systems < 0 || n_systems > 65535) return NSR_ERR_ARGUMENT;
  if (n_systems == 0) return 0;
  const size_t need = nsr_precondition_workspace_size(grid, n_systems);
  if (need == 0) return NSR_ERR_ARGUMENT;
  if (need > NSR_STATIC_SCRATCH_BYTES) return NSR_ERR_CAPACITY;
  void* scratch = nullptr;
  err = scratch_address(&scratch);
  if (err) return err;
  // The tables are rewritten and every transformed field is fully written by
  // the row pass before it is read, so no part of the array needs clearing.
  return nsr_precondition(grid, freq_hz, n_systems, shift, adjoint, x, y, scratch, NSR_STATIC_SCRATCH_BYTES,
                          stream);
}
