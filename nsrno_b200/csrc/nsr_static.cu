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

#include <mutex>

// 16 MiB: tables plus two 1024 x 768 complex64 fields, or 32 fields of 256 x 256.
#define NSR_STATIC_SCRATCH_BYTES ((size_t)16 << 20)
#define NSR_STATIC_MAX_DEVICES 64

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_prec_scratch[NSR_STATIC_SCRATCH_BYTES];

namespace {
std::mutex g_scratch_mutex;
void* g_scratch_addr[NSR_STATIC_MAX_DEVICES] = {nullptr};

// Device address of g_prec_scratch on the current device.  In host code the
// symbol name is only a host-side handle, so the address is looked up once
// per device, with that device current, and cached.
int scratch_address(void** out) {
  int dev = -1;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess) return (int)ce;
  if (dev < 0 || dev >= NSR_STATIC_MAX_DEVICES) return NSR_ERR_CAPACITY;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    ce = cudaGetSymbolAddress(&p, g_prec_scratch);
    if (ce != cudaSuccess) return (int)ce;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
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
