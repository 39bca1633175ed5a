// Allocation-free dot products.
//
// ddx_pcg_dots_rz needs two caller-allocated scratch buffers (per-CTA partial
// sums and an arrival ticket). Some callers cannot allocate device memory at
// the point where they need a dot product: hosts that reach this library
// through a plain C FFI with no device allocator of their own, and real-time
// loops that must not touch the allocator after start-up.
// ddx_dot_noalloc gives them the same deterministic reduction with the scratch
// in a fixed array inside this library instead.
#include <atomic>

#include "common.cuh"

namespace ddx {
namespace {

constexpr int kNoAllocMaxR = 64;

// One partial per CTA and right-hand side, plus the arrival ticket:
// 592 * 64 doubles + one counter, about 296 KiB. Every GPU that loads the
// library keeps this array until the process exits.
struct DotScratch {
  double partials[(size_t)kRedCtas * kNoAllocMaxR];
  unsigned int ticket;
};

static __device__ __align__(256) DotScratch g_dot_scratch;

constexpr int kMaxDevices = 64;
std::atomic<DotScratch*> g_scratch_addr[kMaxDevices];

// out[j] = sum_i x[i*R + j] * y[i*R + j]; the same fixed-order two-stage
// reduction as k_dots_rz (CTA tree, then the last CTA sums the CTA partials).
__global__ void __launch_bounds__(kThreads) k_dot_noalloc(int64_t n, int R, const double* __restrict__ x,
                                                          const double* __restrict__ y, double* __restrict__ out,
                                                          DotScratch* s) {
  __shared__ double red[kThreads];
  const int64_t total = n * R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double acc[1] = {0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
    acc[0] = fma(x[i], y[i], acc[0]);
  write_cta_partials<1>(acc, red, R, s->partials);
  if (!last_cta_arrival(&s->ticket)) return;
  double tot[1];
  final_sums<1>(s->partials, R, red, tot, &s->ticket);
  if (threadIdx.x < R) out[threadIdx.x] = tot[0];
}

// Device address of the scratch array for the current device, looked up once
// per device (cudaGetSymbolAddress with that device current) and kept for the
// process: a cudaDeviceReset unloads the module, after which the process must
// restart before calling ddx_dot_noalloc again.
int scratch_for_current_device(DotScratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("ddx_dot_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return DDX_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("ddx_dot_noalloc: device %d beyond the %d supported", dev, kMaxDevices);
    return DDX_ERR_UNSUPPORTED;
  }
  DotScratch* p = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (p == nullptr) {
    void* addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_dot_scratch);
    if (e != cudaSuccess || addr == nullptr) {
      set_error("ddx_dot_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev, cudaGetErrorString(e));
      return DDX_ERR_CUDA;
    }
    p = static_cast<DotScratch*>(addr);
    g_scratch_addr[dev].store(p, std::memory_order_release);
  }
  *out = p;
  return DDX_OK;
}

}  // namespace
}  // namespace ddx

using namespace ddx;

extern "C" int ddx_dot_noalloc(int64_t n, int R, const double* x, const double* y, double* out,
                               ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R) && R <= kNoAllocMaxR,
              "ddx_dot_noalloc: R=%d is not supported (1, 2, 4, ..., %d right-hand sides)", R, kNoAllocMaxR);
  DDX_REQUIRE(n >= 0, "ddx_dot_noalloc: n < 0");
  DDX_REQUIRE(x && y && out, "ddx_dot_noalloc: null pointer");
  DotScratch* s = nullptr;
  int st = scratch_for_current_device(&s);
  if (st != DDX_OK) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  // The ticket must start at zero; a call cut short earlier could have left it set.
  cudaError_t e = cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned int), cs);
  if (e != cudaSuccess) {
    set_error("ddx_dot_noalloc: clearing the ticket failed: %s", cudaGetErrorString(e));
    return DDX_ERR_CUDA;
  }
  k_dot_noalloc<<<red_grid(n * R), kThreads, 0, cs>>>(n, R, x, y, out, s);
  DDX_LAUNCH_CHECK("ddx_dot_noalloc");
  return DDX_OK;
}
