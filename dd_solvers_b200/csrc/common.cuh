// Shared device/host helpers for the ddx library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <stdio.h>

#include <type_traits>

#include "../../include/ddx.h"

namespace ddx {

// ---------------------------------------------------------------------------
// Error reporting: every C entry point returns a status and records a message
// retrievable with ddx_last_error() (thread-local).
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);

#define DDX_REQUIRE(cond, ...)                 \
  do {                                         \
    if (!(cond)) {                             \
      ::ddx::set_error(__VA_ARGS__);           \
      return DDX_ERR_ARG;                      \
    }                                          \
  } while (0)

#define DDX_LAUNCH_CHECK(name)                                                     \
  do {                                                                             \
    cudaError_t e_ = cudaGetLastError();                                           \
    if (e_ != cudaSuccess) {                                                       \
      ::ddx::set_error("%s: launch failed: %s", name, cudaGetErrorString(e_));     \
      return DDX_ERR_CUDA;                                                         \
    }                                                                              \
  } while (0)

constexpr int kThreads = 256;   // block size of every reducing kernel
constexpr int kRedCtas = 592;   // 148 SMs x 4: max grid of a reducing kernel
constexpr int kMaxNV = 4;       // max partial sums per RHS in one reduction

// Device error word (bounded-wait timeouts); read by ddx_device_error().
extern __device__ int g_device_error;
enum { DEVERR_MBAR_TIMEOUT = 1, DEVERR_BAD_SIZE = 2 };

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

inline bool valid_rhs_count(int R) {
  return R == 1 || R == 2 || R == 4 || R == 8 || R == 16 || R == 32 || R == 64;
}

inline int red_grid(int64_t work_items) {
  int64_t g = ceil_div(work_items, kThreads);
  if (g < 1) g = 1;
  if (g > kRedCtas) g = kRedCtas;
  return (int)g;
}

// Grid for a grid-stride kernel: at most the CTAs that are resident at once on
// this device (SM count x occupancy of `kernel` at kThreads threads), at most
// `cap`, at least 1, at most `need`.
template <typename Kernel>
inline int resident_grid(Kernel kernel, int64_t need, int64_t cap) {
  int dev = 0, nsm = 1, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  int64_t g = (int64_t)per_sm * nsm;
  if (g > cap) g = cap;
  if (g > need) g = need;
  return (int)(g < 1 ? 1 : g);
}

// ---------------------------------------------------------------------------
// Value conversions
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ float to_f32(T v);
template <> __device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }

// 16-bit conversions of the tensor-core B panels (through FP32, round to nearest)
template <typename T> __device__ __forceinline__ uint16_t to_bits(double v);
template <> __device__ __forceinline__ uint16_t to_bits<__nv_bfloat16>(double v) {
  return __bfloat16_as_ushort(__float2bfloat16_rn((float)v));
}
template <> __device__ __forceinline__ uint16_t to_bits<__half>(double v) {
  return __half_as_ushort(__float2half_rn((float)v));
}
template <typename T> __device__ __forceinline__ double from_bits(uint16_t b);
template <> __device__ __forceinline__ double from_bits<__nv_bfloat16>(uint16_t b) {
  return (double)__bfloat162float(__ushort_as_bfloat16(b));
}
template <> __device__ __forceinline__ double from_bits<__half>(uint16_t b) {
  return (double)__half2float(__ushort_as_half(b));
}


// Power-of-two scale applied to RHS j of r before the 16-bit conversion, from
// the PCG's current ||r_j||^2 (1 without PCG state): ||s r_j|| lands in
// [2^(top-1), 2^top) with top = 14 for FP16 (every entry stays below 2^14, far
// from the FP16 maximum 65504, while entries down to ~2^-10 ||r_j|| keep full
// precision instead of falling into FP16 subnormals) and top = 0 for BF16,
// whose exponent range needs no help.
template <typename T>
__device__ __forceinline__ float rhs_scale(const double* st, int R, int j) {
  if (st == nullptr) return 1.0f;
  const double rr = st[DDX_ST_RR * R + j];
  if (!(rr > 0.0) || !(rr < 1e300)) return 1.0f;
  int e;
  frexp(sqrt(rr), &e);  // sqrt(rr) in [2^(e-1), 2^e)
  e = max(-100, min(100, e));
  constexpr int top = std::is_same<T, __half>::value ? 14 : 0;
  return ldexpf(1.0f, top - e);
}

// ---------------------------------------------------------------------------
// Deterministic reductions.
//
// A fused kernel accumulates NV per-RHS partial sums in fixed thread order,
// reduces them inside the CTA in a fixed tree, and writes one partial per CTA
// to partials[(cta * NV + v) * R + j]. The CTA that arrives last (ticket
// counter) sums the per-CTA partials in a fixed order and runs the finalize
// step. The order of every floating-point addition is fixed by the launch
// shape, so repeated runs are bitwise identical. The ticket resets itself, so
// the kernel can be replayed from a CUDA graph.
// ---------------------------------------------------------------------------

// Sum `val` over the threads of the CTA that share the column tid % R (R a
// power of two dividing blockDim). Result valid in threads tid < R.
__device__ __forceinline__ double block_sum_by_col(double val, double* red, int R) {
  const int tid = threadIdx.x;
  red[tid] = val;
  __syncthreads();
  for (int s = blockDim.x >> 1; s >= R; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  double out = red[tid];
  __syncthreads();
  return out;
}

template <int NV>
__device__ __forceinline__ void write_cta_partials(const double (&v)[NV], double* red, int R,
                                                   double* partials) {
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = block_sum_by_col(v[k], red, R);
    if (threadIdx.x < R) partials[((size_t)blockIdx.x * NV + k) * R + threadIdx.x] = s;
  }
}

// True in exactly one CTA, the last to arrive; it then sees all partials.
__device__ __forceinline__ bool last_cta_arrival(unsigned int* ticket) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// In the last CTA: totals over all CTAs, valid in threads tid < R (column tid).
// Resets the ticket.
template <int NV>
__device__ __forceinline__ void final_sums(const double* partials, int R, double* red,
                                           double (&out)[NV], unsigned int* ticket) {
  const int t = threadIdx.x;
  const int j = t % R, g = t / R, G = blockDim.x / R;
  const int ncta = gridDim.x;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double acc = 0.0;
    for (int c = g; c < ncta; c += G) acc += __ldcg(partials + ((size_t)c * NV + v) * R + j);
    out[v] = block_sum_by_col(acc, red, R);
  }
  if (t == 0) *ticket = 0u;
}

// ---------------------------------------------------------------------------
// PCG state accessors (layout documented in ddx.h)
// ---------------------------------------------------------------------------
struct PcgState {
  double* st;
  int* ist;
  double* hist;
  int R;
  __device__ __forceinline__ double& s(int slot, int j) const { return st[slot * R + j]; }
  __device__ __forceinline__ int& a(int slot, int j) const { return ist[slot * R + j]; }
  __device__ __forceinline__ int& g(int slot) const { return ist[DDX_IST_COUNT * R + slot]; }
};

// A sharded solve (DDX_G_DEFER set): the last CTA of a fused reduction parks
// its NV column totals (valid in threads tid < R) in st slots T0.. and leaves
// the epilogue to ddx_pcg_finalize. True when parked (the caller returns).
template <int NV>
__device__ __forceinline__ bool park_totals(PcgState S, const double (&tot)[NV]) {
  if (S.ist == nullptr || S.g(DDX_G_DEFER) == 0) return false;
  if (threadIdx.x < S.R) {
#pragma unroll
    for (int v = 0; v < NV; ++v) S.s(DDX_ST_T0 + v, threadIdx.x) = tot[v];
  }
  return true;
}

__device__ __forceinline__ int n_active(const int* ist, int R) {
  return ist == nullptr ? 1 : *((volatile const int*)ist + DDX_IST_COUNT * R + DDX_G_NACTIVE);
}

// Count active RHS into the global counter (all threads of the CTA call it;
// threads tid < R pass their flag).
__device__ __forceinline__ void publish_nactive(PcgState S, int flag) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  if (threadIdx.x < S.R && flag) atomicAdd(&cnt, 1);
  __syncthreads();
  if (threadIdx.x == 0) S.g(DDX_G_NACTIVE) = cnt;
}

// Finalize steps shared by the fused kernels (threads tid < R, column tid).
__device__ __forceinline__ void fin_rz(PcgState S, int j, double rho, double zq) {
  if (!S.a(DDX_IST_ACTIVE, j)) return;
  S.s(DDX_ST_RHO, j) = rho;
  S.s(DDX_ST_ZQ, j) = zq;
  double beta = 0.0;
  if (S.a(DDX_IST_ITERS, j) > 0) {
    const double rho_prev = S.s(DDX_ST_RHO_PREV, j);
    if (rho_prev != 0.0) {
      beta = S.g(DDX_G_FLEXIBLE) ? -S.s(DDX_ST_ALPHA, j) * zq / rho_prev : rho / rho_prev;
    }
  }
  S.s(DDX_ST_BETA, j) = beta;
}

__device__ __forceinline__ int fin_pq(PcgState S, int j, double pq) {
  S.s(DDX_ST_PQ, j) = pq;
  S.s(DDX_ST_ALPHA_X, j) = 0.0;  // a parked x step was applied by the p update before this product
  int act = S.a(DDX_IST_ACTIVE, j);
  double alpha = 0.0;
  if (act) {
    if (pq > 0.0) {
      alpha = S.s(DDX_ST_RHO, j) / pq;
    } else {
      act = 0;
      S.a(DDX_IST_ACTIVE, j) = 0;
      S.g(DDX_G_BREAKDOWN) = 1;
    }
    S.s(DDX_ST_RHO_PREV, j) = S.s(DDX_ST_RHO, j);
  }
  S.s(DDX_ST_ALPHA, j) = alpha;
  return act;
}

// defer_x: x was not updated with this alpha; park it for the next p update
// (inactive RHS have alpha = 0 here, so parking is harmless for them).
__device__ __forceinline__ int fin_rr(PcgState S, int j, double rr, bool defer_x = false) {
  if (defer_x) S.s(DDX_ST_ALPHA_X, j) = S.s(DDX_ST_ALPHA, j);
  int act = S.a(DDX_IST_ACTIVE, j);
  if (act) {
    const int it = ++S.a(DDX_IST_ITERS, j);
    const double rn = sqrt(rr);
    S.s(DDX_ST_RR, j) = rr;
    S.hist[(size_t)it * S.R + j] = rn;
    if (rn < S.s(DDX_ST_ATOL, j) || it >= S.g(DDX_G_MAXITER)) {
      act = 0;
      S.a(DDX_IST_ACTIVE, j) = 0;
    }
  }
  return act;
}

// r = b - A x at the start of a solve: tolerance from ||b||, first stop test.
__device__ __forceinline__ int fin_init(PcgState S, int j, double bb, double rr) {
  const double rtol = S.s(DDX_ST_BB, j);  // ddx_pcg_reset parks rtol here
  const double atol = fmax(S.s(DDX_ST_ATOL, j), rtol * sqrt(bb));
  S.s(DDX_ST_ATOL, j) = atol;
  S.s(DDX_ST_BB, j) = bb;
  S.s(DDX_ST_RR, j) = rr;
  const double rn = sqrt(rr);
  S.hist[j] = rn;
  S.a(DDX_IST_ITERS, j) = 0;
  // A zero right-hand side with a zero residual has nothing to solve.
  const int act = !(rn < atol) && !(bb == 0.0 && rr == 0.0) && S.g(DDX_G_MAXITER) > 0;
  S.a(DDX_IST_ACTIVE, j) = act;
  return act;
}

// Residual replacement: r was recomputed as b - A x; redo the stop test.
__device__ __forceinline__ int fin_replace(PcgState S, int j, double rr) {
  int act = S.a(DDX_IST_ACTIVE, j);
  if (!act) return 0;  // converged RHS keep their recorded history
  const double rn = sqrt(rr);
  S.s(DDX_ST_RR, j) = rr;
  S.hist[(size_t)S.a(DDX_IST_ITERS, j) * S.R + j] = rn;
  if (rn < S.s(DDX_ST_ATOL, j)) {
    act = 0;
    S.a(DDX_IST_ACTIVE, j) = 0;
  }
  return act;
}

}  // namespace ddx
