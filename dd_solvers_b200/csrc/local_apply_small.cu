// Schwarz local-inverse apply for small subdomains (a few to a few dozen DOFs).
//
// Same product and block layout as ddx_schwarz_local_apply (column-major
// blocks, leading dimension round_up(k, 16 B / element), per-block scale):
//   ylocal[sub_ptr[i] + t, j] = scale[i] * sum_c Q_i[t, c] * r[sub_idx[sub_ptr[i] + c], j],
// for the reference's DG layouts (src/dd_solvers/dd_solvers/solvers.py:355-359 on
// equal blocks of 3-48 DOFs, the BMV-I regime of src/dd_solvers/cpp/gemv_kernels.cu:31-57),
// where the streaming kernel's per-subdomain pipeline set-up would dominate.
// Equal subdomains (k <= 256): a CTA owns whole subdomains and stages their
// inputs in shared memory once; otherwise one thread per output entry (row t
// of block i, right-hand side j, j fastest) with the inputs read through L1.
// Either way a warp reads consecutive rows of one block column per step and
// the column loop runs in ascending c, so results are deterministic.
#include <algorithm>

#include "common.cuh"

namespace ddx {
namespace {

template <typename TB, typename ACC> __device__ __forceinline__ ACC load_as(const TB* p);
template <> __device__ __forceinline__ double load_as<double, double>(const double* p) { return __ldg(p); }
template <> __device__ __forceinline__ double load_as<float, double>(const float* p) { return (double)__ldg(p); }
template <> __device__ __forceinline__ float load_as<float, float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float load_as<__nv_bfloat16, float>(const __nv_bfloat16* p) {
  return __bfloat162float(*p);
}
template <> __device__ __forceinline__ float load_as<__half, float>(const __half* p) { return __half2float(*p); }

template <typename TB, typename ACC>
__global__ void __launch_bounds__(256)
    k_local_apply_small(int n_sub, int R, int k_equal, int64_t rows, const int64_t* __restrict__ sub_ptr,
                        const int* __restrict__ sub_idx, const int64_t* __restrict__ blk_off,
                        const TB* __restrict__ blocks, const float* __restrict__ scale,
                        const double* __restrict__ r, ACC* __restrict__ y, const int* ist) {
  if (ist != nullptr && n_active(ist, R) == 0) return;
  constexpr int V = 16 / (int)sizeof(TB);
  const int64_t total = rows * R;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = g / R;
    const int j = (int)(g - row * R);
    int64_t i;
    if (k_equal > 0) {
      i = row / k_equal;
    } else {  // last i with sub_ptr[i] <= row
      int64_t lo = 0, hi = n_sub;
      while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (sub_ptr[mid] <= row) lo = mid;
        else hi = mid;
      }
      i = lo;
    }
    const int64_t p0 = sub_ptr[i];
    const int k = (int)(sub_ptr[i + 1] - p0);
    const int t = (int)(row - p0);
    const int64_t ld = (k + V - 1) / V * V;
    const TB* q = blocks + blk_off[i] + t;
    const int* idx = sub_idx + p0;
    ACC acc = ACC(0);
    for (int c = 0; c < k; ++c) acc = fma(load_as<TB, ACC>(q + c * ld), (ACC)r[(int64_t)idx[c] * R + j], acc);
    const ACC sc = scale ? (ACC)scale[i] : ACC(1);
    y[row * R + j] = sc * acc;
  }
}

// Equal subdomains of k <= 256 DOFs: a CTA owns floor(256 / k) whole
// subdomains, stages their inputs in shared memory once per right-hand side,
// then each thread produces one output row.
template <typename TB, typename ACC>
__global__ void __launch_bounds__(256)
    k_local_apply_small_eq(int n_sub, int R, int k, const int* __restrict__ sub_idx,
                           const int64_t* __restrict__ blk_off, const TB* __restrict__ blocks,
                           const float* __restrict__ scale, const double* __restrict__ r, ACC* __restrict__ y,
                           const int* ist) {
  if (ist != nullptr && n_active(ist, R) == 0) return;
  constexpr int V = 16 / (int)sizeof(TB);
  __shared__ ACC xs[256];
  const int bpc = 256 / k;
  const int64_t ld = (k + V - 1) / V * V;
  for (int64_t i0 = (int64_t)blockIdx.x * bpc; i0 < n_sub; i0 += (int64_t)gridDim.x * bpc) {
    const int nb = (int)(n_sub - i0 < bpc ? n_sub - i0 : bpc);
    const int rows = nb * k;
    const int64_t p0 = i0 * k;
    for (int j = 0; j < R; ++j) {
      if (threadIdx.x < rows) xs[threadIdx.x] = (ACC)r[(int64_t)sub_idx[p0 + threadIdx.x] * R + j];
      __syncthreads();
      if (threadIdx.x < rows) {
        const int bl = threadIdx.x / k, t = threadIdx.x - bl * k;
        const int64_t i = i0 + bl;
        const TB* q = blocks + blk_off[i] + t;
        const ACC* xv = xs + bl * k;
        ACC acc = ACC(0);
        for (int c = 0; c < k; ++c) acc = fma(load_as<TB, ACC>(q + c * ld), xv[c], acc);
        const ACC sc = scale ? (ACC)scale[i] : ACC(1);
        y[(p0 + threadIdx.x) * R + j] = sc * acc;
      }
      __syncthreads();
    }
  }
}

template <typename TB, typename ACC>
int launch_small(int n_sub, int R, int k_equal, int64_t rows, const int64_t* sub_ptr, const int* sub_idx,
                 const int64_t* blk_off, const void* blocks, const float* scale, const double* r, void* ylocal,
                 const int* ist, cudaStream_t s) {
  if (k_equal > 0 && k_equal <= 256) {
    const int grid = resident_grid(k_local_apply_small_eq<TB, ACC>, ceil_div(n_sub, 256 / k_equal), 1 << 20);
    k_local_apply_small_eq<TB, ACC><<<grid, 256, 0, s>>>(n_sub, R, k_equal, sub_idx, blk_off, (const TB*)blocks,
                                                         scale, r, (ACC*)ylocal, ist);
  } else {
    const int grid = resident_grid(k_local_apply_small<TB, ACC>, ceil_div(rows * R, 256), 1 << 20);
    k_local_apply_small<TB, ACC><<<grid, 256, 0, s>>>(n_sub, R, k_equal, rows, sub_ptr, sub_idx, blk_off,
                                                      (const TB*)blocks, scale, r, (ACC*)ylocal, ist);
  }
  DDX_LAUNCH_CHECK("ddx_schwarz_local_apply_small");
  return DDX_OK;
}

}  // namespace
}  // namespace ddx

using namespace ddx;

extern "C" int ddx_schwarz_local_apply_small(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                             const int64_t* blk_off, const void* blocks, int block_dtype,
                                             const float* scale, int kmax, int k_equal, int64_t rows,
                                             const double* r, void* ylocal, int acc_dtype, const int* ist,
                                             ddx_stream_t stream) {
  DDX_REQUIRE(R >= 1 && n_sub >= 0 && kmax >= 0 && rows >= 0, "ddx_schwarz_local_apply_small: bad sizes");
  if (n_sub == 0 || rows == 0) return DDX_OK;
  DDX_REQUIRE(sub_ptr && sub_idx && blk_off && blocks && r && ylocal, "ddx_schwarz_local_apply_small: null pointer");
  DDX_REQUIRE(k_equal <= 0 || (int64_t)k_equal * n_sub == rows,
              "ddx_schwarz_local_apply_small: k_equal * n_sub must equal rows");
  cudaStream_t s = (cudaStream_t)stream;
  switch (block_dtype) {
    case DDX_F64:
      DDX_REQUIRE(acc_dtype == DDX_F64, "ddx_schwarz_local_apply_small: F64 blocks accumulate in F64");
      return launch_small<double, double>(n_sub, R, k_equal, rows, sub_ptr, sub_idx, blk_off, blocks, scale, r,
                                          ylocal, ist, s);
    case DDX_F32:
      if (acc_dtype == DDX_F64)
        return launch_small<float, double>(n_sub, R, k_equal, rows, sub_ptr, sub_idx, blk_off, blocks, scale, r,
                                           ylocal, ist, s);
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply_small: F32 blocks accumulate in F32 or F64");
      return launch_small<float, float>(n_sub, R, k_equal, rows, sub_ptr, sub_idx, blk_off, blocks, scale, r,
                                        ylocal, ist, s);
    case DDX_BF16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply_small: BF16 blocks accumulate in F32");
      return launch_small<__nv_bfloat16, float>(n_sub, R, k_equal, rows, sub_ptr, sub_idx, blk_off, blocks, scale,
                                                r, ylocal, ist, s);
    case DDX_F16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply_small: F16 blocks accumulate in F32");
      return launch_small<__half, float>(n_sub, R, k_equal, rows, sub_ptr, sub_idx, blk_off, blocks, scale, r,
                                         ylocal, ist, s);
    default:
      set_error("ddx_schwarz_local_apply_small: unknown block dtype %d", block_dtype);
      return DDX_ERR_ARG;
  }
}
