// Reference op gemv_strided_batched: out[b] = M_b v_b for column-major (N, k, k)
// matrices, matrix entries converted to the vector type and accumulated in it
// (src/dd_solvers/cpp/gemv.cpp:9-53; src/dd_solvers/cpp/gemv_kernels.cu:31-139).
//
// A CTA owns floor(rows / k) consecutive batches (rows = 256 threads' rows,
// more for small k and for row pairs) or one batch; the batches' vectors are
// staged in shared memory; each thread produces one
// output row, so a warp reads 32 consecutive rows of one column per step
// (coalesced). The column loop runs in ascending c, like the reference.
#include <algorithm>

#include "common.cuh"

namespace ddx {

template <typename T> __device__ __forceinline__ double as_f64(T v) { return (double)to_f32<T>(v); }
template <> __device__ __forceinline__ double as_f64<double>(double v) { return v; }

template <typename TM, typename TV>
__device__ __forceinline__ TV up(TM m) {
  if constexpr (std::is_same<TV, double>::value) return as_f64<TM>(m);
  else return to_f32<TM>(m);
}

template <typename TM, typename TV>
__global__ void k_gemv_batched(int64_t N, int k, int bpc, const TM* __restrict__ mat,
                               const TV* __restrict__ vec, TV* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char sm[];
  TV* vs = reinterpret_cast<TV*>(sm);
  const int64_t b0 = (int64_t)blockIdx.x * bpc;
  const int nb = (int)std::min<int64_t>(bpc, N - b0);
  for (int t = threadIdx.x; t < nb * k; t += blockDim.x) vs[t] = vec[b0 * k + t];
  __syncthreads();
  for (int t = threadIdx.x; t < nb * k; t += blockDim.x) {
    const int bl = t / k, row = t - bl * k;
    const TM* m = mat + (b0 + bl) * (int64_t)k * k + row;
    const TV* v = vs + bl * k;
    TV acc = TV(0);
    for (int c = 0; c < k; ++c) acc += up<TM, TV>(m[(int64_t)c * k]) * v[c];
    out[(b0 + bl) * k + row] = acc;
  }
}

// 16-bit matrices with even k: each thread produces the row pair (2j, 2j+1)
// of a batch from one 4-byte load per column (the pair is 4-byte aligned: k
// even makes every column start even), halving the load instructions of the
// narrow type; each row keeps the ascending-c sum of the scalar kernel.
template <typename TM> struct Pair;
template <> struct Pair<__half> { using T = __half2; };
template <> struct Pair<__nv_bfloat16> { using T = __nv_bfloat162; };

template <typename TM, typename TV>
__global__ void k_gemv_pairs(int64_t N, int k, int bpc, const TM* __restrict__ mat, const TV* __restrict__ vec,
                             TV* __restrict__ out) {
  using TM2 = typename Pair<TM>::T;
  extern __shared__ __align__(16) unsigned char sm[];
  TV* vs = reinterpret_cast<TV*>(sm);
  const int64_t b0 = (int64_t)blockIdx.x * bpc;
  const int nb = (int)std::min<int64_t>(bpc, N - b0);
  const int kh = k / 2;
  for (int t = threadIdx.x; t < nb * k; t += blockDim.x) vs[t] = vec[b0 * k + t];
  __syncthreads();
  for (int t = threadIdx.x; t < nb * kh; t += blockDim.x) {
    const int bl = t / kh, row = 2 * (t - bl * kh);
    const TM2* m = reinterpret_cast<const TM2*>(mat + (b0 + bl) * (int64_t)k * k + row);
    const TV* v = vs + bl * k;
    TV a0 = TV(0), a1 = TV(0);
    for (int c = 0; c < k; ++c) {
      const TM2 w = m[(int64_t)c * kh];
      a0 += up<TM, TV>(w.x) * v[c];
      a1 += up<TM, TV>(w.y) * v[c];
    }
    out[(b0 + bl) * k + row] = a0;
    out[(b0 + bl) * k + row + 1] = a1;
  }
}

template <typename TM, typename TV>
static int launch_gemv(int64_t N, int k, const void* mat, const void* vec, void* out, cudaStream_t s) {
  constexpr bool narrow = sizeof(TM) == 2;
  const bool pairs = narrow && k % 2 == 0 && ((uintptr_t)mat & 3u) == 0;
  // rows per CTA: 256 threads x 1 row (x 2 rows for pairs), x 8 for k <= 8 so
  // that small matrices do not make thousands of tiny CTAs
  const int rows = 256 * (pairs ? 2 : 1) * (k <= 8 ? 8 : 1);
  const int bpc = k <= rows ? std::max(1, rows / k) : 1;
  const int64_t grid = ceil_div(N, bpc);
  const size_t smem = (size_t)bpc * k * sizeof(TV);
  if (smem > 200 * 1024) {
    set_error("ddx_gemv_strided_batched: k=%d too large", k);
    return DDX_ERR_UNSUPPORTED;
  }
  if constexpr (narrow) {
    if (pairs) {
      if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_gemv_pairs<TM, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_gemv_pairs<TM, TV><<<(unsigned)grid, 256, smem, s>>>(N, k, bpc, (const TM*)mat, (const TV*)vec, (TV*)out);
      DDX_LAUNCH_CHECK("ddx_gemv_strided_batched");
      return DDX_OK;
    }
  }
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_gemv_batched<TM, TV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_gemv_batched<TM, TV><<<(unsigned)grid, 256, smem, s>>>(N, k, bpc, (const TM*)mat, (const TV*)vec, (TV*)out);
  DDX_LAUNCH_CHECK("ddx_gemv_strided_batched");
  return DDX_OK;
}

}  // namespace ddx

using namespace ddx;

extern "C" int ddx_gemv_strided_batched(int64_t N, int k, const void* mat, int mat_dtype, const void* vec,
                                        void* out, int vec_dtype, ddx_stream_t stream) {
  DDX_REQUIRE(N >= 0 && k >= 0, "ddx_gemv_strided_batched: bad sizes");
  if (N == 0 || k == 0) return DDX_OK;
  DDX_REQUIRE(mat && vec && out, "ddx_gemv_strided_batched: null pointer");
  DDX_REQUIRE(vec_dtype == DDX_F32 || vec_dtype == DDX_F64, "ddx_gemv_strided_batched: vector dtype must be F32/F64");
  DDX_REQUIRE(!(mat_dtype == DDX_F64 && vec_dtype == DDX_F32),
              "Double-Float mixed precision is not supported.");
  cudaStream_t s = (cudaStream_t)stream;
  if (vec_dtype == DDX_F64) {
    switch (mat_dtype) {
      case DDX_F64: return launch_gemv<double, double>(N, k, mat, vec, out, s);
      case DDX_F32: return launch_gemv<float, double>(N, k, mat, vec, out, s);
      case DDX_BF16: return launch_gemv<__nv_bfloat16, double>(N, k, mat, vec, out, s);
      case DDX_F16: return launch_gemv<__half, double>(N, k, mat, vec, out, s);
    }
  } else {
    switch (mat_dtype) {
      case DDX_F32: return launch_gemv<float, float>(N, k, mat, vec, out, s);
      case DDX_BF16: return launch_gemv<__nv_bfloat16, float>(N, k, mat, vec, out, s);
      case DDX_F16: return launch_gemv<__half, float>(N, k, mat, vec, out, s);
    }
  }
  set_error("ddx_gemv_strided_batched: unknown matrix dtype %d", mat_dtype);
  return DDX_ERR_ARG;
}
