// Schwarz local-inverse apply for small subdomains (a few to a few dozen DOFs).
//
// Same product and block layout as ddx_schwarz_local_apply (column-major
// blocks, leading dimension round_up(k, 16 B / element), per-block scale):
//   ylocal[sub_ptr[i] + t, j] = scale[i] * sum_c Q_i[t, c] * r[sub_idx[sub_ptr[i] + c], j],
// for the reference's DG layouts (src/dd_solvers/dd_solvers/solvers.py:355-359 on
// equal blocks of 3-48 DOFs, the BMV-I regime of src/dd_solvers/cpp/gemv_kernels.cu:31-57),
// where the streaming kernel's per-subdomain pipeline set-up would dominate.
// Equal subdomains: a thread owns 16 bytes of rows of one block (one vector
// load per column), a CTA owns whole subdomains and stages their inputs in
// shared memory once; otherwise one thread per output entry (row t of block
// i, right-hand side j, j fastest) with the inputs read through L1. Either way
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

// 16 bytes of a block column -> V accumulator-type values.
template <typename TB, typename ACC> struct Unpack;
template <> struct Unpack<double, double> {
  static constexpr int V = 2;
  __device__ __forceinline__ static void run(const uint4& u, double* o) {
    const double2 d = *reinterpret_cast<const double2*>(&u);
    o[0] = d.x; o[1] = d.y;
  }
};
template <> struct Unpack<float, double> {
  static constexpr int V = 4;
  __device__ __forceinline__ static void run(const uint4& u, double* o) {
    const float4 f = *reinterpret_cast<const float4*>(&u);
    o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = f.w;
  }
};
template <> struct Unpack<float, float> {
  static constexpr int V = 4;
  __device__ __forceinline__ static void run(const uint4& u, float* o) {
    const float4 f = *reinterpret_cast<const float4*>(&u);
    o[0] = f.x; o[1] = f.y; o[2] = f.z; o[3] = f.w;
  }
};
template <> struct Unpack<__half, float> {
  static constexpr int V = 8;
  __device__ __forceinline__ static void run(const uint4& u, float* o) {
    const __half2* h = reinterpret_cast<const __half2*>(&u);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const float2 f = __half22float2(h[e]);
      o[2 * e] = f.x; o[2 * e + 1] = f.y;
    }
  }
};
template <> struct Unpack<__nv_bfloat16, float> {
  static constexpr int V = 8;
  __device__ __forceinline__ static void run(const uint4& u, float* o) {
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {  // BF16 -> FP32 is exact: the upper half of the FP32 bits
      o[2 * e] = __uint_as_float(w[e] << 16);
      o[2 * e + 1] = __uint_as_float(w[e] & 0xffff0000u);
    }
  }
};

// Equal subdomains of k DOFs (column-major blocks, ld = round_up(k, V), V =
// 16 B / element): a thread owns V consecutive rows of one block and reads one
// 16-byte vector per column; a CTA owns floor(256 / (ld / V)) whole blocks and
// stages their inputs in shared memory once per right-hand side.
template <typename TB, typename ACC>
__global__ void __launch_bounds__(256, 4)
    k_local_apply_small_eq(int n_sub, int R, int k, const int* __restrict__ sub_idx,
                           const int64_t* __restrict__ blk_off, const TB* __restrict__ blocks,
                           const float* __restrict__ scale, const double* __restrict__ r, ACC* __restrict__ y,
                           const int* ist) {
  if (ist != nullptr && n_active(ist, R) == 0) return;
  using U = Unpack<TB, ACC>;
  constexpr int V = U::V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ACC* xs = reinterpret_cast<ACC*>(smem_raw);
  const int ld = (k + V - 1) / V * V;
  const int tpb = ld / V;
  const int bpc = 256 / tpb;
  const int bl = threadIdx.x / tpb, tv = threadIdx.x - bl * tpb;
  for (int64_t i0 = (int64_t)blockIdx.x * bpc; i0 < n_sub; i0 += (int64_t)gridDim.x * bpc) {
    const int nb = (int)(n_sub - i0 < bpc ? n_sub - i0 : bpc);
    const int64_t p0 = i0 * k;
    for (int j = 0; j < R; ++j) {
      for (int e = threadIdx.x; e < nb * k; e += 256) xs[e] = (ACC)r[(int64_t)sub_idx[p0 + e] * R + j];
      __syncthreads();
      if (bl < nb) {
        const int64_t i = i0 + bl;
        const TB* q = blocks + blk_off[i] + tv * V;
        const ACC* xv = xs + bl * k;
        ACC acc[V];
#pragma unroll
        for (int e = 0; e < V; ++e) acc[e] = ACC(0);
#pragma unroll 4
        for (int c = 0; c < k; ++c) {
          const uint4 u = __ldg(reinterpret_cast<const uint4*>(q + (int64_t)c * ld));
          ACC v[V];
          U::run(u, v);
          const ACC x = xv[c];
#pragma unroll
          for (int e = 0; e < V; ++e) acc[e] = fma(v[e], x, acc[e]);
        }
        const ACC sc = scale ? (ACC)scale[i] : ACC(1);
#pragma unroll
        for (int e = 0; e < V; ++e) {
          const int row = tv * V + e;
          if (row < k) y[(p0 + (int64_t)bl * k + row) * R + j] = sc * acc[e];
        }
      }
      __syncthreads();
    }
  }
}

template <typename TB, typename ACC>
int launch_small(int n_sub, int R, int k_equal, int64_t rows, const int64_t* sub_ptr, const int* sub_idx,
                 const int64_t* blk_off, const void* blocks, const float* scale, const double* r, void* ylocal,
                 const int* ist, cudaStream_t s) {
  constexpr int V = Unpack<TB, ACC>::V;
  const int ld = k_equal > 0 ? (k_equal + V - 1) / V * V : 0;
  if (k_equal > 0 && ld / V <= 256) {
    const int bpc = 256 / (ld / V);
    const size_t smem = (size_t)bpc * k_equal * sizeof(ACC);  // <= 256 * V values
    const int grid = resident_grid(k_local_apply_small_eq<TB, ACC>, ceil_div(n_sub, bpc), 1 << 20);
    k_local_apply_small_eq<TB, ACC><<<grid, 256, smem, s>>>(n_sub, R, k_equal, sub_idx, blk_off,
                                                            (const TB*)blocks, scale, r, (ACC*)ylocal, ist);
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
  DDX_REQUIRE(((uintptr_t)blocks & 15u) == 0, "ddx_schwarz_local_apply_small: blocks must be 16-byte aligned");
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
