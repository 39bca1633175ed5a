// Schwarz preconditioner kernels.
//
// Replaces Inv.solve -> gemv_strided_batched (src/dd_solvers/dd_solvers/solvers.py:355-359,
// src/dd_solvers/cpp/gemv_kernels.cu:59-139) and the reshape/sum/segment_reduce/
// repeat_interleave glue of AdditiveSchwarz.solve / HybridSchwarz.solve
// (solvers.py:811-826, 874-888), generalised to overlapping index-set
// subdomains of uneven size.
//
// local_apply: persistent CTAs walk a size-sorted subdomain list. Per CTA, one
// producer warp streams each inverse block (column-major, 16-byte columns)
// through a ring of shared-memory stages with cp.async.bulk (the TMA engine)
// and mbarrier completion; four consumer warps gather r[idx] into shared
// memory, then each thread owns fixed 16-byte row groups and accumulates
// acc[rows] += Q[rows, c] * x[c] column by column (no cross-thread reduction).
//
// combine: the prolongation is a gather over the transpose map (DOF ->
// positions in the subdomain-major ylocal) summed in ascending subdomain
// order, so it is atomic-free and deterministic; it also adds the coarse
// prolongation and forms the PCG dots.
#include <algorithm>

#include "common.cuh"

namespace ddx {

// ---------------------------------------------------------------------------
// mbarrier / bulk-copy primitives (sm_90+ PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait: gives up after ~2 s, records the timeout in the device error
// word and returns false (the caller then leaves its loops).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 1023u) == 0) {
      const uint64_t t = global_timer_ns();
      if (t0 == 0) t0 = t;
      else if (t - t0 > 2000000000ull) {
        atomicOr(&g_device_error, DEVERR_MBAR_TIMEOUT);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void consumer_sync(int nthreads) {
  asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

// ---------------------------------------------------------------------------
// Block element helpers: V elements per 16-byte vector, FMA into ACC.
// ---------------------------------------------------------------------------
template <typename TB> struct Vec16;
template <> struct Vec16<double> { static constexpr int V = 2; };
template <> struct Vec16<float> { static constexpr int V = 4; };
template <> struct Vec16<__nv_bfloat16> { static constexpr int V = 8; };
template <> struct Vec16<__half> { static constexpr int V = 8; };

template <typename TB, typename ACC>
__device__ __forceinline__ void fma_vec(const void* p, ACC xv, ACC* acc);

template <>
__device__ __forceinline__ void fma_vec<double, double>(const void* p, double xv, double* acc) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  acc[0] = fma(v.x, xv, acc[0]);
  acc[1] = fma(v.y, xv, acc[1]);
}
template <>
__device__ __forceinline__ void fma_vec<float, float>(const void* p, float xv, float* acc) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  acc[0] = fmaf(v.x, xv, acc[0]);
  acc[1] = fmaf(v.y, xv, acc[1]);
  acc[2] = fmaf(v.z, xv, acc[2]);
  acc[3] = fmaf(v.w, xv, acc[3]);
}
template <>
__device__ __forceinline__ void fma_vec<float, double>(const void* p, double xv, double* acc) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  acc[0] = fma((double)v.x, xv, acc[0]);
  acc[1] = fma((double)v.y, xv, acc[1]);
  acc[2] = fma((double)v.z, xv, acc[2]);
  acc[3] = fma((double)v.w, xv, acc[3]);
}
template <>
__device__ __forceinline__ void fma_vec<__nv_bfloat16, float>(const void* p, float xv, float* acc) {
  const uint4 u = *reinterpret_cast<const uint4*>(p);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    // bf16 -> f32 is exact: the bf16 bits are the top half of the f32 bits
    const float lo = __uint_as_float(w[k] << 16);
    const float hi = __uint_as_float(w[k] & 0xffff0000u);
    acc[2 * k] = fmaf(lo, xv, acc[2 * k]);
    acc[2 * k + 1] = fmaf(hi, xv, acc[2 * k + 1]);
  }
}
template <>
__device__ __forceinline__ void fma_vec<__half, float>(const void* p, float xv, float* acc) {
  const uint4 u = *reinterpret_cast<const uint4*>(p);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[k]));
    acc[2 * k] = fmaf(f.x, xv, acc[2 * k]);
    acc[2 * k + 1] = fmaf(f.y, xv, acc[2 * k + 1]);
  }
}

constexpr int kConsumers = 128;           // 4 consumer warps
constexpr int kApplyThreads = kConsumers + 32;  // + 1 producer warp
constexpr int kStages = 4;

struct ApplyArgs {
  int n_sub, R, j0;
  const int64_t* sub_ptr;
  const int* sub_idx;
  const int* order;
  const int64_t* blk_off;
  const void* blocks;
  const float* scale;
  const double* r;
  void* ylocal;
  const int* ist;
  uint32_t stage_bytes;
  int kmax;
};

template <typename TB>
__device__ __forceinline__ void chunk_geometry(int k, uint32_t stage_bytes, int& ld, int& cs, int& nchunk) {
  constexpr int V = Vec16<TB>::V;
  ld = (k + V - 1) / V * V;
  const uint32_t colbytes = (uint32_t)ld * sizeof(TB);
  cs = (int)(stage_bytes / colbytes);
  if (cs < 1) cs = 1;
  nchunk = (k + cs - 1) / cs;
}

template <typename TB, typename ACC, int G>
__global__ void __launch_bounds__(kApplyThreads) k_local_apply(ApplyArgs a) {
  constexpr int V = Vec16<TB>::V;
  extern __shared__ __align__(128) unsigned char smem[];
  if (a.ist != nullptr && n_active(a.ist, a.R) == 0) return;

  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kStages;
  __shared__ int abort_flag;
  unsigned char* stage_base = smem + 128;  // after the barriers
  ACC* xs = reinterpret_cast<ACC*>(stage_base + (size_t)kStages * a.stage_bytes);

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumers / 32);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const TB* blocks = reinterpret_cast<const TB*>(a.blocks);

  if (tid >= kConsumers) {
    // ------------------------------ producer ------------------------------
    if (tid != kConsumers) return;
    uint32_t g = 0;
    for (int w = blockIdx.x; w < a.n_sub; w += gridDim.x) {
      const int i = a.order[w];
      const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
      if (k == 0 || k > a.kmax) continue;
      int ld, cs, nchunk;
      chunk_geometry<TB>(k, a.stage_bytes, ld, cs, nchunk);
      const TB* src = blocks + a.blk_off[i];
      for (int q = 0; q < nchunk; ++q, ++g) {
        const int s = g % kStages;
        const uint32_t phase = (g / kStages) & 1u;
        if (!mbar_wait(&empty[s], phase ^ 1u)) { abort_flag = 1; return; }
        const int c0 = q * cs;
        const int nc = min(cs, k - c0);
        const uint32_t bytes = (uint32_t)nc * (uint32_t)ld * (uint32_t)sizeof(TB);
        mbar_arrive_expect_tx(&full[s], bytes);
        bulk_g2s(stage_base + (size_t)s * a.stage_bytes, src + (int64_t)c0 * ld, bytes, &full[s]);
      }
    }
    return;
  }

  // ------------------------------ consumers ------------------------------
  const int R = a.R;
  uint32_t g = 0;
  for (int w = blockIdx.x; w < a.n_sub; w += gridDim.x) {
    const int i = a.order[w];
    const int64_t p0 = a.sub_ptr[i];
    const int k = (int)(a.sub_ptr[i + 1] - p0);
    if (k == 0) continue;
    if (k > a.kmax) {  // would overflow the shared-memory gather buffer
      if (tid == 0) atomicOr(&g_device_error, DEVERR_BAD_SIZE);
      continue;
    }
    int ld, cs, nchunk;
    chunk_geometry<TB>(k, a.stage_bytes, ld, cs, nchunk);
    consumer_sync(kConsumers);  // previous subdomain done with xs
    for (int c = tid; c < k; c += kConsumers)
      xs[c] = (ACC)a.r[(int64_t)a.sub_idx[p0 + c] * R + a.j0];
    consumer_sync(kConsumers);

    ACC acc[G][V];
#pragma unroll
    for (int gg = 0; gg < G; ++gg)
#pragma unroll
      for (int e = 0; e < V; ++e) acc[gg][e] = ACC(0);
    const int nvr = ld / V;  // 16-byte row groups per column

    bool ok = true;
    for (int q = 0; q < nchunk; ++q, ++g) {
      const int s = g % kStages;
      const uint32_t phase = (g / kStages) & 1u;
      if (!mbar_wait(&full[s], phase)) { ok = false; break; }
      const unsigned char* st = stage_base + (size_t)s * a.stage_bytes;
      const int c0 = q * cs;
      const int nc = min(cs, k - c0);
#pragma unroll 4
      for (int cl = 0; cl < nc; ++cl) {
        const ACC xv = xs[c0 + cl];
        const unsigned char* col = st + (size_t)cl * ld * sizeof(TB);
#pragma unroll
        for (int gg = 0; gg < G; ++gg) {
          const int vr = tid + gg * kConsumers;
          if (vr < nvr) fma_vec<TB, ACC>(col + (size_t)vr * 16, xv, acc[gg]);
        }
      }
      __syncwarp();
      if ((tid & 31) == 0) mbar_arrive(&empty[s]);
    }
    if (!ok || abort_flag) return;

    const ACC sc = a.scale ? (ACC)a.scale[i] : ACC(1);
    ACC* y = reinterpret_cast<ACC*>(a.ylocal);
#pragma unroll
    for (int gg = 0; gg < G; ++gg) {
      const int vr = tid + gg * kConsumers;
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const int row = vr * V + e;
        if (row < k) y[(p0 + row) * R + a.j0] = sc * acc[gg][e];
      }
    }
  }
}

template <typename TB, typename ACC>
static int launch_apply_typed(const ApplyArgs& base, cudaStream_t s) {
  constexpr int V = Vec16<TB>::V;
  const int ldmax = (base.kmax + V - 1) / V * V;
  const int nvr = ldmax / V;
  const int G = (int)ceil_div(nvr, kConsumers);
  ApplyArgs a = base;
  const uint32_t colbytes = (uint32_t)ldmax * sizeof(TB);
  a.stage_bytes = std::max<uint32_t>(20480u, (colbytes + 15u) / 16u * 16u);
  const size_t smem = 128 + (size_t)kStages * a.stage_bytes + (size_t)ldmax * sizeof(ACC) + 16;
  if (smem > 227 * 1024) {
    set_error("ddx_schwarz_local_apply: subdomain size %d needs %zu bytes of shared memory", base.kmax, smem);
    return DDX_ERR_UNSUPPORTED;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  auto go = [&](auto kernel) -> int {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kApplyThreads, smem);
    per_sm = std::max(1, std::min(per_sm, 2));
    const int grid = std::max(1, std::min(a.n_sub, nsm * per_sm));
    for (int j = 0; j < base.R; ++j) {
      a.j0 = j;
      kernel<<<grid, kApplyThreads, smem, s>>>(a);
    }
    DDX_LAUNCH_CHECK("ddx_schwarz_local_apply");
    return DDX_OK;
  };
  if (G <= 1) return go(k_local_apply<TB, ACC, 1>);
  if (G <= 2) return go(k_local_apply<TB, ACC, 2>);
  if (G <= 4) return go(k_local_apply<TB, ACC, 4>);
  if (G <= 8) return go(k_local_apply<TB, ACC, 8>);
  if (G <= 16) return go(k_local_apply<TB, ACC, 16>);
  set_error("ddx_schwarz_local_apply: kmax %d too large", base.kmax);
  return DDX_ERR_UNSUPPORTED;
}

// ---------------------------------------------------------------------------
// combine
// ---------------------------------------------------------------------------
template <typename ACC>
__global__ void __launch_bounds__(kThreads)
    k_combine(int64_t n, PcgState S, const int* __restrict__ dof_ptr, const int* __restrict__ dof_src,
              const ACC* __restrict__ ylocal, const double* u, const int* __restrict__ p_ptr,
              const int* __restrict__ p_col, const double* __restrict__ p_val,
              const double* __restrict__ yc, double sign, double* z, int dots,
              const double* __restrict__ r, const double* __restrict__ q, double* partials,
              unsigned int* ticket) {
  __shared__ double red[kThreads];
  const int R = S.R;
  if (S.ist != nullptr && n_active(S.ist, R) == 0) return;
  const int64_t total = n * R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int j = threadIdx.x % R;
  double acc[2] = {0.0, 0.0};
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += stride) {
    const int64_t d = e / R;
    double v = 0.0;
    if (ylocal != nullptr) {
      const int t0 = dof_ptr[d], t1 = dof_ptr[d + 1];
      for (int t = t0; t < t1; ++t) v += (double)ylocal[(int64_t)dof_src[t] * R + j];
    }
    if (u != nullptr) v += u[e];
    if (p_ptr != nullptr) {
      double c = 0.0;
      const int k0 = p_ptr[d], k1 = p_ptr[d + 1];
      for (int k = k0; k < k1; ++k) c = fma(p_val[k], yc[(int64_t)p_col[k] * R + j], c);
      v = fma(sign, c, v);
    }
    z[e] = v;
    if (dots) {
      acc[0] = fma(r[e], v, acc[0]);
      if (q != nullptr) acc[1] = fma(v, q[e], acc[1]);
    }
  }
  if (!dots) return;
  write_cta_partials<2>(acc, red, R, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[2];
  final_sums<2>(partials, R, red, tot, ticket);
  if (threadIdx.x < R) fin_rz(S, threadIdx.x, tot[0], tot[1]);
}

// ---------------------------------------------------------------------------
// dense coarse solve: yc = Ainv w  (Ainv symmetric, row-major)
// ---------------------------------------------------------------------------
// R = 1: one warp per row, lanes stride the row, shuffle-tree reduction.
__global__ void k_coarse_gemv1(int n_c, const double* __restrict__ Ainv, const double* __restrict__ w,
                               double* __restrict__ yc, const int* ist) {
  if (ist != nullptr && n_active(ist, 1) == 0) return;
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n_c) return;
  const double* a = Ainv + row * n_c;
  double s = 0.0;
  for (int c = lane; c < n_c; c += 32) s = fma(__ldcs(a + c), __ldg(w + c), s);
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) yc[row] = s;
}

// R > 1: CTA of 256 threads = (256/R) rows x R columns; row entries broadcast.
__global__ void k_coarse_gemvR(int n_c, int R, const double* __restrict__ Ainv, const double* __restrict__ w,
                               double* __restrict__ yc, const int* ist) {
  if (ist != nullptr && n_active(ist, R) == 0) return;
  const int j = threadIdx.x % R;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / R) + threadIdx.x / R;
  if (row >= n_c) return;
  const double* a = Ainv + row * n_c;
  double s = 0.0;
  for (int c = 0; c < n_c; ++c) s = fma(__ldg(a + c), __ldg(w + (int64_t)c * R + j), s);
  yc[row * R + j] = s;
}

}  // namespace ddx

using namespace ddx;

extern "C" {

int ddx_schwarz_local_apply(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx, const int* order,
                            const int64_t* blk_off, const void* blocks, int block_dtype, const float* scale,
                            int kmax, const double* r, void* ylocal, int acc_dtype, const int* ist,
                            ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_schwarz_local_apply: unsupported R=%d", R);
  DDX_REQUIRE(n_sub >= 0 && kmax >= 0, "ddx_schwarz_local_apply: bad sizes");
  if (n_sub == 0 || kmax == 0) return DDX_OK;
  DDX_REQUIRE(sub_ptr && sub_idx && order && blk_off && blocks && r && ylocal,
              "ddx_schwarz_local_apply: null pointer");
  DDX_REQUIRE(((uintptr_t)blocks & 15u) == 0, "ddx_schwarz_local_apply: blocks must be 16-byte aligned");
  ApplyArgs a{};
  a.n_sub = n_sub; a.R = R; a.j0 = 0;
  a.sub_ptr = sub_ptr; a.sub_idx = sub_idx; a.order = order; a.blk_off = blk_off;
  a.blocks = blocks; a.scale = scale; a.r = r; a.ylocal = ylocal; a.ist = ist; a.kmax = kmax;
  cudaStream_t s = (cudaStream_t)stream;
  switch (block_dtype) {
    case DDX_F64:
      DDX_REQUIRE(acc_dtype == DDX_F64, "ddx_schwarz_local_apply: F64 blocks accumulate in F64");
      return launch_apply_typed<double, double>(a, s);
    case DDX_F32:
      // FP64 accumulation matches the reference's rule for FP32 blocks with
      // FP64 vectors (accumulate in the vector type)
      if (acc_dtype == DDX_F64) return launch_apply_typed<float, double>(a, s);
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply: F32 blocks accumulate in F32 or F64");
      return launch_apply_typed<float, float>(a, s);
    case DDX_BF16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply: BF16 blocks accumulate in F32");
      return launch_apply_typed<__nv_bfloat16, float>(a, s);
    case DDX_F16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply: F16 blocks accumulate in F32");
      return launch_apply_typed<__half, float>(a, s);
    default:
      set_error("ddx_schwarz_local_apply: unknown block dtype %d", block_dtype);
      return DDX_ERR_ARG;
  }
}

int ddx_schwarz_combine(int64_t n, int R, const int* dof_ptr, const int* dof_src, const void* ylocal,
                        int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                        const double* p_val, const double* yc, double sign, double* z, int dots,
                        const double* r, const double* q, double* st, int* ist, double* partials,
                        unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_schwarz_combine: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && z, "ddx_schwarz_combine: bad arguments");
  if (ylocal) DDX_REQUIRE(dof_ptr && dof_src, "ddx_schwarz_combine: ylocal needs the transpose map");
  if (p_ptr) DDX_REQUIRE(p_col && p_val && yc, "ddx_schwarz_combine: prolongation needs P and yc");
  if (dots) DDX_REQUIRE(r && st && ist && partials && tickets, "ddx_schwarz_combine: dots need PCG state");
  PcgState S{st, ist, nullptr, R};
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = dots ? red_grid(n * R) : (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(n * R, kThreads), 148 * 16));
  unsigned int* t = tickets ? tickets + 4 : nullptr;
  if (ylocal == nullptr || acc_dtype == DDX_F64) {
    k_combine<double><<<grid, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, (const double*)ylocal, u, p_ptr, p_col,
                                                p_val, yc, sign, z, dots, r, q, partials, t);
  } else if (acc_dtype == DDX_F32) {
    k_combine<float><<<grid, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, (const float*)ylocal, u, p_ptr, p_col,
                                               p_val, yc, sign, z, dots, r, q, partials, t);
  } else {
    set_error("ddx_schwarz_combine: acc dtype %d", acc_dtype);
    return DDX_ERR_ARG;
  }
  DDX_LAUNCH_CHECK("ddx_schwarz_combine");
  return DDX_OK;
}

int ddx_coarse_gemv_f64(int n_c, int R, const double* Ainv, const double* w, double* yc, const int* ist,
                        ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_coarse_gemv_f64: unsupported R=%d", R);
  DDX_REQUIRE(n_c >= 0 && Ainv && w && yc, "ddx_coarse_gemv_f64: bad arguments");
  if (n_c == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (R == 1) {
    k_coarse_gemv1<<<(int)ceil_div(n_c, 8), 256, 0, s>>>(n_c, Ainv, w, yc, ist);
  } else {
    k_coarse_gemvR<<<(int)ceil_div((int64_t)n_c * R, 256), 256, 0, s>>>(n_c, R, Ainv, w, yc, ist);
  }
  DDX_LAUNCH_CHECK("ddx_coarse_gemv_f64");
  return DDX_OK;
}

}  // extern "C"
