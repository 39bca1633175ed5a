// Schwarz local-inverse apply, SIMT streaming kernel (one or a few RHS).
//
// Replaces Inv.solve -> gemv_strided_batched (src/dd_solvers/dd_solvers/solvers.py:355-359,
// src/dd_solvers/cpp/gemv_kernels.cu:59-139) for index-set subdomains of any size:
//   ylocal[sub_ptr[i] + t, j] = scale[i] * sum_c Q_i[t, c] * r[sub_idx[sub_ptr[i] + c], j].
//
// Persistent CTAs walk a size-sorted subdomain list. In each CTA one producer
// thread streams every block (column-major, 16-byte columns) through a ring of
// four shared-memory stages with cp.async.bulk + mbarriers. NG consumer groups
// of four warps split the columns: group g takes the ring chunks whose global
// index is g mod NG, so NG x 4 warps per CTA hide the shared-memory latency.
// Inside a group each thread owns fixed 16-byte row groups and accumulates
// acc[rows] += Q[rows, c] * x[c] column by column (packed FP32x2 FMAs for
// BF16/FP16/FP32 blocks; FP64 FMAs for FP64 blocks and for FP32 blocks with FP64
// vectors). Group partials are added in a fixed order through shared memory, so
// results do not depend on timing. The group count and stage size are run-time
// choices (ddx_schwarz_local_apply_ex) for the setup-time autotuner.
#include <algorithm>

#include "pipeline.cuh"

namespace ddx {
using namespace pipe;

namespace {

constexpr int kGroup = 128;  // threads per consumer group (4 warps)
constexpr int kStages = 4;   // ring stages; a multiple of every group count used

template <typename TB> struct Vec16;
template <> struct Vec16<double> { static constexpr int V = 2; };
template <> struct Vec16<float> { static constexpr int V = 4; };
template <> struct Vec16<__nv_bfloat16> { static constexpr int V = 8; };
template <> struct Vec16<__half> { static constexpr int V = 8; };

// Accumulator slots per 16-byte vector: FP32 accumulators are float2 pairs
// (one packed FMA per pair), FP64 accumulators are scalars.
template <typename TB, typename ACC> struct Slot { using T = ACC; static constexpr int N = Vec16<TB>::V; };
template <> struct Slot<float, float> { using T = float2; static constexpr int N = 2; };
template <> struct Slot<__nv_bfloat16, float> { using T = float2; static constexpr int N = 4; };
template <> struct Slot<__half, float> { using T = float2; static constexpr int N = 4; };

template <typename TB, typename ACC>
__device__ __forceinline__ void fma_vec(const unsigned char* p, ACC xv, typename Slot<TB, ACC>::T* acc);

template <>
__device__ __forceinline__ void fma_vec<double, double>(const unsigned char* p, double xv, double* acc) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  acc[0] = fma(v.x, xv, acc[0]);
  acc[1] = fma(v.y, xv, acc[1]);
}
template <>
__device__ __forceinline__ void fma_vec<float, double>(const unsigned char* p, double xv, double* acc) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  acc[0] = fma((double)v.x, xv, acc[0]);
  acc[1] = fma((double)v.y, xv, acc[1]);
  acc[2] = fma((double)v.z, xv, acc[2]);
  acc[3] = fma((double)v.w, xv, acc[3]);
}
template <>
__device__ __forceinline__ void fma_vec<float, float>(const unsigned char* p, float xv, float2* acc) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  const float2 x2 = make_float2(xv, xv);
  acc[0] = __ffma2_rn(make_float2(v.x, v.y), x2, acc[0]);
  acc[1] = __ffma2_rn(make_float2(v.z, v.w), x2, acc[1]);
}
template <>
__device__ __forceinline__ void fma_vec<__nv_bfloat16, float>(const unsigned char* p, float xv, float2* acc) {
  const uint4 u = *reinterpret_cast<const uint4*>(p);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
  const float2 x2 = make_float2(xv, xv);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    // BF16 -> FP32 is exact: the BF16 bits are the upper half of the FP32 bits
    const float2 f = make_float2(__uint_as_float(w[k] << 16), __uint_as_float(w[k] & 0xffff0000u));
    acc[k] = __ffma2_rn(f, x2, acc[k]);
  }
}
template <>
__device__ __forceinline__ void fma_vec<__half, float>(const unsigned char* p, float xv, float2* acc) {
  const uint4 u = *reinterpret_cast<const uint4*>(p);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
  const float2 x2 = make_float2(xv, xv);
#pragma unroll
  for (int k = 0; k < 4; ++k) acc[k] = __ffma2_rn(__half22float2(*reinterpret_cast<const __half2*>(&w[k])), x2, acc[k]);
}

template <typename T> __device__ __forceinline__ T zero_slot();
template <> __device__ __forceinline__ double zero_slot<double>() { return 0.0; }
template <> __device__ __forceinline__ float2 zero_slot<float2>() { return make_float2(0.f, 0.f); }

// Element e of a thread's V accumulated rows.
__device__ __forceinline__ double slot_get(const double* s, int e) { return s[e]; }
__device__ __forceinline__ float slot_get(const float2* s, int e) { return (e & 1) ? s[e >> 1].y : s[e >> 1].x; }
__device__ __forceinline__ void slot_add(double* s, int e, double v) { s[e] += v; }
__device__ __forceinline__ void slot_add(float2* s, int e, float v) {
  if (e & 1) s[e >> 1].y += v;
  else s[e >> 1].x += v;
}

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
  int ldmax;
  int red_elems;  // capacity of the group-reduction buffer (elements)
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

template <typename TB, typename ACC, int G, int NG>
__global__ void __launch_bounds__(NG * kGroup + 32) k_local_apply(ApplyArgs a) {
  constexpr int V = Vec16<TB>::V;
  using ST = typename Slot<TB, ACC>::T;
  constexpr int NS = Slot<TB, ACC>::N;
  constexpr int NC = NG * kGroup;
  extern __shared__ __align__(128) unsigned char smem[];
  if (a.ist != nullptr && n_active(a.ist, a.R) == 0) return;

  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kStages;
  __shared__ int abort_s;
  volatile int& abort_flag = abort_s;
  unsigned char* stage_base = smem + 128;
  ACC* xs = reinterpret_cast<ACC*>(stage_base + (size_t)kStages * a.stage_bytes);
  ACC* red = xs + a.ldmax;  // (NG - 1) x G x V x kGroup partials of groups 1..NG-1

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kGroup / 32);  // the four warps of the group that owns the stage
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const TB* blocks = reinterpret_cast<const TB*>(a.blocks);

  if (tid >= NC) {
    // ------------------------------ producer ------------------------------
    if (tid != NC) return;
    uint32_t g = 0;
    for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
      const int i = a.order[w];
      const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
      if (k == 0 || k > a.kmax) continue;
      int ld, cs, nchunk;
      chunk_geometry<TB>(k, a.stage_bytes, ld, cs, nchunk);
      const TB* src = blocks + a.blk_off[i];
      for (int q = 0; q < nchunk; ++q, ++g) {
        const int s = g % kStages;
        if (!mbar_wait(&empty[s], ((g / kStages) & 1u) ^ 1u)) { abort_flag = 1; return; }
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
  const int grp = tid / kGroup, gt = tid % kGroup;
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
    named_sync(1, NC);  // previous subdomain done with xs and red
    if (abort_flag) break;
    for (int c = tid; c < k; c += NC) xs[c] = (ACC)a.r[(int64_t)a.sub_idx[p0 + c] * R + a.j0];
    named_sync(1, NC);

    ST acc[G][NS];
#pragma unroll
    for (int gg = 0; gg < G; ++gg)
#pragma unroll
      for (int e = 0; e < NS; ++e) acc[gg][e] = zero_slot<ST>();
    const int nvr = ld / V;  // 16-byte row groups per column

    for (int q = 0; q < nchunk; ++q) {
      const uint32_t gq = g + (uint32_t)q;
      if ((int)(gq % NG) != grp) continue;
      const int s = gq % kStages;
      if (abort_flag) break;  // another role gave up: stop waiting, leave at the next barrier
      if (!mbar_wait(&full[s], (gq / kStages) & 1u)) { abort_flag = 1; break; }
      const unsigned char* st = stage_base + (size_t)s * a.stage_bytes;
      const int c0 = q * cs;
      const int nc = min(cs, k - c0);
#pragma unroll 4
      for (int cl = 0; cl < nc; ++cl) {
        const ACC xv = xs[c0 + cl];
        const unsigned char* col = st + (size_t)cl * ld * sizeof(TB);
#pragma unroll
        for (int gg = 0; gg < G; ++gg) {
          const int vr = gt + gg * kGroup;
          if (vr < nvr) fma_vec<TB, ACC>(col + (size_t)vr * 16, xv, acc[gg]);
        }
      }
      __syncwarp();
      if ((tid & 31) == 0) mbar_arrive(&empty[s]);
    }
    g += (uint32_t)nchunk;

    if (NG > 1) {
      if (grp > 0) {
#pragma unroll
        for (int gg = 0; gg < G; ++gg)
#pragma unroll
          for (int e = 0; e < V; ++e) {
            const int ri = (((grp - 1) * G + gg) * V + e) * kGroup + gt;
            if (ri < a.red_elems) red[ri] = slot_get(acc[gg], e);  // checked: a sizing bug records, never faults
            else atomicOr(&g_device_error, DEVERR_BAD_SIZE);
          }
      }
      named_sync(1, NC);
      if (grp == 0) {
        for (int og = 1; og < NG; ++og)
#pragma unroll
          for (int gg = 0; gg < G; ++gg)
#pragma unroll
            for (int e = 0; e < V; ++e) {
              const int ri = (((og - 1) * G + gg) * V + e) * kGroup + gt;
              if (ri < a.red_elems) slot_add(acc[gg], e, red[ri]);
            }
      }
    }
    // (an abort is acted on at the barrier at the top of the next subdomain,
    // where every consumer reads the flag at the same point)
    if (grp == 0) {
      const ACC sc = a.scale ? (ACC)a.scale[i] : ACC(1);
      ACC* y = reinterpret_cast<ACC*>(a.ylocal);
#pragma unroll
      for (int gg = 0; gg < G; ++gg) {
        const int vr = gt + gg * kGroup;
#pragma unroll
        for (int e = 0; e < V; ++e) {
          const int row = vr * V + e;
          if (row < k) y[(p0 + row) * R + a.j0] = sc * slot_get(acc[gg], e);
        }
      }
    }
  }
}

template <typename TB, typename ACC, int NG>
int dispatch_g(const ApplyArgs& a, int G, size_t smem, cudaStream_t s) {
  auto go = [&](auto kernel) -> int {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, NG * kGroup + 32, smem);
    per_sm = std::max(1, std::min(per_sm, 3));
    const int grid = std::max(1, std::min(a.n_sub, nsm * per_sm));
    ApplyArgs b = a;
    for (int j = 0; j < a.R; ++j) {
      b.j0 = j;
      kernel<<<grid, NG * kGroup + 32, smem, s>>>(b);
    }
    DDX_LAUNCH_CHECK("ddx_schwarz_local_apply");
    return DDX_OK;
  };
  if (G <= 1) return go(k_local_apply<TB, ACC, 1, NG>);
  if (G <= 2) return go(k_local_apply<TB, ACC, 2, NG>);
  if (G <= 4) return go(k_local_apply<TB, ACC, 4, NG>);
  if (G <= 8) return go(k_local_apply<TB, ACC, 8, NG>);
  if (G <= 16) return go(k_local_apply<TB, ACC, 16, NG>);
  set_error("ddx_schwarz_local_apply: kmax %d too large", a.kmax);
  return DDX_ERR_UNSUPPORTED;
}

template <typename TB, typename ACC>
int launch_apply_typed(ApplyArgs a, int groups, int stage_kb, cudaStream_t s) {
  constexpr int V = Vec16<TB>::V;
  a.ldmax = (a.kmax + V - 1) / V * V;
  const int g_need = (int)ceil_div(a.ldmax / V, kGroup);
  // row groups per thread as instantiated (dispatch_g rounds up to a power of two);
  // every per-thread buffer below is sized for this instantiated count
  int G = 1;
  while (G < g_need) G *= 2;
  if (groups <= 0) groups = 2;
  if (stage_kb <= 0) stage_kb = 20;
  if (groups != 1 && groups != 2 && groups != 4) {
    set_error("ddx_schwarz_local_apply: groups must be 1, 2 or 4 (got %d)", groups);
    return DDX_ERR_ARG;
  }
  const uint32_t colbytes = (uint32_t)a.ldmax * sizeof(TB);
  a.stage_bytes = std::max<uint32_t>((uint32_t)stage_kb * 1024u, (colbytes + 15u) / 16u * 16u);
  const size_t red_bytes = (size_t)(groups - 1) * G * V * kGroup * sizeof(ACC);
  a.red_elems = (int)((groups - 1) * G * V * kGroup);
  const size_t smem = 128 + (size_t)kStages * a.stage_bytes + (size_t)a.ldmax * sizeof(ACC) + red_bytes + 16;
  if (smem > 227 * 1024) {
    set_error("ddx_schwarz_local_apply: subdomain size %d with %d groups needs %zu bytes of shared memory", a.kmax,
              groups, smem);
    return DDX_ERR_UNSUPPORTED;
  }
  if (groups == 1) return dispatch_g<TB, ACC, 1>(a, G, smem, s);
  if (groups == 2) return dispatch_g<TB, ACC, 2>(a, G, smem, s);
  return dispatch_g<TB, ACC, 4>(a, G, smem, s);
}

}  // namespace
}  // namespace ddx

using namespace ddx;

extern "C" int ddx_schwarz_local_apply_ex(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                          const int* order, const int64_t* blk_off, const void* blocks,
                                          int block_dtype, const float* scale, int kmax, const double* r,
                                          void* ylocal, int acc_dtype, const int* ist, int groups, int stage_kb,
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
      return launch_apply_typed<double, double>(a, groups, stage_kb, s);
    case DDX_F32:
      // FP64 accumulation matches the reference's rule for FP32 blocks with
      // FP64 vectors (accumulate in the vector type)
      if (acc_dtype == DDX_F64) return launch_apply_typed<float, double>(a, groups, stage_kb, s);
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply: F32 blocks accumulate in F32 or F64");
      return launch_apply_typed<float, float>(a, groups, stage_kb, s);
    case DDX_BF16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply: BF16 blocks accumulate in F32");
      return launch_apply_typed<__nv_bfloat16, float>(a, groups, stage_kb, s);
    case DDX_F16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply: F16 blocks accumulate in F32");
      return launch_apply_typed<__half, float>(a, groups, stage_kb, s);
    default:
      set_error("ddx_schwarz_local_apply: unknown block dtype %d", block_dtype);
      return DDX_ERR_ARG;
  }
}

extern "C" int ddx_schwarz_local_apply(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                       const int* order, const int64_t* blk_off, const void* blocks, int block_dtype,
                                       const float* scale, int kmax, const double* r, void* ylocal, int acc_dtype,
                                       const int* ist, ddx_stream_t stream) {
  return ddx_schwarz_local_apply_ex(n_sub, R, sub_ptr, sub_idx, order, blk_off, blocks, block_dtype, scale, kmax, r,
                                    ylocal, acc_dtype, ist, 0, 0, stream);
}
