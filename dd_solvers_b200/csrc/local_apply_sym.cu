// Schwarz local-inverse apply on symmetric blocks stored as upper-triangle
// tiles: about half the bytes of the full blocks for the HBM-bound stream.
//
// Replaces Inv.solve -> gemv_strided_batched (src/dd_solvers/dd_solvers/solvers.py:355-359,
// src/dd_solvers/cpp/gemv_kernels.cu:59-139) for index-set subdomains:
//   ylocal[sub_ptr[i] + t, j] = scale[i] * sum_c Q_i[t, c] * r[sub_idx[sub_ptr[i] + c], j].
// The stored Q_i is exactly symmetric (the FP64 inverse is symmetrised before
// rounding), so only its 32 x 32 tiles (I, J), I <= J, are kept (row-major
// order of (I, J); each tile row-major with its 16-byte chunks XOR-swizzled by
// the row, see setup_ops.sym_tile_index). Tile (I, J) contributes
//   y_I += T x_J                 and, for I < J,   y_J += T^T x_I.
//
// Persistent CTAs walk a size-sorted list of work items (block, part): with
// parts > 1 (few, large blocks: not enough blocks to fill the SMs) part s of a
// block takes tiles [s T / parts, (s + 1) T / parts) of its T tiles and writes
// its partial y to ylocal slice s (slices sum_i k_i x R apart; the combine adds
// them). One producer thread streams the tiles through a ring of four
// shared-memory stages
// (cp.async.bulk + mbarriers). W consumer warps take the tiles round-robin; in
// a warp, lane t loads row t of the tile (16-byte loads, conflict-free thanks
// to the swizzle) for the row sum sum_c T[t, c] x_J[c] -> y_I[t], and the
// lanes read the tile's columns (ColProd) for sum_t T[t, c] x_I[t] -> y_J[c]:
// each tile crosses HBM once and shared memory twice. Each warp adds into its
// own slice of a shared-memory y (no atomics); the slices are summed in warp
// order at the end of the block, so results are bitwise repeatable.
// Every wait is bounded (device error word).
#include <algorithm>

#include "pipeline.cuh"

namespace ddx {
using namespace pipe;

namespace {

constexpr int kT = 32;           // tile edge
constexpr int kTE = kT * kT;     // elements per tile
constexpr int kSymStages = 4;

// Row t of a tile as 32 accumulator-type values, undoing the chunk swizzle
// (16-bit types: 4 chunks of 8, XOR (t >> 1) & 3; FP32: 8 chunks of 4, XOR t & 7;
// FP64: 16 chunks of 2, XOR t & 7).
template <typename TB, typename ACC> struct RowLoad;

template <> struct RowLoad<__nv_bfloat16, float> {
  static __device__ __forceinline__ void load(const unsigned char* tile, int t, float* v) {
    const unsigned char* row = tile + t * 64;
    const int sw = (t >> 1) & 3;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 u = *reinterpret_cast<const uint4*>(row + ((q ^ sw) << 4));
      const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        // BF16 -> FP32 is exact: the BF16 bits are the upper half of the FP32 bits
        v[q * 8 + 2 * h] = __uint_as_float(w[h] << 16);
        v[q * 8 + 2 * h + 1] = __uint_as_float(w[h] & 0xffff0000u);
      }
    }
  }
};
template <> struct RowLoad<__half, float> {
  static __device__ __forceinline__ void load(const unsigned char* tile, int t, float* v) {
    const unsigned char* row = tile + t * 64;
    const int sw = (t >> 1) & 3;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 u = *reinterpret_cast<const uint4*>(row + ((q ^ sw) << 4));
      const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[h]));
        v[q * 8 + 2 * h] = f.x;
        v[q * 8 + 2 * h + 1] = f.y;
      }
    }
  }
};
template <typename ACC> struct RowLoad<float, ACC> {
  static __device__ __forceinline__ void load(const unsigned char* tile, int t, ACC* v) {
    const unsigned char* row = tile + t * 128;
    const int sw = t & 7;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 f = *reinterpret_cast<const float4*>(row + ((q ^ sw) << 4));
      v[q * 4] = (ACC)f.x;
      v[q * 4 + 1] = (ACC)f.y;
      v[q * 4 + 2] = (ACC)f.z;
      v[q * 4 + 3] = (ACC)f.w;
    }
  }
};
template <> struct RowLoad<double, double> {
  static __device__ __forceinline__ void load(const unsigned char* tile, int t, double* v) {
    const unsigned char* row = tile + t * 256;
    const int sw = t & 7;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const double2 d = *reinterpret_cast<const double2*>(row + ((q ^ sw) << 4));
      v[q * 2] = d.x;
      v[q * 2 + 1] = d.y;
    }
  }
};

// Column product y_J[c] += sum_t T[t, c] x_I[t] read straight from the
// shared-memory tile (no cross-lane reduction of 32 values).
//  16-bit types: lane l takes the column pair (2 cp, 2 cp + 1), cp = l % 16, over
//    the rows of parity h = l / 16: one 32-bit load per row (the swizzle of row
//    2i + h is i & 3, so lanes 0-15 and 16-31 read the two halves of the bank
//    range: conflict-free), packed FP32x2 FMAs, then the two parities are added
//    with one exchange; lanes 0-15 update y_J.
//  FP32 / FP64: lane l takes column l over all 32 rows (row r is read by the
//    whole warp at once: conflict-free).
template <typename TB, typename ACC> struct ColProd;

template <typename TB> struct ColProd16 {
  static __device__ __forceinline__ float2 cvt(uint32_t w);
  static __device__ __forceinline__ void add(const unsigned char* tile, int lane, const float* xI, float* yJ) {
    const int h = lane >> 4, cp = lane & 15, q = cp >> 2;
    const unsigned char* base = tile + h * 64 + ((cp & 3) << 2);
    const unsigned char* b4[4] = {base + ((q ^ 0) << 4), base + ((q ^ 1) << 4), base + ((q ^ 2) << 4),
                                  base + ((q ^ 3) << 4)};
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const uint32_t w = *reinterpret_cast<const uint32_t*>(b4[i & 3] + i * 128);
      const float xv = xI[2 * i + h];
      acc = __ffma2_rn(cvt(w), make_float2(xv, xv), acc);
    }
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 16);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 16);
    if (lane < 16) {
      float2* y2 = reinterpret_cast<float2*>(yJ) + cp;
      float2 t = *y2;
      t.x += acc.x;
      t.y += acc.y;
      *y2 = t;
    }
  }
};
template <> __device__ __forceinline__ float2 ColProd16<__nv_bfloat16>::cvt(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}
template <> __device__ __forceinline__ float2 ColProd16<__half>::cvt(uint32_t w) {
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}
template <> struct ColProd<__nv_bfloat16, float> : ColProd16<__nv_bfloat16> {};
template <> struct ColProd<__half, float> : ColProd16<__half> {};

template <typename ACC> struct ColProd<float, ACC> {
  static __device__ __forceinline__ void add(const unsigned char* tile, int lane, const ACC* xI, ACC* yJ) {
    const float* t = reinterpret_cast<const float*>(tile);
    const int q = lane >> 2, e = lane & 3;
    ACC acc0 = ACC(0), acc1 = ACC(0);
#pragma unroll
    for (int r = 0; r < kT; r += 2) {
      acc0 = fma((ACC)t[r * 32 + ((q ^ (r & 7)) << 2) + e], xI[r], acc0);
      acc1 = fma((ACC)t[(r + 1) * 32 + ((q ^ ((r + 1) & 7)) << 2) + e], xI[r + 1], acc1);
    }
    yJ[lane] += acc0 + acc1;
  }
};
template <> struct ColProd<double, double> {
  static __device__ __forceinline__ void add(const unsigned char* tile, int lane, const double* xI, double* yJ) {
    const double* t = reinterpret_cast<const double*>(tile);
    const int q = lane >> 1, e = lane & 1;
    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
    for (int r = 0; r < kT; r += 2) {
      acc0 = fma(t[r * 32 + ((q ^ (r & 7)) << 1) + e], xI[r], acc0);
      acc1 = fma(t[(r + 1) * 32 + ((q ^ ((r + 1) & 7)) << 1) + e], xI[r + 1], acc1);
    }
    yJ[lane] += acc0 + acc1;
  }
};

// Row product sum_c v[c] x_J[c] (x_J 16-byte aligned in shared memory).
__device__ __forceinline__ float row_dot(const float (&v)[kT], const float* xj) {
  float2 acc0 = make_float2(0.f, 0.f), acc1 = make_float2(0.f, 0.f);
  const float4* x4 = reinterpret_cast<const float4*>(xj);
#pragma unroll
  for (int c = 0; c < kT; c += 4) {
    const float4 x = x4[c / 4];
    acc0 = __ffma2_rn(make_float2(v[c], v[c + 1]), make_float2(x.x, x.y), acc0);
    acc1 = __ffma2_rn(make_float2(v[c + 2], v[c + 3]), make_float2(x.z, x.w), acc1);
  }
  return (acc0.x + acc1.x) + (acc0.y + acc1.y);
}
__device__ __forceinline__ double row_dot(const double (&v)[kT], const double* xj) {
  double acc0 = 0.0, acc1 = 0.0;
  const double2* x2 = reinterpret_cast<const double2*>(xj);
#pragma unroll
  for (int c = 0; c < kT; c += 2) {
    const double2 x = x2[c / 2];
    acc0 = fma(v[c], x.x, acc0);
    acc1 = fma(v[c + 1], x.y, acc1);
  }
  return acc0 + acc1;
}

struct SymArgs {
  int n_sub, R, j0;
  const int64_t* sub_ptr;
  const int* sub_idx;
  const int* order;
  const int64_t* blk_off;  // elements
  const void* blocks;
  const float* scale;
  const double* r;
  void* ylocal;
  const int* ist;
  int tiles_per_stage;
  int kpad_max;  // ceil(kmax / 32) * 32
  int kmax;
  int parts;  // tile ranges per block (work items = blocks x parts); the ylocal
             // slice of part s starts s * sub_ptr[n_sub] * R elements in
};

// Tile range [ta, tb) of part s of a block with ntiles tiles.
__device__ __forceinline__ void part_range(int ntiles, int parts, int s, int& ta, int& tb) {
  ta = (int)((int64_t)ntiles * s / parts);
  tb = (int)((int64_t)ntiles * (s + 1) / parts);
}

template <typename TB, typename ACC, int W>
__global__ void __launch_bounds__(W * 32 + 32) k_local_apply_sym(SymArgs a) {
  constexpr int NC = W * 32;
  constexpr int TILE_BYTES = kTE * (int)sizeof(TB);
  extern __shared__ __align__(128) unsigned char smem[];
  if (a.ist != nullptr && n_active(a.ist, a.R) == 0) return;

  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kSymStages;
  __shared__ int abort_s;
  volatile int& abort_flag = abort_s;
  const uint32_t stage_bytes = (uint32_t)a.tiles_per_stage * TILE_BYTES;
  unsigned char* stage_base = smem + 128;
  ACC* xs = reinterpret_cast<ACC*>(stage_base + (size_t)kSymStages * stage_bytes);
  ACC* ys = xs + a.kpad_max;  // W slices of kpad_max

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kSymStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], W);  // one arrival per consumer warp
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
    for (int w = blockIdx.x; w < a.n_sub * a.parts && !abort_flag; w += gridDim.x) {
      const int i = a.order[w / a.parts];
      const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
      if (k == 0 || k > a.kmax) continue;
      const int nt = (k + kT - 1) / kT;
      int ta, tb;
      part_range(nt * (nt + 1) / 2, a.parts, w % a.parts, ta, tb);
      const int nchunk = (tb - ta + a.tiles_per_stage - 1) / a.tiles_per_stage;
      const TB* src = blocks + a.blk_off[i];
      for (int q = 0; q < nchunk; ++q, ++g) {
        const int s = g % kSymStages;
        if (!mbar_wait(&empty[s], ((g / kSymStages) & 1u) ^ 1u)) { abort_flag = 1; return; }
        const int t0 = ta + q * a.tiles_per_stage;
        const int nt_here = min(a.tiles_per_stage, tb - t0);
        const uint32_t bytes = (uint32_t)nt_here * TILE_BYTES;
        mbar_arrive_expect_tx(&full[s], bytes);
        bulk_g2s(stage_base + (size_t)s * stage_bytes, src + (int64_t)t0 * kTE, bytes, &full[s]);
      }
    }
    return;
  }

  // ------------------------------ consumers ------------------------------
  const int warp = tid >> 5, lane = tid & 31;
  const int R = a.R;
  ACC* yw = ys + (size_t)warp * a.kpad_max;
  uint32_t g = 0;
  for (int w = blockIdx.x; w < a.n_sub * a.parts; w += gridDim.x) {
    const int i = a.order[w / a.parts];
    const int part = w % a.parts;
    const int64_t p0 = a.sub_ptr[i];
    const int k = (int)(a.sub_ptr[i + 1] - p0);
    if (k == 0) continue;
    if (k > a.kmax) {  // would overflow the shared-memory buffers
      if (tid == 0) atomicOr(&g_device_error, DEVERR_BAD_SIZE);
      continue;
    }
    const int nt = (k + kT - 1) / kT;
    const int kp = nt * kT;
    int ta, tb;
    part_range(nt * (nt + 1) / 2, a.parts, part, ta, tb);
    const int nchunk = (tb - ta + a.tiles_per_stage - 1) / a.tiles_per_stage;
    named_sync(1, NC);  // previous subdomain done with xs and ys
    if (abort_flag) break;
    for (int c = tid; c < kp; c += NC) xs[c] = c < k ? (ACC)a.r[(int64_t)a.sub_idx[p0 + c] * R + a.j0] : ACC(0);
    for (int e = tid; e < W * kp; e += NC) ys[(e / kp) * a.kpad_max + e % kp] = ACC(0);
    named_sync(1, NC);

    // this warp's tiles: tau = ta + warp, ta + warp + W, ... in row-major
    // (I, J >= I) order; row I holds J = I..nt-1 and starts at tile
    // I nt - I (I - 1) / 2, so stepping past its end continues at J - nt + I + 1
    // of row I + 1
    int tau = ta + warp;
    int I = 0, row_start = 0;
    while (I < nt && row_start + (nt - I) <= tau) {
      row_start += nt - I;
      ++I;
    }
    int J = I + (tau - row_start);
    for (int q = 0; q < nchunk; ++q) {
      const uint32_t gq = g + (uint32_t)q;
      const int s = gq % kSymStages;
      const int t0 = ta + q * a.tiles_per_stage;
      const int t1 = min(t0 + a.tiles_per_stage, tb);
      if (abort_flag) break;
      // every warp waits for every stage before releasing it, with or without
      // tiles of its own there: a warp can then never arrive twice on one
      // phase of `empty` (which would free the stage while another warp reads it)
      if (!mbar_wait(&full[s], (gq / kSymStages) & 1u)) { abort_flag = 1; break; }
      {
        const unsigned char* st = stage_base + (size_t)s * stage_bytes;
        for (; tau < t1; tau += W) {
          const unsigned char* tile = st + (size_t)(tau - t0) * TILE_BYTES;
          ACC v[kT];
          RowLoad<TB, ACC>::load(tile, lane, v);
          yw[I * kT + lane] += row_dot(v, xs + J * kT);
          if (I != J) ColProd<TB, ACC>::add(tile, lane, xs + I * kT, yw + J * kT);
          // next tile of this warp: advance W positions in row-major (I, J >= I) order
          J += W;
          while (J >= nt && I < nt) { ++I; J = J - nt + I; }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);  // every warp releases every stage of the block
    }
    g += (uint32_t)nchunk;
    named_sync(1, NC);  // all warps' slices complete
    if (abort_flag) break;
    const ACC sc = a.scale ? (ACC)a.scale[i] : ACC(1);
    ACC* y = reinterpret_cast<ACC*>(a.ylocal) + (int64_t)part * a.sub_ptr[a.n_sub] * R;
    for (int row = tid; row < k; row += NC) {
      ACC sum = ACC(0);
#pragma unroll
      for (int ww = 0; ww < W; ++ww) sum += ys[(size_t)ww * a.kpad_max + row];
      y[(p0 + row) * R + a.j0] = sc * sum;
    }
  }
}

template <typename TB, typename ACC, int W>
int launch_sym_w(SymArgs a, int stage_kb, cudaStream_t s) {
  constexpr int TILE_BYTES = kTE * (int)sizeof(TB);
  a.tiles_per_stage = std::max(1, stage_kb * 1024 / TILE_BYTES);
  const size_t smem = 128 + (size_t)kSymStages * a.tiles_per_stage * TILE_BYTES +
                      (size_t)(W + 1) * a.kpad_max * sizeof(ACC) + 16;
  if (smem > 227 * 1024) {
    set_error("ddx_schwarz_local_apply_sym: subdomain size %d with %d warps needs %zu bytes of shared memory",
              a.kmax, W, smem);
    return DDX_ERR_UNSUPPORTED;
  }
  auto kernel = k_local_apply_sym<TB, ACC, W>;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, nsm = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, W * 32 + 32, smem);
  per_sm = std::max(1, std::min(per_sm, 4));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)a.n_sub * a.parts, (int64_t)nsm * per_sm));
  for (int j = 0; j < a.R; ++j) {
    a.j0 = j;
    kernel<<<grid, W * 32 + 32, smem, s>>>(a);
  }
  DDX_LAUNCH_CHECK("ddx_schwarz_local_apply_sym");
  return DDX_OK;
}

template <typename TB, typename ACC>
int launch_sym(SymArgs a, int warps, int stage_kb, cudaStream_t s) {
  if (warps <= 0) warps = 8;
  if (stage_kb <= 0) stage_kb = 16;
  if (warps == 4) return launch_sym_w<TB, ACC, 4>(a, stage_kb, s);
  if (warps == 8) return launch_sym_w<TB, ACC, 8>(a, stage_kb, s);
  if (warps == 16) return launch_sym_w<TB, ACC, 16>(a, stage_kb, s);
  set_error("ddx_schwarz_local_apply_sym: warps must be 4, 8 or 16 (got %d)", warps);
  return DDX_ERR_ARG;
}

}  // namespace
}  // namespace ddx

using namespace ddx;

extern "C" int ddx_schwarz_local_apply_sym(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                           const int* order, const int64_t* blk_off, const void* blocks,
                                           int block_dtype, const float* scale, int kmax, const double* r,
                                           void* ylocal, int acc_dtype, const int* ist, int warps, int stage_kb,
                                           int parts, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_schwarz_local_apply_sym: unsupported R=%d", R);
  DDX_REQUIRE(n_sub >= 0 && kmax >= 0, "ddx_schwarz_local_apply_sym: bad sizes");
  if (n_sub == 0 || kmax == 0) return DDX_OK;
  DDX_REQUIRE(sub_ptr && sub_idx && order && blk_off && blocks && r && ylocal,
              "ddx_schwarz_local_apply_sym: null pointer");
  DDX_REQUIRE(((uintptr_t)blocks & 15u) == 0, "ddx_schwarz_local_apply_sym: blocks must be 16-byte aligned");
  SymArgs a{};
  a.n_sub = n_sub;
  a.R = R;
  a.sub_ptr = sub_ptr;
  a.sub_idx = sub_idx;
  a.order = order;
  a.blk_off = blk_off;
  a.blocks = blocks;
  a.scale = scale;
  a.r = r;
  a.ylocal = ylocal;
  a.ist = ist;
  DDX_REQUIRE(parts >= 1 && parts <= 64, "ddx_schwarz_local_apply_sym: parts must be 1..64 (got %d)", parts);
  a.kmax = kmax;
  a.kpad_max = (kmax + kT - 1) / kT * kT;
  a.parts = parts;
  cudaStream_t s = (cudaStream_t)stream;
  switch (block_dtype) {
    case DDX_F64:
      DDX_REQUIRE(acc_dtype == DDX_F64, "ddx_schwarz_local_apply_sym: FP64 blocks accumulate in FP64");
      return launch_sym<double, double>(a, warps, stage_kb, s);
    case DDX_F32:
      if (acc_dtype == DDX_F64) return launch_sym<float, double>(a, warps, stage_kb, s);
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply_sym: bad acc dtype %d", acc_dtype);
      return launch_sym<float, float>(a, warps, stage_kb, s);
    case DDX_BF16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply_sym: BF16 blocks accumulate in FP32");
      return launch_sym<__nv_bfloat16, float>(a, warps, stage_kb, s);
    case DDX_F16:
      DDX_REQUIRE(acc_dtype == DDX_F32, "ddx_schwarz_local_apply_sym: FP16 blocks accumulate in FP32");
      return launch_sym<__half, float>(a, warps, stage_kb, s);
    default:
      set_error("ddx_schwarz_local_apply_sym: block dtype %d", block_dtype);
      return DDX_ERR_ARG;
  }
}
