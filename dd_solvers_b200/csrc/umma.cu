// Multi-RHS Schwarz local apply on the 5th-generation tensor cores (tcgen05).
//
// For many right-hand sides the local solve of subdomain i is a dense product
// Y_i (k x R) = Q_i (k x k) * X_i (k x R), X_i = r[idx_i, :], i.e. a GEMM with
// N = R, which the SIMT streaming kernel cannot feed at HBM speed. Layout per
// persistent CTA (one per SM):
//   warp 0      producer: per subdomain, the B panel X_i (written by
//               ddx_pack_panels16 already gathered, converted to 16 bits and
//               in the MN-major swizzled UMMA layout) with one cp.async.bulk
//               per 64-row chunk into the resident panel buffer, then the
//               128x64 BF16/FP16 tiles of Q_i, stored in HBM already in the
//               K-major 128-byte-swizzled layout, one cp.async.bulk per tile
//               into a 4-stage ring.
//   warp 1      allocates TMEM; one lane issues tcgen05.mma (M=128, N=R, K=16)
//               and tcgen05.commit to release ring stages / the panel and to
//               publish results.
//   warps 2..5  drain each 128-row accumulator from TMEM (tcgen05.ld), scale,
//               and store ylocal (FP32).
// Two TMEM accumulators (2 x R columns) let the epilogue of row tile m overlap
// the MMAs of row tile m+1. Every wait is bounded (device error word). No
// thread of this kernel issues a dependent global load on the B path: the
// gather through the subdomain index map happens in the pack kernel, where
// every thread has its own independent loads in flight.
//
// Residual terms. Rounding r to 16 bits perturbs Q_i r by up to
// cond(A_i) * 2^-p relative (p = 8 for BF16, 11 for FP16), which stalls PCG
// once the local blocks are ill conditioned (high-contrast coefficients,
// large 2D subdomains). With TERMS = 2 the pack writes r ~ hi + lo (hi the
// 16-bit rounding of r, lo that of r - hi) as two panels, and each K step
// issues one MMA per panel into the same accumulator: the product sees r to
// ~2^-2p, the A stream (the HBM cost) is read once.
#include <algorithm>

#include "common.cuh"

namespace ddx {
namespace umma {

constexpr int kM = 128;
constexpr int kK = 64;              // 16-bit elements per 128-byte swizzle row
constexpr int kStages = 4;
constexpr int kTileBytes = kM * 128; // 16 KB
constexpr int kThreads = 192;
constexpr int kEpiThreads = 128;
constexpr int kPanelSlack = 2048;

// 64-row chunks per residual term of a subdomain's B panel in HBM: whole pairs
// (128 rows), so the symmetric kernel's 128-row K steps stay inside the panel.
__host__ __device__ __forceinline__ int panel_chunks(int k) { return 2 * ((k + 127) / 128); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait (2 s); false on timeout (recorded in the device error word).
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
      const uint64_t t = gtimer();
      if (t0 == 0) t0 = t;
      else if (t - t0 > 2000000000ull) {
        atomicOr(&g_device_error, DEVERR_MBAR_TIMEOUT);
        return false;
      }
    }
  }
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (sm_100 format):
// start address >> 4 in bits 0-13, leading byte offset (unused for swizzled
// K-major, 16 B) in 16-29, stride byte offset 1024 B (8 rows x 128 B) in 32-45,
// descriptor version 1 in 46-47, layout type 2 (128B swizzle) in 61-63.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

// MN-major B panel: one row of N 16-bit values (2N bytes) per K index, the
// swizzle as wide as a row (128 / 64 / 32 bytes for N = 64 / 32 / 16), atoms of
// 8 rows at stride SBO = 16 N bytes. LBO (stride between MN atoms) is unused
// because N fits in one atom. Layout codes: 2 = 128B, 4 = 64B, 6 = 32B.
template <int N>
__device__ __forceinline__ uint64_t mn_desc(uint32_t saddr) {
  constexpr uint32_t sbo = 16u * N;
  constexpr uint64_t layout = N == 64 ? 2u : (N == 32 ? 4u : 6u);
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(sbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         ((uint64_t)1u << 46) | (layout << 61);
}

// Byte offset of 16-byte chunk q of panel row c under the row-wide swizzle
// (address bits [4,7) XOR bits [7,10), masked to the swizzle width).
template <int N>
__device__ __forceinline__ uint32_t mn_offset(int c, int q) {
  constexpr uint32_t mask = N == 64 ? 7u : (N == 32 ? 3u : 1u);
  const uint32_t L = (uint32_t)c * (2u * N) + (uint32_t)q * 16u;
  return L ^ (((L >> 7) & mask) << 4);
}

// Instruction descriptor, kind::f16: D F32 (bits 4-5 = 1), A/B format in bits
// 7-9 / 10-12 (F16 = 0, BF16 = 1), A K-major (bit 15 = 0), B MN-major
// (bit 16 = 1), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_f16(int ab_fmt, int N) {
  return (1u << 4) | ((uint32_t)ab_fmt << 7) | ((uint32_t)ab_fmt << 10) | (1u << 16) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(kM >> 4) << 24);
}


__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 32 lanes x 16 consecutive columns of FP32 from TMEM; the wait is tied to the
// destination registers so no use can be scheduled before it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t u0, u1, u2, u3, u4, u5, u6, u7, u8, u9, u10, u11, u12, u13, u14, u15;
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(u0), "=r"(u1), "=r"(u2), "=r"(u3), "=r"(u4), "=r"(u5), "=r"(u6), "=r"(u7), "=r"(u8), "=r"(u9),
        "=r"(u10), "=r"(u11), "=r"(u12), "=r"(u13), "=r"(u14), "=r"(u15)
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(u0), "+r"(u1), "+r"(u2), "+r"(u3), "+r"(u4), "+r"(u5), "+r"(u6), "+r"(u7), "+r"(u8),
                 "+r"(u9), "+r"(u10), "+r"(u11), "+r"(u12), "+r"(u13), "+r"(u14), "+r"(u15)
               :
               : "memory");
  v[0] = __uint_as_float(u0); v[1] = __uint_as_float(u1); v[2] = __uint_as_float(u2); v[3] = __uint_as_float(u3);
  v[4] = __uint_as_float(u4); v[5] = __uint_as_float(u5); v[6] = __uint_as_float(u6); v[7] = __uint_as_float(u7);
  v[8] = __uint_as_float(u8); v[9] = __uint_as_float(u9); v[10] = __uint_as_float(u10);
  v[11] = __uint_as_float(u11); v[12] = __uint_as_float(u12); v[13] = __uint_as_float(u13);
  v[14] = __uint_as_float(u14); v[15] = __uint_as_float(u15);
}

struct Args {
  int n_sub;
  const int64_t* sub_ptr;
  const int* order;
  const int64_t* tile_off;  // bytes
  const unsigned char* tiles;
  const float* scale;
  const unsigned char* b16;    // per-subdomain B panels (ddx_pack_panels16)
  const int64_t* panel_off;    // bytes
  float* ylocal;
  const int* ist;
  const double* st;  // PCG state (||r_j||^2 scales the 16-bit conversion); may be null
  int kmax;
};

using ::ddx::from_bits;
using ::ddx::rhs_scale;
using ::ddx::to_bits;

template <typename T, int N, int TERMS>
__global__ void __launch_bounds__(kThreads, 1) k_apply_tc(Args a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* ring = smem;                                  // kStages x 16 KB
  unsigned char* bbuf = smem + kStages * kTileBytes;           // TERMS x nK x (N x 128 B)
  const int nk_max = (a.kmax + kK - 1) / kK;
  const uint32_t panel_bytes = (uint32_t)nk_max * N * 128;    // a multiple of 1024: every panel is atom aligned
  // 2 KiB of slack after the B panels keeps every operand read inside this CTA's shared memory
  uint64_t* bars = reinterpret_cast<uint64_t*>(bbuf + (size_t)TERMS * panel_bytes + kPanelSlack);
  uint64_t* a_full = bars;
  uint64_t* a_empty = bars + kStages;
  uint64_t* b_full = bars + 2 * kStages;
  uint64_t* b_empty = b_full + 1;
  uint64_t* acc_full = b_full + 2;   // [2]
  uint64_t* acc_empty = b_full + 4;  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(b_full + 6);
  __shared__ int abort_flag_s;
  volatile int& abort_flag = abort_flag_s;
  __shared__ float rhs_unscale[64];  // 1 / (per-RHS conversion scale)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (a.ist != nullptr && n_active(a.ist, N) == 0) return;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&a_full[s], 1);
      mbar_init(&a_empty[s], 1);
    }
    mbar_init(b_full, 1);
    mbar_init(b_empty, 1);
    for (int s = 0; s < 2; ++s) {
      mbar_init(&acc_full[s], 1);
      mbar_init(&acc_empty[s], kEpiThreads / 32);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < N) rhs_unscale[threadIdx.x] = 1.0f / rhs_scale<T>(a.st, N, threadIdx.x);
  constexpr uint32_t kCols = (2 * N < 32) ? 32 : 2 * N;  // power of two >= 32
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      uint32_t g = 0, sub_n = 0;
      for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
        const int i = a.order[w];
        const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
        if (k == 0 || k > a.kmax) continue;
        const int nK = (k + kK - 1) / kK;
        // B panel: the previous subdomain's MMAs must have finished reading it
        if (!mbar_wait(b_empty, (sub_n & 1u) ^ 1u)) { abort_flag = 1; break; }
        ++sub_n;
        constexpr uint32_t chunk_bytes = (uint32_t)kK * 2u * N;  // 64 panel rows
        const int nKp = panel_chunks(k);                           // chunks per term in HBM
        mbar_expect_tx(b_full, (uint32_t)TERMS * (uint32_t)nK * chunk_bytes);
        for (int tt = 0; tt < TERMS; ++tt) {
          const unsigned char* psrc = a.b16 + a.panel_off[i] + (size_t)tt * nKp * chunk_bytes;
          for (int t = 0; t < nK; ++t, psrc += chunk_bytes)
            bulk_g2s(bbuf + (size_t)tt * panel_bytes + (size_t)t * chunk_bytes, psrc, chunk_bytes, b_full);
        }
        const unsigned char* src = a.tiles + a.tile_off[i];
        for (int m0 = 0; m0 < k; m0 += kM) {
          const int rows = (min(kM, k - m0) + 7) / 8 * 8;
          const uint32_t bytes = (uint32_t)rows * 128u;
          for (int t = 0; t < nK; ++t, ++g) {
            const int s = g % kStages;
            if (!mbar_wait(&a_empty[s], ((g / kStages) & 1u) ^ 1u)) { abort_flag = 1; break; }
            mbar_expect_tx(&a_full[s], bytes);
            bulk_g2s(ring + (size_t)s * kTileBytes, src, bytes, &a_full[s]);
            src += bytes;
          }
          if (abort_flag) break;
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------ MMA issuer -----------------------------
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_f16(std::is_same<T, __nv_bfloat16>::value ? 1 : 0, N);
      uint32_t g = 0, acc_n = 0, sub_n = 0;
      for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
        const int i = a.order[w];
        const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
        if (k == 0 || k > a.kmax) continue;
        const int nK = (k + kK - 1) / kK;
        if (!mbar_wait(b_full, sub_n & 1u)) { abort_flag = 1; break; }
        fence_after();
        for (int m0 = 0; m0 < k; m0 += kM, ++acc_n) {
          const uint32_t ab = acc_n & 1u;
          if (!mbar_wait(&acc_empty[ab], ((acc_n >> 1) & 1u) ^ 1u)) { abort_flag = 1; break; }
          fence_after();
          const uint32_t d = tmem + ab * N;
          for (int t = 0; t < nK; ++t, ++g) {
            const int s = g % kStages;
            if (!mbar_wait(&a_full[s], (g / kStages) & 1u)) { abort_flag = 1; break; }
            fence_after();
            const uint32_t sa = smem_u32(ring + (size_t)s * kTileBytes);
            const uint32_t sb = smem_u32(bbuf + (size_t)t * N * 128);
#pragma unroll
            for (int kk = 0; kk < kK / 16; ++kk)
#pragma unroll
              for (int tt = 0; tt < TERMS; ++tt)
                mma_f16(d, sw128_desc(sa + kk * 32), mn_desc<N>(sb + tt * panel_bytes + kk * 32 * N), idesc,
                        (t > 0 || kk > 0 || tt > 0) ? 1u : 0u);
            mma_commit(&a_empty[s]);
          }
          if (abort_flag) break;
          mma_commit(&acc_full[ab]);
        }
        if (abort_flag) break;
        mma_commit(b_empty);
        ++sub_n;
      }
    }
  } else {
    // ------------------------------ epilogue --------------------------------
    const int e = threadIdx.x - 64;   // 0..127
    const int quarter = warp & 3;     // TMEM lane quarter this warp may access
    uint32_t acc_n = 0;
    for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
      const int i = a.order[w];
      const int64_t p0 = a.sub_ptr[i];
      const int k = (int)(a.sub_ptr[i + 1] - p0);
      if (k == 0) continue;
      if (k > a.kmax) {
        if (e == 0) atomicOr(&g_device_error, DEVERR_BAD_SIZE);
        continue;
      }
      // epilogue per 128-row tile
      const float sc = a.scale ? a.scale[i] : 1.0f;
      for (int m0 = 0; m0 < k; m0 += kM, ++acc_n) {
        const uint32_t ab = acc_n & 1u;
        if (!mbar_wait(&acc_full[ab], (acc_n >> 1) & 1u)) { abort_flag = 1; break; }
        fence_after();
        float v[N];
#pragma unroll
        for (int c = 0; c < N; c += 16) tmem_ld16(tmem + ab * N + c + ((uint32_t)(quarter * 32) << 16), v + c);
        fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[ab]);
        const int row = m0 + quarter * 32 + lane;
        if (row < k) {
          float4* dst = reinterpret_cast<float4*>(a.ylocal + (p0 + row) * N);
#pragma unroll
          for (int c = 0; c < N; c += 4)
            dst[c / 4] = make_float4(sc * rhs_unscale[c] * v[c], sc * rhs_unscale[c + 1] * v[c + 1],
                                     sc * rhs_unscale[c + 2] * v[c + 2], sc * rhs_unscale[c + 3] * v[c + 3]);
        }
      }
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

template <typename T, int N, int TERMS>
static int launch(const Args& a, cudaStream_t s) {
  const int nk_max = (a.kmax + kK - 1) / kK;
  const size_t smem =
      1024 + (size_t)kStages * kTileBytes + (size_t)TERMS * nk_max * N * 128 + kPanelSlack + 16 * 8 + 64;
  if (smem > 227 * 1024) {
    set_error("ddx_schwarz_local_apply_tc: k=%d with R=%d and %d residual terms needs %zu bytes of shared memory",
              a.kmax, N, TERMS, smem);
    return DDX_ERR_UNSUPPORTED;
  }
  auto kern = k_apply_tc<T, N, TERMS>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min(a.n_sub, nsm));
  kern<<<grid, kThreads, smem, s>>>(a);
  DDX_LAUNCH_CHECK("ddx_schwarz_local_apply_tc");
  return DDX_OK;
}

// ---------------------------------------------------------------------------
// Symmetric blocks: upper-triangle 128 x 128 tiles
// ---------------------------------------------------------------------------
// Q_i (exactly symmetric) stored as its tiles (I, J), I <= J, of 128 x 128,
// row-major order of (I, J), each as two 128 x 64 halves (columns 0-63, 64-127
// of the tile) in the K-major 128-byte-swizzled layout of the full-block kernel,
// zero beyond k: 32 KB per tile, one bulk copy per tile. Tile (I, J) serves
//   D_I += T X_J   (A = the tile, K-major: rows along I, K along J) and, for I < J,
//   D_J += T^T X_I (A = the same shared memory read MN-major: its 128-byte rows
//                   run along J (M), its rows along I (K); the two halves are
//                   M-atoms 16 KB apart (LBO), 8-row groups 1 KB apart (SBO)).
// The swizzle is a function of the shared-memory address, so one layout serves
// both readings. Every row-tile accumulator of a block lives in TMEM at once
// (nt x N columns, nt = ceil(k / 128)); the epilogue drains them after the
// block's last MMA.

// MN-major 128-byte-swizzle descriptor: LBO = stride between 64-element
// M-atoms, SBO = stride between 8-row K groups (1024 B), version 1, layout 2.
__device__ __forceinline__ uint64_t sw128_mn_desc(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(1024u >> 4) << 32) | ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

// Instruction descriptor as idesc_f16 with A MN-major (bit 15).
__host__ __device__ constexpr uint32_t idesc_f16_amn(int ab_fmt, int N) { return idesc_f16(ab_fmt, N) | (1u << 15); }

constexpr int kSymTile = 128;
constexpr int kSymTileBytes = kSymTile * kSymTile * 2;  // 32 KB
constexpr int kHalfBytes = kSymTileBytes / 2;           // 16 KB
constexpr int kSymMaxStages = 6;
// Shared memory after the panels, never addressed by an operand descriptor
// (a margin between the last panel byte and the end of the allocation).
constexpr int kSymSlack = 1024;

// Row tiles (128 rows) of the largest block: all their accumulators live in
// TMEM at once (nt x N of the 512 columns); at most 24, so the barriers and
// the per-RHS scales fit in the 1 KB control area.
template <int N>
__host__ __device__ constexpr int sym_max_row_tiles() { return 512 / N < 24 ? 512 / N : 24; }

// Control area at the start of the (1024-byte aligned) dynamic shared memory:
// a_full/a_empty per ring stage, p_full/p_empty per 128-row panel chunk,
// acc_full/acc_empty per row-tile accumulator, the TMEM address, the abort flag
// and the per-RHS unscale factors.
template <int N>
struct SymCtl {
  static constexpr int MT = sym_max_row_tiles<N>();
  uint64_t a_full[kSymMaxStages], a_empty[kSymMaxStages];
  uint64_t p_full[MT], p_empty[MT];
  uint64_t acc_full[MT], acc_empty[MT];
  uint32_t tmem_slot;
  int abort_flag;
  float rhs_unscale[N];
};
static_assert(sizeof(SymCtl<16>) <= 1024 && sizeof(SymCtl<32>) <= 1024 && sizeof(SymCtl<64>) <= 1024,
              "control area exceeds 1 KB");

// Dynamic shared memory of the symmetric kernel: alignment margin, control
// area, STAGES tiles of 32 KB, TERMS B panels of the largest block, slack.
__host__ __device__ inline size_t sym_smem_bytes(int stages, int terms, int kmax, int N) {
  return 1024 + 1024 + (size_t)stages * kSymTileBytes + (size_t)terms * panel_chunks(kmax) * N * 128 + kSymSlack;
}

// Per block (k rows, nt = ceil(k / 128) row tiles):
//   producer  loads panel chunk J (rows 128 J .. 128 J + 127 of every residual
//             term) just before tile (0, J), then the remaining tiles in
//             row-major order of (I, J), I <= J, through the STAGES-deep ring;
//   MMA       row I = 0 waits for each chunk J as its tile (0, J) comes up, so
//             the first MMA needs only chunk 0; after row I, chunk I is read
//             by no later row and is released (p_empty[I]) for the next
//             block, whose panel therefore streams in while this block's
//             last rows multiply;
//   epilogue  drains D_I once row I is complete.
template <typename T, int N, int TERMS, int STAGES>
__global__ void __launch_bounds__(kThreads, 1) k_apply_tc_sym(Args a) {
  constexpr int MT = sym_max_row_tiles<N>();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  SymCtl<N>& ctl = *reinterpret_cast<SymCtl<N>*>(smem);
  unsigned char* ring = smem + 1024;                            // STAGES x 32 KB
  unsigned char* bbuf = ring + (size_t)STAGES * kSymTileBytes;  // TERMS x panel
  const int nt_max = (a.kmax + kSymTile - 1) / kSymTile;
  const uint32_t panel_bytes = (uint32_t)panel_chunks(a.kmax) * N * 128;  // nt_max x 128 rows
  constexpr uint32_t chunk_bytes = (uint32_t)kK * 2u * N;                  // 64 panel rows
  constexpr uint32_t chunk128 = 2u * chunk_bytes;                          // 128 panel rows
  volatile int& abort_flag = ctl.abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (a.ist != nullptr && n_active(a.ist, N) == 0) return;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&ctl.a_full[s], 1);
      mbar_init(&ctl.a_empty[s], 1);
    }
    for (int m = 0; m < MT; ++m) {
      mbar_init(&ctl.p_full[m], 1);
      mbar_init(&ctl.p_empty[m], 1);
      mbar_init(&ctl.acc_full[m], 1);
      mbar_init(&ctl.acc_empty[m], kEpiThreads / 32);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < N) ctl.rhs_unscale[threadIdx.x] = 1.0f / rhs_scale<T>(a.st, N, threadIdx.x);
  uint32_t cols = 32;
  while (cols < (uint32_t)(nt_max * N)) cols <<= 1;  // power of two >= 32, <= 512 (checked at launch)
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&ctl.tmem_slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = ctl.tmem_slot;

  if (warp == 0) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      uint32_t g = 0;
      uint32_t pu = 0;  // bit c: parity of the loads into panel chunk c so far
      for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
        const int i = a.order[w];
        const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
        if (k == 0 || k > a.kmax) continue;
        const int nKp = panel_chunks(k);  // 64-row chunks per term in HBM (whole 128-row pairs, zero beyond k)
        const int nt = (k + kSymTile - 1) / kSymTile;
        const unsigned char* pbase = a.b16 + a.panel_off[i];
        const unsigned char* src = a.tiles + a.tile_off[i];
        const int ntiles = nt * (nt + 1) / 2;
        for (int t = 0; t < ntiles; ++t, ++g) {
          if (t < nt) {
            // panel chunk J = t, needed from tile (0, J) on
            if (!mbar_wait(&ctl.p_empty[t], ((pu >> t) & 1u) ^ 1u)) { abort_flag = 1; break; }
            pu ^= 1u << t;
            mbar_expect_tx(&ctl.p_full[t], (uint32_t)TERMS * chunk128);
#pragma unroll
            for (int tt = 0; tt < TERMS; ++tt)
              bulk_g2s(bbuf + (size_t)tt * panel_bytes + (size_t)t * chunk128,
                       pbase + ((size_t)tt * nKp * chunk_bytes + (size_t)t * chunk128), chunk128, &ctl.p_full[t]);
          }
          const int s = g % STAGES;
          if (!mbar_wait(&ctl.a_empty[s], ((g / STAGES) & 1u) ^ 1u)) { abort_flag = 1; break; }
          mbar_expect_tx(&ctl.a_full[s], (uint32_t)kSymTileBytes);
          bulk_g2s(ring + (size_t)s * kSymTileBytes, src, (uint32_t)kSymTileBytes, &ctl.a_full[s]);
          src += kSymTileBytes;
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------ MMA issuer -----------------------------
    if (lane == 0) {
      constexpr int fmt = std::is_same<T, __nv_bfloat16>::value ? 1 : 0;
      constexpr uint32_t idesc_k = idesc_f16(fmt, N);
      constexpr uint32_t idesc_mn = idesc_f16_amn(fmt, N);
      uint32_t g = 0;
      uint32_t ph = 0;  // bit m: parity of the completed uses of accumulator D_m
      uint32_t pm = 0;  // bit c: parity of the completed loads of panel chunk c
      for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
        const int i = a.order[w];
        const int k = (int)(a.sub_ptr[i + 1] - a.sub_ptr[i]);
        if (k == 0 || k > a.kmax) continue;
        const int nt = (k + kSymTile - 1) / kSymTile;
        uint64_t touched = 0;  // row tiles whose accumulator already holds a partial sum
        // before the first MMA into D_m in this block, the epilogue must have
        // drained D_m of the previous block
        auto claim = [&](int m) -> bool {
          if ((touched >> m) & 1u) return true;
          if (!mbar_wait(&ctl.acc_empty[m], ((ph >> m) & 1u) ^ 1u)) return false;
          fence_after();
          return true;
        };
        for (int I = 0; I < nt && !abort_flag; ++I) {
          for (int J = I; J < nt; ++J, ++g) {
            const int s = g % STAGES;
            if (!mbar_wait(&ctl.a_full[s], (g / STAGES) & 1u)) { abort_flag = 1; break; }
            if (I == 0) {
              if (!mbar_wait(&ctl.p_full[J], (pm >> J) & 1u)) { abort_flag = 1; break; }
              pm ^= 1u << J;
            }
            if (!claim(I) || (I != J && !claim(J))) { abort_flag = 1; break; }
            fence_after();
            const uint32_t sa = smem_u32(ring + (size_t)s * kSymTileBytes);
            // D_I += T X_J: K runs over the 128 columns of J (two 64-column halves)
            {
              const uint32_t d = tmem + (uint32_t)(I * N);
              const uint32_t acc0 = (touched >> I) & 1u;
#pragma unroll
              for (int kk = 0; kk < kSymTile / 16; ++kk) {
                const uint32_t a_addr = sa + (uint32_t)(kk >> 2) * kHalfBytes + (uint32_t)(kk & 3) * 32u;
                const int prow = J * kSymTile + kk * 16;  // panel row of this K step
                const uint32_t sb = smem_u32(bbuf + (size_t)(prow / kK) * N * 128) + (uint32_t)(prow % kK) * 2u * N;
#pragma unroll
                for (int tt = 0; tt < TERMS; ++tt)
                  mma_f16(d, sw128_desc(a_addr), mn_desc<N>(sb + tt * panel_bytes), idesc_k,
                          (acc0 || kk > 0 || tt > 0) ? 1u : 0u);
              }
              touched |= 1ull << I;
            }
            // D_J += T^T X_I: K runs over the 128 rows of I (16 rows = 2 KB per step)
            if (I != J) {
              const uint32_t d = tmem + (uint32_t)(J * N);
              const uint32_t acc0 = (touched >> J) & 1u;
#pragma unroll
              for (int kk = 0; kk < kSymTile / 16; ++kk) {
                const uint32_t a_addr = sa + (uint32_t)kk * 2048u;
                const int prow = I * kSymTile + kk * 16;
                const uint32_t sb = smem_u32(bbuf + (size_t)(prow / kK) * N * 128) + (uint32_t)(prow % kK) * 2u * N;
#pragma unroll
                for (int tt = 0; tt < TERMS; ++tt)
                  mma_f16(d, sw128_mn_desc(a_addr, (uint32_t)kHalfBytes), mn_desc<N>(sb + tt * panel_bytes), idesc_mn,
                          (acc0 || kk > 0 || tt > 0) ? 1u : 0u);
              }
              touched |= 1ull << J;
            }
            mma_commit(&ctl.a_empty[s]);
          }
          if (abort_flag) break;
          // D_I is complete once row I is done: its other contributions (T^T X of
          // tiles (I', I), I' < I) came from earlier rows; panel chunk I is read
          // by no later row
          mma_commit(&ctl.acc_full[I]);
          mma_commit(&ctl.p_empty[I]);
        }
        if (abort_flag) break;
        ph ^= (nt >= 32) ? 0xffffffffu : ((1u << nt) - 1u);
      }
    }
  } else {
    // ------------------------------ epilogue --------------------------------
    const int e = threadIdx.x - 64;
    const int quarter = warp & 3;
    uint32_t ph = 0;  // bit m: parity of the completed uses of accumulator D_m
    for (int w = blockIdx.x; w < a.n_sub && !abort_flag; w += gridDim.x) {
      const int i = a.order[w];
      const int64_t p0 = a.sub_ptr[i];
      const int k = (int)(a.sub_ptr[i + 1] - p0);
      if (k == 0) continue;
      if (k > a.kmax) {
        if (e == 0) atomicOr(&g_device_error, DEVERR_BAD_SIZE);
        continue;
      }
      const int nt = (k + kSymTile - 1) / kSymTile;
      const float sc = a.scale ? a.scale[i] : 1.0f;
      for (int m = 0; m < nt; ++m) {
        // drain D_m as soon as its row is done, while later rows still multiply
        if (!mbar_wait(&ctl.acc_full[m], (ph >> m) & 1u)) { abort_flag = 1; break; }
        fence_after();
        float v[N];
#pragma unroll
        for (int c = 0; c < N; c += 16) tmem_ld16(tmem + (uint32_t)(m * N + c) + ((uint32_t)(quarter * 32) << 16), v + c);
        const int row = m * kSymTile + quarter * 32 + lane;
        if (row < k) {
          float4* dst = reinterpret_cast<float4*>(a.ylocal + (p0 + row) * N);
#pragma unroll
          for (int c = 0; c < N; c += 4)
            dst[c / 4] = make_float4(sc * ctl.rhs_unscale[c] * v[c], sc * ctl.rhs_unscale[c + 1] * v[c + 1],
                                     sc * ctl.rhs_unscale[c + 2] * v[c + 2], sc * ctl.rhs_unscale[c + 3] * v[c + 3]);
        }
        fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&ctl.acc_empty[m]);
      }
      if (abort_flag) break;
      ph ^= (nt >= 32) ? 0xffffffffu : ((1u << nt) - 1u);
    }
  }
  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
  }
}

template <typename T, int N, int TERMS, int STAGES>
static void launch_sym_stages(const Args& a, cudaStream_t s, size_t smem, int grid) {
  auto kern = k_apply_tc_sym<T, N, TERMS, STAGES>;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  kern<<<grid, kThreads, smem, s>>>(a);
}

// Ring depth of the symmetric kernel: the deepest ring (2..6 stages of 32 KB)
// that fits next to the B panels of the largest block; 0 if none does.
inline int sym_stages(int terms, int kmax, int N) {
  for (int st = kSymMaxStages; st >= 2; --st)
    if (sym_smem_bytes(st, terms, kmax, N) <= 227 * 1024) return st;
  return 0;
}

template <typename T, int N, int TERMS>
static int launch_sym(const Args& a, cudaStream_t s, int stages_req) {
  constexpr int MT = sym_max_row_tiles<N>();
  const int nt_max = (a.kmax + kSymTile - 1) / kSymTile;
  if (nt_max > MT) {
    set_error("ddx_schwarz_local_apply_tc_sym: %d row tiles of 128 with R=%d exceed the %d accumulators in TMEM",
              nt_max, N, MT);
    return DDX_ERR_UNSUPPORTED;
  }
  const int max_st = sym_stages(TERMS, a.kmax, N);
  if (max_st == 0) {
    set_error("ddx_schwarz_local_apply_tc_sym: k=%d with R=%d and %d residual terms needs %zu bytes of shared memory",
              a.kmax, N, TERMS, sym_smem_bytes(2, TERMS, a.kmax, N));
    return DDX_ERR_UNSUPPORTED;
  }
  const int stages = stages_req > 0 ? std::min(stages_req, max_st) : max_st;
  if (stages < 2) {
    set_error("ddx_schwarz_local_apply_tc_sym: %d ring stages requested (at least 2)", stages_req);
    return DDX_ERR_ARG;
  }
  // at least 120 KB of shared memory keeps one CTA per SM (its accumulators may take all 512 TMEM columns)
  const size_t smem = std::max<size_t>(sym_smem_bytes(stages, TERMS, a.kmax, N), 120 * 1024);
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, std::min(a.n_sub, nsm));
  switch (stages) {
    case 2: launch_sym_stages<T, N, TERMS, 2>(a, s, smem, grid); break;
    case 3: launch_sym_stages<T, N, TERMS, 3>(a, s, smem, grid); break;
    case 4: launch_sym_stages<T, N, TERMS, 4>(a, s, smem, grid); break;
    case 5: launch_sym_stages<T, N, TERMS, 5>(a, s, smem, grid); break;
    default: launch_sym_stages<T, N, TERMS, 6>(a, s, smem, grid); break;
  }
  DDX_LAUNCH_CHECK("ddx_schwarz_local_apply_tc_sym");
  return DDX_OK;
}

}  // namespace umma
}  // namespace ddx

using namespace ddx;

template <typename T, int TERMS>
static int launch_r(int R, const umma::Args& a, cudaStream_t s) {
  if (R == 16) return umma::launch<T, 16, TERMS>(a, s);
  if (R == 32) return umma::launch<T, 32, TERMS>(a, s);
  return umma::launch<T, 64, TERMS>(a, s);
}

extern "C" int ddx_schwarz_local_apply_tc(int n_sub, int R, const int64_t* sub_ptr, const int* order,
                                          const int64_t* tile_off, const void* tiles, int block_dtype,
                                          const float* scale, int kmax, const void* b16,
                                          const int64_t* panel_off, int terms, float* ylocal, const int* ist,
                                          const double* st, ddx_stream_t stream) {
  DDX_REQUIRE(R == 16 || R == 32 || R == 64, "ddx_schwarz_local_apply_tc: R must be 16, 32 or 64 (got %d)", R);
  DDX_REQUIRE(terms == 1 || terms == 2, "ddx_schwarz_local_apply_tc: terms must be 1 or 2 (got %d)", terms);
  DDX_REQUIRE(n_sub >= 0 && kmax >= 0, "ddx_schwarz_local_apply_tc: bad sizes");
  if (n_sub == 0 || kmax == 0) return DDX_OK;
  DDX_REQUIRE(sub_ptr && order && tile_off && tiles && b16 && panel_off && ylocal,
              "ddx_schwarz_local_apply_tc: null pointer");
  DDX_REQUIRE(((uintptr_t)tiles & 15u) == 0 && ((uintptr_t)ylocal & 15u) == 0 && ((uintptr_t)b16 & 15u) == 0,
              "ddx_schwarz_local_apply_tc: tiles, b16 and ylocal must be 16-byte aligned");
  umma::Args a{n_sub, sub_ptr, order, tile_off, (const unsigned char*)tiles, scale,
               (const unsigned char*)b16, panel_off, ylocal, ist, st, kmax};
  cudaStream_t s = (cudaStream_t)stream;
  if (block_dtype == DDX_BF16)
    return terms == 1 ? launch_r<__nv_bfloat16, 1>(R, a, s) : launch_r<__nv_bfloat16, 2>(R, a, s);
  if (block_dtype == DDX_F16) return terms == 1 ? launch_r<__half, 1>(R, a, s) : launch_r<__half, 2>(R, a, s);
  set_error("ddx_schwarz_local_apply_tc: block dtype must be BF16 or F16");
  return DDX_ERR_ARG;
}

template <typename T, int TERMS>
static int launch_sym_r(int R, const umma::Args& a, cudaStream_t s, int stages) {
  if (R == 16) return umma::launch_sym<T, 16, TERMS>(a, s, stages);
  if (R == 32) return umma::launch_sym<T, 32, TERMS>(a, s, stages);
  return umma::launch_sym<T, 64, TERMS>(a, s, stages);
}

extern "C" int ddx_schwarz_local_apply_tc_sym(int n_sub, int R, const int64_t* sub_ptr, const int* order,
                                              const int64_t* tile_off, const void* tiles, int block_dtype,
                                              const float* scale, int kmax, const void* b16,
                                              const int64_t* panel_off, int terms, float* ylocal, const int* ist,
                                              const double* st, ddx_stream_t stream) {
  return ddx_schwarz_local_apply_tc_sym_ex(n_sub, R, sub_ptr, order, tile_off, tiles, block_dtype, scale, kmax, b16,
                                           panel_off, terms, ylocal, ist, st, 0, stream);
}

extern "C" int ddx_schwarz_local_apply_tc_sym_ex(int n_sub, int R, const int64_t* sub_ptr, const int* order,
                                                 const int64_t* tile_off, const void* tiles, int block_dtype,
                                                 const float* scale, int kmax, const void* b16,
                                                 const int64_t* panel_off, int terms, float* ylocal, const int* ist,
                                                 const double* st, int stages, ddx_stream_t stream) {
  DDX_REQUIRE(stages == 0 || (stages >= 2 && stages <= 6),
              "ddx_schwarz_local_apply_tc_sym: stages must be 0 or 2..6 (got %d)", stages);
  DDX_REQUIRE(R == 16 || R == 32 || R == 64, "ddx_schwarz_local_apply_tc_sym: R must be 16, 32 or 64 (got %d)", R);
  DDX_REQUIRE(terms == 1 || terms == 2, "ddx_schwarz_local_apply_tc_sym: terms must be 1 or 2 (got %d)", terms);
  DDX_REQUIRE(n_sub >= 0 && kmax >= 0, "ddx_schwarz_local_apply_tc_sym: bad sizes");
  if (n_sub == 0 || kmax == 0) return DDX_OK;
  DDX_REQUIRE(sub_ptr && order && tile_off && tiles && b16 && panel_off && ylocal,
              "ddx_schwarz_local_apply_tc_sym: null pointer");
  DDX_REQUIRE(((uintptr_t)tiles & 15u) == 0 && ((uintptr_t)ylocal & 15u) == 0 && ((uintptr_t)b16 & 15u) == 0,
              "ddx_schwarz_local_apply_tc_sym: tiles, b16 and ylocal must be 16-byte aligned");
  umma::Args a{n_sub, sub_ptr, order, tile_off, (const unsigned char*)tiles, scale,
               (const unsigned char*)b16, panel_off, ylocal, ist, st, kmax};
  cudaStream_t s = (cudaStream_t)stream;
  if (block_dtype == DDX_BF16)
    return terms == 1 ? launch_sym_r<__nv_bfloat16, 1>(R, a, s, stages) : launch_sym_r<__nv_bfloat16, 2>(R, a, s, stages);
  if (block_dtype == DDX_F16)
    return terms == 1 ? launch_sym_r<__half, 1>(R, a, s, stages) : launch_sym_r<__half, 2>(R, a, s, stages);
  set_error("ddx_schwarz_local_apply_tc_sym: block dtype must be BF16 or F16");
  return DDX_ERR_ARG;
}

namespace ddx {
namespace umma {
// B panels of the tensor-core apply. Subdomain i (k rows, nKp = panel_chunks(k)
// = 2 ceil(k / 128) chunks of 64 rows) occupies TERMS x nKp x 64 x 2N bytes at
// panel_off[i], term-major;
// within a term, panel row c (= DOF sub_idx[sub_ptr[i] + c]) holds its N
// 16-bit values at the MN-major swizzled offsets mn_offset<N>(c, q) (q = 16-byte
// chunk), the layout the UMMA B descriptor reads. Term 0 = 16-bit(s_j r[d, j]),
// term 1 = 16-bit(s_j r[d, j] - term 0), s_j = rhs_scale<T>. Rows k..64 nKp - 1
// are never written (the caller zeroes them once). One CTA walks subdomains;
// each thread converts one 16-byte chunk (8 RHS) of one row per step.
template <typename T, int N, int TERMS>
__global__ void __launch_bounds__(256) k_pack_panels(int n_sub, const int64_t* __restrict__ sub_ptr,
                                                     const int* __restrict__ sub_idx,
                                                     const int64_t* __restrict__ panel_off,
                                                     const double* __restrict__ r, const double* __restrict__ st,
                                                     unsigned char* __restrict__ out) {
  __shared__ double sc[N];
  if (threadIdx.x < N) sc[threadIdx.x] = (double)rhs_scale<T>(st, N, threadIdx.x);
  __syncthreads();
  constexpr int CPR = N / 8;  // 16-byte chunks per row
  for (int i = blockIdx.x; i < n_sub; i += gridDim.x) {
    const int64_t p0 = sub_ptr[i];
    const int k = (int)(sub_ptr[i + 1] - p0);
    unsigned char* base = out + panel_off[i];
    const size_t term_bytes = (size_t)panel_chunks(k) * kK * 2 * N;
    for (int u = threadIdx.x; u < k * CPR; u += blockDim.x) {
      const int c = u / CPR, q = u % CPR;
      const double2* src = reinterpret_cast<const double2*>(r + (int64_t)sub_idx[p0 + c] * N + q * 8);
      double v[8];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const double2 d = __ldg(src + h);
        v[2 * h] = d.x * sc[q * 8 + 2 * h];
        v[2 * h + 1] = d.y * sc[q * 8 + 2 * h + 1];
      }
      uint16_t hi[8];
#pragma unroll
      for (int h = 0; h < 8; ++h) hi[h] = to_bits<T>(v[h]);
      const uint32_t off = mn_offset<N>(c, q);
      *reinterpret_cast<uint4*>(base + off) =
          make_uint4(hi[0] | ((uint32_t)hi[1] << 16), hi[2] | ((uint32_t)hi[3] << 16), hi[4] | ((uint32_t)hi[5] << 16),
                     hi[6] | ((uint32_t)hi[7] << 16));
      if (TERMS == 2) {
        uint16_t lo[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) lo[h] = to_bits<T>(v[h] - from_bits<T>(hi[h]));
        *reinterpret_cast<uint4*>(base + term_bytes + off) =
            make_uint4(lo[0] | ((uint32_t)lo[1] << 16), lo[2] | ((uint32_t)lo[3] << 16),
                       lo[4] | ((uint32_t)lo[5] << 16), lo[6] | ((uint32_t)lo[7] << 16));
      }
    }
  }
}

template <typename T, int TERMS>
static void launch_pack(int N, int grid, cudaStream_t s, int n_sub, const int64_t* sub_ptr, const int* sub_idx,
                        const int64_t* panel_off, const double* r, const double* st, unsigned char* out) {
  if (N == 16) k_pack_panels<T, 16, TERMS><<<grid, 256, 0, s>>>(n_sub, sub_ptr, sub_idx, panel_off, r, st, out);
  else if (N == 32) k_pack_panels<T, 32, TERMS><<<grid, 256, 0, s>>>(n_sub, sub_ptr, sub_idx, panel_off, r, st, out);
  else k_pack_panels<T, 64, TERMS><<<grid, 256, 0, s>>>(n_sub, sub_ptr, sub_idx, panel_off, r, st, out);
}
}  // namespace umma
}  // namespace ddx

extern "C" int ddx_pack_panels16(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                 const int64_t* panel_off, const double* r, const double* st, void* b16,
                                 int dtype, int terms, ddx_stream_t stream) {
  DDX_REQUIRE(R == 16 || R == 32 || R == 64, "ddx_pack_panels16: R must be 16, 32 or 64 (got %d)", R);
  DDX_REQUIRE(terms == 1 || terms == 2, "ddx_pack_panels16: terms must be 1 or 2 (got %d)", terms);
  DDX_REQUIRE(n_sub >= 0, "ddx_pack_panels16: bad sizes");
  if (n_sub == 0) return DDX_OK;
  DDX_REQUIRE(sub_ptr && sub_idx && panel_off && r && b16, "ddx_pack_panels16: null pointer");
  DDX_REQUIRE(((uintptr_t)r & 15u) == 0 && ((uintptr_t)b16 & 15u) == 0,
              "ddx_pack_panels16: r and b16 must be 16-byte aligned");
  const int grid = std::min(n_sub, 148 * 8);
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* o = (unsigned char*)b16;
  if (dtype == DDX_BF16) {
    if (terms == 1) umma::launch_pack<__nv_bfloat16, 1>(R, grid, s, n_sub, sub_ptr, sub_idx, panel_off, r, st, o);
    else umma::launch_pack<__nv_bfloat16, 2>(R, grid, s, n_sub, sub_ptr, sub_idx, panel_off, r, st, o);
  } else if (dtype == DDX_F16) {
    if (terms == 1) umma::launch_pack<__half, 1>(R, grid, s, n_sub, sub_ptr, sub_idx, panel_off, r, st, o);
    else umma::launch_pack<__half, 2>(R, grid, s, n_sub, sub_ptr, sub_idx, panel_off, r, st, o);
  } else {
    set_error("ddx_pack_panels16: dtype must be BF16 or F16");
    return DDX_ERR_ARG;
  }
  DDX_LAUNCH_CHECK("ddx_pack_panels16");
  return DDX_OK;
}
