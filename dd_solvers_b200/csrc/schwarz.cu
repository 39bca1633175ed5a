// Schwarz preconditioner: prolongation/combination and dense coarse solve.
//
// Replaces the reshape/sum/segment_reduce/repeat_interleave glue of
// AdditiveSchwarz.solve / HybridSchwarz.solve (src/dd_solvers/dd_solvers/solvers.py:811-826,
// 874-888) and the CUDSS solve (solvers.py:106-110), generalised to overlapping
// index-set subdomains of uneven size. (The local-inverse apply is in
// local_apply.cu and umma.cu.)
//
// combine: the prolongation is a gather over the transpose map (DOF ->
// positions in the subdomain-major ylocal) summed in ascending subdomain
// order, so it is atomic-free and deterministic; it also adds the coarse
// prolongation and forms the PCG dots.
#include <algorithm>

#include "common.cuh"

namespace ddx {

// ---------------------------------------------------------------------------
// combine
// ---------------------------------------------------------------------------
// R = 1: one DOF per thread and U DOFs in flight per step (index loads, the
// first transpose-map entry, u and the prolongation of all U issued before
// any store). Every combine kernel here sums an element in one fixed order:
// the ylocal entries in ascending subdomain order, then u, then sign * (P yc).
template <typename ACC>
__global__ void __launch_bounds__(kThreads, 4)
    k_combine1(int64_t n, PcgState S, const int* __restrict__ dof_ptr, const int* __restrict__ dof_src,
               const ACC* __restrict__ ylocal, const double* u, const int* __restrict__ p_ptr,
               const int* __restrict__ p_col, const double* __restrict__ p_val,
               const double* __restrict__ yc, double sign, double* z, int dots,
               const double* __restrict__ r, const double* __restrict__ q, double* partials,
               unsigned int* ticket) {
  constexpr int U = 4;
  __shared__ double red[kThreads];
  if (S.ist != nullptr && n_active(S.ist, 1) == 0) return;
  const int64_t pass = (int64_t)gridDim.x * blockDim.x;
  double acc[2] = {0.0, 0.0};
  for (int64_t d0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d0 < n; d0 += pass * U) {
    int64_t d[U];
    bool ok[U];
    double v[U];
#pragma unroll
    for (int uu = 0; uu < U; ++uu) {
      d[uu] = d0 + uu * pass;
      ok[uu] = d[uu] < n;
      v[uu] = 0.0;
    }
    if (ylocal != nullptr && dof_ptr == nullptr) {  // identity map: ylocal is DOF-ordered
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (ok[uu]) v[uu] += (double)__ldg(ylocal + d[uu]);
    } else if (ylocal != nullptr) {
      int t0[U], t1[U], s0[U];
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        t0[uu] = ok[uu] ? __ldg(dof_ptr + d[uu]) : 0;
        t1[uu] = ok[uu] ? __ldg(dof_ptr + d[uu] + 1) : 0;
      }
#pragma unroll
      for (int uu = 0; uu < U; ++uu) s0[uu] = t0[uu] < t1[uu] ? __ldg(dof_src + t0[uu]) : -1;
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (s0[uu] >= 0) v[uu] += (double)__ldg(ylocal + s0[uu]);
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        for (int t = t0[uu] + 1; t < t1[uu]; ++t) v[uu] += (double)__ldg(ylocal + __ldg(dof_src + t));
    }
    if (u != nullptr) {
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (ok[uu]) v[uu] += u[d[uu]];
    }
    if (p_ptr == nullptr && p_col != nullptr) {  // one unit entry per DOF: P0 aggregates
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (ok[uu]) v[uu] = fma(sign, __ldg(yc + __ldg(p_col + d[uu])), v[uu]);
    } else if (p_ptr != nullptr) {
      int k0[U], k1[U];
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        k0[uu] = ok[uu] ? __ldg(p_ptr + d[uu]) : 0;
        k1[uu] = ok[uu] ? __ldg(p_ptr + d[uu] + 1) : 0;
      }
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        double c = 0.0;
        for (int k = k0[uu]; k < k1[uu]; ++k) c = fma(__ldg(p_val + k), __ldg(yc + __ldg(p_col + k)), c);
        if (ok[uu]) v[uu] = fma(sign, c, v[uu]);
      }
    }
#pragma unroll
    for (int uu = 0; uu < U; ++uu)
      if (ok[uu]) {
        if (dots) {
          acc[0] = fma(__ldg(r + d[uu]), v[uu], acc[0]);
          if (q != nullptr) acc[1] = fma(v[uu], __ldg(q + d[uu]), acc[1]);
        }
        z[d[uu]] = v[uu];
      }
  }
  if (!dots) return;
  write_cta_partials<2>(acc, red, 1, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[2];
  final_sums<2>(partials, 1, red, tot, ticket);
  if (park_totals<2>(S, tot)) return;
  if (threadIdx.x == 0) fin_rz(S, 0, tot[0], tot[1]);
}

template <typename ACC> __device__ __forceinline__ double2 load_pair(const ACC* p);
template <> __device__ __forceinline__ double2 load_pair<double>(const double* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}
template <> __device__ __forceinline__ double2 load_pair<float>(const float* p) {
  const float2 f = __ldg(reinterpret_cast<const float2*>(p));
  return make_double2((double)f.x, (double)f.y);
}

// R >= 2: R/2 threads per DOF, each owning two adjacent RHS columns (8/16-byte
// loads), and U (DDX_COMBINE_U) DOFs per thread in flight per step: the index loads, the first
// transpose-map entry, u and the prolongation of all U DOFs are issued before
// any store. (u may alias z, so a one-element loop cannot
// start the next element's loads before the previous store: every element
// then waits out a chain of three dependent loads.) Each element is summed in
// the same order as in k_combine1, so every column of z has the bits of an
// R = 1 combine.
// MODE 0: store z (and reduce it when dots); MODE 1: reduce z without storing
// it; MODE 2: the direction update on the recomputed z (same bits as MODE 0's
// z): x += alpha_x p (x may be null), p = z + beta p, no reduction. In MODE 2
// the `z` argument is p and `r` is x.
// dof_first (may be null): per DOF its only position (>= 0), -1 when it has
// none, -2 when it has several; a DOF in one subdomain then costs a chain of
// two dependent loads (dof_first, ylocal) instead of three (dof_ptr, dof_src,
// ylocal). Same sums in the same order either way.
// CTAs per SM the multi-RHS combine is compiled for (5 or 6, which spill a few
// registers, measured slower on C3 and C5), and DOFs in flight per thread (4:
// C3 2.664 -> 2.645 ms per iteration against 3; 2, or 4 at three CTAs per SM,
// slower)
#ifndef DDX_COMBINE_MIN_CTAS
#define DDX_COMBINE_MIN_CTAS 4
#endif
#ifndef DDX_COMBINE_U
#define DDX_COMBINE_U 4
#endif
template <typename ACC, int MODE>
__global__ void __launch_bounds__(kThreads, DDX_COMBINE_MIN_CTAS)
    k_combine2(int64_t n, PcgState S, const int* __restrict__ dof_ptr, const int* __restrict__ dof_src,
               const int* __restrict__ dof_first, const ACC* __restrict__ ylocal, const double* u, const int* __restrict__ p_ptr,
               const int* __restrict__ p_col, const double* __restrict__ p_val,
               const double* __restrict__ yc, double sign, double* z, int dots,
               const double* r, const double* __restrict__ q, double* partials,
               unsigned int* ticket) {
  constexpr int U = DDX_COMBINE_U;
  __shared__ double red[kThreads];
  const int R = S.R;
  if (S.ist != nullptr && n_active(S.ist, R) == 0) return;
  const int tpr = R / 2;
  const int jc = 2 * (threadIdx.x % tpr);  // first of this thread's two columns
  double beta0 = 0.0, beta1 = 0.0, ax0 = 0.0, ax1 = 0.0;
  if (MODE == 2) {
    beta0 = S.st[DDX_ST_BETA * R + jc];
    beta1 = S.st[DDX_ST_BETA * R + jc + 1];
    ax0 = S.st[DDX_ST_ALPHA_X * R + jc];
    ax1 = S.st[DDX_ST_ALPHA_X * R + jc + 1];
  }
  const int64_t rows_per_pass = (int64_t)gridDim.x * (blockDim.x / tpr);
  double acc_rz[2] = {0.0, 0.0}, acc_zq[2] = {0.0, 0.0};
  for (int64_t d0 = (int64_t)blockIdx.x * (blockDim.x / tpr) + threadIdx.x / tpr; d0 < n; d0 += rows_per_pass * U) {
    int64_t d[U];
    bool ok[U];
    double2 v[U];
#pragma unroll
    for (int uu = 0; uu < U; ++uu) {
      d[uu] = d0 + uu * rows_per_pass;
      ok[uu] = d[uu] < n;
      v[uu] = make_double2(0.0, 0.0);
    }
    if (ylocal != nullptr && dof_ptr == nullptr) {  // identity map
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (ok[uu]) {
          const double2 y = load_pair<ACC>(ylocal + d[uu] * R + jc);
          v[uu].x += y.x;
          v[uu].y += y.y;
        }
    } else if (ylocal != nullptr && dof_first != nullptr) {
      int f[U], t0[U], t1[U];
#pragma unroll
      for (int uu = 0; uu < U; ++uu) f[uu] = ok[uu] ? __ldg(dof_first + d[uu]) : -1;
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        const bool multi = f[uu] <= -2;
        t0[uu] = multi ? __ldg(dof_ptr + d[uu]) : 0;
        t1[uu] = multi ? __ldg(dof_ptr + d[uu] + 1) : 0;
      }
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (f[uu] >= 0) {
          const double2 y = load_pair<ACC>(ylocal + (int64_t)f[uu] * R + jc);
          v[uu].x += y.x;
          v[uu].y += y.y;
        }
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        for (int t = t0[uu]; t < t1[uu]; ++t) {
          const double2 y = load_pair<ACC>(ylocal + (int64_t)__ldg(dof_src + t) * R + jc);
          v[uu].x += y.x;
          v[uu].y += y.y;
        }
    } else if (ylocal != nullptr) {
      int t0[U], t1[U], s0[U];
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        t0[uu] = ok[uu] ? __ldg(dof_ptr + d[uu]) : 0;
        t1[uu] = ok[uu] ? __ldg(dof_ptr + d[uu] + 1) : 0;
      }
#pragma unroll
      for (int uu = 0; uu < U; ++uu) s0[uu] = t0[uu] < t1[uu] ? __ldg(dof_src + t0[uu]) : -1;
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (s0[uu] >= 0) {
          const double2 y = load_pair<ACC>(ylocal + (int64_t)s0[uu] * R + jc);
          v[uu].x += y.x;
          v[uu].y += y.y;
        }
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        for (int t = t0[uu] + 1; t < t1[uu]; ++t) {
          const double2 y = load_pair<ACC>(ylocal + (int64_t)__ldg(dof_src + t) * R + jc);
          v[uu].x += y.x;
          v[uu].y += y.y;
        }
    }
    if (u != nullptr) {
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (ok[uu]) {
          const double2 uv = *reinterpret_cast<const double2*>(u + d[uu] * R + jc);
          v[uu].x += uv.x;
          v[uu].y += uv.y;
        }
    }
    if (p_ptr == nullptr && p_col != nullptr) {  // one unit entry per DOF
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (ok[uu]) {
          const double2 y = __ldg(reinterpret_cast<const double2*>(yc + (int64_t)__ldg(p_col + d[uu]) * R + jc));
          v[uu].x = fma(sign, y.x, v[uu].x);
          v[uu].y = fma(sign, y.y, v[uu].y);
        }
    } else if (p_ptr != nullptr) {
      int k0[U], k1[U];
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        k0[uu] = ok[uu] ? __ldg(p_ptr + d[uu]) : 0;
        k1[uu] = ok[uu] ? __ldg(p_ptr + d[uu] + 1) : 0;
      }
#pragma unroll
      for (int uu = 0; uu < U; ++uu) {
        double2 c = make_double2(0.0, 0.0);
        for (int k = k0[uu]; k < k1[uu]; ++k) {
          const double pv = __ldg(p_val + k);
          const double2 y = __ldg(reinterpret_cast<const double2*>(yc + (int64_t)__ldg(p_col + k) * R + jc));
          c.x = fma(pv, y.x, c.x);
          c.y = fma(pv, y.y, c.y);
        }
        if (ok[uu]) {
          v[uu].x = fma(sign, c.x, v[uu].x);
          v[uu].y = fma(sign, c.y, v[uu].y);
        }
      }
    }
#pragma unroll
    for (int uu = 0; uu < U; ++uu)
      if (ok[uu]) {
        if (MODE == 2) {
          double* pp = z + d[uu] * R + jc;
          const double2 pv = *reinterpret_cast<const double2*>(pp);
          if (r != nullptr) {
            double* xp = const_cast<double*>(r) + d[uu] * R + jc;
            const double2 xv = *reinterpret_cast<const double2*>(xp);
            *reinterpret_cast<double2*>(xp) = make_double2(fma(ax0, pv.x, xv.x), fma(ax1, pv.y, xv.y));
          }
          *reinterpret_cast<double2*>(pp) = make_double2(fma(beta0, pv.x, v[uu].x), fma(beta1, pv.y, v[uu].y));
          continue;
        }
        if (dots) {
          const double2 rv = __ldg(reinterpret_cast<const double2*>(r + d[uu] * R + jc));
          acc_rz[0] = fma(rv.x, v[uu].x, acc_rz[0]);
          acc_rz[1] = fma(rv.y, v[uu].y, acc_rz[1]);
          if (q != nullptr) {
            const double2 qv = __ldg(reinterpret_cast<const double2*>(q + d[uu] * R + jc));
            acc_zq[0] = fma(v[uu].x, qv.x, acc_zq[0]);
            acc_zq[1] = fma(v[uu].y, qv.y, acc_zq[1]);
          }
        }
        if (MODE == 0) *reinterpret_cast<double2*>(z + d[uu] * R + jc) = v[uu];
      }
  }
  if constexpr (MODE == 2) return;
  if (!dots) return;
  // CTA sums per column, partials[(cta * 2 + v) * R + column], v = 0: r.z, 1: z.q
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const double a = block_sum_by_col(acc_rz[h], red, tpr);
    if (threadIdx.x < tpr) partials[((size_t)blockIdx.x * 2 + 0) * R + 2 * threadIdx.x + h] = a;
    const double b = block_sum_by_col(acc_zq[h], red, tpr);
    if (threadIdx.x < tpr) partials[((size_t)blockIdx.x * 2 + 1) * R + 2 * threadIdx.x + h] = b;
  }
  if (!last_cta_arrival(ticket)) return;
  double tot[2];
  final_sums<2>(partials, R, red, tot, ticket);
  if (park_totals<2>(S, tot)) return;
  if (threadIdx.x < R) fin_rz(S, threadIdx.x, tot[0], tot[1]);
}

// ---------------------------------------------------------------------------
// dense coarse solve: yc = Ainv w  (Ainv symmetric, row-major)
// ---------------------------------------------------------------------------
// R = 1: one warp per row, lanes stride the row in 16-byte pairs (eight pairs
// in flight per lane, then four), shuffle-tree reduction. A row of odd length n_c starts
// 8 bytes off a 16-byte boundary on every other row: its first entry is
// taken as a scalar head.
__global__ void k_coarse_gemv1(int n_c, const double* __restrict__ Ainv, const double* __restrict__ w,
                               double* __restrict__ yc, const int* ist) {
  if (ist != nullptr && n_active(ist, 1) == 0) return;
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n_c) return;
  const double* a = Ainv + row * n_c;
  const int head = (int)(((uintptr_t)a >> 3) & 1u);  // 0 or 1 scalar before the first aligned pair
  const int m = (n_c - head) >> 1;                    // aligned pairs
  const double2* a2 = reinterpret_cast<const double2*>(a + head);
  const double* wh = w + head;
  double s0 = 0.0, s1 = 0.0;
  int c = lane;
  // eight pairs in flight per lane
  for (; c + 224 < m; c += 256) {
    double2 v[8];
#pragma unroll
    for (int h = 0; h < 8; ++h) v[h] = __ldcs(a2 + c + 32 * h);
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      s0 = fma(v[h].x, __ldg(wh + 2 * c + 64 * h), s0);
      s1 = fma(v[h].y, __ldg(wh + 2 * c + 64 * h + 1), s1);
    }
  }
  for (; c + 96 < m; c += 128) {
    const double2 v0 = __ldcs(a2 + c), v1 = __ldcs(a2 + c + 32), v2 = __ldcs(a2 + c + 64), v3 = __ldcs(a2 + c + 96);
    s0 = fma(v0.x, __ldg(wh + 2 * c), s0);
    s1 = fma(v0.y, __ldg(wh + 2 * c + 1), s1);
    s0 = fma(v1.x, __ldg(wh + 2 * c + 64), s0);
    s1 = fma(v1.y, __ldg(wh + 2 * c + 65), s1);
    s0 = fma(v2.x, __ldg(wh + 2 * c + 128), s0);
    s1 = fma(v2.y, __ldg(wh + 2 * c + 129), s1);
    s0 = fma(v3.x, __ldg(wh + 2 * c + 192), s0);
    s1 = fma(v3.y, __ldg(wh + 2 * c + 193), s1);
  }
  for (; c < m; c += 32) {
    const double2 v = __ldcs(a2 + c);
    s0 = fma(v.x, __ldg(wh + 2 * c), s0);
    s1 = fma(v.y, __ldg(wh + 2 * c + 1), s1);
  }
  double s = s0 + s1;
  if (lane == 0) {
    if (head) s = fma(a[0], w[0], s);
    if ((n_c - head) & 1) s = fma(a[n_c - 1], w[n_c - 1], s);
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) yc[row] = s;
}

// R > 1: CTA of 8 warps = 8 rows x G = min(R, 16) RHS columns (blockIdx.y
// picks the column group). w is staged in shared memory in tiles of kTC rows,
// shared by the CTA's 8 rows (every row needs all of w: staging cuts the L2
// reads of w by 8x against one warp per row); each lane loads its Ainv entries
// of the tile before the barrier, keeps one partial sum per column, and the
// warp reduces them with a shuffle tree; lane j < G writes column j.
template <int G>
__global__ void __launch_bounds__(256) k_coarse_gemvT(int n_c, int R, const double* __restrict__ Ainv,
                                                      const double* __restrict__ w, double* __restrict__ yc,
                                                      const int* ist) {
  constexpr int kTC = 256;
  constexpr int kPer = kTC / 32;
  __shared__ double ws[kTC][G + 1];  // +1 double per row: lanes at stride G + 1 spread over the banks
  if (ist != nullptr && n_active(ist, R) == 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * 8 + warp;
  const int g0 = blockIdx.y * G;
  const bool live = row < n_c;
  const double* arow = Ainv + (live ? row : 0) * n_c;
  double s[G];
#pragma unroll
  for (int j = 0; j < G; ++j) s[j] = 0.0;
  for (int c0 = 0; c0 < n_c; c0 += kTC) {
    const int tc = min(kTC, n_c - c0);
    double av[kPer];
#pragma unroll
    for (int h = 0; h < kPer; ++h) {
      const int c = lane + 32 * h;
      av[h] = (live && c < tc) ? __ldcs(arow + c0 + c) : 0.0;
    }
    __syncthreads();  // previous tile fully consumed
    for (int e = threadIdx.x; e < tc * G; e += blockDim.x) {
      const int c = e / G, j = e % G;
      ws[c][j] = __ldg(w + (int64_t)(c0 + c) * R + g0 + j);
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < kPer; ++h) {
      const int c = lane + 32 * h;
      if (c < tc) {
#pragma unroll
        for (int j = 0; j < G; ++j) s[j] = fma(av[h], ws[c][j], s[j]);
      }
    }
  }
  double out = 0.0;
#pragma unroll
  for (int j = 0; j < G; ++j) {
    double t = s[j];
    for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    if (lane == j) out = t;
  }
  if (live && lane < G) yc[row * R + g0 + lane] = out;
}

// R in {16, 32, 64}: yc = Ainv w as a tiled FP64 GEMM. A CTA of 256 threads
// computes a tile of BM rows (64 for R = 64, else 128) x all R columns, each
// thread an RM x 4 block (rows ty, ty + TR, ...; four adjacent columns), over
// one K range of kc columns of Ainv, in 32-wide K steps staged in shared
// memory (Ainv transposed into As[k][row], w as Bs[k][col]). Every Ainv entry is
// read once per solve (not once per 16 columns), every w row once per row tile.
// With more K ranges than one (few row tiles: n_c / BM CTAs would leave SMs
// idle), each range writes its own partial tile and k_coarse_ksum adds them in
// ascending range order. Each output is summed over k in ascending order, then
// over the ranges in order: deterministic.
template <int R>
__global__ void __launch_bounds__(256) k_coarse_gemm(int n_c, const double* __restrict__ Ainv,
                                                     const double* __restrict__ w, double* __restrict__ out,
                                                     int kc, const int* ist) {
  constexpr int BK = 32;
  constexpr int TC = R / 4;          // thread columns
  constexpr int TR = 256 / TC;       // thread rows
  constexpr int RM = R == 16 ? 2 : 4;  // rows per thread
  constexpr int BM = RM * TR;        // rows per tile
  __shared__ double As[BK][BM + 1];
  __shared__ __align__(16) double Bs[BK][R];
  if (ist != nullptr && n_active(ist, R) == 0) return;
  const int tx = threadIdx.x % TC, ty = threadIdx.x / TC;
  const int row0 = blockIdx.x * BM;
  const int k_begin = blockIdx.y * kc;
  const int k_end = min(n_c, k_begin + kc);
  double acc[RM][4];
#pragma unroll
  for (int i = 0; i < RM; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int k0 = k_begin; k0 < k_end; k0 += BK) {
    const int kt = min(BK, k_end - k0);
    __syncthreads();  // previous tile consumed
    // A tile: BM rows x kt columns of Ainv (row-major), lanes along k
    for (int e = threadIdx.x; e < BM * BK; e += 256) {
      const int r = e / BK, k = e % BK;
      const int gr = row0 + r;
      As[k][r] = (gr < n_c && k < kt) ? __ldg(Ainv + (int64_t)gr * n_c + k0 + k) : 0.0;
    }
    // B tile: kt rows of w, R columns each
    for (int e = threadIdx.x; e < BK * R; e += 256) {
      const int k = e / R, c = e % R;
      Bs[k][c] = k < kt ? __ldg(w + (int64_t)(k0 + k) * R + c) : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < BK; ++k) {
      double a[RM];
#pragma unroll
      for (int i = 0; i < RM; ++i) a[i] = As[k][ty + i * TR];
      const double2 b01 = *reinterpret_cast<const double2*>(&Bs[k][4 * tx]);
      const double2 b23 = *reinterpret_cast<const double2*>(&Bs[k][4 * tx + 2]);
      const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
      for (int i = 0; i < RM; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
  double* o = out + (int64_t)blockIdx.y * n_c * R;
#pragma unroll
  for (int i = 0; i < RM; ++i) {
    const int gr = row0 + ty + i * TR;
    if (gr < n_c) {
      double2* d = reinterpret_cast<double2*>(o + (int64_t)gr * R + 4 * tx);
      d[0] = make_double2(acc[i][0], acc[i][1]);
      d[1] = make_double2(acc[i][2], acc[i][3]);
    }
  }
}

// yc = sum over the K ranges s = 0..S-1 of part[s], in that order.
__global__ void __launch_bounds__(256) k_coarse_ksum(int64_t total, int S, const double* __restrict__ part,
                                                     double* __restrict__ yc, const int* ist, int R) {
  if (ist != nullptr && n_active(ist, R) == 0) return;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int s = 0; s < S; ++s) acc += __ldg(part + (int64_t)s * total + t);
    yc[t] = acc;
  }
}

// ---------------------------------------------------------------------------
// hybrid restriction per subdomain: w = A_R y = sum_i (A_R R_i^T) y_i
// ---------------------------------------------------------------------------
// The coarse rows that subdomain i touches (A_R[c, idx_i] != 0) are its slots
// 0..n_slots[i]-1 (ascending c), the pairs q = slot_base[i] + slot. Row p of
// the subdomain-major ylocal carries its entries (slot, A_R[c, sub_idx[p]]) in
// ascending slot: the first two directly at p (f_slot[2p + e], f_val[2p + e],
// e = 0, 1; slot 255: none), the others in [ov_ptr[p], ov_ptr[p+1]) of
// ov_slot / ov_val (on a 2D P0 coarse space only the rows at an aggregate's
// corner have more than two).
//
// Pass 1, one CTA per subdomain (grid-stride): R/2 threads per row, two columns
// each, G = 512 / R row groups; group g takes the rows g, g + G, ... in order,
// eight at a time with all their loads (ylocal, first entry, overflow range)
// issued before any use, and adds val * ylocal[p, :] into its own
// shared-memory accumulators acc[g][slot][:] (every thread touches only its
// own columns of its own group: no atomics, no barrier while streaming); then
// the groups are summed in ascending g into partial[q, :]. ylocal streams
// once, row by row, with no transpose-map gathers.
constexpr int kRestrictMaxSlots = 16;
// rows in flight per row group, and CTAs per SM the kernel is compiled for:
// eight rows took 142 registers (one CTA per SM); four rows at three CTAs (78
// registers) measured C3 2.78 -> 2.61 ms and C5 4.17 -> 3.99 ms per iteration
#ifndef DDX_RESTRICT_ROWS
#define DDX_RESTRICT_ROWS 4
#endif
#ifndef DDX_RESTRICT_MIN_CTAS
#define DDX_RESTRICT_MIN_CTAS 3
#endif
template <typename ACC>
__global__ void __launch_bounds__(kThreads, DDX_RESTRICT_MIN_CTAS)
    k_restrict_sub(int n_sub, int R, const int64_t* __restrict__ sub_ptr, const int* __restrict__ slot_base,
                   const int* __restrict__ n_slots, const unsigned char* __restrict__ f_slot,
                   const double* __restrict__ f_val, const int* __restrict__ ov_ptr,
                   const unsigned char* __restrict__ ov_slot, const double* __restrict__ ov_val,
                   const ACC* __restrict__ ylocal, int slices, int64_t slice_rows, double* __restrict__ partial,
                   const int* ist) {
  constexpr int U = DDX_RESTRICT_ROWS;
  extern __shared__ double acc_sm[];  // [G][kRestrictMaxSlots][R]
  if (ist != nullptr && n_active(ist, R) == 0) return;
  const int tpr = R / 2;
  const int c2 = threadIdx.x % tpr;
  const int G = blockDim.x / tpr;
  const int g = threadIdx.x / tpr;
  double* mine = acc_sm + (size_t)g * kRestrictMaxSlots * R + 2 * c2;
  for (int i = blockIdx.x; i < n_sub; i += gridDim.x) {
    const int ns = n_slots[i];
    if (ns > kRestrictMaxSlots) {
      if (threadIdx.x == 0) atomicOr(&g_device_error, DEVERR_BAD_SIZE);
      continue;
    }
    for (int sl = 0; sl < ns; ++sl) *reinterpret_cast<double2*>(mine + sl * R) = make_double2(0.0, 0.0);
    for (int sc = 0; sc < slices; ++sc)
      for (int64_t p0 = sub_ptr[i] + sc * slice_rows, p1 = sub_ptr[i + 1] + sc * slice_rows, pb = p0 + g; pb < p1;
           pb += (int64_t)U * G) {
        double2 y[U], fv[U];
        int fs[U], o0[U], o1[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t p = pb + (int64_t)u * G;
          const bool ok = p < p1;
          y[u] = ok ? load_pair<ACC>(ylocal + p * R + 2 * c2) : make_double2(0.0, 0.0);
          // both direct entries: a 2-byte slot pair, a 16-byte value pair
          fs[u] = ok ? (int)__ldg(reinterpret_cast<const unsigned short*>(f_slot) + p) : 0xffff;
          fv[u] = ok ? __ldg(reinterpret_cast<const double2*>(f_val) + p) : make_double2(0.0, 0.0);
          o0[u] = ok ? __ldg(ov_ptr + p) : 0;
          o1[u] = ok ? __ldg(ov_ptr + p + 1) : 0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int s0 = fs[u] & 0xff, s1 = fs[u] >> 8;
          if (s0 != 255) {
            double2* a = reinterpret_cast<double2*>(mine + s0 * R);
            double2 cur = *a;
            cur.x = fma(fv[u].x, y[u].x, cur.x);
            cur.y = fma(fv[u].x, y[u].y, cur.y);
            *a = cur;
          }
          if (s1 != 255) {
            double2* a = reinterpret_cast<double2*>(mine + s1 * R);
            double2 cur = *a;
            cur.x = fma(fv[u].y, y[u].x, cur.x);
            cur.y = fma(fv[u].y, y[u].y, cur.y);
            *a = cur;
          }
          for (int t = o0[u]; t < o1[u]; ++t) {
            const double v = __ldg(ov_val + t);
            double2* a = reinterpret_cast<double2*>(mine + (int)__ldg(ov_slot + t) * R);
            double2 cur = *a;
            cur.x = fma(v, y[u].x, cur.x);
            cur.y = fma(v, y[u].y, cur.y);
            *a = cur;
          }
        }
      }
    __syncthreads();
    // groups summed in ascending order: thread t takes (slot, column) items
    const int base = slot_base[i];
    for (int it = threadIdx.x; it < ns * R; it += blockDim.x) {
      const int sl = it / R, col = it % R;
      double sum = 0.0;
      for (int gg = 0; gg < G; ++gg) sum += acc_sm[((size_t)gg * kRestrictMaxSlots + sl) * R + col];
      partial[(int64_t)(base + sl) * R + col] = sum;
    }
    __syncthreads();
  }
}

// Pass 2: w[c, j] = sum of partial[q, j] over the pairs q of coarse row c in
// ascending subdomain order (sum_pair[sum_ptr[c] .. sum_ptr[c+1])), one
// thread per (c, j).
__global__ void __launch_bounds__(kThreads)
    k_restrict_sum(int64_t n_coarse, int R, const int* __restrict__ sum_ptr, const int* __restrict__ sum_pair,
                   const double* __restrict__ partial, double* __restrict__ w, const int* ist) {
  if (ist != nullptr && n_active(ist, R) == 0) return;
  const int64_t total = n_coarse * R;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / R;
    const int j = (int)(t % R);
    double acc = 0.0;
    for (int u = __ldg(sum_ptr + c); u < __ldg(sum_ptr + c + 1); ++u)
      acc += __ldg(partial + (int64_t)__ldg(sum_pair + u) * R + j);
    w[t] = acc;
  }
}

}  // namespace ddx

using namespace ddx;

extern "C" {

int ddx_schwarz_restrict_sub(int n_sub, int64_t n_pairs, int64_t n_coarse, int R, const int64_t* sub_ptr,
                             const int* slot_base, const int* n_slots, const unsigned char* f_slot,
                             const double* f_val, const int* ov_ptr, const unsigned char* ov_slot,
                             const double* ov_val, const void* ylocal, int acc_dtype, int slices, int64_t slice_rows,
                             const int* sum_ptr, const int* sum_pair, double* partial, double* w, const int* ist,
                             ddx_stream_t stream) {
  DDX_REQUIRE(R >= 2 && R <= 64 && valid_rhs_count(R), "ddx_schwarz_restrict_sub: R must be 2, 4, ..., 64 (got %d)",
              R);
  DDX_REQUIRE(n_sub >= 0 && n_pairs >= 0 && n_coarse >= 0 && slices >= 1 && (slices == 1 || slice_rows >= 0),
              "ddx_schwarz_restrict_sub: bad sizes");
  DDX_REQUIRE(acc_dtype == DDX_F64 || acc_dtype == DDX_F32, "ddx_schwarz_restrict_sub: acc dtype %d", acc_dtype);
  if (n_coarse == 0) return DDX_OK;
  DDX_REQUIRE(sum_ptr && w && (n_pairs == 0 || (sub_ptr && slot_base && n_slots && f_slot && f_val && ov_ptr &&
                                                ylocal && sum_pair && partial)),
              "ddx_schwarz_restrict_sub: null pointer");
  DDX_REQUIRE(((uintptr_t)partial & 15u) == 0 && ((uintptr_t)ylocal & (acc_dtype == DDX_F64 ? 15u : 7u)) == 0 &&
                  ((uintptr_t)f_val & 15u) == 0 && ((uintptr_t)f_slot & 1u) == 0,
              "ddx_schwarz_restrict_sub: partial and f_val must be 16-byte aligned, f_slot 2-byte aligned, ylocal "
              "aligned to two columns");
  cudaStream_t s = (cudaStream_t)stream;
  if (n_pairs > 0 && n_sub > 0) {
    const size_t smem = (size_t)(512 / R) * kRestrictMaxSlots * R * sizeof(double);  // 64 KB
    auto go = [&](auto kern, const auto* yl) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      int dev = 0, nsm = 148, per = 1;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kThreads, smem) != cudaSuccess || per < 1) per = 1;
      const int grid = (int)std::min<int64_t>(n_sub, (int64_t)per * nsm);
      kern<<<grid, kThreads, smem, s>>>(n_sub, R, sub_ptr, slot_base, n_slots, f_slot, f_val, ov_ptr, ov_slot, ov_val,
                                        yl, slices, slice_rows, partial, ist);
    };
    if (acc_dtype == DDX_F64) go(k_restrict_sub<double>, (const double*)ylocal);
    else go(k_restrict_sub<float>, (const float*)ylocal);
    DDX_LAUNCH_CHECK("ddx_schwarz_restrict_sub");
  }
  const int grid2 = (int)std::min<int64_t>(ceil_div(n_coarse * R, kThreads), 4096);
  k_restrict_sum<<<grid2, kThreads, 0, s>>>(n_coarse, R, sum_ptr, sum_pair, partial, w, ist);
  DDX_LAUNCH_CHECK("ddx_schwarz_restrict_sub");
  return DDX_OK;
}

int ddx_schwarz_combine(int64_t n, int R, const int* dof_ptr, const int* dof_src, const void* ylocal,
                        int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                        const double* p_val, const double* yc, double sign, double* z, int dots,
                        const double* r, const double* q, double* st, int* ist, double* partials,
                        unsigned int* tickets, ddx_stream_t stream) {
  return ddx_schwarz_combine_ex(n, R, dof_ptr, dof_src, nullptr, ylocal, acc_dtype, u, p_ptr, p_col, p_val, yc,
                                sign, z, dots, r, q, st, ist, partials, tickets, stream);
}

int ddx_schwarz_combine_ex(int64_t n, int R, const int* dof_ptr, const int* dof_src, const int* dof_first,
                           const void* ylocal, int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                           const double* p_val, const double* yc, double sign, double* z, int dots,
                           const double* r, const double* q, double* st, int* ist, double* partials,
                           unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_schwarz_combine: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && (z || (dots && R >= 2)), "ddx_schwarz_combine: bad arguments (z is required unless "
              "R >= 2 and the combine only reduces)");
  if (ylocal && dof_ptr) DDX_REQUIRE(dof_src, "ddx_schwarz_combine: transpose map without dof_src");
  if (dof_first) DDX_REQUIRE(dof_ptr && dof_src, "ddx_schwarz_combine: dof_first needs the transpose map");
  if (p_ptr) DDX_REQUIRE(p_col && p_val && yc, "ddx_schwarz_combine: prolongation needs P and yc");
  if (!p_ptr && p_col) DDX_REQUIRE(yc, "ddx_schwarz_combine: P0 prolongation needs yc");
  if (dots) DDX_REQUIRE(r && st && ist && partials && tickets, "ddx_schwarz_combine: dots need PCG state");
  PcgState S{st, ist, nullptr, R};
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int* t = tickets ? tickets + 4 : nullptr;
  if (ylocal != nullptr && acc_dtype != DDX_F64 && acc_dtype != DDX_F32) {
    set_error("ddx_schwarz_combine: acc dtype %d", acc_dtype);
    return DDX_ERR_ARG;
  }
  const bool f64 = ylocal == nullptr || acc_dtype == DDX_F64;
  if (R >= 2) {
    DDX_REQUIRE(((uintptr_t)z & 15u) == 0 && ((uintptr_t)u & 15u) == 0 && ((uintptr_t)r & 15u) == 0 &&
                    ((uintptr_t)q & 15u) == 0 && ((uintptr_t)yc & 15u) == 0 &&
                    ((uintptr_t)ylocal & (f64 ? 15u : 7u)) == 0,
                "ddx_schwarz_combine: vectors must be 16-byte aligned for R >= 2");
    const int grid2 = red_grid(ceil_div(n * (R / 2), DDX_COMBINE_U));
    if (z != nullptr) {
      if (f64)
        k_combine2<double, 0><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, dof_first, (const double*)ylocal, u, p_ptr,
                                                         p_col, p_val, yc, sign, z, dots, r, q, partials, t);
      else
        k_combine2<float, 0><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, dof_first, (const float*)ylocal, u, p_ptr,
                                                        p_col, p_val, yc, sign, z, dots, r, q, partials, t);
    } else {
      if (f64)
        k_combine2<double, 1><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, dof_first, (const double*)ylocal, u, p_ptr,
                                                         p_col, p_val, yc, sign, z, dots, r, q, partials, t);
      else
        k_combine2<float, 1><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, dof_first, (const float*)ylocal, u, p_ptr,
                                                        p_col, p_val, yc, sign, z, dots, r, q, partials, t);
    }
  } else {
    const int grid1 = red_grid(ceil_div(n, 4));
    if (f64)
      k_combine1<double><<<grid1, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, (const double*)ylocal, u, p_ptr,
                                                    p_col, p_val, yc, sign, z, dots, r, q, partials, t);
    else
      k_combine1<float><<<grid1, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, (const float*)ylocal, u, p_ptr,
                                                   p_col, p_val, yc, sign, z, dots, r, q, partials, t);
  }
  DDX_LAUNCH_CHECK("ddx_schwarz_combine");
  return DDX_OK;
}

int ddx_schwarz_combine_update(int64_t n, int R, const int* dof_ptr, const int* dof_src, const int* dof_first,
                               const void* ylocal, int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                               const double* p_val, const double* yc, double sign, double* x, double* p,
                               const double* st, const int* ist, ddx_stream_t stream) {
  DDX_REQUIRE(R >= 2 && valid_rhs_count(R), "ddx_schwarz_combine_update: R must be 2, 4, ..., 64 (got %d)", R);
  DDX_REQUIRE(n >= 0 && p && st && ist, "ddx_schwarz_combine_update: bad arguments");
  if (ylocal && dof_ptr) DDX_REQUIRE(dof_src, "ddx_schwarz_combine_update: transpose map without dof_src");
  if (dof_first) DDX_REQUIRE(dof_ptr && dof_src, "ddx_schwarz_combine_update: dof_first needs the transpose map");
  if (p_ptr) DDX_REQUIRE(p_col && p_val && yc, "ddx_schwarz_combine_update: prolongation needs P and yc");
  if (!p_ptr && p_col) DDX_REQUIRE(yc, "ddx_schwarz_combine_update: P0 prolongation needs yc");
  if (ylocal != nullptr && acc_dtype != DDX_F64 && acc_dtype != DDX_F32) {
    set_error("ddx_schwarz_combine_update: acc dtype %d", acc_dtype);
    return DDX_ERR_ARG;
  }
  const bool f64 = ylocal == nullptr || acc_dtype == DDX_F64;
  DDX_REQUIRE(((uintptr_t)p & 15u) == 0 && ((uintptr_t)x & 15u) == 0 && ((uintptr_t)u & 15u) == 0 &&
                  ((uintptr_t)yc & 15u) == 0 && ((uintptr_t)ylocal & (f64 ? 15u : 7u)) == 0,
              "ddx_schwarz_combine_update: vectors must be 16-byte aligned");
  if (n == 0) return DDX_OK;
  // same launch shape as ddx_schwarz_combine (the per-element arithmetic does
  // not depend on it, but keeping it keeps the memory behaviour alike)
  PcgState S{const_cast<double*>(st), const_cast<int*>(ist), nullptr, R};
  cudaStream_t s = (cudaStream_t)stream;
  const int grid2 = red_grid(ceil_div(n * (R / 2), DDX_COMBINE_U));
  if (f64)
    k_combine2<double, 2><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, dof_first, (const double*)ylocal, u, p_ptr, p_col,
                                                     p_val, yc, sign, p, 0, x, nullptr, nullptr, nullptr);
  else
    k_combine2<float, 2><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, dof_first, (const float*)ylocal, u, p_ptr, p_col,
                                                    p_val, yc, sign, p, 0, x, nullptr, nullptr, nullptr);
  DDX_LAUNCH_CHECK("ddx_schwarz_combine_update");
  return DDX_OK;
}

int ddx_coarse_gemm_f64(int n_c, int R, const double* Ainv, const double* w, double* yc, double* scratch,
                        int64_t scratch_len, const int* ist, ddx_stream_t stream) {
  DDX_REQUIRE(R == 16 || R == 32 || R == 64, "ddx_coarse_gemm_f64: R must be 16, 32 or 64 (got %d)", R);
  DDX_REQUIRE(n_c >= 0 && Ainv && w && yc && scratch_len >= 0, "ddx_coarse_gemm_f64: bad arguments");
  DDX_REQUIRE(scratch_len == 0 || scratch, "ddx_coarse_gemm_f64: scratch_len > 0 with a null scratch");
  DDX_REQUIRE(((uintptr_t)yc & 15u) == 0 && ((uintptr_t)scratch & 15u) == 0,
              "ddx_coarse_gemm_f64: yc and scratch must be 16-byte aligned");
  if (n_c == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int bm = (R == 16 ? 2 : 4) * (256 / (R / 4));
  const int row_tiles = (int)ceil_div(n_c, bm);
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  // K ranges (multiples of 32 columns) so that about two CTAs per SM run, as
  // many as the scratch holds (S x n_c x R doubles)
  const int64_t k_tiles = ceil_div(n_c, 32);
  int64_t S = std::min<int64_t>(k_tiles, std::max<int64_t>(1, ceil_div(2 * nsm, row_tiles)));
  S = std::min<int64_t>(S, scratch_len / ((int64_t)n_c * R));
  if (S < 1) S = 1;
  const int kc = (int)(ceil_div(k_tiles, S) * 32);
  S = ceil_div(n_c, kc);
  double* out = S == 1 ? yc : scratch;
  const dim3 grid((unsigned)row_tiles, (unsigned)S);
  if (R == 16) k_coarse_gemm<16><<<grid, 256, 0, s>>>(n_c, Ainv, w, out, kc, ist);
  else if (R == 32) k_coarse_gemm<32><<<grid, 256, 0, s>>>(n_c, Ainv, w, out, kc, ist);
  else k_coarse_gemm<64><<<grid, 256, 0, s>>>(n_c, Ainv, w, out, kc, ist);
  DDX_LAUNCH_CHECK("ddx_coarse_gemm_f64");
  if (S > 1) {
    const int64_t total = (int64_t)n_c * R;
    k_coarse_ksum<<<(int)std::min<int64_t>(ceil_div(total, 256), 4096), 256, 0, s>>>(total, (int)S, scratch, yc,
                                                                                       ist, R);
    DDX_LAUNCH_CHECK("ddx_coarse_gemm_f64");
  }
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
    const int G = R < 16 ? R : 16;
    const dim3 grid((unsigned)ceil_div(n_c, 8), (unsigned)(R / G));
    if (G == 2) k_coarse_gemvT<2><<<grid, 256, 0, s>>>(n_c, R, Ainv, w, yc, ist);
    else if (G == 4) k_coarse_gemvT<4><<<grid, 256, 0, s>>>(n_c, R, Ainv, w, yc, ist);
    else if (G == 8) k_coarse_gemvT<8><<<grid, 256, 0, s>>>(n_c, R, Ainv, w, yc, ist);
    else k_coarse_gemvT<16><<<grid, 256, 0, s>>>(n_c, R, Ainv, w, yc, ist);
  }
  DDX_LAUNCH_CHECK("ddx_coarse_gemv_f64");
  return DDX_OK;
}

}  // extern "C"
