// Sparse matrix-vector products for the PCG loop.
//
// Replaces FastBSR's RPT-I kernel (src/dd_solvers/dd_solvers/bsr.py:40-76, one
// thread per scalar row over a BSR matrix) and torch's CSR matvec
// (solvers.py:264, 880). The continuous Q1/P1 matrices of the measured
// problems are scalar (9/27/7-point rows), so the main kernel uses SELL-32:
// each warp owns a 32-row slice whose entries are stored column by column, so
// every value/column load of the warp is one contiguous 256/128-byte segment;
// x is read through the read-only cache (its reuse across neighbouring rows is
// served by L1/L2). The PCG epilogues (p.q, b - A x and its norms) are fused
// with deterministic CTA partials and a last-CTA finalize. The DG matrices of
// the reference's experiments are block-dense: their PCG products run in BSR
// form (8 bytes per entry instead of 12), followed by the same epilogue as a
// separate grid-stride pass.
#include <algorithm>
#include <exception>
#include <vector>
#include <type_traits>

#include "common.cuh"

namespace ddx {

// 4 CTAs per SM (64 registers): twice the loads in flight of the unbounded
// 84-92-register build, without spills.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 4)
    k_spmv_sell(int64_t n, int64_t nslices, const int64_t* __restrict__ slice_ptr,
                const int* __restrict__ slice_width, const int* __restrict__ cols,
                const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y,
                const double* __restrict__ b, PcgState S, double* partials, unsigned int* ticket) {
  __shared__ double red[kThreads];
  if (MODE != DDX_SPMV_PLAIN && n_active(S.ist, 1) == 0) return;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  double acc[2] = {0.0, 0.0};
  for (int64_t s = (int64_t)blockIdx.x * wpb + warp; s < nslices; s += (int64_t)gridDim.x * wpb) {
    const int64_t row = s * 32 + lane;
    const int64_t base = slice_ptr[s] + lane;
    const int w = slice_width[s];
    double sum = 0.0;
    if (row < n) {
      int jj = 0;
      for (; jj + 4 <= w; jj += 4) {
        const int64_t o = base + (int64_t)jj * 32;
        const double v0 = __ldcs(vals + o), v1 = __ldcs(vals + o + 32), v2 = __ldcs(vals + o + 64),
                     v3 = __ldcs(vals + o + 96);
        const int c0 = __ldcs(cols + o), c1 = __ldcs(cols + o + 32), c2 = __ldcs(cols + o + 64),
                  c3 = __ldcs(cols + o + 96);
        sum = fma(v0, __ldg(x + c0), sum);
        sum = fma(v1, __ldg(x + c1), sum);
        sum = fma(v2, __ldg(x + c2), sum);
        sum = fma(v3, __ldg(x + c3), sum);
      }
      for (; jj < w; ++jj) {
        const int64_t o = base + (int64_t)jj * 32;
        sum = fma(__ldcs(vals + o), __ldg(x + __ldcs(cols + o)), sum);
      }
      if (MODE == DDX_SPMV_PLAIN || MODE == DDX_SPMV_PQ) {
        y[row] = sum;
        if (MODE == DDX_SPMV_PQ) acc[0] = fma(x[row], sum, acc[0]);
      } else {
        const double bi = b[row];
        const double ri = bi - sum;
        y[row] = ri;
        if (MODE == DDX_SPMV_RES_INIT) acc[1] = fma(bi, bi, acc[1]);
        acc[0] = fma(ri, ri, acc[0]);
      }
    }
  }
  if (MODE == DDX_SPMV_PLAIN) return;
  constexpr int NV = (MODE == DDX_SPMV_RES_INIT) ? 2 : 1;
  double part[NV];
  part[0] = acc[0];
  if (NV == 2) part[NV - 1] = acc[1];
  write_cta_partials<NV>(part, red, 1, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[NV];
  final_sums<NV>(partials, 1, red, tot, ticket);
  if (park_totals<NV>(S, tot)) return;
  int act = 0;
  if (threadIdx.x == 0) {
    if (MODE == DDX_SPMV_PQ) act = fin_pq(S, 0, tot[0]);
    if (MODE == DDX_SPMV_RES_INIT) act = fin_init(S, 0, tot[NV - 1], tot[0]);
    if (MODE == DDX_SPMV_RES_REPLACE) act = fin_replace(S, 0, tot[0]);
    if (MODE >= DDX_SPMV_RES_INIT) S.s(DDX_ST_RR_PACK, 0) = S.s(DDX_ST_RR, 0);  // panels packed from this r
  }
  if (MODE != DDX_SPMV_PQ) publish_nactive(S, act);
  else {
    // alpha step can deactivate a RHS on breakdown; keep the counter exact.
    publish_nactive(S, threadIdx.x == 0 ? act : 0);
  }
}

// The PCG epilogue of a product that another kernel computed (the BSR product
// for DG block matrices): y = A v is already in y. PQ: p.q -> alpha (x is p);
// RES_*: y = b - y and its norms. Same partials, ticket and finalize as the
// fused SELL kernel; grid-stride over rows with at most kRedCtas CTAs.
template <int MODE>
__global__ void __launch_bounds__(kThreads)
    k_spmv_epilogue(int64_t n, const double* __restrict__ x, double* __restrict__ y,
                    const double* __restrict__ b, PcgState S, double* partials, unsigned int* ticket) {
  __shared__ double red[kThreads];
  if (n_active(S.ist, 1) == 0) return;
  double acc[2] = {0.0, 0.0};
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n;
       row += (int64_t)gridDim.x * blockDim.x) {
    const double q = y[row];
    if (MODE == DDX_SPMV_PQ) {
      acc[0] = fma(x[row], q, acc[0]);
    } else {
      const double bi = b[row];
      const double ri = bi - q;
      y[row] = ri;
      if (MODE == DDX_SPMV_RES_INIT) acc[1] = fma(bi, bi, acc[1]);
      acc[0] = fma(ri, ri, acc[0]);
    }
  }
  constexpr int NV = (MODE == DDX_SPMV_RES_INIT) ? 2 : 1;
  double part[NV];
  part[0] = acc[0];
  if (NV == 2) part[NV - 1] = acc[1];
  write_cta_partials<NV>(part, red, 1, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[NV];
  final_sums<NV>(partials, 1, red, tot, ticket);
  if (park_totals<NV>(S, tot)) return;
  int act = 0;
  if (threadIdx.x == 0) {
    if (MODE == DDX_SPMV_PQ) act = fin_pq(S, 0, tot[0]);
    if (MODE == DDX_SPMV_RES_INIT) act = fin_init(S, 0, tot[NV - 1], tot[0]);
    if (MODE == DDX_SPMV_RES_REPLACE) act = fin_replace(S, 0, tot[0]);
    if (MODE >= DDX_SPMV_RES_INIT) S.s(DDX_ST_RR_PACK, 0) = S.s(DDX_ST_RR, 0);
  }
  if (MODE != DDX_SPMV_PQ) publish_nactive(S, act);
  else publish_nactive(S, threadIdx.x == 0 ? act : 0);
}

// CSR, R threads per row (R in {1..64}, power of two), (n, R) vector layout.
template <int MODE>
__global__ void __launch_bounds__(kThreads)
    k_spmv_csr(int64_t n, const int* __restrict__ row_ptr, const int* __restrict__ cols,
               const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y,
               const double* __restrict__ b, PcgState S, double* partials, unsigned int* ticket) {
  __shared__ double red[kThreads];
  const int R = S.R;
  if (MODE != DDX_SPMV_PLAIN && n_active(S.ist, R) == 0) return;
  const int j = threadIdx.x % R;
  const int rpb = blockDim.x / R;
  double acc[2] = {0.0, 0.0};
  for (int64_t row = (int64_t)blockIdx.x * rpb + threadIdx.x / R; row < n; row += (int64_t)gridDim.x * rpb) {
    const int k0 = row_ptr[row], k1 = row_ptr[row + 1];
    double sum = 0.0;
    for (int k = k0; k < k1; ++k) sum = fma(__ldg(vals + k), __ldg(x + (int64_t)__ldg(cols + k) * R + j), sum);
    const int64_t o = row * R + j;
    if (MODE == DDX_SPMV_PLAIN || MODE == DDX_SPMV_PQ) {
      y[o] = sum;
      if (MODE == DDX_SPMV_PQ) acc[0] = fma(x[o], sum, acc[0]);
    } else {
      const double bi = b[o];
      const double ri = bi - sum;
      y[o] = ri;
      if (MODE == DDX_SPMV_RES_INIT) acc[1] = fma(bi, bi, acc[1]);
      acc[0] = fma(ri, ri, acc[0]);
    }
  }
  if (MODE == DDX_SPMV_PLAIN) return;
  constexpr int NV = (MODE == DDX_SPMV_RES_INIT) ? 2 : 1;
  double part[NV];
  part[0] = acc[0];
  if (NV == 2) part[NV - 1] = acc[1];
  write_cta_partials<NV>(part, red, R, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[NV];
  final_sums<NV>(partials, R, red, tot, ticket);
  if (park_totals<NV>(S, tot)) return;
  int act = 0;
  if (threadIdx.x < R) {
    const int jj = threadIdx.x;
    if (MODE == DDX_SPMV_PQ) act = fin_pq(S, jj, tot[0]);
    if (MODE == DDX_SPMV_RES_INIT) act = fin_init(S, jj, tot[NV - 1], tot[0]);
    if (MODE == DDX_SPMV_RES_REPLACE) act = fin_replace(S, jj, tot[0]);
    if (MODE >= DDX_SPMV_RES_INIT) S.s(DDX_ST_RR_PACK, jj) = S.s(DDX_ST_RR, jj);  // panels packed from this r
  }
  publish_nactive(S, act);
}

// CSR SpMM for R >= 2 right-hand sides: R/2 threads per row, each owning two
// adjacent RHS columns (16-byte loads of x rows), entries walked four at a
// time with independent loads. Column sums for the PCG epilogues are reduced
// as even/odd halves and written in the standard partials layout.
// Work order: with order == NULL, the rows in their own order, rpb = 256 /
// (R/2) consecutive rows per CTA step and grid-stride steps. With a row order
// (a permutation of the rows cut into clusters of `chunk` graph-adjacent
// rows, ddx_row_clusters), a CTA takes a whole cluster at a time, its rows in
// consecutive steps, so the x rows the cluster's neighbourhood shares are read
// from L2 once and then hit in L1 (a stencil row is read by up to 27 rows in
// 3D; in the natural order only the ~3 neighbours along a grid line share L1).
// CTAs per SM the multi-RHS SpMM is compiled for (register cap 65536 / (256 x
// this)): the kernel is latency-bound, so occupancy pays; 6 CTAs (40 registers,
// no spills) measured 0.354 / 1.482 / 0.353 ms against 0.414 / 1.631 / 0.405
// with 4 on C3's 9-point rows at 64 RHS, a 27-point 128^3 problem at 64 RHS
// and C5's P1 mesh at 16 RHS (5 CTAs: no gain)
#ifndef DDX_SPMM_MIN_CTAS
#define DDX_SPMM_MIN_CTAS 6
#endif
template <int MODE, bool ORDERED>
__global__ void __launch_bounds__(kThreads, DDX_SPMM_MIN_CTAS)
    k_spmm_csr2(int64_t n, const int* __restrict__ row_ptr, const int* __restrict__ cols,
                const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y,
                const double* __restrict__ b, PcgState S, double* partials, unsigned int* ticket,
                const int* __restrict__ order, int chunk) {
  __shared__ double red[kThreads];
  const int R = S.R;
  if (MODE != DDX_SPMV_PLAIN && n_active(S.ist, R) == 0) return;
  const int tpr = R / 2;
  const int c2 = threadIdx.x % tpr;  // this thread's column pair
  const int rpb = blockDim.x / tpr;
  double acc0[2] = {0.0, 0.0}, acc1[2] = {0.0, 0.0};  // [even, odd] column partials
  auto do_row = [&](int64_t row) {
    const int k0 = row_ptr[row], k1 = row_ptr[row + 1];
    double2 sum = make_double2(0.0, 0.0);
    int k = k0;
    for (; k + 4 <= k1; k += 4) {
      const int cA = __ldg(cols + k), cB = __ldg(cols + k + 1), cC = __ldg(cols + k + 2), cD = __ldg(cols + k + 3);
      const double vA = __ldg(vals + k), vB = __ldg(vals + k + 1), vC = __ldg(vals + k + 2), vD = __ldg(vals + k + 3);
      const double2 xA = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cA * R) + c2);
      const double2 xB = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cB * R) + c2);
      const double2 xC = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cC * R) + c2);
      const double2 xD = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cD * R) + c2);
      sum.x = fma(vA, xA.x, sum.x); sum.y = fma(vA, xA.y, sum.y);
      sum.x = fma(vB, xB.x, sum.x); sum.y = fma(vB, xB.y, sum.y);
      sum.x = fma(vC, xC.x, sum.x); sum.y = fma(vC, xC.y, sum.y);
      sum.x = fma(vD, xD.x, sum.x); sum.y = fma(vD, xD.y, sum.y);
    }
    for (; k < k1; ++k) {
      const double v = __ldg(vals + k);
      const double2 xv = __ldg(reinterpret_cast<const double2*>(x + (int64_t)__ldg(cols + k) * R) + c2);
      sum.x = fma(v, xv.x, sum.x);
      sum.y = fma(v, xv.y, sum.y);
    }
    double2* yo = reinterpret_cast<double2*>(y + row * R) + c2;
    if (MODE == DDX_SPMV_PLAIN || MODE == DDX_SPMV_PQ) {
      *yo = sum;
      if (MODE == DDX_SPMV_PQ) {
        const double2 xo = reinterpret_cast<const double2*>(x + row * R)[c2];
        acc0[0] = fma(xo.x, sum.x, acc0[0]);
        acc0[1] = fma(xo.y, sum.y, acc0[1]);
      }
    } else {
      const double2 bi = reinterpret_cast<const double2*>(b + row * R)[c2];
      const double2 ri = make_double2(bi.x - sum.x, bi.y - sum.y);
      *yo = ri;
      if (MODE == DDX_SPMV_RES_INIT) {
        acc1[0] = fma(bi.x, bi.x, acc1[0]);
        acc1[1] = fma(bi.y, bi.y, acc1[1]);
      }
      acc0[0] = fma(ri.x, ri.x, acc0[0]);
      acc0[1] = fma(ri.y, ri.y, acc0[1]);
    }
  };
  if constexpr (!ORDERED) {
    for (int64_t row = (int64_t)blockIdx.x * rpb + threadIdx.x / tpr; row < n; row += (int64_t)gridDim.x * rpb)
      do_row(row);
  } else {
    // chunk is a multiple of rpb: the CTA walks one cluster in consecutive steps
    for (int64_t c0 = (int64_t)blockIdx.x * chunk; c0 < n; c0 += (int64_t)gridDim.x * chunk)
      for (int st = 0; st < chunk; st += rpb) {
        const int64_t t = c0 + st + threadIdx.x / tpr;
        if (t >= n) break;
        do_row((int64_t)__ldg(order + t));
      }
  }
  if (MODE == DDX_SPMV_PLAIN) return;
  constexpr int NV = (MODE == DDX_SPMV_RES_INIT) ? 2 : 1;
  // CTA sums of each column, written as partials[(cta * NV + v) * R + column]
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double* a = v == 0 ? acc0 : acc1;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const double s = block_sum_by_col(a[h], red, tpr);
      if (threadIdx.x < tpr) partials[((size_t)blockIdx.x * NV + v) * R + 2 * threadIdx.x + h] = s;
    }
  }
  if (!last_cta_arrival(ticket)) return;
  double tot[NV];
  final_sums<NV>(partials, R, red, tot, ticket);
  if (park_totals<NV>(S, tot)) return;
  int act = 0;
  if (threadIdx.x < R) {
    const int jj = threadIdx.x;
    if (MODE == DDX_SPMV_PQ) act = fin_pq(S, jj, tot[0]);
    if (MODE == DDX_SPMV_RES_INIT) act = fin_init(S, jj, tot[NV - 1], tot[0]);
    if (MODE == DDX_SPMV_RES_REPLACE) act = fin_replace(S, jj, tot[0]);
    if (MODE >= DDX_SPMV_RES_INIT) S.s(DDX_ST_RR_PACK, jj) = S.s(DDX_ST_RR, jj);  // panels packed from this r
  }
  publish_nactive(S, act);
}

// One CTA per (long) row for R >= 2: R/2 threads per entry, each owning two
// RHS columns (16-byte x loads), 256/(R/2) entries per step, unrolled by 4;
// fixed-order reduction of the per-thread sums (even and odd columns).
__global__ void __launch_bounds__(kThreads)
    k_spmv_rowblock2(int64_t n_rows, int R, const int* __restrict__ row_ptr, const int* __restrict__ cols,
                     const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double red[kThreads];
  const int tpr = R / 2;
  const int c2 = threadIdx.x % tpr;
  const int G = blockDim.x / tpr;  // entries per step
  const int e0 = threadIdx.x / tpr;
  for (int64_t row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const int k0 = row_ptr[row], k1 = row_ptr[row + 1];
    double2 s = make_double2(0.0, 0.0);
    int k = k0 + e0;
    for (; k + 3 * G < k1; k += 4 * G) {
      const int cA = __ldg(cols + k), cB = __ldg(cols + k + G), cC = __ldg(cols + k + 2 * G),
                cD = __ldg(cols + k + 3 * G);
      const double vA = __ldg(vals + k), vB = __ldg(vals + k + G), vC = __ldg(vals + k + 2 * G),
                   vD = __ldg(vals + k + 3 * G);
      const double2 xA = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cA * R) + c2);
      const double2 xB = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cB * R) + c2);
      const double2 xC = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cC * R) + c2);
      const double2 xD = __ldg(reinterpret_cast<const double2*>(x + (int64_t)cD * R) + c2);
      s.x = fma(vA, xA.x, s.x); s.y = fma(vA, xA.y, s.y);
      s.x = fma(vB, xB.x, s.x); s.y = fma(vB, xB.y, s.y);
      s.x = fma(vC, xC.x, s.x); s.y = fma(vC, xC.y, s.y);
      s.x = fma(vD, xD.x, s.x); s.y = fma(vD, xD.y, s.y);
    }
    for (; k < k1; k += G) {
      const double v = __ldg(vals + k);
      const double2 xv = __ldg(reinterpret_cast<const double2*>(x + (int64_t)__ldg(cols + k) * R) + c2);
      s.x = fma(v, xv.x, s.x);
      s.y = fma(v, xv.y, s.y);
    }
    const double se = block_sum_by_col(s.x, red, tpr);
    const double so = block_sum_by_col(s.y, red, tpr);
    if (threadIdx.x < tpr) reinterpret_cast<double2*>(y + row * R)[threadIdx.x] = make_double2(se, so);
  }
}

// k_spmv_rowblock2 with x = the sum of the local products through the
// transpose map, x[d, :] = sum_{t in [dof_ptr[d], dof_ptr[d+1])} ylocal[src[t], :]
// (identity map when dof_ptr is null), each x value summed in FP64 in ascending
// t from 0.0, as ddx_schwarz_combine sums it: the result equals
// ddx_spmv_csr_rowblock_f64 applied to the materialised x, bit for bit, without
// writing and re-reading that vector (the hybrid Schwarz restriction A_R y).
template <typename ACC>
__device__ __forceinline__ double2 ypair(const ACC* p);
template <> __device__ __forceinline__ double2 ypair<double>(const double* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}
template <> __device__ __forceinline__ double2 ypair<float>(const float* p) {
  const float2 f = __ldg(reinterpret_cast<const float2*>(p));
  return make_double2((double)f.x, (double)f.y);
}

template <typename ACC>
__device__ __forceinline__ double2 mapped_x(int64_t d, int R, int c2, const int* __restrict__ dof_ptr,
                                            const int* __restrict__ dof_src, const ACC* __restrict__ ylocal) {
  double2 v = make_double2(0.0, 0.0);
  if (dof_ptr == nullptr) {
    const double2 y = ypair<ACC>(ylocal + d * R + 2 * c2);
    v.x += y.x;
    v.y += y.y;
    return v;
  }
  const int t0 = __ldg(dof_ptr + d), t1 = __ldg(dof_ptr + d + 1);
  for (int t = t0; t < t1; ++t) {
    const double2 y = ypair<ACC>(ylocal + (int64_t)__ldg(dof_src + t) * R + 2 * c2);
    v.x += y.x;
    v.y += y.y;
  }
  return v;
}

template <typename ACC>
__global__ void __launch_bounds__(kThreads)
    k_spmv_rowblock2_mapped(int64_t n_rows, int R, const int* __restrict__ row_ptr, const int* __restrict__ cols,
                            const double* __restrict__ vals, const int* __restrict__ dof_ptr,
                            const int* __restrict__ dof_src, const ACC* __restrict__ ylocal, double* __restrict__ y) {
  __shared__ double red[kThreads];
  const int tpr = R / 2;
  const int c2 = threadIdx.x % tpr;
  const int G = blockDim.x / tpr;  // entries per step
  const int e0 = threadIdx.x / tpr;
  for (int64_t row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const int k0 = row_ptr[row], k1 = row_ptr[row + 1];
    double2 s = make_double2(0.0, 0.0);
    int k = k0 + e0;
    for (; k + 3 * G < k1; k += 4 * G) {
      const int cA = __ldg(cols + k), cB = __ldg(cols + k + G), cC = __ldg(cols + k + 2 * G),
                cD = __ldg(cols + k + 3 * G);
      const double vA = __ldg(vals + k), vB = __ldg(vals + k + G), vC = __ldg(vals + k + 2 * G),
                   vD = __ldg(vals + k + 3 * G);
      const double2 xA = mapped_x<ACC>(cA, R, c2, dof_ptr, dof_src, ylocal);
      const double2 xB = mapped_x<ACC>(cB, R, c2, dof_ptr, dof_src, ylocal);
      const double2 xC = mapped_x<ACC>(cC, R, c2, dof_ptr, dof_src, ylocal);
      const double2 xD = mapped_x<ACC>(cD, R, c2, dof_ptr, dof_src, ylocal);
      s.x = fma(vA, xA.x, s.x); s.y = fma(vA, xA.y, s.y);
      s.x = fma(vB, xB.x, s.x); s.y = fma(vB, xB.y, s.y);
      s.x = fma(vC, xC.x, s.x); s.y = fma(vC, xC.y, s.y);
      s.x = fma(vD, xD.x, s.x); s.y = fma(vD, xD.y, s.y);
    }
    for (; k < k1; k += G) {
      const double v = __ldg(vals + k);
      const double2 xv = mapped_x<ACC>(__ldg(cols + k), R, c2, dof_ptr, dof_src, ylocal);
      s.x = fma(v, xv.x, s.x);
      s.y = fma(v, xv.y, s.y);
    }
    const double se = block_sum_by_col(s.x, red, tpr);
    const double so = block_sum_by_col(s.y, red, tpr);
    if (threadIdx.x < tpr) reinterpret_cast<double2*>(y + row * R)[threadIdx.x] = make_double2(se, so);
  }
}

// One CTA per (long) row; threads stride over the row's entries.
__global__ void __launch_bounds__(kThreads)
    k_spmv_rowblock(int64_t n_rows, int R, const int* __restrict__ row_ptr, const int* __restrict__ cols,
                    const double* __restrict__ vals, const double* __restrict__ x, double* __restrict__ y) {
  __shared__ double red[kThreads];
  const int j = threadIdx.x % R;
  const int G = blockDim.x / R;
  for (int64_t row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const int k0 = row_ptr[row], k1 = row_ptr[row + 1];
    double sum = 0.0;
    for (int k = k0 + threadIdx.x / R; k < k1; k += G)
      sum = fma(__ldg(vals + k), __ldg(x + (int64_t)__ldg(cols + k) * R + j), sum);
    sum = block_sum_by_col(sum, red, R);
    if (threadIdx.x < R) y[row * R + threadIdx.x] = sum;
  }
}

// Rows of moderate length (R = 1): L lanes per row (L = 4..32), lane l sums
// the entries k0 + l, k0 + l + L, ...; the L partial sums are combined by a
// fixed xor tree, so the result does not depend on timing.
template <int L, typename TX>
__global__ void __launch_bounds__(kThreads)
    k_spmv_rowwarp(int64_t n_rows, const int* __restrict__ row_ptr, const int* __restrict__ cols,
                   const double* __restrict__ vals, const TX* __restrict__ x, double* __restrict__ y) {
  constexpr int RPW = 32 / L;  // rows per warp and step
  const int lane = threadIdx.x & 31;
  const int sub = lane % L;
  const int64_t warps = (int64_t)gridDim.x * (kThreads / 32);
  // the loop bound depends on the warp only, so every lane reaches the shuffles
  for (int64_t base = ((int64_t)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)) * RPW; base < n_rows;
       base += warps * RPW) {
    const int64_t row = base + lane / L;
    double sum = 0.0;
    if (row < n_rows) {
      const int k0 = row_ptr[row], k1 = row_ptr[row + 1];
      for (int k = k0 + sub; k < k1; k += L)
        sum = fma(__ldg(vals + k), (double)__ldg(x + __ldg(cols + k)), sum);
    }
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, L);
    if (sub == 0 && row < n_rows) y[row] = sum;
  }
}

// BSR SpMV, row per lane: a warp covers G = floor(32 / BS) block rows, lane
// (g, r) computes scalar row r of block row g:
//   y[br BS + r] = sum_{blk in row br} sum_c vals[blk][c][r] * x[cols[blk] BS + c]
// with column-major blocks, so the BS lanes of a block row read BS consecutive
// values per column c (coalesced) and x[cols[blk] BS + c] is a broadcast; no
// cross-lane reduction. The next block's column index is loaded ahead.
// CTAs per SM the BSR kernel is compiled for: the unrolled block columns took
// up to ~180 registers at bs = 20 without a cap (one CTA per SM); with three
// CTAs (at most 80 registers, no spills) the kernel measured 0.75 -> 0.88 of
// the copy peak at bs = 6, 0.74 -> 1.04 at bs = 15, 0.69 -> 0.96 at bs = 20,
// and with five for bs <= 4 (48 registers) 0.72 -> 0.79 at bs = 3 and
// 0.76 -> 0.91 at bs = 4
#ifndef DDX_BSR_MIN_CTAS
#define DDX_BSR_MIN_CTAS 3
#endif
#ifndef DDX_BSR_MIN_CTAS_SMALL  // bs <= 4
#define DDX_BSR_MIN_CTAS_SMALL 5
#endif
template <typename T, int BS>
__global__ void __launch_bounds__(256, BS <= 4 ? DDX_BSR_MIN_CTAS_SMALL : DDX_BSR_MIN_CTAS) k_spmv_bsr(int64_t nbr, const int* __restrict__ row_ptr,
                                                  const int* __restrict__ cols, const T* __restrict__ vals,
                                                  const T* __restrict__ x, T* __restrict__ y) {
  constexpr int G = 32 / BS;
  constexpr int B2 = BS * BS;
  const int lane = threadIdx.x & 31;
  const int g = lane / BS, r = lane - g * BS;
  const int64_t br = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * G + g;
  if (g >= G || br >= nbr) return;
  const int k0 = row_ptr[br], k1 = row_ptr[br + 1];
  T acc0 = T(0), acc1 = T(0);
  int col = k0 < k1 ? __ldg(cols + k0) : 0;
  for (int k = k0; k < k1; ++k) {
    const int next = k + 1 < k1 ? __ldg(cols + k + 1) : 0;
    const T* vb = vals + (int64_t)k * B2 + r;
    const T* xb = x + (int64_t)col * BS;
#pragma unroll
    for (int c = 0; c + 1 < BS; c += 2) {
      acc0 = fma(__ldg(vb + c * BS), __ldg(xb + c), acc0);
      acc1 = fma(__ldg(vb + (c + 1) * BS), __ldg(xb + c + 1), acc1);
    }
    if (BS & 1) acc0 = fma(__ldg(vb + (BS - 1) * BS), __ldg(xb + BS - 1), acc0);
    col = next;
  }
  y[br * BS + r] = acc0 + acc1;
}

template <typename T>
static int launch_bsr(int64_t nbr, int bs, const int* rp, const int* ci, const T* v, const T* x, T* y,
                      cudaStream_t s) {
  const int wpb = 8;
  switch (bs) {
#define DDX_BSR_CASE(B)                                                             \
  case B: {                                                                         \
    const int grid = (int)ceil_div(nbr, (int64_t)wpb * (32 / B));                  \
    k_spmv_bsr<T, B><<<grid, wpb * 32, 0, s>>>(nbr, rp, ci, v, x, y);               \
    break;                                                                          \
  }
    DDX_BSR_CASE(1) DDX_BSR_CASE(2) DDX_BSR_CASE(3) DDX_BSR_CASE(4) DDX_BSR_CASE(5) DDX_BSR_CASE(6)
    DDX_BSR_CASE(7) DDX_BSR_CASE(8) DDX_BSR_CASE(9) DDX_BSR_CASE(10) DDX_BSR_CASE(11) DDX_BSR_CASE(12)
    DDX_BSR_CASE(13) DDX_BSR_CASE(14) DDX_BSR_CASE(15) DDX_BSR_CASE(16) DDX_BSR_CASE(17) DDX_BSR_CASE(18)
    DDX_BSR_CASE(19) DDX_BSR_CASE(20) DDX_BSR_CASE(21) DDX_BSR_CASE(22) DDX_BSR_CASE(23) DDX_BSR_CASE(24)
#undef DDX_BSR_CASE
    default: set_error("ddx_spmv_bsr: block size %d not in 1..24", bs); return DDX_ERR_UNSUPPORTED;
  }
  DDX_LAUNCH_CHECK("ddx_spmv_bsr");
  return DDX_OK;
}

// Launch of k_spmm_csr2 (grid-stride: one wave of resident CTAs).
template <bool ORDERED>
static int spmm2_launch_t(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                          const double* x, double* y, const double* b, int mode, PcgState S, double* partials,
                          unsigned int* t, const int* order, int chunk, cudaStream_t s) {
  const int rpb2 = kThreads / (R / 2);
  const int64_t need2 = ORDERED ? ceil_div(n_rows, chunk) : ceil_div(n_rows, rpb2);
  switch (mode) {
    case DDX_SPMV_PLAIN: {
      auto k = k_spmm_csr2<DDX_SPMV_PLAIN, ORDERED>;
      k<<<resident_grid(k, need2, 1 << 20), kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S, partials, t,
                                                              order, chunk);
      break;
    }
    case DDX_SPMV_PQ: {
      auto k = k_spmm_csr2<DDX_SPMV_PQ, ORDERED>;
      k<<<resident_grid(k, need2, kRedCtas), kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S, partials, t,
                                                               order, chunk);
      break;
    }
    case DDX_SPMV_RES_INIT: {
      auto k = k_spmm_csr2<DDX_SPMV_RES_INIT, ORDERED>;
      k<<<resident_grid(k, need2, kRedCtas), kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S, partials, t,
                                                               order, chunk);
      break;
    }
    default: {
      auto k = k_spmm_csr2<DDX_SPMV_RES_REPLACE, ORDERED>;
      k<<<resident_grid(k, need2, kRedCtas), kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S, partials, t,
                                                               order, chunk);
    }
  }
  DDX_LAUNCH_CHECK("ddx_spmv_csr_f64");
  return DDX_OK;
}

static int spmm2_launch(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                        const double* x, double* y, const double* b, int mode, PcgState S, double* partials,
                        unsigned int* t, const int* order, int chunk, cudaStream_t s) {
  if (order != nullptr)
    return spmm2_launch_t<true>(n_rows, R, row_ptr, cols, vals, x, y, b, mode, S, partials, t, order, chunk, s);
  return spmm2_launch_t<false>(n_rows, R, row_ptr, cols, vals, x, y, b, mode, S, partials, t, nullptr, 0, s);
}

}  // namespace ddx

using namespace ddx;

extern "C" {

int ddx_spmv_sell_f64(int64_t n, int64_t nslices, const int64_t* slice_ptr, const int* slice_width,
                      const int* cols, const double* vals, const double* x, double* y, const double* b,
                      int mode, double* st, int* ist, double* hist, double* partials,
                      unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(n >= 0 && nslices == ceil_div(n, 32), "ddx_spmv_sell_f64: nslices must be ceil(n/32)");
  DDX_REQUIRE(slice_ptr && slice_width && x && y, "ddx_spmv_sell_f64: null pointer");
  DDX_REQUIRE(mode >= 0 && mode <= 3, "ddx_spmv_sell_f64: bad mode %d", mode);
  if (mode != DDX_SPMV_PLAIN)
    DDX_REQUIRE(st && ist && hist && partials && tickets, "ddx_spmv_sell_f64: PCG mode needs state");
  if (mode >= DDX_SPMV_RES_INIT) DDX_REQUIRE(b, "ddx_spmv_sell_f64: residual mode needs b");
  if (n == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  PcgState S{st, ist, hist, 1};
  const int wpb = kThreads / 32;
  const int grid = (int)std::min<int64_t>(ceil_div(nslices, wpb), kRedCtas);
  unsigned int* t = tickets ? tickets + 2 : nullptr;
  switch (mode) {
    case DDX_SPMV_PLAIN:
      k_spmv_sell<DDX_SPMV_PLAIN><<<(int)ceil_div(nslices, wpb), kThreads, 0, s>>>(
          n, nslices, slice_ptr, slice_width, cols, vals, x, y, b, S, partials, t);
      break;
    case DDX_SPMV_PQ:
      k_spmv_sell<DDX_SPMV_PQ><<<grid, kThreads, 0, s>>>(n, nslices, slice_ptr, slice_width, cols, vals,
                                                         x, y, b, S, partials, t);
      break;
    case DDX_SPMV_RES_INIT:
      k_spmv_sell<DDX_SPMV_RES_INIT><<<grid, kThreads, 0, s>>>(n, nslices, slice_ptr, slice_width, cols,
                                                               vals, x, y, b, S, partials, t);
      break;
    default:
      k_spmv_sell<DDX_SPMV_RES_REPLACE><<<grid, kThreads, 0, s>>>(n, nslices, slice_ptr, slice_width,
                                                                  cols, vals, x, y, b, S, partials, t);
  }
  DDX_LAUNCH_CHECK("ddx_spmv_sell_f64");
  return DDX_OK;
}

int ddx_spmv_csr_f64(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                     const double* x, double* y, const double* b, int mode, double* st, int* ist,
                     double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_spmv_csr_f64: unsupported R=%d", R);
  DDX_REQUIRE(n_rows >= 0 && row_ptr && x && y, "ddx_spmv_csr_f64: bad arguments");
  DDX_REQUIRE(mode >= 0 && mode <= 3, "ddx_spmv_csr_f64: bad mode %d", mode);
  if (mode != DDX_SPMV_PLAIN)
    DDX_REQUIRE(st && ist && hist && partials && tickets, "ddx_spmv_csr_f64: PCG mode needs state");
  if (mode >= DDX_SPMV_RES_INIT) DDX_REQUIRE(b, "ddx_spmv_csr_f64: residual mode needs b");
  if (n_rows == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  PcgState S{st, ist, hist, R};
  unsigned int* t = tickets ? tickets + 3 : nullptr;
  if (R >= 2) {
    DDX_REQUIRE(((uintptr_t)x & 15u) == 0 && ((uintptr_t)y & 15u) == 0 && (b == nullptr || ((uintptr_t)b & 15u) == 0),
                "ddx_spmv_csr_f64: x, y and b must be 16-byte aligned for R >= 2");
    return spmm2_launch(n_rows, R, row_ptr, cols, vals, x, y, b, mode, S, partials, t, nullptr, 0, s);
  }
  const int rpb = kThreads / R;
  const int64_t need = ceil_div(n_rows, rpb);
  const int grid = (int)std::min<int64_t>(need, kRedCtas);
  switch (mode) {
    case DDX_SPMV_PLAIN:
      k_spmv_csr<DDX_SPMV_PLAIN><<<(int)std::min<int64_t>(need, 148 * 64), kThreads, 0, s>>>(
          n_rows, row_ptr, cols, vals, x, y, b, S, partials, t);
      break;
    case DDX_SPMV_PQ:
      k_spmv_csr<DDX_SPMV_PQ><<<grid, kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S, partials, t);
      break;
    case DDX_SPMV_RES_INIT:
      k_spmv_csr<DDX_SPMV_RES_INIT><<<grid, kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S,
                                                              partials, t);
      break;
    default:
      k_spmv_csr<DDX_SPMV_RES_REPLACE><<<grid, kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, x, y, b, S,
                                                                 partials, t);
  }
  DDX_LAUNCH_CHECK("ddx_spmv_csr_f64");
  return DDX_OK;
}

int ddx_spmv_csr_rowblock_f64(int64_t n_rows, int R, const int* row_ptr, const int* cols,
                              const double* vals, const double* x, double* y, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_spmv_csr_rowblock_f64: unsupported R=%d", R);
  DDX_REQUIRE(n_rows >= 0 && row_ptr && x && y, "ddx_spmv_csr_rowblock_f64: bad arguments");
  if (n_rows == 0) return DDX_OK;
  const int grid = (int)std::min<int64_t>(n_rows, 148 * 8);
  if (R >= 2) {
    DDX_REQUIRE(((uintptr_t)x & 15u) == 0 && ((uintptr_t)y & 15u) == 0,
                "ddx_spmv_csr_rowblock_f64: x and y must be 16-byte aligned for R >= 2");
    k_spmv_rowblock2<<<grid, kThreads, 0, (cudaStream_t)stream>>>(n_rows, R, row_ptr, cols, vals, x, y);
  } else {
    k_spmv_rowblock<<<grid, kThreads, 0, (cudaStream_t)stream>>>(n_rows, R, row_ptr, cols, vals, x, y);
  }
  DDX_LAUNCH_CHECK("ddx_spmv_csr_rowblock_f64");
  return DDX_OK;
}

int ddx_spmv_csr_rowblock_mapped(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                                 const int* dof_ptr, const int* dof_src, const void* ylocal, int acc_dtype,
                                 double* y, ddx_stream_t stream) {
  DDX_REQUIRE(R >= 2 && valid_rhs_count(R), "ddx_spmv_csr_rowblock_mapped: R must be 2, 4, ..., 64 (got %d)", R);
  DDX_REQUIRE(n_rows >= 0 && row_ptr && cols && vals && ylocal && y, "ddx_spmv_csr_rowblock_mapped: bad arguments");
  DDX_REQUIRE((dof_ptr == nullptr) == (dof_src == nullptr),
              "ddx_spmv_csr_rowblock_mapped: dof_ptr and dof_src are given together");
  DDX_REQUIRE(acc_dtype == DDX_F64 || acc_dtype == DDX_F32, "ddx_spmv_csr_rowblock_mapped: ylocal must be F64 or F32");
  DDX_REQUIRE(((uintptr_t)y & 15u) == 0 && ((uintptr_t)ylocal & 15u) == 0,
              "ddx_spmv_csr_rowblock_mapped: ylocal and y must be 16-byte aligned");
  if (n_rows == 0) return DDX_OK;
  const int grid = (int)std::min<int64_t>(n_rows, 148 * 8);
  cudaStream_t s = (cudaStream_t)stream;
  if (acc_dtype == DDX_F64)
    k_spmv_rowblock2_mapped<double><<<grid, kThreads, 0, s>>>(n_rows, R, row_ptr, cols, vals, dof_ptr, dof_src,
                                                              (const double*)ylocal, y);
  else
    k_spmv_rowblock2_mapped<float><<<grid, kThreads, 0, s>>>(n_rows, R, row_ptr, cols, vals, dof_ptr, dof_src,
                                                             (const float*)ylocal, y);
  DDX_LAUNCH_CHECK("ddx_spmv_csr_rowblock_mapped");
  return DDX_OK;
}

int ddx_spmv_csr_ordered_f64(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                             const int* order, int chunk, const double* x, double* y, const double* b, int mode,
                             double* st, int* ist, double* hist, double* partials, unsigned int* tickets,
                             ddx_stream_t stream) {
  DDX_REQUIRE(R >= 2 && valid_rhs_count(R), "ddx_spmv_csr_ordered_f64: R must be 2, 4, ..., 64 (got %d)", R);
  DDX_REQUIRE(n_rows >= 0 && row_ptr && x && y && order, "ddx_spmv_csr_ordered_f64: bad arguments");
  DDX_REQUIRE(chunk > 0 && chunk % (kThreads / (R / 2)) == 0,
              "ddx_spmv_csr_ordered_f64: chunk %d must be a positive multiple of %d rows", chunk,
              kThreads / (R / 2));
  DDX_REQUIRE(mode >= 0 && mode <= 3, "ddx_spmv_csr_ordered_f64: bad mode %d", mode);
  if (mode != DDX_SPMV_PLAIN)
    DDX_REQUIRE(st && ist && hist && partials && tickets, "ddx_spmv_csr_ordered_f64: PCG mode needs state");
  if (mode >= DDX_SPMV_RES_INIT) DDX_REQUIRE(b, "ddx_spmv_csr_ordered_f64: residual mode needs b");
  DDX_REQUIRE(((uintptr_t)x & 15u) == 0 && ((uintptr_t)y & 15u) == 0 && (b == nullptr || ((uintptr_t)b & 15u) == 0),
              "ddx_spmv_csr_ordered_f64: x, y and b must be 16-byte aligned");
  if (n_rows == 0) return DDX_OK;
  PcgState S{st, ist, hist, R};
  return spmm2_launch(n_rows, R, row_ptr, cols, vals, x, y, b, mode, S, partials, tickets ? tickets + 3 : nullptr,
                      order, chunk, (cudaStream_t)stream);
}

// Greedy breadth-first clusters of `cluster` rows: a BFS over the unassigned
// rows of the (symmetric) pattern from the lowest unassigned row, cut every
// `cluster` rows; when a BFS runs out before the cut, the next lowest
// unassigned row seeds the rest of the same cluster. Every cluster but the
// last has exactly `cluster` rows (so clusters line up with the SpMM's
// chunks); each cluster's rows ascending. On a structured grid the clusters
// are bricks (BFS balls of a 27- or 9-point stencil are cubes / squares).
static int row_clusters_impl(int64_t n, const int64_t* indptr, const int64_t* indices, int cluster, int* order) {
  DDX_REQUIRE(n >= 0 && n < (int64_t)1 << 31 && indptr && indices && order && cluster >= 1,
              "ddx_row_clusters: bad arguments");
  std::vector<unsigned char> taken((size_t)n, 0);
  std::vector<int> queue;
  queue.reserve((size_t)cluster);
  int64_t out = 0, seed = 0;
  while (out < n) {
    queue.clear();
    size_t head = 0;
    while ((int)queue.size() < cluster) {
      if (head == queue.size()) {  // BFS exhausted: next unassigned row
        while (seed < n && taken[seed]) ++seed;
        if (seed == n) break;
        taken[seed] = 1;
        queue.push_back((int)seed);
      }
      const int v = queue[head++];
      DDX_REQUIRE(indptr[v] <= indptr[v + 1], "ddx_row_clusters: indptr decreases at row %d", v);
      for (int64_t e = indptr[v]; e < indptr[v + 1] && (int)queue.size() < cluster; ++e) {
        const int64_t u = indices[e];
        DDX_REQUIRE(u >= 0 && u < n, "ddx_row_clusters: column %lld out of range", (long long)u);
        if (!taken[u]) {
          taken[u] = 1;
          queue.push_back((int)u);
        }
      }
    }
    std::sort(queue.begin(), queue.end());
    for (int v : queue) order[out++] = v;
  }
  return DDX_OK;
}

int ddx_row_clusters(int64_t n, const int64_t* indptr, const int64_t* indices, int cluster, int* order) {
  try {
    return row_clusters_impl(n, indptr, indices, cluster, order);
  } catch (const std::exception& ex) {
    set_error("ddx_row_clusters: %s", ex.what());
    return DDX_ERR_ARG;
  }
}

int ddx_spmv_csr_lanes(int64_t n_rows, int lanes, const int* row_ptr, const int* cols, const double* vals,
                       const void* x, int x_dtype, double* y, ddx_stream_t stream) {
  DDX_REQUIRE(n_rows >= 0 && row_ptr && x && y, "ddx_spmv_csr_lanes: bad arguments");
  DDX_REQUIRE(lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32,
              "ddx_spmv_csr_lanes: lanes must be 4, 8, 16 or 32 (got %d)", lanes);
  DDX_REQUIRE(x_dtype == DDX_F64 || x_dtype == DDX_F32, "ddx_spmv_csr_lanes: x must be F64 or F32");
  if (n_rows == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  auto go = [&](auto kernel, auto* xt) {
    const int grid = resident_grid(kernel, ceil_div(n_rows * lanes, kThreads), 1 << 20);
    kernel<<<grid, kThreads, 0, s>>>(n_rows, row_ptr, cols, vals, xt, y);
  };
  auto by_lanes = [&](auto* xt) {
    using TX = typename std::remove_const<typename std::remove_pointer<decltype(xt)>::type>::type;
    if (lanes == 4) go(k_spmv_rowwarp<4, TX>, xt);
    else if (lanes == 8) go(k_spmv_rowwarp<8, TX>, xt);
    else if (lanes == 16) go(k_spmv_rowwarp<16, TX>, xt);
    else go(k_spmv_rowwarp<32, TX>, xt);
  };
  if (x_dtype == DDX_F64) by_lanes((const double*)x);
  else by_lanes((const float*)x);
  DDX_LAUNCH_CHECK("ddx_spmv_csr_lanes");
  return DDX_OK;
}

int ddx_spmv_csr_lanes_f64(int64_t n_rows, int lanes, const int* row_ptr, const int* cols, const double* vals,
                           const double* x, double* y, ddx_stream_t stream) {
  return ddx_spmv_csr_lanes(n_rows, lanes, row_ptr, cols, vals, x, DDX_F64, y, stream);
}

int ddx_spmv_epilogue_f64(int64_t n, const double* x, double* y, const double* b, int mode, double* st, int* ist,
                          double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(n >= 0 && y, "ddx_spmv_epilogue_f64: bad arguments");
  DDX_REQUIRE(mode >= DDX_SPMV_PQ && mode <= DDX_SPMV_RES_REPLACE, "ddx_spmv_epilogue_f64: bad mode %d", mode);
  DDX_REQUIRE(st && ist && hist && partials && tickets, "ddx_spmv_epilogue_f64: PCG mode needs state");
  if (mode == DDX_SPMV_PQ) DDX_REQUIRE(x, "ddx_spmv_epilogue_f64: p.q needs p");
  else DDX_REQUIRE(b, "ddx_spmv_epilogue_f64: residual mode needs b");
  if (n == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  PcgState S{st, ist, hist, 1};
  const int grid = (int)std::min<int64_t>(ceil_div(n, kThreads), kRedCtas);
  unsigned int* t = tickets + 2;
  switch (mode) {
    case DDX_SPMV_PQ:
      k_spmv_epilogue<DDX_SPMV_PQ><<<grid, kThreads, 0, s>>>(n, x, y, b, S, partials, t);
      break;
    case DDX_SPMV_RES_INIT:
      k_spmv_epilogue<DDX_SPMV_RES_INIT><<<grid, kThreads, 0, s>>>(n, x, y, b, S, partials, t);
      break;
    default:
      k_spmv_epilogue<DDX_SPMV_RES_REPLACE><<<grid, kThreads, 0, s>>>(n, x, y, b, S, partials, t);
  }
  DDX_LAUNCH_CHECK("ddx_spmv_epilogue_f64");
  return DDX_OK;
}

int ddx_spmv_bsr(int64_t n_block_rows, int bs, const int* row_ptr, const int* cols, const void* vals,
                 const void* x, void* y, int dtype, ddx_stream_t stream) {
  DDX_REQUIRE(n_block_rows >= 0 && row_ptr && x && y, "ddx_spmv_bsr: bad arguments");
  if (n_block_rows == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == DDX_F64)
    return launch_bsr<double>(n_block_rows, bs, row_ptr, cols, (const double*)vals, (const double*)x,
                              (double*)y, s);
  if (dtype == DDX_F32)
    return launch_bsr<float>(n_block_rows, bs, row_ptr, cols, (const float*)vals, (const float*)x,
                             (float*)y, s);
  set_error("ddx_spmv_bsr: dtype %d not supported (F64 or F32)", dtype);
  return DDX_ERR_UNSUPPORTED;
}

}  // extern "C"
