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
// loads), and U DOFs per thread in flight per step: the index loads, the first
// transpose-map entry, u and the prolongation of all U DOFs are issued before
// any store. (u may alias z, so a one-element loop cannot
// start the next element's loads before the previous store: every element
// then waits out a chain of three dependent loads.) Each element is summed in
// the same order as in k_combine1, so every column of z has the bits of an
// R = 1 combine.
template <typename ACC>
__global__ void __launch_bounds__(kThreads, 4)
    k_combine2(int64_t n, PcgState S, const int* __restrict__ dof_ptr, const int* __restrict__ dof_src,
               const ACC* __restrict__ ylocal, const double* u, const int* __restrict__ p_ptr,
               const int* __restrict__ p_col, const double* __restrict__ p_val,
               const double* __restrict__ yc, double sign, double* z, int dots,
               const double* __restrict__ r, const double* __restrict__ q, double* partials,
               unsigned int* ticket) {
  constexpr int U = 3;
  __shared__ double red[kThreads];
  const int R = S.R;
  if (S.ist != nullptr && n_active(S.ist, R) == 0) return;
  const int tpr = R / 2;
  const int jc = 2 * (threadIdx.x % tpr);  // first of this thread's two columns
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
        *reinterpret_cast<double2*>(z + d[uu] * R + jc) = v[uu];
      }
  }
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
// R = 1: one warp per row, lanes stride the row in 16-byte pairs (four pairs
// in flight per lane), shuffle-tree reduction. A row of odd length n_c starts
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

}  // namespace ddx

using namespace ddx;

extern "C" {

int ddx_schwarz_combine(int64_t n, int R, const int* dof_ptr, const int* dof_src, const void* ylocal,
                        int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                        const double* p_val, const double* yc, double sign, double* z, int dots,
                        const double* r, const double* q, double* st, int* ist, double* partials,
                        unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_schwarz_combine: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && z, "ddx_schwarz_combine: bad arguments");
  if (ylocal && dof_ptr) DDX_REQUIRE(dof_src, "ddx_schwarz_combine: transpose map without dof_src");
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
    const int grid2 = red_grid(ceil_div(n * (R / 2), 3));
    if (f64)
      k_combine2<double><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, (const double*)ylocal, u, p_ptr,
                                                    p_col, p_val, yc, sign, z, dots, r, q, partials, t);
    else
      k_combine2<float><<<grid2, kThreads, 0, s>>>(n, S, dof_ptr, dof_src, (const float*)ylocal, u, p_ptr,
                                                   p_col, p_val, yc, sign, z, dots, r, q, partials, t);
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
