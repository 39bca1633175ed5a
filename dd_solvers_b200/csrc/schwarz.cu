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
