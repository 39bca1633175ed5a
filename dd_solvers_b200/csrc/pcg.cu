// PCG vector updates with fused deterministic reductions and a device-side
// stop test. Replaces the per-iteration torch ops of CG.solve
// (src/dd_solvers/dd_solvers/solvers.py:243-268): the norm + .item() host
// sync (244), torch.dot (256, 265) and the compiled axpy updates (170-189).
#include <stdarg.h>

#include "common.cuh"

namespace ddx {

static thread_local char g_msg[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
}

__device__ int g_device_error = 0;

__global__ void k_pcg_reset(PcgState S, int maxiter, int flexible, double rtol, double atol) {
  const int j = threadIdx.x;
  if (j < S.R) {
#pragma unroll
    for (int s = 0; s < DDX_ST_COUNT; ++s) S.s(s, j) = 0.0;
    S.s(DDX_ST_ATOL, j) = atol;
    S.s(DDX_ST_BB, j) = rtol;
    S.a(DDX_IST_ACTIVE, j) = 1;
    S.a(DDX_IST_ITERS, j) = 0;
  }
  if (j == 0) {
    S.g(DDX_G_NACTIVE) = S.R;
    S.g(DDX_G_MAXITER) = maxiter;
    S.g(DDX_G_FLEXIBLE) = flexible;
    S.g(DDX_G_BREAKDOWN) = 0;
    S.g(DDX_G_DEFER) = 0;
  }
}

// Epilogue of a deferred reduction on the totals parked in T0 / T1 (summed
// over the ranks by the caller): the same fin_* step as the fused kernels.
__global__ void k_pcg_finalize(PcgState S, int kind) {
  const int j = threadIdx.x;
  int act = 0;
  if (j < S.R) {
    const double t0 = S.s(DDX_ST_T0, j), t1 = S.s(DDX_ST_T1, j);
    if (kind == DDX_FIN_RZ) fin_rz(S, j, t0, t1);
    else if (kind == DDX_FIN_PQ) act = fin_pq(S, j, t0);
    else if (kind == DDX_FIN_RR) act = fin_rr(S, j, t0);
    else if (kind == DDX_FIN_INIT) act = fin_init(S, j, t1, t0);
    else act = fin_replace(S, j, t0);
    if (kind == DDX_FIN_INIT || kind == DDX_FIN_REPLACE) S.s(DDX_ST_RR_PACK, j) = S.s(DDX_ST_RR, j);
  }
  if (kind != DDX_FIN_RZ) publish_nactive(S, act);
}

// p = z + beta p; with x: first x += alpha_x p (a deferred x update)
__global__ void k_update_p(int64_t n, int R, const double* __restrict__ z, double* __restrict__ p,
                           double* __restrict__ x, const double* __restrict__ st, const int* __restrict__ ist) {
  if (n_active(ist, R) == 0) return;
  const int64_t total = n * R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int j = threadIdx.x % R;  // stride is a multiple of R
  const double beta = st[DDX_ST_BETA * R + j];
  if (x != nullptr) {
    const double ax = st[DDX_ST_ALPHA_X * R + j];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      const double pi = p[i];
      x[i] = fma(ax, pi, x[i]);
      p[i] = fma(beta, pi, z[i]);
    }
    return;
  }
  if (R == 1 && (((uintptr_t)z | (uintptr_t)p) & 15u) == 0) {
    // one right-hand side: element pairs with 16-byte loads
    const int64_t npair = total / 2;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t i = t0; i < npair; i += stride) {
      const double2 pv = reinterpret_cast<const double2*>(p)[i], zv = reinterpret_cast<const double2*>(z)[i];
      reinterpret_cast<double2*>(p)[i] = make_double2(fma(beta, pv.x, zv.x), fma(beta, pv.y, zv.y));
    }
    if ((total & 1) && t0 == 0) p[total - 1] = fma(beta, p[total - 1], z[total - 1]);
    return;
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    p[i] = fma(beta, p[i], z[i]);
  }
}

// x += alpha_x p, the parked step of a deferred x update, then alpha_x = 0
// (by the last CTA, after every CTA has read it). Runs even when no RHS is
// active: it completes the solution after the last update.
__global__ void __launch_bounds__(kThreads) k_flush_x(int64_t n, int R, double* __restrict__ x,
                                                      const double* __restrict__ p, double* st,
                                                      unsigned int* ticket) {
  const int64_t total = n * R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int j = threadIdx.x % R;
  const double ax = st[DDX_ST_ALPHA_X * R + j];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride)
    x[i] = fma(ax, p[i], x[i]);
  if (!last_cta_arrival(ticket)) return;
  if (threadIdx.x < R) st[DDX_ST_ALPHA_X * R + threadIdx.x] = 0.0;
  if (threadIdx.x == 0) *ticket = 0u;
}

// x += alpha p; r -= alpha q; rr = ||r||^2 -> stop test
__global__ void __launch_bounds__(kThreads) k_update_xr(int64_t n, PcgState S, double* __restrict__ x,
                                                        double* __restrict__ r, const double* __restrict__ p,
                                                        const double* __restrict__ q, double* partials,
                                                        unsigned int* ticket) {
  __shared__ double red[kThreads];
  const int R = S.R;
  if (n_active(S.ist, R) == 0) return;
  const int64_t total = n * R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int j = threadIdx.x % R;
  const double alpha = S.st[DDX_ST_ALPHA * R + j];
  const bool defer_x = x == nullptr;  // x += alpha p left to the next p update
  double acc[1] = {0.0};
  const bool aligned = (((uintptr_t)x | (uintptr_t)r | (uintptr_t)p | (uintptr_t)q) & 15u) == 0;
  if (R == 1 && aligned) {
    // one right-hand side: element pairs with 16-byte loads, two pairs in flight
    const int64_t npair = total / 2;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t i = t0; i < npair; i += 2 * stride) {
      const bool two = i + stride < npair;
      const double2 qa = reinterpret_cast<const double2*>(q)[i], ra = reinterpret_cast<const double2*>(r)[i];
      double2 qb = make_double2(0.0, 0.0), rb = qb;
      if (two) {
        qb = reinterpret_cast<const double2*>(q)[i + stride];
        rb = reinterpret_cast<const double2*>(r)[i + stride];
      }
      if (!defer_x) {
        const double2 pa = reinterpret_cast<const double2*>(p)[i], xa = reinterpret_cast<const double2*>(x)[i];
        reinterpret_cast<double2*>(x)[i] = make_double2(fma(alpha, pa.x, xa.x), fma(alpha, pa.y, xa.y));
        if (two) {
          const double2 pb = reinterpret_cast<const double2*>(p)[i + stride];
          const double2 xb = reinterpret_cast<const double2*>(x)[i + stride];
          reinterpret_cast<double2*>(x)[i + stride] = make_double2(fma(alpha, pb.x, xb.x), fma(alpha, pb.y, xb.y));
        }
      }
      const double2 na = make_double2(fma(-alpha, qa.x, ra.x), fma(-alpha, qa.y, ra.y));
      reinterpret_cast<double2*>(r)[i] = na;
      acc[0] = fma(na.x, na.x, acc[0]);
      acc[0] = fma(na.y, na.y, acc[0]);
      if (two) {
        const double2 nb = make_double2(fma(-alpha, qb.x, rb.x), fma(-alpha, qb.y, rb.y));
        reinterpret_cast<double2*>(r)[i + stride] = nb;
        acc[0] = fma(nb.x, nb.x, acc[0]);
        acc[0] = fma(nb.y, nb.y, acc[0]);
      }
    }
    if ((total & 1) && t0 == 0) {  // an odd length: the last element
      const int64_t i = total - 1;
      if (!defer_x) x[i] = fma(alpha, p[i], x[i]);
      const double ri = fma(-alpha, q[i], r[i]);
      r[i] = ri;
      acc[0] = fma(ri, ri, acc[0]);
    }
  } else {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
      if (!defer_x) x[i] = fma(alpha, p[i], x[i]);
      const double ri = fma(-alpha, q[i], r[i]);
      r[i] = ri;
      acc[0] = fma(ri, ri, acc[0]);
    }
  }
  write_cta_partials<1>(acc, red, R, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[1];
  final_sums<1>(partials, R, red, tot, ticket);
  if (park_totals<1>(S, tot)) return;
  int act = 0;
  if (threadIdx.x < R) act = fin_rr(S, threadIdx.x, tot[0], defer_x);
  publish_nactive(S, act);
}

// k_update_xr for R in {16, 32, 64} right-hand sides that also writes the
// tensor-core B panels of the next local apply (BF16, one residual term, scale
// 1). Same layout as the multi-RHS SpMM: R/2 threads per DOF, each owning two
// adjacent columns (16-byte loads, a warp reads whole rows), so x, p, r, q
// stream exactly as in the plain update; each thread then stores its two
// columns of r rounded to BF16 (4 bytes) into every panel row that holds the
// DOF (pan_row[e] for e in [pan_ptr[d], pan_ptr[d+1]): the row's byte offset in
// b16), in 16-byte chunk (c2 / 4) ^ ((offset >> 7) & mask), the panel's row
// swizzle (mask 7 / 3 / 1 for R = 64 / 32 / 16): the threads of a DOF write
// its panel row whole. The pack pass and its re-read of r through the subdomain
// index maps disappear. rr = ||r||^2 per column in a fixed order (CTA trees of
// the even and odd columns, then the last CTA).
// T16 = __half: the FP16 panels of ddx_pack_panels16 (per-RHS power-of-two
// scale from the squared norm in st slot RR when the update starts, the norm
// kept in slot RR_PACK for the apply); T16 = __nv_bfloat16: scale 1.
template <typename T16, int R>
__global__ void __launch_bounds__(kThreads) k_update_xr_pack(int64_t n, PcgState S, double* __restrict__ x,
                                                             double* __restrict__ r, const double* __restrict__ p,
                                                             const double* __restrict__ q,
                                                             const int* __restrict__ pan_ptr,
                                                             const int64_t* __restrict__ pan_row,
                                                             unsigned char* __restrict__ b16, double* partials,
                                                             unsigned int* ticket) {
  constexpr int TPR = R / 2;  // threads per DOF, two columns each
  constexpr uint32_t kMask = R == 64 ? 7u : (R == 32 ? 3u : 1u);
  __shared__ double red[kThreads];
  if (n_active(S.ist, R) == 0) return;
  const int c2 = threadIdx.x % TPR;  // the stride is a multiple of TPR
  const double a0 = S.st[DDX_ST_ALPHA * R + 2 * c2], a1 = S.st[DDX_ST_ALPHA * R + 2 * c2 + 1];
  constexpr bool kF16 = std::is_same<T16, __half>::value;
  // the 16-bit conversion scales (FP16), from the norm before this update
  const double sc0 = kF16 ? (double)rhs_scale<T16>(S.st, R, 2 * c2) : 1.0;
  const double sc1 = kF16 ? (double)rhs_scale<T16>(S.st, R, 2 * c2 + 1) : 1.0;
  const double rr_old = threadIdx.x < R ? S.st[DDX_ST_RR * R + threadIdx.x] : 0.0;
  const int inrow = ((c2 >> 2) << 4) | ((c2 & 3) << 2);  // byte of this thread's pair in an unswizzled row
  double acc0 = 0.0, acc1 = 0.0;
  const int64_t total = n * TPR;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const bool defer_x = x == nullptr;  // x += alpha p left to the next p update
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int64_t d = i / TPR;
    const int64_t o = d * R + 2 * c2;
    if (!defer_x) {
      const double2 xv = *reinterpret_cast<const double2*>(x + o);
      const double2 pv = *reinterpret_cast<const double2*>(p + o);
      *reinterpret_cast<double2*>(x + o) = make_double2(fma(a0, pv.x, xv.x), fma(a1, pv.y, xv.y));
    }
    const double2 rv = *reinterpret_cast<const double2*>(r + o);
    const double2 qv = *reinterpret_cast<const double2*>(q + o);
    const double2 rn = make_double2(fma(-a0, qv.x, rv.x), fma(-a1, qv.y, rv.y));
    *reinterpret_cast<double2*>(r + o) = rn;
    acc0 = fma(rn.x, rn.x, acc0);
    acc1 = fma(rn.y, rn.y, acc1);
    const uint32_t bits = (uint32_t)to_bits<T16>(rn.x * sc0) | ((uint32_t)to_bits<T16>(rn.y * sc1) << 16);
    const int e1 = __ldg(pan_ptr + d + 1);
    for (int e = __ldg(pan_ptr + d); e < e1; ++e) {
      const int64_t off = __ldg(pan_row + e);
      *reinterpret_cast<uint32_t*>(b16 + off + (inrow ^ (int)(((off >> 7) & kMask) << 4))) = bits;
    }
  }
  // CTA sums of each column, written as partials[cta * R + column]
  const double s0 = block_sum_by_col(acc0, red, TPR);
  if (threadIdx.x < TPR) partials[(size_t)blockIdx.x * R + 2 * threadIdx.x] = s0;
  const double s1 = block_sum_by_col(acc1, red, TPR);
  if (threadIdx.x < TPR) partials[(size_t)blockIdx.x * R + 2 * threadIdx.x + 1] = s1;
  if (!last_cta_arrival(ticket)) return;
  double tot[1];
  final_sums<1>(partials, R, red, tot, ticket);
  if (park_totals<1>(S, tot)) return;
  int act = 0;
  if (threadIdx.x < R) {
    if (kF16) S.s(DDX_ST_RR_PACK, threadIdx.x) = rr_old;  // the norm the panels were scaled with
    act = fin_rr(S, threadIdx.x, tot[0], defer_x);
  }
  publish_nactive(S, act);
}

// rho = r.z, zq = z.q -> beta
__global__ void __launch_bounds__(kThreads) k_dots_rz(int64_t n, PcgState S, const double* __restrict__ r,
                                                      const double* __restrict__ z,
                                                      const double* __restrict__ q, double* partials,
                                                      unsigned int* ticket) {
  __shared__ double red[kThreads];
  const int R = S.R;
  if (n_active(S.ist, R) == 0) return;
  const int64_t total = n * R;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
    const double zi = z[i];
    acc[0] = fma(r[i], zi, acc[0]);
    if (q != nullptr) acc[1] = fma(zi, q[i], acc[1]);
  }
  write_cta_partials<2>(acc, red, R, partials);
  if (!last_cta_arrival(ticket)) return;
  double tot[2];
  final_sums<2>(partials, R, red, tot, ticket);
  if (park_totals<2>(S, tot)) return;
  if (threadIdx.x < R) fin_rz(S, threadIdx.x, tot[0], tot[1]);
}

}  // namespace ddx

using namespace ddx;

extern "C" {

const char* ddx_last_error(void) { return g_msg; }

int ddx_version(void) { return 100; }

size_t ddx_partials_len(int R) { return (size_t)kRedCtas * kMaxNV * (size_t)R; }

int ddx_device_error(int* code) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_device_error, sizeof(int));
  if (e != cudaSuccess) {
    set_error("ddx_device_error: %s", cudaGetErrorString(e));
    return DDX_ERR_CUDA;
  }
  int zero = 0;
  e = cudaMemcpyToSymbol(g_device_error, &zero, sizeof(int));
  if (e != cudaSuccess) {
    set_error("ddx_device_error: %s", cudaGetErrorString(e));
    return DDX_ERR_CUDA;
  }
  if (code) *code = v;
  return DDX_OK;
}

int ddx_pcg_reset(int R, double* st, int* ist, int maxiter, int flexible, double rtol, double atol,
                  ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_reset: unsupported R=%d", R);
  DDX_REQUIRE(st && ist, "ddx_pcg_reset: null state");
  DDX_REQUIRE(maxiter >= 0, "ddx_pcg_reset: maxiter < 0");
  PcgState S{st, ist, nullptr, R};
  k_pcg_reset<<<1, 64, 0, (cudaStream_t)stream>>>(S, maxiter, flexible, rtol, atol);
  DDX_LAUNCH_CHECK("ddx_pcg_reset");
  return DDX_OK;
}

int ddx_pcg_finalize(int R, int kind, double* st, int* ist, double* hist, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_finalize: unsupported R=%d", R);
  DDX_REQUIRE(st && ist && hist, "ddx_pcg_finalize: null state");
  DDX_REQUIRE(kind >= DDX_FIN_RZ && kind <= DDX_FIN_REPLACE, "ddx_pcg_finalize: unknown kind %d", kind);
  PcgState S{st, ist, hist, R};
  k_pcg_finalize<<<1, 64, 0, (cudaStream_t)stream>>>(S, kind);
  DDX_LAUNCH_CHECK("ddx_pcg_finalize");
  return DDX_OK;
}

int ddx_pcg_update_p(int64_t n, int R, const double* z, double* p, const double* st, const int* ist,
                     ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_update_p: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && z && p && st && ist, "ddx_pcg_update_p: bad arguments");
  if (n == 0) return DDX_OK;
  int grid = (int)std::min<int64_t>(ceil_div(n * R, kThreads), 148 * 16);
  k_update_p<<<grid, kThreads, 0, (cudaStream_t)stream>>>(n, R, z, p, nullptr, st, ist);
  DDX_LAUNCH_CHECK("ddx_pcg_update_p");
  return DDX_OK;
}

int ddx_pcg_update_px(int64_t n, int R, const double* z, double* p, double* x, const double* st, const int* ist,
                      ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_update_px: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && z && p && x && st && ist, "ddx_pcg_update_px: bad arguments");
  if (n == 0) return DDX_OK;
  int grid = (int)std::min<int64_t>(ceil_div(n * R, kThreads), 148 * 16);
  k_update_p<<<grid, kThreads, 0, (cudaStream_t)stream>>>(n, R, z, p, x, st, ist);
  DDX_LAUNCH_CHECK("ddx_pcg_update_px");
  return DDX_OK;
}

int ddx_pcg_flush_x(int64_t n, int R, double* x, const double* p, double* st, unsigned int* tickets,
                    ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_flush_x: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && x && p && st && tickets, "ddx_pcg_flush_x: bad arguments");
  k_flush_x<<<red_grid(n * R), kThreads, 0, (cudaStream_t)stream>>>(n, R, x, p, st, tickets + 5);
  DDX_LAUNCH_CHECK("ddx_pcg_flush_x");
  return DDX_OK;
}

int ddx_pcg_update_xr(int64_t n, int R, double* x, double* r, const double* p, const double* q,
                      double* st, int* ist, double* hist, double* partials, unsigned int* tickets,
                      ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_update_xr: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && r && p && q && st && ist && hist && partials && tickets,
              "ddx_pcg_update_xr: bad arguments");
  PcgState S{st, ist, hist, R};
  k_update_xr<<<red_grid(n * R), kThreads, 0, (cudaStream_t)stream>>>(n, S, x, r, p, q, partials,
                                                                       tickets + 0);
  DDX_LAUNCH_CHECK("ddx_pcg_update_xr");
  return DDX_OK;
}

int ddx_pcg_update_xr_pack16(int64_t n, int R, double* x, double* r, const double* p, const double* q,
                             const int* pan_ptr, const int64_t* pan_row, void* b16, double* st, int* ist,
                             double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream) {
  return ddx_pcg_update_xr_pack16_ex(n, R, x, r, p, q, pan_ptr, pan_row, b16, DDX_BF16, st, ist, hist, partials,
                                     tickets, stream);
}

int ddx_pcg_update_xr_pack16_ex(int64_t n, int R, double* x, double* r, const double* p, const double* q,
                                const int* pan_ptr, const int64_t* pan_row, void* b16, int dtype, double* st,
                                int* ist, double* hist, double* partials, unsigned int* tickets,
                                ddx_stream_t stream) {
  DDX_REQUIRE(dtype == DDX_BF16 || dtype == DDX_F16, "ddx_pcg_update_xr_pack16: dtype must be BF16 or F16");
  DDX_REQUIRE(R == 16 || R == 32 || R == 64, "ddx_pcg_update_xr_pack16: R must be 16, 32 or 64 (got %d)", R);
  DDX_REQUIRE(n >= 0 && r && p && q && pan_ptr && pan_row && b16 && st && ist && hist && partials && tickets,
              "ddx_pcg_update_xr_pack16: bad arguments");
  DDX_REQUIRE(((uintptr_t)x & 15u) == 0 && ((uintptr_t)r & 15u) == 0 && ((uintptr_t)p & 15u) == 0 &&
                  ((uintptr_t)q & 15u) == 0 && ((uintptr_t)b16 & 15u) == 0,
              "ddx_pcg_update_xr_pack16: x, r, p, q and b16 must be 16-byte aligned");
  if (n == 0) return DDX_OK;
  PcgState S{st, ist, hist, R};
  const int grid = red_grid(n * (R / 2));
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* b = (unsigned char*)b16;
  auto go = [&](auto t16) {
    using T16 = decltype(t16);
    if (R == 16)
      k_update_xr_pack<T16, 16><<<grid, kThreads, 0, s>>>(n, S, x, r, p, q, pan_ptr, pan_row, b, partials, tickets);
    else if (R == 32)
      k_update_xr_pack<T16, 32><<<grid, kThreads, 0, s>>>(n, S, x, r, p, q, pan_ptr, pan_row, b, partials, tickets);
    else
      k_update_xr_pack<T16, 64><<<grid, kThreads, 0, s>>>(n, S, x, r, p, q, pan_ptr, pan_row, b, partials, tickets);
  };
  if (dtype == DDX_F16) go(__half());
  else go(__nv_bfloat16());
  DDX_LAUNCH_CHECK("ddx_pcg_update_xr_pack16");
  return DDX_OK;
}

int ddx_pcg_dots_rz(int64_t n, int R, const double* r, const double* z, const double* q, double* st,
                    int* ist, double* partials, unsigned int* tickets, ddx_stream_t stream) {
  DDX_REQUIRE(valid_rhs_count(R), "ddx_pcg_dots_rz: unsupported R=%d", R);
  DDX_REQUIRE(n >= 0 && r && z && st && ist && partials && tickets, "ddx_pcg_dots_rz: bad arguments");
  PcgState S{st, ist, nullptr, R};
  k_dots_rz<<<red_grid(n * R), kThreads, 0, (cudaStream_t)stream>>>(n, S, r, z, q, partials,
                                                                     tickets + 1);
  DDX_LAUNCH_CHECK("ddx_pcg_dots_rz");
  return DDX_OK;
}

}  // extern "C"
