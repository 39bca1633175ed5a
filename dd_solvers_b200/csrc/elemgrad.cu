// Per-element coefficient gradient of a Q1 diffusion solve.
//
// For A(kappa) u = b with A = sum_e kappa_e K_e (K_e the unit-coefficient
// element stiffness on the interior nodes) and an adjoint lambda solving
// A lambda = dL/du, dL/dkappa_e = -lambda_e^T K_e u_e. On a uniform grid
// K_e = h^(dim-2) K_ref, so one thread per cell gathers the 2^dim nodal values
// of u and lambda (zero on Dirichlet nodes) and contracts them with K_ref.
// Cells are numbered x fastest, matching the kappa layout [ez][ey][ex].
#include <algorithm>

#include "common.cuh"

namespace ddx {

template <int DIM>
__global__ void k_elem_grad_q1(int n_el, const double* __restrict__ u, const double* __restrict__ lam,
                               const double* __restrict__ kref, double scale, double* __restrict__ grad) {
  constexpr int NL = 1 << DIM;
  // K_ref ((2^dim)^2, row-major; local node bit d = offset along axis d, x = bit 0)
  __shared__ double c_kref[NL * NL];
  for (int q = threadIdx.x; q < NL * NL; q += blockDim.x) c_kref[q] = kref[q];
  __syncthreads();
  const int64_t ncell = DIM == 2 ? (int64_t)n_el * n_el : (int64_t)n_el * n_el * n_el;
  const int m = n_el - 1;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ncell; e += (int64_t)gridDim.x * blockDim.x) {
    int c[3] = {0, 0, 0};  // x, y, z cell coordinates
    int64_t t = e;
    c[0] = (int)(t % n_el); t /= n_el;
    c[1] = (int)(t % n_el); t /= n_el;
    if (DIM == 3) c[2] = (int)t;
    double ul[NL], ll[NL];
#pragma unroll
    for (int a = 0; a < NL; ++a) {
      bool interior = true;
      int64_t idx = 0;
#pragma unroll
      for (int d = DIM - 1; d >= 0; --d) {
        const int p = c[d] + ((a >> d) & 1);
        interior &= (p >= 1 && p <= m);
        idx = idx * m + (p - 1);
      }
      ul[a] = interior ? u[idx] : 0.0;
      ll[a] = interior ? lam[idx] : 0.0;
    }
    double g = 0.0;
#pragma unroll
    for (int a = 0; a < NL; ++a) {
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < NL; ++b) s = fma(c_kref[a * NL + b], ul[b], s);
      g = fma(ll[a], s, g);
    }
    grad[e] = -scale * g;
  }
}

}  // namespace ddx

using namespace ddx;

extern "C" int ddx_elem_grad_q1(int dim, int n_el, const double* u, const double* lam, const double* kref,
                                double* grad, ddx_stream_t stream) {
  DDX_REQUIRE(dim == 2 || dim == 3, "ddx_elem_grad_q1: dim must be 2 or 3");
  DDX_REQUIRE(n_el >= 2 && u && lam && kref && grad, "ddx_elem_grad_q1: bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  const double h = 1.0 / n_el;
  const double scale = dim == 2 ? 1.0 : h;  // h^(dim-2)
  const int64_t ncell = dim == 2 ? (int64_t)n_el * n_el : (int64_t)n_el * n_el * n_el;
  const int grid = (int)std::min<int64_t>(ceil_div(ncell, 256), 148 * 16);
  if (dim == 2) k_elem_grad_q1<2><<<grid, 256, 0, s>>>(n_el, u, lam, kref, scale, grad);
  else k_elem_grad_q1<3><<<grid, 256, 0, s>>>(n_el, u, lam, kref, scale, grad);
  DDX_LAUNCH_CHECK("ddx_elem_grad_q1");
  return DDX_OK;
}
