// Sparse SPD direct solve for large coarse problems: nested-dissection
// ordering (host) and the per-level multifrontal solve kernels (device).
//
// Replaces the cuDSS factor/solve behind the reference's CUDSS coarse solver
// (src/dd_solvers/dd_solvers/solvers.py:85-113, src/dd_solvers/cpp/cudss.cpp:64-105)
// for coarse spaces too large for a dense inverse. The numeric factorisation
// (dense fronts, batched Cholesky) runs in torch at setup; what it leaves for
// every front t is G_t = [Linv; M] ((s+u) x s, row-major FP64) with
// Linv = chol(F_SS)^-1 and M = F_US F_SS^-1, so both solve sweeps are dense
// GEMVs with no triangular recurrences:
//
//   forward  (leaves -> root): f = [w_S; 0] + children's update vectors
//            y_S = Linv f_S,  u_t = f_U - M f_S
//   backward (root -> leaves): x_S = Linv^T y_S - M^T x_U
//
// The backward sweep reads the transposed copy G_t^T, so both sweeps are
// row-wise GEMVs (a warp per row, lanes along the row: coalesced, short
// per-lane chains). One launch per tree level and sweep; every front is split
// into work items of a few rows sized by bytes. All sums run in a fixed order.
//
// On levels whose fronts are cut into many forward items, a gather launch
// first assembles each front's vector f = [w_S; 0] + children's updates once
// (into fb, front-position order), so the forward items read it contiguously
// instead of each repeating the index-chained gather of the whole f_S.
//
// The sweeps are latency-bound (a few hundred items per level, one level after
// another), so each item copies its operator rows into shared memory and
// reads its static index maps before waiting on the previous level: after the
// wait only the right-hand-side reads remain on its critical path.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <exception>
#include <system_error>
#include <thread>
#include <vector>

#include "common.cuh"

namespace ddx {
namespace {

constexpr int kNdThreads = 256;
constexpr int kNdWarps = kNdThreads / 32;
constexpr int kNdSmemMax = 96 * 1024;     // the staged vector (front rows x RHS group)
constexpr int kNdSmemOptin = 227 * 1024;  // a CTA's shared memory on sm_100
constexpr int kNdItemRows = 256;          // forward rows whose f_U is gathered up front (items hold <= 128)

// Programmatic dependent launch: each level's kernel is launched so that it
// may start while the previous one runs. Before griddepcontrol.wait it reads
// only the static plan and operators (staging its operator rows into shared
// memory); the wait returns once the previous grid has finished and its writes
// are visible. With `release`, each grid lets its successor launch right after
// its own wait, so a successor's prologue overlaps at most this grid's
// dependent phase; without it the successor launches when this grid ends.
__device__ __forceinline__ void wait_previous_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void release_next_grid() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Operator rows global -> shared with cp.async (8 bytes each: the rows of a
// front start at any double), all of a thread's copies in flight together.
__device__ __forceinline__ void stage_operator(double* dst, const double* __restrict__ src, int n) {
  for (int e = threadIdx.x; e < n; e += kNdThreads) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst + e);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src + e) : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void staged_operator_ready() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename Kernel, typename... Args>
cudaError_t launch_after_previous(Kernel kernel, unsigned grid, size_t smem, cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kNdThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct NdArgs {
  const int* items;
  const int* front_s;
  const int* front_u;
  const int64_t* g_off;
  const int64_t* idx_off;
  const int64_t* upd_off;
  const int* fidx;
  const int64_t* gptr;
  const int64_t* gsrc;
  const double* G;   // forward operator, (s+u) x s row-major per front
  const double* GT;  // its transpose, s x (s+u) row-major per front (backward sweep)
  const int64_t* s_first;  // elimination position of each front's first separator vertex
  const int* fpos;         // elimination position of every front position
};

// The static part of one front position's gather, read before the wait: its
// right-hand-side row (separator positions), its range in the gather map and
// the first two update rows it adds (the two children of a binary separator
// tree; positions of the merged top front may add more, read after the wait).
struct GatherSlot {
  int64_t v = 0, q0 = 0, q1 = 0, g0 = 0, g1 = 0;
  __device__ __forceinline__ void load(const NdArgs& A, int64_t io, int p, int s) {
    if (p < s) v = A.fidx[io + p];
    q0 = A.gptr[io + p];
    q1 = A.gptr[io + p + 1];
    if (q1 > q0) g0 = A.gsrc[q0];
    if (q1 > q0 + 1) g1 = A.gsrc[q0 + 1];
  }
  // f[p] for right-hand sides r0 .. r0+ng: w (separator rows), then the
  // update entries in gather-map order
  template <int RG>
  __device__ __forceinline__ void sum(const NdArgs& A, int p, int s, int R, int r0, int ng,
                                      const double* __restrict__ w, const double* __restrict__ upd,
                                      double (&acc)[RG]) const {
#pragma unroll
    for (int r = 0; r < RG; ++r) acc[r] = (p < s && r < ng) ? w[v * R + r0 + r] : 0.0;
    if (q1 > q0) {
#pragma unroll
      for (int r = 0; r < RG; ++r)
        if (r < ng) acc[r] += upd[g0 * R + r0 + r];
    }
    if (q1 > q0 + 1) {
#pragma unroll
      for (int r = 0; r < RG; ++r)
        if (r < ng) acc[r] += upd[g1 * R + r0 + r];
    }
    for (int64_t q = q0 + 2; q < q1; ++q) {
      const int64_t src = A.gsrc[q] * R + r0;
#pragma unroll
      for (int r = 0; r < RG; ++r)
        if (r < ng) acc[r] += upd[src + r];
    }
  }
};

// Forward item: rows row0 .. row0+nrows of G_t; a warp per row, lanes along
// the row. f_S (and f_U of the item's update rows) come from fb when the
// level's gather launch assembled them, else they are gathered here. With
// STAGE the item's operator rows (one contiguous range of G) are copied to
// shared memory before the wait.
// 4 CTAs per SM for the narrow RHS groups (latency-bound sweeps want warps in flight)
template <int RG, bool STAGE>
__global__ void __launch_bounds__(kNdThreads, RG <= 2 ? 4 : 1)
    k_nd_fwd(NdArgs A, int64_t item0, int R, const double* __restrict__ w, const double* __restrict__ fb,
             double* __restrict__ y, double* __restrict__ upd, const int* ist, int release) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double fu[kNdItemRows * RG];
  const int64_t it = item0 + blockIdx.x;
  const int t = A.items[3 * it], row0 = A.items[3 * it + 1], nrows = A.items[3 * it + 2];
  const int s = A.front_s[t];
  const int64_t io = A.idx_off[t], go = A.g_off[t], uo = A.upd_off[t];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* fs = sm;                   // f_S, s x RG
  double* gs = sm + (int64_t)s * RG;  // the item's operator rows, nrows x s
  if constexpr (STAGE) stage_operator(gs, A.G + go + (int64_t)row0 * s, nrows * s);
  // gather slots: the s separator positions, then the item's update rows
  // whose f_U goes to fu (u0 .. u1)
  const int u0 = max(row0, s), u1 = min(row0 + nrows, row0 + kNdItemRows);
  const int nslots = s + max(u1 - u0, 0);
  GatherSlot pre;
  if (fb == nullptr && (int)threadIdx.x < nslots) {
    const int k = threadIdx.x;
    pre.load(A, io, k < s ? k : u0 + (k - s), s);
  }
  wait_previous_grid();
  if (release) release_next_grid();
  if (ist != nullptr && n_active(ist, R) == 0) {
    if constexpr (STAGE) staged_operator_ready();
    return;
  }
  for (int r0 = 0; r0 < R; r0 += RG) {
    const int ng = min(RG, R - r0);
    for (int k = threadIdx.x; k < nslots; k += kNdThreads) {
      const int p = k < s ? k : u0 + (k - s);
      double acc[RG];
      if (fb != nullptr) {
#pragma unroll
        for (int r = 0; r < RG; ++r) acc[r] = r < ng ? fb[(io + p) * R + r0 + r] : 0.0;
      } else if (k == (int)threadIdx.x) {
        pre.sum<RG>(A, p, s, R, r0, ng, w, upd, acc);
      } else {
        GatherSlot g;
        g.load(A, io, p, s);
        g.sum<RG>(A, p, s, R, r0, ng, w, upd, acc);
      }
      double* dst = k < s ? fs + k * RG : fu + (p - row0) * RG;
#pragma unroll
      for (int r = 0; r < RG; ++r) dst[r] = acc[r];
    }
    if constexpr (STAGE) {
      if (r0 == 0) staged_operator_ready();
    }
    __syncthreads();
    for (int p = row0 + warp; p < row0 + nrows; p += kNdWarps) {
      double acc[RG];
#pragma unroll
      for (int r = 0; r < RG; ++r) acc[r] = 0.0;
      if constexpr (STAGE) {
        const double* g = gs + (int64_t)(p - row0) * s;
        for (int j = lane; j < s; j += 32) {
          const double gv = g[j];
#pragma unroll
          for (int r = 0; r < RG; ++r) acc[r] = fma(gv, fs[j * RG + r], acc[r]);
        }
      } else {
        const double* g = A.G + go + (int64_t)p * s;
        for (int j = lane; j < s; j += 32) {
          const double gv = __ldg(g + j);
#pragma unroll
          for (int r = 0; r < RG; ++r) acc[r] = fma(gv, fs[j * RG + r], acc[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < RG; ++r) acc[r] = warp_sum_d(acc[r]);
      if (p < s) {
        const int64_t e = A.s_first[t] + p;  // y is kept in elimination order
#pragma unroll
        for (int r = 0; r < RG; ++r)
          if (lane == r && r < ng) y[e * R + r0 + r] = acc[r];
      } else {
        // f_U of this row (gathered above unless the item is longer than
        // kNdItemRows), then u_t = f_U - M f_S
        double f[RG];
        if (p < u1) {
#pragma unroll
          for (int r = 0; r < RG; ++r) f[r] = fu[(p - row0) * RG + r];
        } else if (fb != nullptr) {
#pragma unroll
          for (int r = 0; r < RG; ++r) f[r] = r < ng ? fb[(io + p) * R + r0 + r] : 0.0;
        } else {
          GatherSlot g;
          g.load(A, io, p, s);
          g.sum<RG>(A, p, s, R, r0, ng, w, upd, f);
        }
        const int64_t dst = (uo + p - s) * R + r0;
#pragma unroll
        for (int r = 0; r < RG; ++r)
          if (lane == r && r < ng) upd[dst + r] = f[r] - acc[r];
      }
    }
    __syncthreads();
  }
}

// Gather item (t, p0, np): f at positions p0 .. p0+np of front t, all R
// right-hand sides, f[p] = (p < s ? w[fidx[p]] : 0) + the children's update
// entries in gather-map order (the order the forward items use on their own).
__global__ void __launch_bounds__(kNdThreads)
    k_nd_gather(NdArgs A, const int* __restrict__ gitems, int64_t item0, int R, const double* __restrict__ w,
                const double* __restrict__ upd, double* __restrict__ fb, const int* ist, int release) {
  const int64_t it = item0 + blockIdx.x;
  const int t = gitems[3 * it], p0 = gitems[3 * it + 1], np = gitems[3 * it + 2];
  const int s = A.front_s[t];
  const int64_t io = A.idx_off[t];
  GatherSlot pre;
  if ((int)threadIdx.x < np) pre.load(A, io, p0 + threadIdx.x, s);
  wait_previous_grid();
  if (release) release_next_grid();
  if (ist != nullptr && n_active(ist, R) == 0) return;
  for (int k = threadIdx.x; k < np; k += kNdThreads) {
    const int p = p0 + k;
    GatherSlot g = pre;
    if (k != (int)threadIdx.x) g.load(A, io, p, s);
    for (int r = 0; r < R; ++r) {
      double acc[1];
      g.sum<1>(A, p, s, R, r, 1, w, upd, acc);
      fb[(io + p) * R + r] = acc[0];
    }
  }
}

// Backward item: rows c0 .. c0+nc of G_t^T (columns of G_t); a warp per row,
// lanes over the s+u entries, v = [y_S; -x_U] staged in shared memory. With
// STAGE the item's rows of G_t^T (one contiguous range) are copied to shared
// memory before the wait.
template <int RG, bool STAGE>
__global__ void __launch_bounds__(kNdThreads, RG <= 2 ? 4 : 1)
    k_nd_bwd(NdArgs A, int64_t item0, int R, const double* __restrict__ y, double* __restrict__ xe,
             double* __restrict__ x, const int* ist, int release) {
  extern __shared__ __align__(16) double sm[];
  const int64_t it = item0 + blockIdx.x;
  const int t = A.items[3 * it], c0 = A.items[3 * it + 1], nc = A.items[3 * it + 2];
  const int s = A.front_s[t], m = s + A.front_u[t];
  const int64_t io = A.idx_off[t], go = A.g_off[t];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* vs = sm;                   // v, m x RG
  double* gs = sm + (int64_t)m * RG;  // the item's rows of G_t^T, nc x m
  if constexpr (STAGE) stage_operator(gs, A.GT + go + (int64_t)c0 * m, nc * m);
  // y and the solution are read in elimination order: the separator is one
  // range, the update set a few ranges of ancestor separators
  const int64_t sf = A.s_first[t];
  int64_t pre_e = 0;
  if ((int)threadIdx.x < m) {
    const int p = threadIdx.x;
    pre_e = p < s ? sf + p : (int64_t)A.fpos[io + p];
  }
  wait_previous_grid();
  if (release) release_next_grid();
  if (ist != nullptr && n_active(ist, R) == 0) {
    if constexpr (STAGE) staged_operator_ready();
    return;
  }
  for (int r0 = 0; r0 < R; r0 += RG) {
    const int ng = min(RG, R - r0);
    for (int p = threadIdx.x; p < m; p += kNdThreads) {
      const int64_t e = p == (int)threadIdx.x ? pre_e : (p < s ? sf + p : (int64_t)A.fpos[io + p]);
#pragma unroll
      for (int r = 0; r < RG; ++r)
        vs[p * RG + r] = r < ng ? (p < s ? y[e * R + r0 + r] : -xe[e * R + r0 + r]) : 0.0;
    }
    if constexpr (STAGE) {
      if (r0 == 0) staged_operator_ready();
    }
    __syncthreads();
    for (int c = c0 + warp; c < c0 + nc; c += kNdWarps) {
      double acc[RG];
#pragma unroll
      for (int r = 0; r < RG; ++r) acc[r] = 0.0;
      if constexpr (STAGE) {
        const double* g = gs + (int64_t)(c - c0) * m;
        for (int p = lane; p < m; p += 32) {
          const double gv = g[p];
#pragma unroll
          for (int r = 0; r < RG; ++r) acc[r] = fma(gv, vs[p * RG + r], acc[r]);
        }
      } else {
        const double* g = A.GT + go + (int64_t)c * m;
        for (int p = lane; p < m; p += 32) {
          const double gv = __ldg(g + p);
#pragma unroll
          for (int r = 0; r < RG; ++r) acc[r] = fma(gv, vs[p * RG + r], acc[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < RG; ++r) acc[r] = warp_sum_d(acc[r]);
      const int64_t v = A.fidx[io + c];
#pragma unroll
      for (int r = 0; r < RG; ++r)
        if (lane == r && r < ng) {
          xe[(sf + c) * R + r0 + r] = acc[r];  // for the descendants
          x[v * R + r0 + r] = acc[r];          // the result, in the caller's order
        }
    }
    __syncthreads();
  }
}

template <int RG>
int nd_sweeps(const ddx_nd_plan* P, const NdArgs& fa, const NdArgs& ba, int R, const double* w, double* x,
              double* y, double* xe, double* upd, double* fb, const int* ist, cudaStream_t s) {
  // dynamic shared memory: the staged vector, plus (staging kernels) the
  // operator rows where they fit
  const int fwd_cap = kNdSmemOptin - kNdItemRows * RG * (int)sizeof(double);
  const int bwd_cap = kNdSmemOptin;
  cudaFuncSetAttribute(k_nd_fwd<RG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNdSmemMax);
  cudaFuncSetAttribute(k_nd_bwd<RG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNdSmemMax);
  cudaFuncSetAttribute(k_nd_fwd<RG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwd_cap);
  cudaFuncSetAttribute(k_nd_bwd<RG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd_cap);
  const int rel = P->release_early;
  for (int lv = 0; lv < P->n_levels; ++lv) {
    const int64_t a = P->fwd_level_ptr[lv], b = P->fwd_level_ptr[lv + 1];
    if (b == a) continue;
    const size_t smem = (size_t)std::max(P->fwd_level_smax[lv], 1) * RG * sizeof(double);
    const int64_t gmax = P->fwd_level_gmax ? P->fwd_level_gmax[lv] : -1;
    const bool stage = gmax >= 0 && (int64_t)smem + gmax <= fwd_cap;
    const double* f = nullptr;
    if (fb != nullptr && P->gat_level_ptr != nullptr) {
      const int64_t ga = P->gat_level_ptr[lv], gb = P->gat_level_ptr[lv + 1];
      if (gb > ga) {
        launch_after_previous(k_nd_gather, (unsigned)(gb - ga), 0, s, fa, P->gat_items, ga, R, w,
                              (const double*)upd, fb, ist, rel);
        f = fb;
      }
    }
    if (stage)
      launch_after_previous(k_nd_fwd<RG, true>, (unsigned)(b - a), smem + (size_t)gmax, s, fa, a, R, w, f, y,
                            upd, ist, rel);
    else
      launch_after_previous(k_nd_fwd<RG, false>, (unsigned)(b - a), smem, s, fa, a, R, w, f, y, upd, ist, rel);
  }
  for (int lv = 0; lv < P->n_levels; ++lv) {
    const int64_t a = P->bwd_level_ptr[lv], b = P->bwd_level_ptr[lv + 1];
    if (b == a) continue;
    const size_t smem = (size_t)std::max(P->bwd_level_mmax[lv], 1) * RG * sizeof(double);
    const int64_t gmax = P->bwd_level_gmax ? P->bwd_level_gmax[lv] : -1;
    const bool stage = gmax >= 0 && (int64_t)smem + gmax <= bwd_cap;
    if (stage)
      launch_after_previous(k_nd_bwd<RG, true>, (unsigned)(b - a), smem + (size_t)gmax, s, ba, a, R,
                            (const double*)y, xe, x, ist, rel);
    else
      launch_after_previous(k_nd_bwd<RG, false>, (unsigned)(b - a), smem, s, ba, a, R, (const double*)y, xe, x,
                            ist, rel);
  }
  DDX_LAUNCH_CHECK("ddx_coarse_solve_nd");
  return DDX_OK;
}

// ---------------------------------------------------------------------------
// ordering: recursive BFS level-set bisection
// ---------------------------------------------------------------------------
// The two halves below a separator are independent subgraphs, so they are
// ordered on separate threads down to a few levels. The output does not
// depend on the threads: every subtree owns a known slice of perm (its
// vertices, in the sequential order: first half, second half, separator), and
// its nodes are numbered after the parent joins the halves' node lists.

constexpr int64_t kNdParMin = 20000;  // smallest pair of halves worth a thread

// Nodes of one subtree in creation (post-)order: perm offset and size of each
// node's vertex set, and its parent (index in this list; -1 for the roots).
struct NodeList {
  std::vector<int64_t> first, size, parent;
  void append(const NodeList& o) {
    const int64_t base = (int64_t)first.size();
    for (size_t i = 0; i < o.first.size(); ++i) {
      first.push_back(o.first[i]);
      size.push_back(o.size[i]);
      parent.push_back(o.parent[i] < 0 ? -1 : o.parent[i] + base);
    }
  }
  void add(int64_t f, int64_t s) {
    first.push_back(f);
    size.push_back(s);
    parent.push_back(-1);
  }
};

struct NdOrder {
  int64_t n;
  std::vector<int64_t> ptr, adj;  // symmetric adjacency, no self loops
  // current subgraph label of each vertex (-1 eliminated, -2 separator being
  // ordered below). A BFS reads the labels of neighbours that another thread
  // may be relabelling, never to the BFS's own label: relaxed atomics.
  std::vector<int64_t> label;
  std::vector<int64_t> seen, level;  // written only by the thread ordering the vertex's subgraph
  std::atomic<int64_t> stamp{0}, next_label{1};
  int leaf = 128;
  int par_depth = 0;  // recursion depth down to which the halves run on separate threads
  int64_t* perm = nullptr;

  int64_t get_label(int64_t v) { return __atomic_load_n(&label[v], __ATOMIC_RELAXED); }
  void set_label(int64_t v, int64_t l) { __atomic_store_n(&label[v], l, __ATOMIC_RELAXED); }

  // BFS over vertices labelled lab from src; returns the visit order and
  // fills level[] for the visited vertices.
  void bfs(int64_t src, int64_t lab, std::vector<int64_t>& order) {
    const int64_t st = stamp.fetch_add(1) + 1;
    order.clear();
    order.push_back(src);
    seen[src] = st;
    level[src] = 0;
    for (size_t h = 0; h < order.size(); ++h) {
      const int64_t v = order[h];
      for (int64_t e = ptr[v]; e < ptr[v + 1]; ++e) {
        const int64_t w = adj[e];
        if (get_label(w) == lab && seen[w] != st) {
          seen[w] = st;
          level[w] = level[v] + 1;
          order.push_back(w);
        }
      }
    }
  }

  // a node eliminating the vertices S (sorted) from perm[off]
  void put(std::vector<int64_t>& S, int64_t off, NodeList& out) {
    std::sort(S.begin(), S.end());
    for (size_t i = 0; i < S.size(); ++i) {
      perm[off + (int64_t)i] = S[i];
      set_label(S[i], -1);
    }
    out.add(off, (int64_t)S.size());
  }

  // Vertices V (all labelled lab), placed in perm from off: the nodes built for them.
  NodeList process(std::vector<int64_t> V, int64_t lab, int64_t off, int depth) {
    NodeList out;
    std::vector<std::vector<int64_t>> comps;
    std::vector<int64_t> order;
    for (int64_t v : V) {
      if (get_label(v) != lab) continue;
      bfs(v, lab, order);
      const int64_t lc = next_label.fetch_add(1);
      for (int64_t u : order) set_label(u, lc);
      comps.push_back(order);
    }
    for (auto& C : comps) {
      const int64_t lc = get_label(C[0]);
      const int64_t csize = (int64_t)C.size();
      if (csize <= leaf) {
        put(C, off, out);
        off += csize;
        continue;
      }
      bfs(C[0], lc, order);
      const int64_t far = order.back();
      bfs(far, lc, order);
      const int64_t depth_c = level[order.back()];
      if (depth_c < 2) {
        put(C, off, out);
        off += csize;
        continue;
      }
      std::vector<int64_t> cnt(depth_c + 1, 0);
      for (int64_t v : order) ++cnt[level[v]];
      int64_t k = 0, cum = 0;
      while (k <= depth_c && 2 * (cum + cnt[k]) < csize) cum += cnt[k++];
      k = std::min(std::max(k, (int64_t)1), depth_c - 1);
      std::vector<int64_t> S, Av, Bv;
      for (int64_t v : order) {
        if (level[v] == k) S.push_back(v);
        else if (level[v] < k) Av.push_back(v);
        else Bv.push_back(v);
      }
      const int64_t la = next_label.fetch_add(1), lb = next_label.fetch_add(1);
      for (int64_t v : S) set_label(v, -2);  // removed from both halves
      for (int64_t v : Av) set_label(v, la);
      for (int64_t v : Bv) set_label(v, lb);
      const int64_t na = (int64_t)Av.size(), nb = (int64_t)Bv.size();
      NodeList A, B;
      std::exception_ptr err;
      std::thread th;
      if (depth < par_depth && na + nb >= kNdParMin) {
        try {
          th = std::thread([&] {
            try {
              A = process(std::move(Av), la, off, depth + 1);
            } catch (...) {
              err = std::current_exception();
            }
          });
        } catch (const std::system_error&) {
          // no thread available: order this half here (same output)
        }
      }
      if (th.joinable()) {
        try {
          B = process(std::move(Bv), lb, off + na, depth + 1);
        } catch (...) {
          th.join();
          throw;
        }
        th.join();
        if (err) std::rethrow_exception(err);
      } else {
        A = process(std::move(Av), la, off, depth + 1);
        B = process(std::move(Bv), lb, off + na, depth + 1);
      }
      const int64_t base = (int64_t)out.first.size();
      out.append(A);
      out.append(B);
      const int64_t sid = (int64_t)out.first.size();
      for (int64_t i = base; i < sid; ++i)
        if (out.parent[i] < 0) out.parent[i] = sid;
      put(S, off + na + nb, out);
      off += csize;
    }
    return out;
  }
};

// threads for the ordering: DDX_ND_THREADS if set, else the host's
int nd_order_threads() {
  if (const char* e = std::getenv("DDX_ND_THREADS")) {
    const int t = std::atoi(e);
    if (t >= 1) return t;
  }
  const unsigned hw = std::thread::hardware_concurrency();
  return hw ? (int)hw : 1;
}

}  // namespace
}  // namespace ddx

using namespace ddx;

namespace {

int nd_order_impl(int64_t n, const int64_t* indptr, const int64_t* indices, int leaf, int64_t* perm,
                  int64_t* node_first, int64_t* node_parent, int64_t* n_nodes) {
  DDX_REQUIRE(n >= 0 && indptr && indices && perm && node_first && node_parent && n_nodes && leaf >= 1,
              "ddx_nd_order: bad arguments");
  NdOrder o;
  o.n = n;
  o.leaf = leaf;
  o.perm = perm;
  for (int t = nd_order_threads(); t > 1 && o.par_depth < 6; t >>= 1) ++o.par_depth;
  // symmetrised adjacency without the diagonal
  std::vector<int64_t> deg(n + 1, 0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t e = indptr[i]; e < indptr[i + 1]; ++e) {
      const int64_t j = indices[e];
      DDX_REQUIRE(j >= 0 && j < n, "ddx_nd_order: column %lld out of range", (long long)j);
      if (j != i) {
        ++deg[i + 1];
        ++deg[j + 1];
      }
    }
  o.ptr.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) o.ptr[i + 1] = o.ptr[i] + deg[i + 1];
  o.adj.resize(o.ptr[n]);
  std::vector<int64_t> fill(o.ptr.begin(), o.ptr.end() - 1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t e = indptr[i]; e < indptr[i + 1]; ++e) {
      const int64_t j = indices[e];
      if (j != i) {
        o.adj[fill[i]++] = j;
        o.adj[fill[j]++] = i;
      }
    }
  // sort and deduplicate each list (pattern given once or twice per pair)
  std::vector<int64_t> nptr(n + 1, 0);
  int64_t outp = 0;
  for (int64_t i = 0; i < n; ++i) {
    auto b = o.adj.begin() + o.ptr[i], e = o.adj.begin() + o.ptr[i + 1];
    std::sort(b, e);
    auto u = std::unique(b, e);
    nptr[i] = outp;
    for (auto it = b; it != u; ++it) o.adj[outp++] = *it;
  }
  nptr[n] = outp;
  o.adj.resize(outp);
  o.ptr.swap(nptr);
  o.label.assign(n, 0);
  o.seen.assign(n, 0);
  o.level.assign(n, 0);
  std::vector<int64_t> all(n);
  for (int64_t i = 0; i < n; ++i) all[i] = i;
  NodeList nodes;
  try {
    nodes = o.process(std::move(all), 0, 0, 0);
  } catch (const std::exception& ex) {
    ::ddx::set_error("ddx_nd_order: %s", ex.what());
    return DDX_ERR_ARG;
  }
  const int64_t nn = (int64_t)nodes.first.size();
  int64_t end = 0;
  for (int64_t i = 0; i < nn; ++i) {
    DDX_REQUIRE(nodes.first[i] == end, "ddx_nd_order: node %lld out of order", (long long)i);
    node_first[i] = nodes.first[i];
    node_parent[i] = nodes.parent[i];
    end += nodes.size[i];
  }
  node_first[nn] = end;
  *n_nodes = nn;
  DDX_REQUIRE(end == n, "ddx_nd_order: ordering incomplete (%lld of %lld)", (long long)end, (long long)n);
  return DDX_OK;
}

int nd_update_sets_impl(int64_t n, int64_t n_fronts, const int64_t* s_first, const int64_t* s_size,
                        const int64_t* p_ptr, const int64_t* p_pos, const int64_t* parent, int64_t* u_ptr,
                        int64_t* u_pos, int64_t capacity, int64_t* u_total) {
  DDX_REQUIRE(n >= 0 && n_fronts >= 0 && s_first && s_size && p_ptr && p_pos && parent && u_ptr && u_total &&
                  (capacity == 0 || u_pos),
              "ddx_nd_update_sets: bad arguments");
  // every front's separator range lies in [0, n), and p_ptr does not decrease over it
  for (int64_t t = 0; t < n_fronts; ++t) {
    DDX_REQUIRE(s_first[t] >= 0 && s_size[t] >= 0 && s_first[t] + s_size[t] <= n,
                "ddx_nd_update_sets: front %lld covers rows [%lld, %lld) outside [0, %lld)", (long long)t,
                (long long)s_first[t], (long long)(s_first[t] + s_size[t]), (long long)n);
    DDX_REQUIRE(p_ptr[s_first[t]] >= 0, "ddx_nd_update_sets: negative p_ptr at row %lld", (long long)s_first[t]);
    for (int64_t i = s_first[t]; i < s_first[t] + s_size[t]; ++i)
      DDX_REQUIRE(p_ptr[i] <= p_ptr[i + 1], "ddx_nd_update_sets: p_ptr decreases at row %lld", (long long)i);
  }
  // children of each front, in front order (a front's children precede it)
  std::vector<int64_t> cptr(n_fronts + 1, 0), cidx;
  for (int64_t t = 0; t < n_fronts; ++t) {
    DDX_REQUIRE(parent[t] < n_fronts && (parent[t] < 0 || parent[t] > t), "ddx_nd_update_sets: not a post-order");
    if (parent[t] >= 0) ++cptr[parent[t] + 1];
  }
  for (int64_t t = 0; t < n_fronts; ++t) cptr[t + 1] += cptr[t];
  cidx.resize(cptr[n_fronts]);
  {
    std::vector<int64_t> fill(cptr.begin(), cptr.end() - 1);
    for (int64_t t = 0; t < n_fronts; ++t)
      if (parent[t] >= 0) cidx[fill[parent[t]]++] = t;
  }
  // per front: its separator rows' positions and its children's update sets,
  // later than its own separator, sorted and distinct
  std::vector<int64_t> mark(n, -1), cand;
  std::vector<int64_t> store;  // all sets, concatenated as in u_pos (which may be too small to read back)
  u_ptr[0] = 0;
  for (int64_t t = 0; t < n_fronts; ++t) {
    const int64_t last = s_first[t] + s_size[t] - 1;
    cand.clear();
    for (int64_t e = p_ptr[s_first[t]]; e < p_ptr[s_first[t] + s_size[t]]; ++e) {
      const int64_t q = p_pos[e];
      DDX_REQUIRE(q >= 0 && q < n, "ddx_nd_update_sets: position %lld out of range", (long long)q);
      if (q > last && mark[q] != t) {
        mark[q] = t;
        cand.push_back(q);
      }
    }
    for (int64_t k = cptr[t]; k < cptr[t + 1]; ++k) {
      const int64_t c = cidx[k];
      for (int64_t i = u_ptr[c]; i < u_ptr[c + 1]; ++i) {
        const int64_t q = store[i];
        if (q > last && mark[q] != t) {
          mark[q] = t;
          cand.push_back(q);
        }
      }
    }
    std::sort(cand.begin(), cand.end());
    store.insert(store.end(), cand.begin(), cand.end());
    u_ptr[t + 1] = (int64_t)store.size();
  }
  const int64_t total = (int64_t)store.size();
  *u_total = total;
  DDX_REQUIRE(total <= capacity, "ddx_nd_update_sets: %lld update entries exceed the capacity %lld",
              (long long)total, (long long)capacity);
  std::copy(store.begin(), store.end(), u_pos);
  return DDX_OK;
}

}  // namespace

extern "C" {

// Host entry points: a failed allocation (or any other exception) in the host
// code comes back as a status code instead of crossing the C boundary.
int ddx_nd_order(int64_t n, const int64_t* indptr, const int64_t* indices, int leaf, int64_t* perm,
                 int64_t* node_first, int64_t* node_parent, int64_t* n_nodes) {
  try {
    return nd_order_impl(n, indptr, indices, leaf, perm, node_first, node_parent, n_nodes);
  } catch (const std::exception& ex) {
    ::ddx::set_error("ddx_nd_order: %s", ex.what());
    return DDX_ERR_ARG;
  }
}

int ddx_nd_update_sets(int64_t n, int64_t n_fronts, const int64_t* s_first, const int64_t* s_size,
                       const int64_t* p_ptr, const int64_t* p_pos, const int64_t* parent, int64_t* u_ptr,
                       int64_t* u_pos, int64_t capacity, int64_t* u_total) {
  try {
    return nd_update_sets_impl(n, n_fronts, s_first, s_size, p_ptr, p_pos, parent, u_ptr, u_pos, capacity, u_total);
  } catch (const std::exception& ex) {
    ::ddx::set_error("ddx_nd_update_sets: %s", ex.what());
    return DDX_ERR_ARG;
  }
}

int ddx_coarse_solve_nd(const ddx_nd_plan* P, int R, const double* w, double* x, double* y, double* xe,
                        double* upd, double* fb, const int* ist, ddx_stream_t stream) {
  DDX_REQUIRE(P && w && x && y && xe && upd && R >= 1, "ddx_coarse_solve_nd: bad arguments");
  DDX_REQUIRE(fb == nullptr || P->gat_level_ptr == nullptr || P->gat_level_ptr[P->n_levels] == 0 ||
                  P->gat_items != nullptr,
              "ddx_coarse_solve_nd: plan with gather levels but no gather items");
  DDX_REQUIRE(P->s_first && P->fpos, "ddx_coarse_solve_nd: plan without elimination positions");
  DDX_REQUIRE(P->fwd_level_ptr && P->bwd_level_ptr && P->fwd_level_smax && P->bwd_level_mmax,
              "ddx_coarse_solve_nd: plan without level tables");
  if (P->n == 0) return DDX_OK;
  cudaStream_t s = (cudaStream_t)stream;
  DDX_REQUIRE(P->G && P->GT, "ddx_coarse_solve_nd: plan without operators");
  NdArgs fa{P->fwd_items, P->front_s, P->front_u, P->g_off, P->idx_off, P->upd_off, P->fidx, P->gptr,
            P->gsrc, P->G, P->GT, P->s_first, P->fpos};
  NdArgs ba = fa;
  ba.items = P->bwd_items;
  const int64_t mmax = std::max<int64_t>(P->max_front, 1);
  // widest RHS group whose shared-memory vector fits
  int rg = 1;
  while (rg < 16 && rg * 2 <= R && mmax * rg * 2 * (int64_t)sizeof(double) <= kNdSmemMax) rg *= 2;
  DDX_REQUIRE(mmax * (int64_t)sizeof(double) <= kNdSmemMax, "ddx_coarse_solve_nd: front of %lld exceeds %d B",
              (long long)mmax, kNdSmemMax);
  switch (rg) {
    case 1: return nd_sweeps<1>(P, fa, ba, R, w, x, y, xe, upd, fb, ist, s);
    case 2: return nd_sweeps<2>(P, fa, ba, R, w, x, y, xe, upd, fb, ist, s);
    case 4: return nd_sweeps<4>(P, fa, ba, R, w, x, y, xe, upd, fb, ist, s);
    case 8: return nd_sweeps<8>(P, fa, ba, R, w, x, y, xe, upd, fb, ist, s);
    default: return nd_sweeps<16>(P, fa, ba, R, w, x, y, xe, upd, fb, ist, s);
  }
}

}  // extern "C"
