/*
 * ddx.h - C ABI of the B200 (sm_100a) Schwarz-preconditioned CG kernels.
 *
 * Every entry point takes raw device pointers, sizes and a CUDA stream, never
 * allocates device memory, launches asynchronously on `stream`, and returns a
 * ddx_status (0 = success). The message of the last failure on the calling
 * thread is returned by ddx_last_error().
 *
 * Vector blocks of several right-hand sides use the layout (n, R) with the R
 * values of one DOF contiguous ("DOF-major"); R = 1 is a plain vector. The
 * fused PCG kernels support R in {1, 2, 4, 8, 16, 32, 64}.
 *
 * References (paths within mgr0dzicki/dd-solvers) name the interface of the
 * reference that each entry point replaces.
 */
#ifndef DDX_H
#define DDX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* ddx_stream_t; /* same type as cudaStream_t */

enum ddx_status {
  DDX_OK = 0,
  DDX_ERR_ARG = 1,         /* invalid argument (shape, alignment, dtype) */
  DDX_ERR_CUDA = 2,        /* CUDA launch or runtime error */
  DDX_ERR_UNSUPPORTED = 3  /* valid request this build does not implement */
};

enum ddx_dtype { DDX_F64 = 0, DDX_F32 = 1, DDX_BF16 = 2, DDX_F16 = 3 };

/* ---- PCG state (device memory owned by the caller) ----------------------
 * st   : double[DDX_ST_COUNT * R], slot s of RHS j at st[s*R + j]
 * ist  : int[DDX_IST_COUNT * R + DDX_G_COUNT], slot s of RHS j at ist[s*R + j],
 *        global g at ist[DDX_IST_COUNT*R + g]
 * hist : double[(maxiter + 1) * R], residual norm after k updates of RHS j at
 *        hist[k*R + j]
 * partials / tickets: reduction scratch, sized by ddx_partials_len(R) doubles
 *        and DDX_TICKETS unsigned ints (zero-initialised once by the caller;
 *        every kernel leaves its ticket at zero again).
 */
enum {
  DDX_ST_RHO = 0, DDX_ST_RHO_PREV = 1, DDX_ST_ZQ = 2, DDX_ST_PQ = 3, DDX_ST_ALPHA = 4,
  DDX_ST_BETA = 5, DDX_ST_RR = 6, DDX_ST_ATOL = 7, DDX_ST_BB = 8,
  DDX_ST_T0 = 9, DDX_ST_T1 = 10, /* parked column totals (DDX_G_DEFER) */
  DDX_ST_ALPHA_X = 11,            /* step length still to be applied to x (deferred x update) */
  DDX_ST_RR_PACK = 12,            /* ||r||^2 the current 16-bit B panels were scaled with */
  DDX_ST_COUNT = 13
};
enum { DDX_IST_ACTIVE = 0, DDX_IST_ITERS = 1, DDX_IST_COUNT = 2 };
enum {
  DDX_G_NACTIVE = 0,   /* number of RHS still iterating */
  DDX_G_MAXITER = 1,   /* update limit per RHS */
  DDX_G_FLEXIBLE = 2,  /* 1: Polak-Ribiere beta, 0: Fletcher-Reeves */
  DDX_G_BREAKDOWN = 3, /* set when p.q <= 0 stopped a RHS */
  DDX_G_DEFER = 4,     /* 1: reductions park their totals for ddx_pcg_finalize */
  DDX_G_COUNT = 5
};
/* Deferred reductions (a solve sharded over ranks): with DDX_G_DEFER set (the
 * caller writes 1 after ddx_pcg_reset, which clears it), every fused reduction
 * of this header (SpMV modes PQ / RES_INIT / RES_REPLACE, ddx_pcg_update_xr,
 * ddx_pcg_update_xr_pack16, ddx_pcg_dots_rz, ddx_schwarz_combine with dots)
 * stores its column totals of this rank's rows in st slots DDX_ST_T0 (and
 * DDX_ST_T1: r.r for RES_INIT's b.b, z.q for the r.z pair) instead of running
 * the step-length / stop-test epilogue. The caller sums those 2R doubles over
 * the ranks (one all-reduce) and then calls ddx_pcg_finalize with the kind of
 * the reduction, which runs the same epilogue on the summed totals. */
enum {
  DDX_FIN_RZ = 0,      /* T0 = r.z, T1 = z.q      -> beta        */
  DDX_FIN_PQ = 1,      /* T0 = p.q                -> alpha       */
  DDX_FIN_RR = 2,      /* T0 = r.r                -> stop test   */
  DDX_FIN_INIT = 3,    /* T0 = r.r, T1 = b.b      -> tolerance, first stop test */
  DDX_FIN_REPLACE = 4  /* T0 = r.r (replaced r)   -> stop test   */
};
enum { DDX_TICKETS = 16 };

const char* ddx_last_error(void);
int ddx_version(void);
/* doubles needed for the `partials` scratch of the fused reductions */
size_t ddx_partials_len(int R);
/* Reads and clears the device-side error word (bounded-wait timeouts).
 * Synchronous. 0 = no error. */
int ddx_device_error(int* code);

/* ---- PCG state and vector updates ---------------------------------------
 * Replace CG.solve's torch ops: fused_add / fused_sub / fused_mul_add
 * (src/dd_solvers/dd_solvers/solvers.py:170-189), torch.dot (256, 265) and
 * torch.linalg.norm(r).item() (244), which become device-side deterministic
 * reductions with the stop test evaluated on the device. */

/* Initialise st/ist for a new solve: iterations 0, every RHS active,
 * maxiter and flexible flags, tolerance constants. */
int ddx_pcg_reset(int R, double* st, int* ist, int maxiter, int flexible, double rtol, double atol,
                  ddx_stream_t stream);
/* p = z + beta p (beta = 0 on a RHS's first iteration). */
int ddx_pcg_update_p(int64_t n, int R, const double* z, double* p, const double* st, const int* ist,
                     ddx_stream_t stream);
/* x += alpha p; r -= alpha q; then rr = ||r||^2 per RHS, stop test, history.
 * Deferred x update (x = NULL): only r is updated and alpha is parked in st
 * slot DDX_ST_ALPHA_X; the next ddx_pcg_update_px / ddx_schwarz_combine_update,
 * which read p anyway, apply it to x before p changes (one read of p fewer per
 * iteration), and ddx_pcg_flush_x applies what is left after the last update
 * or before a residual replacement. Same x bits as the undeferred update. */
int ddx_pcg_update_xr(int64_t n, int R, double* x, double* r, const double* p, const double* q,
                      double* st, int* ist, double* hist, double* partials, unsigned int* tickets,
                      ddx_stream_t stream);
/* p = z + beta p, after x += alpha_x p with the parked step length of a
 * deferred x update (st slot DDX_ST_ALPHA_X, 0 when nothing is parked): the
 * x update of solvers.py:265 moved into the p update of solvers.py:267. */
int ddx_pcg_update_px(int64_t n, int R, const double* z, double* p, double* x, const double* st, const int* ist,
                      ddx_stream_t stream);
/* x += alpha_x p with the parked step length (DDX_ST_ALPHA_X), which is then
 * cleared; runs whether or not any RHS is still active. */
int ddx_pcg_flush_x(int64_t n, int R, double* x, const double* p, double* st, unsigned int* tickets,
                    ddx_stream_t stream);
/* The epilogue of a deferred reduction (DDX_G_DEFER) on the totals in st slots
 * DDX_ST_T0 / DDX_ST_T1, after the caller summed them over the ranks: kind is a
 * DDX_FIN_* value. One CTA; same arithmetic as the in-kernel epilogue, so every
 * rank that holds the same totals reaches the same alpha, beta and stop
 * decisions. Replaces the host-side scalar steps of CG.solve (solvers.py:244-267)
 * for a solve whose vectors are split over ranks. */
int ddx_pcg_finalize(int R, int kind, double* st, int* ist, double* hist, ddx_stream_t stream);
/* ddx_pcg_update_xr for R in {16, 32, 64} (16-byte aligned vectors) that also
 * writes r, rounded to BF16 with scale 1, into the tensor-core B panels of the
 * next local apply (ddx_pack_panels16's layout with one term): DOF d's row goes
 * to every panel row that holds it, at byte offsets pan_row[e] of b16 for e in
 * [pan_ptr[d], pan_ptr[d+1]) (offset = panel_off[i] + 2R c for DOF d at local
 * row c of subdomain i), its 16-byte chunk q at q ^ ((offset >> 7) & mask),
 * mask 7 / 3 / 1 for R = 64 / 32 / 16. The apply then runs without a pack and
 * with st = NULL (scale 1). rr is summed per column in a fixed order (not the
 * order of ddx_pcg_update_xr). Replaces the same reference updates as
 * ddx_pcg_update_xr (solvers.py:265-267) plus the gather of r into the
 * local solves (Inv.solve's input, solvers.py:355-359). */
/* x = NULL: deferred x update, as for ddx_pcg_update_xr. */
int ddx_pcg_update_xr_pack16(int64_t n, int R, double* x, double* r, const double* p, const double* q,
                             const int* pan_ptr, const int64_t* pan_row, void* b16, double* st, int* ist,
                             double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream);
/* The same for BF16 (dtype DDX_BF16, scale 1, as above) or FP16 (DDX_F16)
 * panels. FP16 panels hold s_j r[d, j] with the power-of-two scale s_j of
 * ddx_pack_panels16 taken from the squared norm this update starts from
 * (st slot DDX_ST_RR before it is replaced); that squared norm is left in slot
 * DDX_ST_RR_PACK, and the tensor-core apply that reads these panels must
 * take its scales from there: pass it st + (DDX_ST_RR_PACK - DDX_ST_RR) * R
 * (the SpMV residual modes also copy RR to RR_PACK, for panels that
 * ddx_pack_panels16 writes from a freshly computed residual). The scale is a
 * power of two, so the products equal those of panels scaled with the new
 * norm except where an entry over- or underflows the 16-bit range. */
int ddx_pcg_update_xr_pack16_ex(int64_t n, int R, double* x, double* r, const double* p, const double* q,
                                const int* pan_ptr, const int64_t* pan_row, void* b16, int dtype, double* st,
                                int* ist, double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream);
/* rho = r.z (and z.q when flexible) -> beta; for preconditioners that write z
 * themselves (generic path). q may be NULL on the first iteration. */
int ddx_pcg_dots_rz(int64_t n, int R, const double* r, const double* z, const double* q, double* st,
                    int* ist, double* partials, unsigned int* tickets, ddx_stream_t stream);
/* out[j] = x_j . y_j for R right-hand sides in (n, R) layout, with the same
 * deterministic two-stage reduction as ddx_pcg_dots_rz, but without any
 * caller-provided scratch: for callers that cannot allocate device memory
 * when they need the product (through a C FFI with no device allocator, in
 * loops that must not allocate after start-up).
 * No counterpart in the reference. The scratch lives in a fixed array inside
 * the library (~296 KiB, held by every GPU that loads it until exit), which
 * limits R to at most 64 (R a power of two); larger R is rejected with
 * DDX_ERR_ARG. The first call on a device looks the array up
 * (cudaGetSymbolAddress) with that device current and keeps the address for
 * the rest of the process; make that first call before any stream capture.
 * A device reset (cudaDeviceReset) unloads the array, so after one the
 * process must restart before calling this again. All calls share the array:
 * calls that can run
 * at the same time on the GPU (other streams, other host threads) race and
 * must be serialised by the caller. Allocates nothing (no cudaMalloc or
 * cudaFree); it clears the array's ticket with cudaMemsetAsync on `stream`. */
int ddx_dot_noalloc(int64_t n, int R, const double* x, const double* y, double* out, ddx_stream_t stream);

/* ---- Sparse matrix-vector products --------------------------------------
 * Replace FastBSR.__matmul__ (src/dd_solvers/dd_solvers/bsr.py:24-25, RPT-I
 * kernel 40-76) and torch's CSR matvec (solvers.py:264, 880).
 *
 * SELL-32 (R = 1): slice s holds rows [32s, 32s+32); entry j of row 32s+l is
 * at slice_ptr[s] + 32*j + l (padding: value 0, column = own row).
 * mode: 0 y = A x
 *       1 y = A x, then p.q -> alpha (x is p, y is q; PCG step)
 *       2 y = b - A x, then ||b||, ||y|| -> tolerance and active flags (PCG start)
 *       3 y = b - A x, then ||y|| -> stop test (residual replacement)
 */
enum { DDX_SPMV_PLAIN = 0, DDX_SPMV_PQ = 1, DDX_SPMV_RES_INIT = 2, DDX_SPMV_RES_REPLACE = 3 };
int ddx_spmv_sell_f64(int64_t n, int64_t nslices, const int64_t* slice_ptr, const int* slice_width,
                      const int* cols, const double* vals, const double* x, double* y,
                      const double* b, int mode, double* st, int* ist, double* hist,
                      double* partials, unsigned int* tickets, ddx_stream_t stream);
/* CSR, R right-hand sides in (n, R) layout (R threads per row). Same modes. */
int ddx_spmv_csr_f64(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                     const double* x, double* y, const double* b, int mode, double* st, int* ist,
                     double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream);
/* The CSR SpMM for R in {2, 4, ..., 64} with a row work order: order is a
 * permutation of the rows cut into clusters of `chunk` rows (ddx_row_clusters;
 * chunk a multiple of 256 / (R/2)), and one CTA computes a whole cluster before
 * its next, so the x rows shared by a cluster's neighbourhood come from L2
 * once. Same modes and results as ddx_spmv_csr_f64 up to the summation order
 * of the fused dot products. Replaces, for a block of right-hand sides,
 * FastBSR's y = A x (src/dd_solvers/dd_solvers/bsr.py:40-76). */
int ddx_spmv_csr_ordered_f64(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                             const int* order, int chunk, const double* x, double* y, const double* b, int mode,
                             double* st, int* ist, double* hist, double* partials, unsigned int* tickets,
                             ddx_stream_t stream);
/* Host: the row order of ddx_spmv_csr_ordered_f64 from the matrix pattern
 * (CSR indptr / indices, symmetric): greedy breadth-first clusters of
 * `cluster` rows, each cluster ascending (order: n ints). No counterpart in
 * the reference, whose SpMV walks the rows in order. */
int ddx_row_clusters(int64_t n, const int64_t* indptr, const int64_t* indices, int cluster, int* order);
/* CSR with long rows, one CTA per row, deterministic block reduction:
 * y[row, j] = sum_k vals[k] x[cols[k], j] (coarse restriction A_R y or R0 r). */
int ddx_spmv_csr_rowblock_f64(int64_t n_rows, int R, const int* row_ptr, const int* cols,
                              const double* vals, const double* x, double* y, ddx_stream_t stream);
/* CSR, R = 1, `lanes` (4, 8, 16 or 32) lanes per row summed by a fixed xor
 * tree: rows of moderate length, e.g. the coarse restriction A_R y when the
 * coarse aggregates are small (the caller picks lanes from the mean row
 * length). */
int ddx_spmv_csr_lanes_f64(int64_t n_rows, int lanes, const int* row_ptr, const int* cols, const double* vals,
                           const double* x, double* y, ddx_stream_t stream);
/* ddx_spmv_csr_rowblock_f64 (R in {2, 4, ..., 64}) with x given as the sum of
 * local products through the transpose map:
 *   x[d, j] = sum_{t in [dof_ptr[d], dof_ptr[d+1])} ylocal[dof_src[t], j]
 * (dof_ptr = dof_src = NULL: x = ylocal), ylocal F64 or F32 (acc_dtype), each
 * x value summed in FP64 from 0.0 in ascending t, exactly as
 * ddx_schwarz_combine sums it. The result equals the product with the
 * materialised x bit for bit; the vector is never written. Replaces, for a
 * block of right-hand sides, HybridSchwarz.solve's y = sum_i R_i^T y_i
 * followed by A_R y (src/dd_solvers/dd_solvers/solvers.py:878-884). */
int ddx_spmv_csr_rowblock_mapped(int64_t n_rows, int R, const int* row_ptr, const int* cols, const double* vals,
                                 const int* dof_ptr, const int* dof_src, const void* ylocal, int acc_dtype,
                                 double* y, ddx_stream_t stream);
/* Same with x in x_dtype (DDX_F64 or DDX_F32, widened to FP64 on load): the
 * hybrid restriction A_R y reads the FP32 local products directly when the
 * subdomains are the reference's contiguous non-overlapping blocks. */
int ddx_spmv_csr_lanes(int64_t n_rows, int lanes, const int* row_ptr, const int* cols, const double* vals,
                       const void* x, int x_dtype, double* y, ddx_stream_t stream);
/* BSR, block size bs (1..24: DG P1..P5 triangles have 3..21 DOFs per
 * element), blocks column-major (bs, bs) as produced by the reference's
 * csr_to_bsr (src/dd_solvers/cpp/cusparse.cpp:22-107); dtype F64 or F32 for
 * vals/x/y. Replaces FastBSR's RPT-I kernel (src/dd_solvers/dd_solvers/bsr.py:40-76):
 * one lane per scalar row, floor(32 / bs) block rows per warp. */
int ddx_spmv_bsr(int64_t n_block_rows, int bs, const int* row_ptr, const int* cols, const void* vals,
                 const void* x, void* y, int dtype, ddx_stream_t stream);
/* PCG epilogue of a product computed by ddx_spmv_bsr (R = 1, F64), for the
 * CG(bsr_matmul=True) path on DG block matrices (src/dd_solvers/dd_solvers/
 * solvers.py:243-268 with the FastBSR product of bsr.py:24-25): y already holds
 * A v. mode 1: x = p, y = q, p.q -> alpha; mode 2/3: y = b - y, then the norms
 * and the stop test of ddx_spmv_sell_f64's modes 2/3. Same state, partials and
 * ticket as ddx_spmv_sell_f64. */
int ddx_spmv_epilogue_f64(int64_t n, const double* x, double* y, const double* b, int mode, double* st, int* ist,
                          double* hist, double* partials, unsigned int* tickets, ddx_stream_t stream);
/* ---- Batched GEMV (reference op) ----------------------------------------
 * Replaces dd_solvers_gemv::gemv_strided_batched
 * (src/dd_solvers/cpp/gemv.cpp:9-53, kernels gemv_kernels.cu:31-139):
 * out[b] = M_b v_b, M (N, k, k) column-major in mat_dtype, v/out (N, k) in
 * vec_dtype (F32/F64); matrix entries are converted to the vector type and
 * accumulated in it. mat F64 with vec F32 is rejected as in the reference. */
int ddx_gemv_strided_batched(int64_t N, int k, const void* mat, int mat_dtype, const void* vec,
                             void* out, int vec_dtype, ddx_stream_t stream);

/* ---- Schwarz preconditioner ---------------------------------------------
 * Replace AdditiveSchwarz.solve (solvers.py:811-826), HybridSchwarz.solve /
 * T0 (861-888) and Inv.solve (355-359).
 *
 * Subdomain i has k_i = sub_ptr[i+1] - sub_ptr[i] DOFs sub_idx[sub_ptr[i]..].
 * Its inverse block is stored column-major with leading dimension
 * ld_i = round_up(k_i, 16 / sizeof(block element)) at element offset
 * blk_off[i] (16-byte aligned); entry (row, col) at blk_off[i] + col*ld_i + row.
 * Low-precision blocks carry a per-block scale: A_i^{-1} ~= scale[i] * Q_i.
 * `order` lists subdomains by decreasing k (work distribution).
 *
 * local_apply: ylocal[sub_ptr[i] + t, j] = scale[i] * sum_c Q_i[t, c] r[sub_idx[sub_ptr[i]+c], j]
 *   blocks are streamed through shared memory by bulk asynchronous copies
 *   (TMA engine); accumulation in FP32 for F32/BF16/F16 blocks, FP64 for F64.
 *   ylocal has element type acc (F32 or F64) and layout (sum k_i, R).
 */
/* Same with explicit tuning knobs (setup-time autotuner): `groups` consumer
 * groups of four warps split each block's columns (1, 2 or 4; 0 = default 2)
 * and `stage_kb` KiB per shared-memory ring stage (0 = default 20). */
int ddx_schwarz_local_apply_ex(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                               const int* order, const int64_t* blk_off, const void* blocks,
                               int block_dtype, const float* scale, int kmax, const double* r,
                               void* ylocal, int acc_dtype, const int* ist, int groups, int stage_kb,
                               ddx_stream_t stream);
int ddx_schwarz_local_apply(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                            const int* order, const int64_t* blk_off, const void* blocks,
                            int block_dtype, const float* scale, int kmax, const double* r,
                            void* ylocal, int acc_dtype, const int* ist, ddx_stream_t stream);
/* Same product and block layout for small subdomains (the reference's DG
 * layouts: equal blocks of a few to a few dozen DOFs), one thread per output
 * entry (equal subdomains: a thread per 16 bytes of block rows). rows =
 * sub_ptr[n_sub]; k_equal > 0 declares every subdomain to have k_equal DOFs
 * (k_equal * n_sub == rows), otherwise each row finds its subdomain by binary
 * search in sub_ptr. Blocks and every block start 16-byte aligned. Any R >= 1. */
int ddx_schwarz_local_apply_small(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                  const int64_t* blk_off, const void* blocks, int block_dtype,
                                  const float* scale, int kmax, int k_equal, int64_t rows, const double* r,
                                  void* ylocal, int acc_dtype, const int* ist, ddx_stream_t stream);
/* Same product for blocks stored as upper-triangle tiles (half the bytes):
 * Q_i exactly symmetric, only its 32 x 32 tiles (I, J), I <= J, kept, in
 * row-major order of (I, J) from element blk_off[i] (16-byte aligned); each
 * tile row-major, 32 elements per row, the 16-byte chunk c of row t stored at
 * chunk c ^ ((t >> 1) & 3) for 16-bit types and c ^ (t & 7) for FP32/FP64;
 * zero beyond k. Tile (I, J) adds T x_J to rows I and, for I < J, T^T x_I to
 * rows J. `warps` (4, 8 or 16; 0 = 8) consumer warps per CTA, `stage_kb`
 * (0 = 16) KiB per shared-memory stage: run-time choices for the autotuner.
 * `parts` (1..64) splits each block's tiles into that many contiguous ranges,
 * processed by different CTAs (for few, large blocks); part s writes its
 * partial product to ylocal slice s, at element offset s * sub_ptr[n_sub] * R,
 * and the caller adds the slices (ddx_schwarz_combine with a transpose map
 * listing every slice). Accumulation and output types as
 * ddx_schwarz_local_apply_ex. No counterpart
 * in the reference, whose inverse blocks are stored in full
 * (src/dd_solvers/dd_solvers/solvers.py:343-359). */
int ddx_schwarz_local_apply_sym(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                                const int* order, const int64_t* blk_off, const void* blocks,
                                int block_dtype, const float* scale, int kmax, const double* r,
                                void* ylocal, int acc_dtype, const int* ist, int warps, int stage_kb,
                                int parts, ddx_stream_t stream);
/* Tensor-core variant for R in {16, 32, 64} right-hand sides and BF16/FP16
 * blocks: Y_i = Q_i X_i as tcgen05.mma (M = 128, N = R, K = 16, FP32
 * accumulators in TMEM). `tiles` holds each block cut into 128-row x 64-column
 * tiles in the K-major 128-byte-swizzled shared-memory layout (row r of a tile
 * at byte 128 r, its 16-byte chunk c stored at chunk c ^ (r % 8)), row-tile
 * major, the last row tile truncated to a multiple of 8 rows, columns >= k
 * zero; subdomain i starts at byte tile_off[i]. X_i comes from b16 at byte
 * panel_off[i], written by ddx_pack_panels16 (same st, same terms). With
 * terms = 2 every K step multiplies the tile by both residual terms into one
 * FP32 accumulator, so the product sees r to about twice the 16-bit precision
 * (needed when the local blocks are ill conditioned; the block stream is read
 * once either way). ylocal is FP32, (sum k_i, R). Needs 66 KB + terms *
 * ceil(kmax / 64) * R * 128 bytes of shared memory (<= 227 KB). */
int ddx_schwarz_local_apply_tc(int n_sub, int R, const int64_t* sub_ptr, const int* order,
                               const int64_t* tile_off, const void* tiles, int block_dtype,
                               const float* scale, int kmax, const void* b16, const int64_t* panel_off,
                               int terms, float* ylocal, const int* ist, const double* st,
                               ddx_stream_t stream);
/* Tensor-core apply for symmetric blocks stored as upper-triangle 128 x 128
 * tiles: tiles (I, J), I <= J, of Q_i in row-major order of (I, J) from byte
 * tile_off[i] (16-byte aligned), each as two 128 x 64 halves (tile
 * columns 0-63, then 64-127) in the K-major 128-byte-swizzled layout of
 * ddx_schwarz_local_apply_tc, zero beyond k_i: 32 KB per tile, about 56% of
 * the full block at k ~ 2000. Each tile is multiplied twice: D_I += T X_J and,
 * for I < J, D_J += T^T X_I (the same shared memory read as an MN-major
 * operand). The B panel of a block arrives in 128-row chunks, each with its
 * own barrier: the first MMA waits for chunk 0 only, and chunk I is released
 * for the next block once tile row I is done. Needs nt = ceil(kmax / 128) row
 * tiles with nt * R <= 512 and nt <= 24 (all row-tile accumulators of a block
 * in TMEM) and 3 KB + S * 32 KB + terms * 2 nt * 64 * 2R bytes of shared
 * memory (<= 227 KB) for a ring of S >= 2 tile stages; the deepest ring that
 * fits (at most 6) is used. Other arguments as ddx_schwarz_local_apply_tc.
 * No counterpart in the reference (full inverse blocks,
 * src/dd_solvers/dd_solvers/solvers.py:343-359). */
int ddx_schwarz_local_apply_tc_sym(int n_sub, int R, const int64_t* sub_ptr, const int* order,
                                   const int64_t* tile_off, const void* tiles, int block_dtype,
                                   const float* scale, int kmax, const void* b16, const int64_t* panel_off,
                                   int terms, float* ylocal, const int* ist, const double* st,
                                   ddx_stream_t stream);
/* ddx_schwarz_local_apply_tc_sym with the ring depth chosen by the caller
 * (stages in 2..6, clamped to the deepest ring that fits; 0 = deepest), for an
 * autotuner. Same results for every depth (the summation order does not
 * depend on it). No counterpart in the reference. */
int ddx_schwarz_local_apply_tc_sym_ex(int n_sub, int R, const int64_t* sub_ptr, const int* order,
                                      const int64_t* tile_off, const void* tiles, int block_dtype,
                                      const float* scale, int kmax, const void* b16, const int64_t* panel_off,
                                      int terms, float* ylocal, const int* ist, const double* st, int stages,
                                      ddx_stream_t stream);
/* Gathers and packs the tensor-core B panels X_i = r[idx_i, :] (r FP64, (n, R),
 * R in {16, 32, 64}) to 16-bit dtype (BF16 or F16). Subdomain i (k_i DOFs,
 * P_i = 2 ceil(k_i / 128) chunks of 64 rows) occupies terms * P_i * 64 * 2R
 * bytes at byte panel_off[i] (16-byte aligned), term-major; within a term, panel row c is DOF
 * sub_idx[sub_ptr[i] + c], its 16-byte chunk q (RHS 8q..8q+7) stored at byte
 * c * 2R + 16 q with bits [4,7) XORed by bits [7,10) masked to the row width
 * (the MN-major swizzle of the UMMA B operand). Term 0 = (dtype) (s_j r[d, j]);
 * for terms = 2, term 1 = (dtype) (s_j r[d, j] - term 0). s_j is a power of two
 * from st (||r_j||^2 slot; 1 when st is NULL) putting ||s_j r_j|| just below
 * 2^14 for F16 and 1 for BF16, so residual entries stay in the normal 16-bit
 * range as the solve converges; the tensor-core apply divides s_j out again.
 * Rows k_i..64 P_i - 1 are not written: zero them once. */
int ddx_pack_panels16(int n_sub, int R, const int64_t* sub_ptr, const int* sub_idx,
                      const int64_t* panel_off, const double* r, const double* st, void* b16,
                      int dtype, int terms, ddx_stream_t stream);
/* combine: z[d, j] = sum_{t in T(d)} ylocal[src[t], j]      (if ylocal)
 *                  + u[d, j]                                (if u)
 *                  + sign * sum_c P[d, c] yc[c, j]          (if p_ptr)
 * where T(d) = dof_ptr[d]..dof_ptr[d+1] lists the positions of DOF d in the
 * subdomain-major ylocal (ascending subdomain order, so the sum order is
 * fixed). With dots != 0 it also forms rho = r.z (and z.q when flexible) and
 * beta on the device. u may alias z. Shortcuts for the reference's own layout
 * (equal contiguous non-overlapping subdomains, P0 coarse aggregates):
 * dof_ptr == NULL with ylocal means the identity map (ylocal is DOF-ordered);
 * p_ptr == NULL with p_col means P has one unit entry per DOF, in column
 * p_col[d] (p_val unused). z = NULL (R >= 2, dots != 0): z is only reduced,
 * not stored; ddx_schwarz_combine_update recomputes it where p needs it. */
int ddx_schwarz_combine(int64_t n, int R, const int* dof_ptr, const int* dof_src, const void* ylocal,
                        int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                        const double* p_val, const double* yc, double sign, double* z, int dots,
                        const double* r, const double* q, double* st, int* ist, double* partials,
                        unsigned int* tickets, ddx_stream_t stream);
/* ddx_schwarz_combine with dof_first (may be NULL): per DOF its only position
 * in ylocal (>= 0), -1 when it has none, -2 when it has several. A DOF in one
 * subdomain then costs two dependent loads (dof_first, ylocal) instead of
 * three (dof_ptr, dof_src, ylocal); the transpose map is still read for the
 * others. Same sums in the same order. Used for R >= 2 (R = 1 reads the map). */
int ddx_schwarz_combine_ex(int64_t n, int R, const int* dof_ptr, const int* dof_src, const int* dof_first,
                           const void* ylocal, int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                           const double* p_val, const double* yc, double sign, double* z, int dots,
                           const double* r, const double* q, double* st, int* ist, double* partials,
                           unsigned int* tickets, ddx_stream_t stream);
/* The PCG direction update on a z that was reduced but not stored (R >= 2):
 * recomputes z exactly as ddx_schwarz_combine_ex does from the same inputs (same
 * operations in the same order, so the same bits), then x += alpha_x p (x may
 * be NULL; see ddx_pcg_update_px) and p = z + beta p. Instead of writing z and
 * reading it back, the local products and the coarse correction are read a
 * second time; fewer bytes when the prolongation is P0 (or absent). Replaces
 * HybridSchwarz.solve's output (solvers.py:885-888) followed by CG.solve's
 * fused_mul_add (solvers.py:267). */
int ddx_schwarz_combine_update(int64_t n, int R, const int* dof_ptr, const int* dof_src, const int* dof_first,
                               const void* ylocal, int acc_dtype, const double* u, const int* p_ptr, const int* p_col,
                               const double* p_val, const double* yc, double sign, double* x, double* p,
                               const double* st, const int* ist, ddx_stream_t stream);
/* Hybrid restriction for a block of R in {2, 4, ..., 64} right-hand sides,
 * computed per subdomain from the local products instead of from y:
 *   w = A_R y = sum_i (A_R R_i^T) y_i.
 * The coarse rows c with A_R[c, idx_i] != 0 are subdomain i's slots
 * 0..n_slots[i]-1 (ascending c, at most 16), the pairs q = slot_base[i] + slot
 * ascending in (i, c). Row p of the subdomain-major ylocal (F64 or F32,
 * acc_dtype) carries its entries (slot, A_R[c, sub_idx[p]]) in ascending slot:
 * the first two as f_slot[2p + e] (255: none; 2-byte aligned) and f_val[2p + e]
 * (16-byte aligned), e = 0, 1, the others in [ov_ptr[p], ov_ptr[p+1]) of
 * ov_slot / ov_val. With slices > 1 (a local apply
 * that splits blocks into parts), ylocal holds `slices` slices of slice_rows =
 * sub_ptr[n_sub] rows each, subdomain i's rows of slice s at s * slice_rows +
 * [sub_ptr[i], sub_ptr[i+1]), and the entry arrays cover all of them (every
 * slice carrying the same entries). Pass 1 streams each subdomain's rows once
 * and writes partial[q, :] (n_pairs x R FP64 scratch, 16-byte aligned) in a
 * fixed order; pass 2 sums, for each coarse row c, the partials of its pairs
 * listed in sum_pair[sum_ptr[c] .. sum_ptr[c+1]) in that order into w[c, :].
 * Deterministic (a fixed summation order, not that of
 * ddx_spmv_csr_rowblock_mapped, so the last bits can differ from it). Skipped
 * when ist says no column is active. Replaces, for a block of right-hand
 * sides, HybridSchwarz.solve's y = sum_i R_i^T y_i followed by A_R y
 * (src/dd_solvers/dd_solvers/solvers.py:878-884). */
int ddx_schwarz_restrict_sub(int n_sub, int64_t n_pairs, int64_t n_coarse, int R, const int64_t* sub_ptr,
                             const int* slot_base, const int* n_slots, const unsigned char* f_slot,
                             const double* f_val, const int* ov_ptr, const unsigned char* ov_slot,
                             const double* ov_val, const void* ylocal, int acc_dtype, int slices, int64_t slice_rows,
                             const int* sum_ptr, const int* sum_pair, double* partial, double* w, const int* ist,
                             ddx_stream_t stream);
/* Dense coarse solve with the explicit FP64 inverse (row-major, symmetric):
 * yc[c, j] = sum_d Ainv[c, d] w[d, j]. */
int ddx_coarse_gemv_f64(int n_c, int R, const double* Ainv, const double* w, double* yc,
                        const int* ist, ddx_stream_t stream);
/* The same for R in {16, 32, 64} as a tiled FP64 GEMM that reads Ainv once
 * per call (ddx_coarse_gemv_f64 reads it once per 16 columns). scratch (16-byte
 * aligned, scratch_len doubles, may be NULL / 0) lets the reduction over
 * Ainv's columns be split into up to scratch_len / (n_c R) ranges, summed in a
 * fixed order by a second pass, so that a coarse space of a few thousand rows
 * still fills the GPU; results differ from ddx_coarse_gemv_f64 in the last
 * bits (another summation order) but not from run to run. Replaces
 * CudssSolver.solve (src/dd_solvers/cpp/cudss.cpp:98-101) for a block of
 * right-hand sides. */
int ddx_coarse_gemm_f64(int n_c, int R, const double* Ainv, const double* w, double* yc, double* scratch,
                        int64_t scratch_len, const int* ist, ddx_stream_t stream);

/* ---- Sparse coarse solve (cuDSS replacement for large coarse spaces) ------
 * Replaces cudssExecute(FACTORIZATION / SOLVE) behind CudssSolver
 * (src/dd_solvers/cpp/cudss.cpp:64-105, called from solvers.py:85-113) when
 * the coarse matrix is too large for a dense inverse.
 *
 * ddx_nd_order (host memory, host computation): nested-dissection ordering of
 * the symmetric pattern (indptr, indices) of an n x n matrix by recursive BFS
 * level-set bisection down to leaves of at most `leaf` vertices. Writes the
 * separator tree in post-order: node t eliminates perm[node_first[t] ..
 * node_first[t+1]), its parent is node_parent[t] (-1 for a root); *n_nodes
 * receives the node count. perm holds n entries; node_first and node_parent
 * need room for n + 1 entries. The halves below large separators are ordered
 * on host threads (the environment variable DDX_ND_THREADS caps them, default
 * the host's hardware threads); the output is the same for any thread count. */
int ddx_nd_order(int64_t n, const int64_t* indptr, const int64_t* indices, int leaf, int64_t* perm,
                 int64_t* node_first, int64_t* node_parent, int64_t* n_nodes);

/* ddx_nd_update_sets (host memory, host computation): the symbolic update
 * sets of the separator tree, the analysis step of the same cuDSS
 * replacement. Positions are elimination-order positions (0 .. n-1); front t
 * eliminates positions s_first[t] .. s_first[t]+s_size[t]-1, fronts in
 * post-order (parent[t] > t, or -1). p_ptr/p_pos hold, for every position,
 * the positions of its matrix row's entries (n+1 pointers). U_t = the
 * positions after front t's separator that its rows or its children's update
 * sets reach, sorted and distinct, written to u_pos[u_ptr[t] .. u_ptr[t+1])
 * (u_ptr: n_fronts+1 entries). *u_total receives the total; if it exceeds
 * capacity the call returns DDX_ERR_ARG and writes no u_pos (call again with
 * capacity >= *u_total). */
int ddx_nd_update_sets(int64_t n, int64_t n_fronts, const int64_t* s_first, const int64_t* s_size,
                       const int64_t* p_ptr, const int64_t* p_pos, const int64_t* parent, int64_t* u_ptr,
                       int64_t* u_pos, int64_t capacity, int64_t* u_total);

/* Multifrontal solve plan. Front t owns the (s_t + u_t) coarse indices
 * fidx[idx_off[t] ...] (its separator, then its update set) and the operator
 * G[g_off[t] ...] = [chol(F_SS)^-1; F_US F_SS^-1] ((s_t+u_t) x s_t, row-major),
 * with its transpose at GT[g_off[t] ...] (s_t x (s_t+u_t), row-major).
 * Its update vector lives at upd[upd_off[t] ...] (u_t rows of R values).
 * gptr/gsrc list, for every front position (idx_off numbering), the update
 * rows of its children to add, in a fixed order. Work items are int triples
 * (front, first row of G_t / of G_t^T, count); fwd_level_ptr / bwd_level_ptr (HOST
 * arrays, n_levels + 1 entries) delimit the items of each level (leaves first
 * for the forward sweep, root first for the backward sweep), and
 * fwd_level_smax / bwd_level_mmax (HOST) give each level's largest s and
 * s + u. All other pointers are device memory. */
typedef struct ddx_nd_plan {
  int n;
  int n_fronts;
  int n_levels;
  int max_front;
  const int64_t* fwd_level_ptr;
  const int64_t* bwd_level_ptr;
  const int* fwd_level_smax;
  const int* bwd_level_mmax;
  const int* fwd_items;
  const int* bwd_items;
  const int* front_s;
  const int* front_u;
  const int64_t* g_off;
  const int64_t* idx_off;
  const int64_t* upd_off;
  const int* fidx;
  const int64_t* gptr;
  const int64_t* gsrc;
  const double* G;
  const double* GT;
  const int64_t* s_first; /* elimination position of front t's first separator vertex */
  const int* fpos;        /* elimination position of every front position (idx_off numbering) */
  const int64_t* gat_level_ptr; /* host, n_levels+1: gather items of each forward level (NULL: none) */
  const int* gat_items;         /* (front, first position, positions) per gather item */
  const int64_t* fwd_level_gmax; /* host, n_levels: largest operator range of a forward item, bytes
                                    (NULL: no staging in shared memory) */
  const int64_t* bwd_level_gmax; /* host, n_levels: the same for the backward items, root level first;
                                    a negative entry leaves that level's operator in global memory */
  int release_early;             /* 1: each level's kernel lets the next one launch right after its wait */
} ddx_nd_plan;

/* x = A^-1 w for w, x of shape (n, R) (DOF-major, FP64). y and xe (n*R
 * doubles each: the forward result and the solution in elimination order),
 * upd (sum_t u_t * R doubles) and fb (sum_t (s_t+u_t) * R doubles: the
 * assembled front vectors of the levels that have gather items; NULL gathers
 * inside the forward items instead, same results) are caller-owned scratch.
 * With ist (PCG state), nothing runs once every right-hand side has
 * converged. Deterministic. */
int ddx_coarse_solve_nd(const ddx_nd_plan* plan, int R, const double* w, double* x, double* y, double* xe,
                        double* upd, double* fb, const int* ist, ddx_stream_t stream);

/* ---- Differentiable solve -----------------------------------------------
 * No counterpart in the reference (it has no autograd). Per-cell coefficient
 * gradient of a Q1 diffusion solve on a uniform n_el^dim grid:
 * grad[e] = -h^(dim-2) lambda_e^T K_ref u_e, with u and lambda on the
 * x-fastest interior nodes (zero on the Dirichlet boundary), kref the
 * (2^dim)^2 unit-cell stiffness (device memory, row-major, local node bit d =
 * offset along axis d), cells numbered x fastest. */
int ddx_elem_grad_q1(int dim, int n_el, const double* u, const double* lam, const double* kref,
                     double* grad, ddx_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* DDX_H */
