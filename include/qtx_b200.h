/*
 * qtx_b200.h -- C ABI of the B200 (sm_100a) NEGF hot-path library
 * (libqtx_b200.so).
 *
 * The library replaces the per-energy hot path of the quatrex/qttools
 * Python package: the block-tridiagonal RGF selected inversion and
 * selected solve, the Sancho-Rubio open-boundary surface Green's function,
 * and the transmission / density reductions. The reference has no foreign
 * function interface of its own (it is NumPy/CuPy Python); each entry point
 * below names the Python routine whose work it performs, and a ctypes
 * binding (quatrex_b200/_native.py) calls it from a GFSolver / OBCSolver
 * subclass with the same Python signature as the reference.
 *
 * Conventions
 *  - Complex numbers are interleaved (re, im): complex128 = 2 x double,
 *    complex64 = 2 x float (numpy / CuPy / torch layout).
 *  - Every matrix argument is a strided stack of dense row-major matrices in
 *    device memory (qtx_mat): element (b, r, c) lives at
 *    ptr + b * stride + r * ld + c (in complex elements). A qtx_mat with a
 *    NULL ptr is an all-zero input block, or an output that is not written.
 *  - A block-tridiagonal stack (qtx_bt) lists its diagonal blocks (i, i),
 *    upper blocks (i, i+1) and lower blocks (i+1, i) in HOST arrays of
 *    qtx_mat; block sizes are a host array.
 *  - All work is enqueued on the given CUDA stream; no call synchronises the
 *    host unless stated. Calls return QTX_OK (0) or a negative error code;
 *    qtx_last_error() describes the last failure of the calling thread.
 *  - Scratch memory is supplied by the caller (workspace pointer + size);
 *    the *_workspace_size functions give the required size in bytes.
 *  - Calls on different streams with disjoint buffers and workspaces are
 *    independent; the library's mutable state is the thread-local error
 *    string, the thread-local GEMM path (qtx_set_gemm_path), the inverse
 *    path knob and the launch profiler.
 */
#ifndef QTX_B200_H
#define QTX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* qtx_stream; /* == cudaStream_t */

enum qtx_status {
  QTX_OK = 0,
  QTX_ERR_ARG = -1,       /* invalid argument / shape */
  QTX_ERR_CUDA = -2,      /* CUDA runtime error */
  QTX_ERR_WORKSPACE = -3, /* workspace too small */
  QTX_ERR_SINGULAR = -4,  /* a block had a zero pivot (see info arrays) */
  QTX_ERR_UNSUPPORTED = -5
};

enum qtx_dtype { QTX_C128 = 0, QTX_C64 = 1 };

typedef struct qtx_mat {
  void* ptr;      /* device pointer to element (0, 0) of stack entry 0 */
  int64_t ld;     /* row stride, complex elements */
  int64_t stride; /* stack stride, complex elements */
} qtx_mat;

typedef struct qtx_bt {
  int32_t num_blocks;
  const int32_t* block_sizes; /* host, num_blocks entries */
  const qtx_mat* diag;        /* host, num_blocks entries: block (i, i) */
  const qtx_mat* upper;       /* host, num_blocks-1 entries: block (i, i+1) */
  const qtx_mat* lower;       /* host, num_blocks-1 entries: block (i+1, i) */
} qtx_bt;

/* Flags of qtx_selected_solve. */
#define QTX_SOLVE_SYMMETRIC_OUT 1 /* X^<, X^> lower blocks are not written
                                     (qttools out.symmetry, rgf.py:358-359) */

/* Library version, e.g. 100 for 0.1.0. */
int qtx_version(void);

/* Message describing the last error returned on this thread. */
const char* qtx_last_error(void);

/* Batched complex128 GEMM, C = alpha op(A) op(B) + beta op(D)
 * (op: 0 = none, 1 = conjugate transpose; D may be NULL). Building block
 * of every `@` of qttools/greens_function_solver/rgf.py:71-110,234-428
 * and boundary_conditions/obc/sancho_rubio.py:64-71. */
int qtx_zgemm_batched(int m, int n, int k, int64_t batch, double alpha_re, double alpha_im,
                      qtx_mat a, int op_a, qtx_mat b, int op_b, double beta_re, double beta_im,
                      qtx_mat d, int op_d, qtx_mat c, qtx_stream stream);

/* Grouped form of qtx_zgemm_batched: entry b reads op(A) at a_ptrs[b],
 * op(B) at b_ptrs[b], D at d_ptrs[b] (NULL table: no addend) and writes C at
 * c_ptrs[b]; row strides lda, ldb, ldd, ldc are shared. The tables are
 * device arrays of `batch` device pointers, each 16-byte aligned; entries may
 * share operands (a broadcast block) and D may equal C (accumulation).
 * k > 0; always the FP64 DMMA products. The batched block products of the
 * reference's bd_matmul / bd_sandwich (qttools/datastructures/
 * routines.py:8-102,354-467) in one launch per band. */
int qtx_zgemm_grouped(int m, int n, int k, int64_t batch, double alpha_re, double alpha_im,
                      const void* const* a_ptrs, int64_t lda, int op_a, const void* const* b_ptrs, int64_t ldb,
                      int op_b, double beta_re, double beta_im, const void* const* d_ptrs, int64_t ldd, int op_d,
                      void* const* c_ptrs, int64_t ldc, qtx_stream stream);

/* Batched complex64 GEMM on the tcgen05 tensor cores, split-TF32 products
 * with FP32 accumulation (mixed precision path):
 * C = alpha op(A) op(B) + beta op(D), complex64 interleaved. err: optional
 * device int set to 1 if an internal wait timed out. */
int qtx_cgemm_batched(int m, int n, int k, int64_t batch, float alpha_re, float alpha_im, qtx_mat a,
                      int op_a, qtx_mat b, int op_b, float beta_re, float beta_im, qtx_mat d,
                      int op_d, qtx_mat c, int* err, qtx_stream stream);

/* Batched complex128 GEMM emulated on the int8 tcgen05 tensor cores,
 * C = alpha op(A) op(B) + beta op(D) as qtx_zgemm_batched. Each operand is
 * split into `slices` (3-8) int8 planes of balanced base-256 digits under a
 * power-of-two scale per row of op(A) / column of op(B); digit pairs are
 * multiplied exactly (int32 tensor-core sums) and combined in FP64
 * (Ozaki-style splitting). Error per element below
 * 2 slices k 2^(4 - 8 slices) max_l|op(A)_il| max_l|op(B)_lj|: ~1e-12 relative
 * at 6 slices, FP64 level at 7. Requires slices * 2k * 2^14 < 2^31.
 * workspace: qtx_zgemm_emulated_workspace bytes for the whole batch; less
 * processes the batch in chunks (too little for one entry is an error).
 * No reference counterpart: a faster evaluation of the same products. */
size_t qtx_zgemm_emulated_workspace(int m, int n, int k, int64_t batch, int slices);
int qtx_zgemm_emulated_batched(int m, int n, int k, int64_t batch, double alpha_re, double alpha_im,
                               qtx_mat a, int op_a, qtx_mat b, int op_b, double beta_re,
                               double beta_im, qtx_mat d, int op_d, qtx_mat c, int slices,
                               void* workspace, size_t workspace_bytes, qtx_stream stream);
/* GEMM path of the CALLING THREAD for the complex128 drivers (selected
 * inversion, selected solve, Sancho-Rubio, OBC refinement, contact
 * self-energy): 0 = FP64 DMMA (default), 3-8 = the int8 emulation with that
 * many slices. With the emulated path the drivers' *_workspace functions
 * include its scratch: query them after selecting the path. */
int qtx_set_gemm_path(int slices);
int qtx_get_gemm_path(void);
/* 1 if a bounded wait inside an emulated GEMM timed out since the last call
 * (the flag is cleared), 0 if not, < 0 on error. Synchronises the device. */
int qtx_emulated_gemm_status(void);

/* Batched complex128 inverse X = A^{-1} (Gauss-Jordan, partial pivoting).
 * Replaces qttools/kernels/linalg/inv.py:6-40 (numpy.linalg.inv /
 * cupy.linalg.solve(a, I)). info: device int[batch], 0 or the 1-based
 * column of a zero pivot (may be NULL). X may equal A. */
int qtx_zinv_batched(int n, int64_t batch, qtx_mat a, qtx_mat x, int* info, qtx_stream stream);

/* Scratch bytes of qtx_zinv_batched_ws. */
size_t qtx_zinv_workspace(int n, int64_t batch);

/* qtx_zinv_batched with scratch: for large blocks and small batches the
 * inverse runs as a multi-CTA blocked Gauss-Jordan (panel factorisation,
 * row interchanges, DMMA trailing update over every SM), otherwise as one CTA
 * per matrix. Same pivot rule and info convention. The library's RGF and
 * Sancho-Rubio drivers invert through this path. Replaces the same
 * qttools/kernels/linalg/inv.py:6-40 call as qtx_zinv_batched. */
int qtx_zinv_batched_ws(int n, int64_t batch, qtx_mat a, qtx_mat x, int* info, void* workspace,
                        size_t workspace_bytes, qtx_stream stream);

/* Inverse path of every inverse in this process: 0 automatic (default),
 * 1 one CTA per matrix, 2 multi-CTA (workspace-backed calls, n > 400 in the
 * automatic choice), 3 one thread-block cluster of ceil(n / 32) CTAs per
 * matrix holding it in distributed shared memory (n <= 256; loaded with
 * TMA), 4 the one-CTA kernel as a cluster of C CTAs per matrix that split
 * its columns (n <= 400; C the largest of 2, 4, 8 leaving 32 columns per
 * CTA). Automatic: the distributed-shared-memory cluster for n <= 256 while
 * batch x ceil(n / 32) is at most half the SM count; else up to n = 400 the
 * column split with the largest C for which batch x C fits the SM count and
 * every cluster is co-resident (C = 1 at full batches); above n = 400 the
 * multi-CTA path for batches up to half the SM count. All paths use the same
 * pivot rule; paths 1 and 4 give bit-identical results. A tuning and test
 * knob; no reference counterpart. */
int qtx_set_inverse_path(int mode);
/* 1 if a bounded wait inside the cluster inverse timed out since the last
 * call (the flag is cleared; those results are invalid), 0 if not, < 0 on
 * error. Synchronises the device. */
int qtx_inverse_status(void);

/* Workspace bytes for qtx_selected_inv on this block layout and batch. */
size_t qtx_selected_inv_workspace(int32_t num_blocks, const int32_t* block_sizes, int64_t batch);

/* RGF selected inversion: diagonal and first off-diagonal blocks of
 * (A - OBC)^{-1}, qttools/greens_function_solver/rgf.py:25-113
 * (RGF.selected_inv). obc_retarded: host array of num_blocks qtx_mat
 * (NULL ptr = no boundary block on that layer), subtracted from A_ii
 * (rgf.py:71-74,83-88). x: output blocks; a NULL output block is skipped.
 * info: device int[batch] singular-pivot report (may be NULL). */
int qtx_selected_inv(const qtx_bt* a, const qtx_mat* obc_retarded, const qtx_bt* x, int64_t batch,
                     int* info, void* workspace, size_t workspace_bytes, qtx_stream stream);

/* qtx_selected_inv without a caller workspace and without any allocation:
 * its scratch is a file-scope 64 MiB device array in the library (held by
 * every GPU that loads it until exit). For callers that cannot call
 * cudaMalloc/cudaFree during a solve (both synchronise the device and fail
 * once another allocator owns the memory). Requests needing more than 64 MiB
 * (sum_i b_i^2 + 6 b_max^2 complex128 per energy) return QTX_ERR_WORKSPACE
 * before anything is enqueued or written. All calls share the array: calls
 * that overlap on the GPU race. A device's first call resolves the array's
 * device address; make it before any stream capture. It always runs the FP64
 * DMMA products (the thread's GEMM path, qtx_set_gemm_path, does not apply)
 * and only the inverses that need no scratch: one CTA per block, the same
 * kernel column-split over a thread-block cluster, or one cluster per block
 * in distributed shared memory, chosen as for qtx_zinv_batched (including
 * qtx_set_inverse_path); the multi-CTA panel inverse (mode 2, or the automatic
 * choice for blocks above 400 at small batches) is replaced by one CTA per
 * block. This entry point has no counterpart in the reference. */
int qtx_selected_inv_static(const qtx_bt* a, const qtx_mat* obc_retarded, const qtx_bt* x,
                            int64_t batch, int* info, qtx_stream stream);

/* Workspace bytes for qtx_selected_solve. */
size_t qtx_selected_solve_workspace(int32_t num_blocks, const int32_t* block_sizes, int64_t batch,
                                    int return_current);

/* RGF selected solve, qttools/greens_function_solver/rgf.py:115-438
 * (RGF.selected_solve): X^R = (A - OBC^R)^{-1} (diagonal blocks only, as in
 * the reference), X^{<,>} = X^R (Sigma^{<,>} + OBC^{<,>}) X^R^H on the
 * diagonal (anti-Hermitian part, rgf.py:305-310,362-364) and first
 * off-diagonal blocks. Only the diagonal and upper blocks of sigma_lesser /
 * sigma_greater are read (rgf.py:222-232,278,291,327-328).
 *  obc_*: host arrays of num_blocks qtx_mat (NULL ptr = none).
 *  xr: may be NULL (return_retarded=False).
 *  current: device complex128 [batch, num_blocks + 1] Meir-Wingreen layer
 *    current (rgf.py:174-181,388-428), or NULL.
 *  g0n: optional output of the corner block G^R_{0,N-1} (NULL ptr = skip),
 *    used for the Caroli transmission.
 *  density: optional device double [batch, sum(block_sizes)] receiving
 *    Im diag X^< (quatrex/core/observables.py:8-31), or NULL. */
int qtx_selected_solve(const qtx_bt* a, const qtx_bt* sigma_lesser, const qtx_bt* sigma_greater,
                       const qtx_mat* obc_retarded, const qtx_mat* obc_lesser,
                       const qtx_mat* obc_greater, const qtx_bt* xl, const qtx_bt* xg,
                       const qtx_bt* xr, void* current, qtx_mat g0n, double* density,
                       int flags, int64_t batch, int* info, void* workspace,
                       size_t workspace_bytes, qtx_stream stream);

/* Workspace bytes for qtx_selected_solve_mixed. */
size_t qtx_selected_solve_mixed_workspace(int32_t num_blocks, const int32_t* block_sizes,
                                          int64_t batch, int return_current);

/* qtx_selected_solve in mixed precision: all block stacks are
 * complex64; block products run on the tcgen05 tensor cores as split-TF32
 * products with FP32 accumulation; every Schur-complement block is inverted
 * in FP64 (upcast, Gauss-Jordan with partial pivoting, rounded back once,
 * so no Newton-Schulz refinement step is applied). The current and the
 * density are accumulated in double. g0n is complex64. The boundary
 * conditions (qtx_sancho_rubio*, qtx_obc_refine, qtx_contact_self_energy)
 * stay complex128 calls. */
int qtx_selected_solve_mixed(const qtx_bt* a, const qtx_bt* sigma_lesser,
                             const qtx_bt* sigma_greater, const qtx_mat* obc_retarded,
                             const qtx_mat* obc_lesser, const qtx_mat* obc_greater, const qtx_bt* xl,
                             const qtx_bt* xg, const qtx_bt* xr, void* current, qtx_mat g0n,
                             double* density, int flags, int64_t batch, int* info, void* workspace,
                             size_t workspace_bytes, qtx_stream stream);

/* Elementwise combination out = sum_k coef_k op_k(term_k) over an m x n
 * stack (1 to 4 terms; coefs: 2 * nterms doubles, re and im of each;
 * conj_trans: NULL or nterms flags, 1 = conjugate transpose, m == n).
 * out may alias a term read without transposition. The block additions of
 * the reference's assembly steps (e.g. quatrex/coulomb_screening/
 * solver.py:473-493, P^R = P^R_h + (P^> - P^<) / 2). */
int qtx_zcombine(int m, int n, int64_t batch, qtx_mat out, int nterms, const qtx_mat* terms,
                 const double* coefs, const int* conj_trans, qtx_stream stream);

/* Converts an m x n stack between complex128 (QTX_C128) and complex64
 * (QTX_C64), or copies it within one type. */
int qtx_convert(int m, int n, int64_t batch, qtx_mat in, int in_dtype, qtx_mat out, int out_dtype,
                qtx_stream stream);

/* Workspace bytes for qtx_sancho_rubio. */
size_t qtx_sancho_rubio_workspace(int n, int64_t batch);

/* Sancho-Rubio surface Green's function,
 * qttools/boundary_conditions/obc/sancho_rubio.py:33-85 (SanchoRubio.__call__).
 * x = inv(eps_s) after at most max_iterations decimation steps.
 *  per_energy = 0: batch-wide stop when max_b delta_b < tol
 *    (sancho_rubio.py:73-78, the reference semantics);
 *  per_energy = 1: entries stop individually once delta_b < tol.
 *  iterations: host int, iterations performed (batch-wide count).
 *  converged: host int, 1 if the stop criterion was met.
 *  delta_out: optional device double[batch], final delta per entry.
 * Synchronises the stream once per iteration to test convergence. */
int qtx_sancho_rubio(int n, int64_t batch, qtx_mat a_ii, qtx_mat a_ij, qtx_mat a_ji, qtx_mat x,
                     int max_iterations, double tol, int per_energy, int* iterations,
                     int* converged, double* delta_out, int* info, void* workspace,
                     size_t workspace_bytes, qtx_stream stream);

/* Sancho-Rubio on several systems of one block size in a single decimation
 * loop (e.g. both contacts of a device, or the leads of several devices):
 * system k has batches[k] entries with inputs a_ii[k], a_ij[k], a_ji[k] and
 * output x[k]. The systems are concatenated, so every launch covers all of
 * them. Workspace: qtx_sancho_rubio_workspace(n, sum(batches)). Stop
 * criteria as qtx_sancho_rubio over the concatenated batch; info (device,
 * optional) has sum(batches) entries in system order. */
int qtx_sancho_rubio_multi(int n, int num_systems, const int64_t* batches, const qtx_mat* a_ii,
                           const qtx_mat* a_ij, const qtx_mat* a_ji, const qtx_mat* x,
                           int max_iterations, double tol, int per_energy, int* iterations,
                           int* converged, int* info, void* workspace, size_t workspace_bytes,
                           qtx_stream stream);

/* qtx_sancho_rubio_multi without host synchronisation: exactly
 * max_iterations decimation steps are enqueued; convergence is tracked on
 * the device (per-energy or batch-wide, as per_energy selects) and retired
 * entries are skipped by every later kernel, so converged steps cost only
 * their launches. The whole sequence can be captured in a CUDA graph.
 * d_iterations / d_converged: device ints receiving the number of steps that
 * still had active entries and whether all entries met the tolerance. */
int qtx_sancho_rubio_multi_async(int n, int num_systems, const int64_t* batches,
                                 const qtx_mat* a_ii, const qtx_mat* a_ij, const qtx_mat* a_ji,
                                 const qtx_mat* x, int max_iterations, double tol, int per_energy,
                                 int* d_iterations, int* d_converged, int* info, void* workspace,
                                 size_t workspace_bytes, qtx_stream stream);

/* Workspace bytes for qtx_beyn_moments. */
size_t qtx_beyn_moments_workspace(int n, int64_t batch, int num_quad_points);

/* Moments of Beyn's contour integral for the spectral open-boundary
 * condition, qttools nevp/beyn.py:166-220 (Beyn._contour_integrate, with
 * kernels/operator.py:117-181): for T(z) = a_ji / z + a_ii + a_ij z and the
 * quadrature points z_j = r exp(2 pi i (j + 1.5) / nq), j < nq, on the
 * circles r = r_o and r = r_i, weight w = 1 / nq,
 *   q0 = sum_j w (z_o,j T(z_o,j)^-1 - z_i,j T(z_i,j)^-1),
 *   q1 = sum_j w (z_o,j^2 T(z_o,j)^-1 - z_i,j^2 T(z_i,j)^-1),
 * for every stack entry (2 nq batched n x n inverses per entry). info
 * (device int[batch], optional): 1-based index of the first singular
 * operator of the entry (outer circle first), 0 if none. */
int qtx_beyn_moments(int n, int64_t batch, qtx_mat a_ji, qtx_mat a_ii, qtx_mat a_ij, double r_o,
                     double r_i, int num_quad_points, qtx_mat q0, qtx_mat q1, int* info,
                     void* workspace, size_t workspace_bytes, qtx_stream stream);

/* Workspace bytes sufficient for qtx_lyapunov_doubling and
 * qtx_lyapunov_refine on n x n blocks. */
size_t qtx_lyapunov_workspace(int n, int64_t batch);

/* Discrete-time Lyapunov equation X = Q + A X A^H by doubling,
 * qttools boundary_conditions/lyapunov/doubling.py:36-91 (Doubling.__call__):
 * X_{k+1} = X_k + A_k X_k A_k^H, A_{k+1} = A_k A_k, stopped when every entry
 * has ||X_{k+1} - X_k||_F / ||X_{k+1}||_F < rel_tol or
 * ||X_{k+1} - X_k||_F < abs_tol. iterations / converged: host ints.
 * Synchronises the stream once per step to test the stop rule. */
int qtx_lyapunov_doubling(int n, int64_t batch, qtx_mat a, qtx_mat q, qtx_mat x, int max_iterations,
                          double rel_tol, double abs_tol, int* iterations, int* converged,
                          void* workspace, size_t workspace_bytes, qtx_stream stream);

/* One fixed-point step of the Lyapunov equation with residuals,
 * qttools boundary_conditions/lyapunov/lyapunov.py:488-579
 * (LyapunovSystem._fixed_point_step / _get_residuals):
 * x_ref = q + a x a^H, abs_res = ||x_ref - x||_F, rel_res = abs_res /
 * ||x_ref||_F (device double[batch]). x_ref may equal x. */
int qtx_lyapunov_refine(int n, int64_t batch, qtx_mat a, qtx_mat q, qtx_mat x, qtx_mat x_ref,
                        double* rel_res, double* abs_res, void* workspace, size_t workspace_bytes,
                        qtx_stream stream);

/* Workspace bytes sufficient for qtx_contact_self_energy, qtx_obc_refine
 * and qtx_transmission (square n x n blocks) on `batch` entries. */
size_t qtx_obc_workspace(int n, int64_t batch);

/* Boundary self-energies of one contact from its surface Green's function
 * (quatrex/electron/solver.py:483-489):
 *   sigma   = a_ji g a_ij
 *   lesser  = i f Gamma,  greater = i (f - 1) Gamma,  Gamma = i (sigma - sigma^H)
 * occupancies: device double[batch]. Any output may have a NULL ptr. */
int qtx_contact_self_energy(int n, int64_t batch, qtx_mat a_ij, qtx_mat a_ji, qtx_mat g,
                            const double* occupancies, qtx_mat sigma, qtx_mat sigma_lesser,
                            qtx_mat sigma_greater, void* workspace, size_t workspace_bytes,
                            qtx_stream stream);

/* One fixed-point refinement step with residuals
 * (qttools/boundary_conditions/obc/obc.py:105-130,156-195):
 *   x_ref = inv(a_ii - a_ji x a_ij), abs_res = ||x_ref - x||_F,
 *   rel_res = abs_res / ||x_ref||_F.  x_ref may equal x. */
int qtx_obc_refine(int n, int64_t batch, qtx_mat a_ii, qtx_mat a_ij, qtx_mat a_ji, qtx_mat x,
                   qtx_mat x_ref, double* rel_res, double* abs_res, int* info, void* workspace,
                   size_t workspace_bytes, qtx_stream stream);

/* Caroli transmission T = Tr[Gamma_L G_{0,N-1} Gamma_R G_{0,N-1}^H] with
 * Gamma = i (Sigma - Sigma^H); g0n is m x n (m = first, n = last block
 * size). The reference computes the same quantity as the boundary
 * Meir-Wingreen current (rgf.py:414-428) divided by (f_L - f_R) in the
 * ballistic case. transmission: device double[batch]. */
int qtx_transmission(int m, int n, int64_t batch, qtx_mat g0n, qtx_mat sigma_left,
                     qtx_mat sigma_right, double* transmission, void* workspace,
                     size_t workspace_bytes, qtx_stream stream);

/* DSDBCOO block densification (qttools datastructures/dsdbcoo.py:333-412,
 * kernels/datastructure/numba/dsdbcoo.py densify_block): the m x n output
 * blocks are zeroed, then out[b, rows[k], cols[k]] = data[b * data_stride + k]
 * for k < nnz. data points at the block's first nonzero (block-sorted
 * storage, dsdbcoo.py:297-331); rows/cols are device int32, block-local. */
int qtx_coo_densify(int64_t batch, const void* data, int64_t data_stride, int64_t nnz,
                    const int32_t* rows, const int32_t* cols, qtx_mat out, int m, int n,
                    qtx_stream stream);

/* Block sparsification (dsdbcoo.py:466-521, sparsify_block):
 * data[b * data_stride + k] = in[b, rows[k], cols[k]]. */
int qtx_coo_sparsify(int64_t batch, qtx_mat in, int64_t nnz, const int32_t* rows,
                     const int32_t* cols, void* data, int64_t data_stride, qtx_stream stream);

/* Copies the byte ranges [offsets[r], offsets[r] + lengths[r]) of each of
 * `rows` rows from src (row pitch src_row_bytes) to dst (row pitch
 * dst_row_bytes), host or device memory in any direction (a pinned host
 * buffer makes it an asynchronous DMA); offsets / lengths are host arrays.
 * The plugin layer moves only the nonzero slices of the DSDBCOO blocks a
 * solve reads or writes (dsdbcoo.py:297-331) with it; replaces the
 * reference's per-block host views of data[stack, nnz]. */
int qtx_copy_ranges(void* dst, int64_t dst_row_bytes, const void* src, int64_t src_row_bytes,
                    int64_t rows, const int64_t* offsets, const int64_t* lengths, int num_ranges,
                    qtx_stream stream);

/* Complex energies z[b] = E[b] + i eta (device double[batch] in, device
 * complex128[batch] out), the scalar part of the system-matrix assembly. */
int qtx_assemble_energies(int64_t batch, const double* energies, double eta, void* z,
                          qtx_stream stream);

/* Diagonal blocks of the system matrix, out[b] = z[b] I - h[b]
 * (the assembly of quatrex/electron/solver.py:668-709 with zero potential
 * and scattering self-energy: A(E) = (E + i eta) I - H). h may have stride
 * 0 (one Hamiltonian block for every energy); z: device complex128[batch]. */
int qtx_assemble_diag(int n, int64_t batch, qtx_mat h, const void* z, qtx_mat out,
                      qtx_stream stream);

/* System matrix of the electron solve in one pass, quatrex
 * electron/solver.py:668-709 (ElectronSolver._assemble_system_matrix with
 * _subtract_hamiltonian_and_self_energy, :611-665; no overlap matrix):
 *   A_ij = delta_ij (z_b I - diag(V_i)) - H_ij - Sigma^R_ij
 *          - (Sigma^>_ij - Sigma^<_ij) / 2
 * for every block of the block-tridiagonal a (a NULL output block is not
 * written). h: Hamiltonian blocks (stride 0 for energy-independent ones);
 * potential: device double[sum(block_sizes)] or NULL; z: device
 * complex128[batch] energies E + i eta; sigma_*: scattering self-energies
 * (Sigma^R is its Hermitian part), NULL or NULL blocks for zero. */
int qtx_assemble_system(const qtx_bt* h, const double* potential, const void* z,
                        const qtx_bt* sigma_retarded, const qtx_bt* sigma_lesser,
                        const qtx_bt* sigma_greater, const qtx_bt* a, int64_t batch,
                        qtx_stream stream);

/* Launch profiler. Kernel classes: */
enum qtx_kernel_class {
  QTX_KERNEL_ZGEMM = 0,    /* batched complex GEMM; work = 8 m n k flops */
  QTX_KERNEL_ZINV = 1,     /* batched inverse; work = 8 n^3 flops */
  QTX_KERNEL_BLOCKOPS = 2, /* elementwise block kernels; work = bytes */
  QTX_KERNEL_REDUCE = 3,   /* traces / norms; work = bytes */
  QTX_KERNEL_FORMAT = 4,   /* assembly, densify / sparsify; work = bytes */
  QTX_KERNEL_CGEMM = 5,    /* complex64 tcgen05 GEMM (split TF32); work = 8 m n k flops */
  QTX_KERNEL_ZGEMM_EMU = 6, /* complex128 GEMM on int8 tcgen05 (digit planes); work = 8 m n k */
  QTX_KERNEL_SPLIT = 7      /* digit-plane split of the emulated GEMM's operands; work = bytes */
};
/* Turns event bracketing of every library kernel launch on or off. */
int qtx_profile_enable(int on);
/* Drops the recorded launches. */
int qtx_profile_reset(void);
/* Sums the recorded launches of one class (kind < 0: all classes):
 * device milliseconds, algorithmic work and launch count. Synchronizes
 * the recorded events. */
int qtx_profile_read(int kind, double* total_ms, double* total_work, int64_t* launches);

#ifdef __cplusplus
}
#endif

#endif /* QTX_B200_H */
