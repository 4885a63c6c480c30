// extern "C" entry points of libqtx_b200.so (declared in include/qtx_b200.h).
//
// Each wrapper validates its arguments, zeroes the caller's status arrays,
// binds the caller's workspace and forwards to the drivers in rgf.cu /
// sr.cu. No C++ exception crosses the ABI; failures return a negative
// qtx_status and leave a message for qtx_last_error().
#include <cstring>
#include <exception>
#include <string>

#include "common.cuh"

namespace qtx {

namespace {
thread_local std::string g_error;
}

void set_error(const std::string& msg) { g_error = msg; }
const char* get_error() { return g_error.c_str(); }

// Drivers (rgf.cu, sr.cu).
int selected_inv_run(const BTRef& a, const MatRef* obc_r, const BTRef& x, int64_t batch, int* info,
                     Workspace& ws, cudaStream_t s);
int selected_solve_run(const SolveIO& io, int64_t batch, int* info, Workspace& ws, cudaStream_t s);
int selected_solve_mixed_run(const SolveIO& io, int64_t batch, int* info, Workspace& ws,
                             cudaStream_t s);
size_t sancho_rubio_ws(int n, int64_t batch);
int sancho_rubio_run(int n, int64_t batch, MatRef aii, MatRef aij, MatRef aji, MatRef x,
                     int max_iterations, double tol, int per_energy, int* iterations,
                     int* converged, double* delta_out, int* info, Workspace& ws, cudaStream_t s);
int sancho_rubio_multi_run(int n, int nsys, const int64_t* batches, const qtx_mat* aii,
                           const qtx_mat* aij, const qtx_mat* aji, const qtx_mat* x,
                           int max_iterations, double tol, int per_energy, int* iterations,
                           int* converged, int* info, Workspace& ws, cudaStream_t s);
int sancho_rubio_multi_async_run(int n, int nsys, const int64_t* batches, const qtx_mat* aii,
                                 const qtx_mat* aij, const qtx_mat* aji, const qtx_mat* x,
                                 int max_iterations, double tol, int per_energy, int* d_iters,
                                 int* d_converged, int* info, Workspace& ws, cudaStream_t s);
size_t obc_refine_ws(int n, int64_t batch);
int obc_refine_run(int n, int64_t batch, MatRef aii, MatRef aij, MatRef aji, MatRef x, MatRef xref,
                   double* rel, double* abs_res, int* info, Workspace& ws, cudaStream_t s);
size_t contact_ws(int n, int64_t batch);
int contact_run(int n, int64_t batch, MatRef aij, MatRef aji, MatRef g, const double* occ,
                MatRef sigma, MatRef sl, MatRef sg, Workspace& ws, cudaStream_t s);
size_t transmission_ws(int m, int n, int64_t batch);
int transmission_run(int m, int n, int64_t batch, MatRef g0n, MatRef sl, MatRef sr, double* T,
                     Workspace& ws, cudaStream_t s);

}  // namespace qtx

using namespace qtx;

namespace {

int check_bt(const qtx_bt* t, const char* name, int n_expected, const int32_t* bs_expected) {
  if (t == nullptr) return QTX_OK;
  if (t->num_blocks <= 0 || t->block_sizes == nullptr) {
    set_error(std::string(name) + ": invalid block layout");
    return QTX_ERR_ARG;
  }
  if (n_expected > 0) {
    if (t->num_blocks != n_expected) {
      set_error(std::string(name) + ": number of blocks differs from the system matrix");
      return QTX_ERR_ARG;
    }
    for (int i = 0; i < n_expected; ++i)
      if (t->block_sizes[i] != bs_expected[i]) {
        set_error(std::string(name) + ": block sizes differ from the system matrix");
        return QTX_ERR_ARG;
      }
  }
  for (int i = 0; i < t->num_blocks; ++i)
    if (t->block_sizes[i] <= 0 || t->block_sizes[i] > 1024) {
      set_error(std::string(name) + ": block sizes must be in [1, 1024]");
      return QTX_ERR_ARG;
    }
  return QTX_OK;
}

std::vector<MatRef> obc_vec(const qtx_mat* o, int n) {
  std::vector<MatRef> v;
  if (o == nullptr) return v;
  v.resize(n);
  for (int i = 0; i < n; ++i) v[i] = from_abi(o[i]);
  return v;
}

template <typename F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    set_error(std::string("internal error: ") + e.what());
    return QTX_ERR_ARG;
  } catch (...) {
    set_error("internal error");
    return QTX_ERR_ARG;
  }
}

Workspace bind(void* base, size_t bytes) {
  Workspace ws;
  ws.base = static_cast<char*>(base);
  ws.cap = bytes;
  return ws;
}

int need_ws(void* base, size_t bytes, size_t need, const char* who) {
  if (need > 0 && (base == nullptr || bytes < need)) {
    set_error(std::string(who) + ": workspace too small (" + std::to_string(bytes) + " < " +
              std::to_string(need) + " bytes)");
    return QTX_ERR_WORKSPACE;
  }
  return QTX_OK;
}

// Workspace of a selected solve: a dry run of the driver's allocations.
size_t solve_ws_bytes(int32_t nb, const int32_t* bs, int64_t batch, int cur, int mixed) {
  SolveIO io;
  io.a.n = nb;
  io.a.bs.assign(bs, bs + nb);
  z64 dummy;
  io.current = cur ? &dummy : nullptr;
  Workspace ws;
  if (mixed)
    selected_solve_mixed_run(io, batch, nullptr, ws, nullptr);
  else
    selected_solve_run(io, batch, nullptr, ws, nullptr);
  return ws.off + 256;
}

size_t inv_ws_bytes(int32_t nb, const int32_t* bs, int64_t batch) {
  Workspace ws;
  int bm = 0;
  for (int i = 0; i < nb; ++i) bm = bs[i] > bm ? bs[i] : bm;
  for (int i = 0; i < nb; ++i) ws.mat(bs[i], bs[i], batch);
  for (int k = 0; k < 6; ++k) ws.mat(bm, bm, batch);
  ws.take(zinv_scratch_bytes(bm, batch));
  ws.take(oz_scratch_bytes(bm, bm, bm, batch, gemm_slices()));
  return ws.off + 256;
}

}  // namespace

extern "C" {

int qtx_version(void) { return 100; }

const char* qtx_last_error(void) { return get_error(); }

int qtx_zgemm_batched(int m, int n, int k, int64_t batch, double alpha_re, double alpha_im,
                      qtx_mat a, int op_a, qtx_mat b, int op_b, double beta_re, double beta_im,
                      qtx_mat d, int op_d, qtx_mat c, qtx_stream stream) {
  return guarded([&] {
    if (m < 0 || n < 0 || k < 0 || batch < 0 || (op_a != 0 && op_a != 1) ||
        (op_b != 0 && op_b != 1) || (op_d != 0 && op_d != 1)) {
      set_error("qtx_zgemm_batched: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    if (c.ptr == nullptr) {
      set_error("qtx_zgemm_batched: null output");
      return (int)QTX_ERR_ARG;
    }
    GemmDesc g;
    g.M = m;
    g.N = n;
    g.K = k;
    g.batch = batch;
    g.A = from_abi(a);
    g.B = from_abi(b);
    g.opA = op_a;
    g.opB = op_b;
    g.alpha = make_double2(alpha_re, alpha_im);
    g.C = from_abi(c);
    if (d.ptr != nullptr) {
      g.add[0] = Addend{from_abi(d), make_double2(beta_re, beta_im), op_d};
      g.nadd = 1;
    }
    return zgemm(g, (cudaStream_t)stream);
  });
}

int qtx_cgemm_batched(int m, int n, int k, int64_t batch, float alpha_re, float alpha_im, qtx_mat a,
                      int op_a, qtx_mat b, int op_b, float beta_re, float beta_im, qtx_mat d,
                      int op_d, qtx_mat c, int* err, qtx_stream stream) {
  return guarded([&] {
    if (m < 0 || n < 0 || k < 0 || batch < 0 || (op_a != 0 && op_a != 1) ||
        (op_b != 0 && op_b != 1) || (op_d != 0 && op_d != 1) || c.ptr == nullptr) {
      set_error("qtx_cgemm_batched: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    CGemmDesc g;
    g.M = m;
    g.N = n;
    g.K = k;
    g.batch = batch;
    g.A = from_abi(a);
    g.B = from_abi(b);
    g.opA = op_a;
    g.opB = op_b;
    g.alpha = make_float2(alpha_re, alpha_im);
    g.C = from_abi(c);
    g.err = err;
    if (d.ptr != nullptr) {
      g.add[0] = CAddend{from_abi(d), make_float2(beta_re, beta_im), op_d};
      g.nadd = 1;
    }
    return cgemm_tc(g, (cudaStream_t)stream);
  });
}

int qtx_zinv_batched(int n, int64_t batch, qtx_mat a, qtx_mat x, int* info, qtx_stream stream) {
  return guarded([&] {
    if (n < 0 || batch < 0 || a.ptr == nullptr || x.ptr == nullptr) {
      set_error("qtx_zinv_batched: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, (cudaStream_t)stream));
    return zinv(n, batch, from_abi(a), from_abi(x), info, nullptr, (cudaStream_t)stream);
  });
}

size_t qtx_zinv_workspace(int n, int64_t batch) { return zinv_scratch_bytes(n, batch) + 256; }

int qtx_zinv_batched_ws(int n, int64_t batch, qtx_mat a, qtx_mat x, int* info, void* workspace,
                        size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (n < 0 || batch < 0 || a.ptr == nullptr || x.ptr == nullptr) {
      set_error("qtx_zinv_batched_ws: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, (cudaStream_t)stream));
    return zinv_ex(n, batch, from_abi(a), from_abi(x), info, nullptr, workspace, workspace_bytes,
                   (cudaStream_t)stream);
  });
}

size_t qtx_zgemm_emulated_workspace(int m, int n, int k, int64_t batch, int slices) {
  if (m <= 0 || n <= 0 || k <= 0 || batch <= 0 || !oz_supported(k, slices)) return 0;
  return oz_scratch_bytes(m, n, k, batch, slices) + 256;
}

int qtx_zgemm_emulated_batched(int m, int n, int k, int64_t batch, double alpha_re, double alpha_im,
                               qtx_mat a, int op_a, qtx_mat b, int op_b, double beta_re,
                               double beta_im, qtx_mat d, int op_d, qtx_mat c, int slices,
                               void* workspace, size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (m < 0 || n < 0 || k < 0 || batch < 0 || (op_a != 0 && op_a != 1) ||
        (op_b != 0 && op_b != 1) || (op_d != 0 && op_d != 1) || c.ptr == nullptr ||
        (k > 0 && (a.ptr == nullptr || b.ptr == nullptr))) {
      set_error("qtx_zgemm_emulated_batched: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    if (!oz_supported(k, slices)) {
      set_error("qtx_zgemm_emulated_batched: slices must be 3-8 and slices * 2k * 2^14 < 2^31");
      return (int)QTX_ERR_ARG;
    }
    if (m == 0 || n == 0 || batch == 0) return (int)QTX_OK;
    GemmDesc g;
    g.M = m;
    g.N = n;
    g.K = k;
    g.batch = batch;
    g.A = from_abi(a);
    g.B = from_abi(b);
    g.opA = op_a;
    g.opB = op_b;
    g.alpha = make_double2(alpha_re, alpha_im);
    g.C = from_abi(c);
    if (d.ptr != nullptr) {
      g.add[0] = Addend{from_abi(d), make_double2(beta_re, beta_im), op_d};
      g.nadd = 1;
    }
    if (k == 0) return zgemm(g, (cudaStream_t)stream);
    return zgemm_oz(g, slices, workspace, workspace_bytes, (cudaStream_t)stream);
  });
}

int qtx_set_gemm_path(int slices) {
  if (slices != 0 && (slices < 3 || slices > 8)) {
    set_error("qtx_set_gemm_path: slices must be 0 (FP64 DMMA) or 3-8 (int8 emulation)");
    return QTX_ERR_ARG;
  }
  set_gemm_slices(slices);
  return QTX_OK;
}

int qtx_get_gemm_path(void) { return gemm_slices(); }

int qtx_emulated_gemm_status(void) {
  int flag = 0;
  const int st = oz_status_take(&flag);
  return st != QTX_OK ? st : flag;
}

int qtx_inverse_status(void) {
  int flag = 0;
  const int st = zinv_cluster_status_take(&flag);
  return st != QTX_OK ? st : flag;
}

int qtx_set_inverse_path(int mode) {
  if (mode < 0 || mode > 4) {
    set_error("qtx_set_inverse_path: mode must be 0, 1, 2, 3 or 4");
    return QTX_ERR_ARG;
  }
  set_inverse_path(mode);
  return QTX_OK;
}

size_t qtx_selected_inv_workspace(int32_t num_blocks, const int32_t* block_sizes, int64_t batch) {
  if (num_blocks <= 0 || block_sizes == nullptr || batch <= 0) return 0;
  return inv_ws_bytes(num_blocks, block_sizes, batch);
}

int qtx_selected_inv(const qtx_bt* a, const qtx_mat* obc_retarded, const qtx_bt* x, int64_t batch,
                     int* info, void* workspace, size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (a == nullptr || x == nullptr || batch <= 0) {
      set_error("qtx_selected_inv: null matrix or empty batch");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(check_bt(a, "a", 0, nullptr));
    QTX_TRY(check_bt(x, "x", a->num_blocks, a->block_sizes));
    const size_t need = inv_ws_bytes(a->num_blocks, a->block_sizes, batch);
    QTX_TRY(need_ws(workspace, workspace_bytes, need, "qtx_selected_inv"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, s));
    BTRef A = bt_from_abi(a), X = bt_from_abi(x);
    std::vector<MatRef> o = obc_vec(obc_retarded, a->num_blocks);
    Workspace ws = bind(workspace, workspace_bytes);
    return selected_inv_run(A, o.empty() ? nullptr : o.data(), X, batch, info, ws, s);
  });
}

size_t qtx_selected_solve_workspace(int32_t num_blocks, const int32_t* block_sizes, int64_t batch,
                                    int return_current) {
  if (num_blocks <= 0 || block_sizes == nullptr || batch <= 0) return 0;
  return solve_ws_bytes(num_blocks, block_sizes, batch, return_current, 0);
}

int qtx_selected_solve(const qtx_bt* a, const qtx_bt* sigma_lesser, const qtx_bt* sigma_greater,
                       const qtx_mat* obc_retarded, const qtx_mat* obc_lesser,
                       const qtx_mat* obc_greater, const qtx_bt* xl, const qtx_bt* xg,
                       const qtx_bt* xr, void* current, qtx_mat g0n, double* density, int flags,
                       int64_t batch, int* info, void* workspace, size_t workspace_bytes,
                       qtx_stream stream) {
  return guarded([&] {
    if (a == nullptr || batch <= 0) {
      set_error("qtx_selected_solve: null system matrix or empty batch");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(check_bt(a, "a", 0, nullptr));
    const int N = a->num_blocks;
    QTX_TRY(check_bt(sigma_lesser, "sigma_lesser", N, a->block_sizes));
    QTX_TRY(check_bt(sigma_greater, "sigma_greater", N, a->block_sizes));
    QTX_TRY(check_bt(xl, "xl", N, a->block_sizes));
    QTX_TRY(check_bt(xg, "xg", N, a->block_sizes));
    QTX_TRY(check_bt(xr, "xr", N, a->block_sizes));
    const size_t need = solve_ws_bytes(N, a->block_sizes, batch, current != nullptr, 0);
    QTX_TRY(need_ws(workspace, workspace_bytes, need, "qtx_selected_solve"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, s));
    if (current)
      QTX_CHECK_CUDA(cudaMemsetAsync(current, 0, sizeof(z64) * batch * (N + 1), s));
    SolveIO io;
    io.a = bt_from_abi(a);
    io.sl = bt_from_abi(sigma_lesser);
    io.sg = bt_from_abi(sigma_greater);
    io.xl = bt_from_abi(xl);
    io.xg = bt_from_abi(xg);
    io.xr = bt_from_abi(xr);
    std::vector<MatRef> orr = obc_vec(obc_retarded, N), ol = obc_vec(obc_lesser, N),
                        og = obc_vec(obc_greater, N);
    io.obc_r = orr.empty() ? nullptr : orr.data();
    io.obc_l = ol.empty() ? nullptr : ol.data();
    io.obc_g = og.empty() ? nullptr : og.data();
    io.current = static_cast<z64*>(current);
    io.g0n = from_abi(g0n);
    io.density = density;
    io.symmetric = (flags & QTX_SOLVE_SYMMETRIC_OUT) ? 1 : 0;
    Workspace ws = bind(workspace, workspace_bytes);
    return selected_solve_run(io, batch, info, ws, s);
  });
}

size_t qtx_selected_solve_mixed_workspace(int32_t num_blocks, const int32_t* block_sizes,
                                          int64_t batch, int return_current) {
  if (num_blocks <= 0 || block_sizes == nullptr || batch <= 0) return 0;
  return solve_ws_bytes(num_blocks, block_sizes, batch, return_current, 1);
}

int qtx_selected_solve_mixed(const qtx_bt* a, const qtx_bt* sigma_lesser,
                             const qtx_bt* sigma_greater, const qtx_mat* obc_retarded,
                             const qtx_mat* obc_lesser, const qtx_mat* obc_greater, const qtx_bt* xl,
                             const qtx_bt* xg, const qtx_bt* xr, void* current, qtx_mat g0n,
                             double* density, int flags, int64_t batch, int* info, void* workspace,
                             size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (a == nullptr || batch <= 0) {
      set_error("qtx_selected_solve_mixed: null system matrix or empty batch");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(check_bt(a, "a", 0, nullptr));
    const int N = a->num_blocks;
    QTX_TRY(check_bt(sigma_lesser, "sigma_lesser", N, a->block_sizes));
    QTX_TRY(check_bt(sigma_greater, "sigma_greater", N, a->block_sizes));
    QTX_TRY(check_bt(xl, "xl", N, a->block_sizes));
    QTX_TRY(check_bt(xg, "xg", N, a->block_sizes));
    QTX_TRY(check_bt(xr, "xr", N, a->block_sizes));
    const size_t need = solve_ws_bytes(N, a->block_sizes, batch, current != nullptr, 1);
    QTX_TRY(need_ws(workspace, workspace_bytes, need, "qtx_selected_solve_mixed"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, s));
    if (current)
      QTX_CHECK_CUDA(cudaMemsetAsync(current, 0, sizeof(z64) * batch * (N + 1), s));
    SolveIO io;
    io.a = bt_from_abi(a);
    io.sl = bt_from_abi(sigma_lesser);
    io.sg = bt_from_abi(sigma_greater);
    io.xl = bt_from_abi(xl);
    io.xg = bt_from_abi(xg);
    io.xr = bt_from_abi(xr);
    std::vector<MatRef> orr = obc_vec(obc_retarded, N), ol = obc_vec(obc_lesser, N),
                        og = obc_vec(obc_greater, N);
    io.obc_r = orr.empty() ? nullptr : orr.data();
    io.obc_l = ol.empty() ? nullptr : ol.data();
    io.obc_g = og.empty() ? nullptr : og.data();
    io.current = static_cast<z64*>(current);
    io.g0n = from_abi(g0n);
    io.density = density;
    io.symmetric = (flags & QTX_SOLVE_SYMMETRIC_OUT) ? 1 : 0;
    Workspace ws = bind(workspace, workspace_bytes);
    return selected_solve_mixed_run(io, batch, info, ws, s);
  });
}

int qtx_zgemm_grouped(int m, int n, int k, int64_t batch, double alpha_re, double alpha_im,
                      const void* const* a_ptrs, int64_t lda, int op_a, const void* const* b_ptrs, int64_t ldb,
                      int op_b, double beta_re, double beta_im, const void* const* d_ptrs, int64_t ldd, int op_d,
                      void* const* c_ptrs, int64_t ldc, qtx_stream stream) {
  return guarded([&] {
    if (m < 0 || n < 0 || k <= 0 || batch < 0 || (op_a != 0 && op_a != 1) || (op_b != 0 && op_b != 1) ||
        (op_d != 0 && op_d != 1) || a_ptrs == nullptr || b_ptrs == nullptr || c_ptrs == nullptr || lda <= 0 ||
        ldb <= 0 || ldc <= 0 || (d_ptrs != nullptr && ldd <= 0)) {
      set_error("qtx_zgemm_grouped: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    GemmDesc g;
    g.M = m;
    g.N = n;
    g.K = k;
    g.batch = batch;
    // the tables stand in for the base pointers (non-null, 16-byte aligned)
    g.A = MatRef{const_cast<void*>(static_cast<const void*>(a_ptrs)), lda, 0};
    g.B = MatRef{const_cast<void*>(static_cast<const void*>(b_ptrs)), ldb, 0};
    g.C = MatRef{const_cast<void*>(static_cast<const void*>(c_ptrs)), ldc, 0};
    g.opA = op_a;
    g.opB = op_b;
    g.alpha = make_double2(alpha_re, alpha_im);
    g.a_ptrs = reinterpret_cast<const z64* const*>(a_ptrs);
    g.b_ptrs = reinterpret_cast<const z64* const*>(b_ptrs);
    g.c_ptrs = reinterpret_cast<z64* const*>(c_ptrs);
    if (d_ptrs != nullptr) {
      g.add[0] = Addend{MatRef{const_cast<void*>(static_cast<const void*>(d_ptrs)), ldd, 0},
                        make_double2(beta_re, beta_im), op_d};
      g.nadd = 1;
      g.d_ptrs = reinterpret_cast<const z64* const*>(d_ptrs);
    }
    return zgemm(g, (cudaStream_t)stream);
  });
}

int qtx_zcombine(int m, int n, int64_t batch, qtx_mat out, int nterms, const qtx_mat* terms,
                 const double* coefs, const int* conj_trans, qtx_stream stream) {
  return guarded([&] {
    if (m < 0 || n < 0 || batch < 0 || out.ptr == nullptr || nterms < 1 || nterms > kMaxAddends ||
        terms == nullptr || coefs == nullptr) {
      set_error("qtx_zcombine: invalid arguments (1 to 4 terms, non-null output)");
      return (int)QTX_ERR_ARG;
    }
    Addend t[kMaxAddends];
    for (int k = 0; k < nterms; ++k) {
      if (terms[k].ptr == nullptr) {
        set_error("qtx_zcombine: null term");
        return (int)QTX_ERR_ARG;
      }
      t[k] = Addend{from_abi(terms[k]), make_double2(coefs[2 * k], coefs[2 * k + 1]),
                    conj_trans ? conj_trans[k] : 0};
    }
    return zcombine(m, n, batch, from_abi(out), t, nterms, nullptr, (cudaStream_t)stream);
  });
}

int qtx_convert(int m, int n, int64_t batch, qtx_mat in, int in_dtype, qtx_mat out, int out_dtype,
                qtx_stream stream) {
  return guarded([&] {
    if (m < 0 || n < 0 || batch < 0 || in.ptr == nullptr || out.ptr == nullptr) {
      set_error("qtx_convert: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (in_dtype == QTX_C64 && out_dtype == QTX_C128)
      return convert_c64_to_c128(m, n, batch, from_abi(in), from_abi(out), s);
    if (in_dtype == QTX_C128 && out_dtype == QTX_C64)
      return convert_c128_to_c64(m, n, batch, from_abi(in), from_abi(out), s);
    Addend t{from_abi(in), make_double2(1.0, 0.0), 0};
    if (in_dtype == QTX_C128 && out_dtype == QTX_C128)
      return zcombine(m, n, batch, from_abi(out), &t, 1, nullptr, s);
    if (in_dtype == QTX_C64 && out_dtype == QTX_C64)
      return ccombine(m, n, batch, from_abi(out), &t, 1, nullptr, s);
    set_error("qtx_convert: unknown dtype");
    return (int)QTX_ERR_ARG;
  });
}

size_t qtx_sancho_rubio_workspace(int n, int64_t batch) {
  if (n <= 0 || batch <= 0) return 0;
  return sancho_rubio_ws(n, batch);
}

int qtx_sancho_rubio(int n, int64_t batch, qtx_mat a_ii, qtx_mat a_ij, qtx_mat a_ji, qtx_mat x,
                     int max_iterations, double tol, int per_energy, int* iterations,
                     int* converged, double* delta_out, int* info, void* workspace,
                     size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (n <= 0 || n > 1024 || batch <= 0 || max_iterations < 0 || a_ii.ptr == nullptr ||
        x.ptr == nullptr) {
      set_error("qtx_sancho_rubio: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(need_ws(workspace, workspace_bytes, sancho_rubio_ws(n, batch), "qtx_sancho_rubio"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, s));
    Workspace ws = bind(workspace, workspace_bytes);
    return sancho_rubio_run(n, batch, from_abi(a_ii), from_abi(a_ij), from_abi(a_ji), from_abi(x),
                            max_iterations, tol, per_energy, iterations, converged, delta_out, info,
                            ws, s);
  });
}

int qtx_sancho_rubio_multi(int n, int num_systems, const int64_t* batches, const qtx_mat* a_ii,
                           const qtx_mat* a_ij, const qtx_mat* a_ji, const qtx_mat* x,
                           int max_iterations, double tol, int per_energy, int* iterations,
                           int* converged, int* info, void* workspace, size_t workspace_bytes,
                           qtx_stream stream) {
  return guarded([&] {
    if (n <= 0 || n > 1024 || num_systems <= 0 || batches == nullptr || a_ii == nullptr ||
        a_ij == nullptr || a_ji == nullptr || x == nullptr || max_iterations < 0) {
      set_error("qtx_sancho_rubio_multi: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    int64_t total = 0;
    for (int k = 0; k < num_systems; ++k) {
      if (batches[k] <= 0 || a_ii[k].ptr == nullptr || x[k].ptr == nullptr) {
        set_error("qtx_sancho_rubio_multi: empty system or null matrix");
        return (int)QTX_ERR_ARG;
      }
      total += batches[k];
    }
    QTX_TRY(need_ws(workspace, workspace_bytes, sancho_rubio_ws(n, total), "qtx_sancho_rubio_multi"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * total, s));
    Workspace ws = bind(workspace, workspace_bytes);
    return sancho_rubio_multi_run(n, num_systems, batches, a_ii, a_ij, a_ji, x, max_iterations, tol,
                                  per_energy, iterations, converged, info, ws, s);
  });
}

int qtx_sancho_rubio_multi_async(int n, int num_systems, const int64_t* batches,
                                 const qtx_mat* a_ii, const qtx_mat* a_ij, const qtx_mat* a_ji,
                                 const qtx_mat* x, int max_iterations, double tol, int per_energy,
                                 int* d_iterations, int* d_converged, int* info, void* workspace,
                                 size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (n <= 0 || n > 1024 || num_systems <= 0 || batches == nullptr || a_ii == nullptr ||
        a_ij == nullptr || a_ji == nullptr || x == nullptr || max_iterations < 0 ||
        d_iterations == nullptr || d_converged == nullptr) {
      set_error("qtx_sancho_rubio_multi_async: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    int64_t total = 0;
    for (int k = 0; k < num_systems; ++k) {
      if (batches[k] <= 0 || a_ii[k].ptr == nullptr || x[k].ptr == nullptr) {
        set_error("qtx_sancho_rubio_multi_async: empty system or null matrix");
        return (int)QTX_ERR_ARG;
      }
      total += batches[k];
    }
    QTX_TRY(need_ws(workspace, workspace_bytes, sancho_rubio_ws(n, total),
                    "qtx_sancho_rubio_multi_async"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * total, s));
    Workspace ws = bind(workspace, workspace_bytes);
    return sancho_rubio_multi_async_run(n, num_systems, batches, a_ii, a_ij, a_ji, x, max_iterations,
                                        tol, per_energy, d_iterations, d_converged, info, ws, s);
  });
}

size_t qtx_obc_workspace(int n, int64_t batch) {
  if (n <= 0 || batch <= 0) return 0;
  size_t w = contact_ws(n, batch);
  const size_t r = obc_refine_ws(n, batch), t = transmission_ws(n, n, batch);
  if (r > w) w = r;
  if (t > w) w = t;
  return w;
}

int qtx_contact_self_energy(int n, int64_t batch, qtx_mat a_ij, qtx_mat a_ji, qtx_mat g,
                            const double* occupancies, qtx_mat sigma, qtx_mat sigma_lesser,
                            qtx_mat sigma_greater, void* workspace, size_t workspace_bytes,
                            qtx_stream stream) {
  return guarded([&] {
    if (n <= 0 || batch <= 0 || g.ptr == nullptr) {
      set_error("qtx_contact_self_energy: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(need_ws(workspace, workspace_bytes, contact_ws(n, batch), "qtx_contact_self_energy"));
    Workspace ws = bind(workspace, workspace_bytes);
    return contact_run(n, batch, from_abi(a_ij), from_abi(a_ji), from_abi(g), occupancies,
                       from_abi(sigma), from_abi(sigma_lesser), from_abi(sigma_greater), ws,
                       (cudaStream_t)stream);
  });
}

int qtx_obc_refine(int n, int64_t batch, qtx_mat a_ii, qtx_mat a_ij, qtx_mat a_ji, qtx_mat x,
                   qtx_mat x_ref, double* rel_res, double* abs_res, int* info, void* workspace,
                   size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (n <= 0 || n > 1024 || batch <= 0 || x.ptr == nullptr || x_ref.ptr == nullptr) {
      set_error("qtx_obc_refine: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(need_ws(workspace, workspace_bytes, obc_refine_ws(n, batch), "qtx_obc_refine"));
    cudaStream_t s = (cudaStream_t)stream;
    if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, s));
    Workspace ws = bind(workspace, workspace_bytes);
    return obc_refine_run(n, batch, from_abi(a_ii), from_abi(a_ij), from_abi(a_ji), from_abi(x),
                          from_abi(x_ref), rel_res, abs_res, info, ws, s);
  });
}

int qtx_transmission(int m, int n, int64_t batch, qtx_mat g0n, qtx_mat sigma_left,
                     qtx_mat sigma_right, double* transmission, void* workspace,
                     size_t workspace_bytes, qtx_stream stream) {
  return guarded([&] {
    if (m <= 0 || n <= 0 || batch <= 0 || g0n.ptr == nullptr || sigma_left.ptr == nullptr ||
        sigma_right.ptr == nullptr || transmission == nullptr) {
      set_error("qtx_transmission: invalid arguments");
      return (int)QTX_ERR_ARG;
    }
    QTX_TRY(need_ws(workspace, workspace_bytes, transmission_ws(m, n, batch), "qtx_transmission"));
    Workspace ws = bind(workspace, workspace_bytes);
    return transmission_run(m, n, batch, from_abi(g0n), from_abi(sigma_left),
                            from_abi(sigma_right), transmission, ws, (cudaStream_t)stream);
  });
}

}  // extern "C"
