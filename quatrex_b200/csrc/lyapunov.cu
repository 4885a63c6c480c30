// Discrete-time Lyapunov equation of the screened-interaction (W) boundary
// conditions, X = Q + A X A^H:
//
//  * qtx_lyapunov_doubling: the doubling iteration of qttools
//    boundary_conditions/lyapunov/doubling.py:36-91,
//      X_{k+1} = X_k + A_k X_k A_k^H,  A_{k+1} = A_k A_k,
//    stopped when every entry has ||X_{k+1} - X_k||_F / ||X_{k+1}||_F below
//    rel_tol or ||X_{k+1} - X_k||_F below abs_tol (the reference's batch-wide
//    rule; the per-step errors are read back once per step, like the
//    Sancho-Rubio stop test);
//  * qtx_lyapunov_refine: one fixed-point step with its residuals,
//    LyapunovSystem._fixed_point_step / _get_residuals (lyapunov.py:488-579).
//
// Products run through the same batched complex GEMM as the RGF (FP64 DMMA,
// or the int8 emulation when the calling thread selected it and scratch is
// bound).
#include <vector>

#include "common.cuh"

namespace qtx {
namespace {

const z64 ONE{1.0, 0.0};

GemmDesc gemm(int n, int64_t batch, MatRef A, int opA, MatRef B, int opB, MatRef C) {
  GemmDesc d;
  d.M = n;
  d.N = n;
  d.K = n;
  d.batch = batch;
  d.A = A;
  d.B = B;
  d.opA = opA;
  d.opB = opB;
  d.C = C;
  d.alpha = ONE;
  return d;
}

size_t doubling_ws(int n, int64_t batch) {
  Workspace ws;
  for (int k = 0; k < 4; ++k) ws.mat(n, n, batch);
  ws.take(2 * sizeof(double) * (size_t)batch);
  ws.take(oz_scratch_bytes(n, n, n, batch, gemm_slices()));
  return ws.off + 256;
}

}  // namespace
}  // namespace qtx

using namespace qtx;

extern "C" size_t qtx_lyapunov_workspace(int n, int64_t batch) {
  if (n <= 0 || batch <= 0) return 0;
  return doubling_ws(n, batch);
}

extern "C" int qtx_lyapunov_doubling(int n, int64_t batch, qtx_mat a, qtx_mat q, qtx_mat x, int max_iterations,
                                     double rel_tol, double abs_tol, int* iterations, int* converged,
                                     void* workspace, size_t workspace_bytes, qtx_stream stream) {
  try {
    if (n <= 0 || batch <= 0) return QTX_OK;
    if (a.ptr == nullptr || q.ptr == nullptr || x.ptr == nullptr || max_iterations < 0) {
      set_error("qtx_lyapunov_doubling: invalid arguments");
      return QTX_ERR_ARG;
    }
    Workspace ws;
    ws.base = static_cast<char*>(workspace);
    ws.cap = workspace_bytes;
    MatRef Ai = ws.mat(n, n, batch), An = ws.mat(n, n, batch), T = ws.mat(n, n, batch), Xn = ws.mat(n, n, batch);
    double* err = static_cast<double*>(ws.take(2 * sizeof(double) * (size_t)batch));
    OzScope oz(ws, n, batch);
    if (workspace == nullptr || ws.overflow) {
      set_error("qtx_lyapunov_doubling: workspace too small");
      return QTX_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const MatRef X = from_abi(x);
    {
      Addend ta{from_abi(a), ONE, 0}, tq{from_abi(q), ONE, 0};
      QTX_TRY(zcombine(n, n, batch, Ai, &ta, 1, nullptr, s));
      QTX_TRY(zcombine(n, n, batch, X, &tq, 1, nullptr, s));
    }
    std::vector<double> h(2 * (size_t)batch);
    int it = 0;
    bool conv = false;
    for (; it < max_iterations;) {
      // X_new = X + A_k X A_k^H
      QTX_TRY(zgemm(gemm(n, batch, Ai, 0, X, 0, T), s));
      GemmDesc d = gemm(n, batch, T, 0, Ai, 1, Xn);
      d.add[d.nadd++] = Addend{X, ONE, 0};
      QTX_TRY(zgemm(d, s));
      QTX_TRY(znorm_diff(n, batch, Xn, X, err, err + batch, nullptr, s));  // ||X_new - X||, ||X_new||
      Addend tx{Xn, ONE, 0};
      QTX_TRY(zcombine(n, n, batch, X, &tx, 1, nullptr, s));
      ++it;
      QTX_CHECK_CUDA(cudaMemcpyAsync(h.data(), err, 2 * sizeof(double) * (size_t)batch, cudaMemcpyDeviceToHost, s));
      QTX_CHECK_CUDA(cudaStreamSynchronize(s));
      bool all = true;
      for (int64_t b = 0; b < batch && all; ++b) {
        const double ab = h[b], rel = h[b] / h[batch + b];
        all = (rel < rel_tol) || (ab < abs_tol);
      }
      if (all) {
        conv = true;
        break;
      }
      // A_{k+1} = A_k A_k
      QTX_TRY(zgemm(gemm(n, batch, Ai, 0, Ai, 0, An), s));
      std::swap(Ai, An);
    }
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
    return QTX_OK;
  } catch (const std::exception& e) {
    set_error(std::string("qtx_lyapunov_doubling: internal error: ") + e.what());
    return QTX_ERR_ARG;
  }
}

extern "C" int qtx_lyapunov_refine(int n, int64_t batch, qtx_mat a, qtx_mat q, qtx_mat x, qtx_mat x_ref,
                                   double* rel_res, double* abs_res, void* workspace, size_t workspace_bytes,
                                   qtx_stream stream) {
  try {
    if (n <= 0 || batch <= 0) return QTX_OK;
    if (a.ptr == nullptr || q.ptr == nullptr || x.ptr == nullptr || x_ref.ptr == nullptr) {
      set_error("qtx_lyapunov_refine: invalid arguments");
      return QTX_ERR_ARG;
    }
    Workspace ws;
    ws.base = static_cast<char*>(workspace);
    ws.cap = workspace_bytes;
    MatRef T = ws.mat(n, n, batch), S = ws.mat(n, n, batch);
    OzScope oz(ws, n, batch);
    if (workspace == nullptr || ws.overflow) {
      set_error("qtx_lyapunov_refine: workspace too small");
      return QTX_ERR_WORKSPACE;
    }
    cudaStream_t s = (cudaStream_t)stream;
    QTX_TRY(zgemm(gemm(n, batch, from_abi(a), 0, from_abi(x), 0, T), s));
    GemmDesc d = gemm(n, batch, T, 0, from_abi(a), 1, S);
    d.add[d.nadd++] = Addend{from_abi(q), ONE, 0};
    QTX_TRY(zgemm(d, s));
    QTX_TRY(znorm_diff(n, batch, S, from_abi(x), abs_res, nullptr, rel_res, s));  // ||S - x||, / ||S||
    Addend t{S, ONE, 0};
    QTX_TRY(zcombine(n, n, batch, from_abi(x_ref), &t, 1, nullptr, s));
    return QTX_OK;
  } catch (const std::exception& e) {
    set_error(std::string("qtx_lyapunov_refine: internal error: ") + e.what());
    return QTX_ERR_ARG;
  }
}
