// Moments of Beyn's contour integral for the spectral open-boundary
// condition (qttools nevp/beyn.py:166-220 with kernels/operator.py:117-181).
//
// For the lead's quadratic eigenvalue problem T(z) = a_ji / z + a_ii + a_ij z
// and quadrature points z_j = r exp(2 pi i (j + 1.5) / nq), j = 0..nq-1, on
// an outer (r_o) and an inner (r_i) circle, with weight w = 1 / nq:
//   q0 = sum_j w (z_o,j T(z_o,j)^-1 - z_i,j T(z_i,j)^-1)
//   q1 = sum_j w (z_o,j^2 T(z_o,j)^-1 - z_i,j^2 T(z_i,j)^-1)
// for every stack entry. The 2 nq operators of all entries are built by one
// elementwise kernel, inverted by the batched Gauss-Jordan inverse (the same
// kernels as every other inverse of the path), and reduced by a second
// elementwise kernel in quadrature order. The small dense problems that
// follow (projection SVD, reduced eigenproblem) are host LAPACK work, as in
// the reference (its default compute location "numpy").
#include "common.cuh"

namespace qtx {
namespace {

struct Quad {
  z64 z, zinv;
};

// Quadrature point j (0..nq-1 outer, nq..2nq-1 inner) and its reciprocal.
__device__ __forceinline__ Quad quad_point(int j, int nq, double r_o, double r_i) {
  const bool outer = j < nq;
  const int jj = outer ? j : j - nq;
  const double r = outer ? r_o : r_i;
  double s, c;
  sincospi(2.0 * ((double)(jj + 1) + 0.5) / (double)nq, &s, &c);
  Quad q;
  q.z = make_double2(r * c, r * s);
  q.zinv = make_double2(c / r, -s / r);
  return q;
}

// W[b * 2nq + j] = a_ji[b] z_j^-1 + a_ii[b] + a_ij[b] z_j
__global__ void contour_operator_kernel(int n, int64_t batch, int nq, double r_o, double r_i, MatRef aji,
                                        MatRef aii, MatRef aij, z64* W) {
  const int64_t per = (int64_t)n * n;
  const int64_t total = per * 2 * nq * batch;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = idx % per;
    const int64_t bj = idx / per;
    const int j = (int)(bj % (2 * nq));
    const int64_t b = bj / (2 * nq);
    const int r = (int)(e / n), c = (int)(e % n);
    const Quad q = quad_point(j, nq, r_o, r_i);
    const z64 m = at<const z64>(aji, b)[(int64_t)r * aji.ld + c];
    const z64 d = at<const z64>(aii, b)[(int64_t)r * aii.ld + c];
    const z64 p = at<const z64>(aij, b)[(int64_t)r * aij.ld + c];
    const z64 t = zadd(zadd(zmul(m, q.zinv), d), zmul(p, q.z));
    W[idx] = t;
  }
}

// q0 = sum_j (w z_o,j W_o,j - w z_i,j W_i,j), q1 likewise with z^2.
__global__ void contour_moments_kernel(int n, int64_t batch, int nq, double r_o, double r_i, const z64* W,
                                       MatRef q0, MatRef q1) {
  const int64_t per = (int64_t)n * n;
  const double w = 1.0 / (double)nq;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < per * batch;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = idx / per, e = idx % per;
    const int r = (int)(e / n), c = (int)(e % n);
    const z64* base = W + (b * 2 * nq) * per + e;
    z64 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
    for (int j = 0; j < nq; ++j) {
      const Quad qo = quad_point(j, nq, r_o, r_i), qi = quad_point(nq + j, nq, r_o, r_i);
      const z64 vo = base[(int64_t)j * per], vi = base[(int64_t)(nq + j) * per];
      const z64 wo = make_double2(w * qo.z.x, w * qo.z.y), wi = make_double2(w * qi.z.x, w * qi.z.y);
      const z64 zo2 = zmul(qo.z, qo.z), zi2 = zmul(qi.z, qi.z);
      const z64 wo2 = make_double2(w * zo2.x, w * zo2.y), wi2 = make_double2(w * zi2.x, w * zi2.y);
      const z64 t0 = zsub(zmul(wo, vo), zmul(wi, vi));
      const z64 t1 = zsub(zmul(wo2, vo), zmul(wi2, vi));
      s0 = zadd(s0, t0);
      s1 = zadd(s1, t1);
    }
    at<z64>(q0, b)[(int64_t)r * q0.ld + c] = s0;
    at<z64>(q1, b)[(int64_t)r * q1.ld + c] = s1;
  }
}

// info[b] = 1-based index of the first singular operator of entry b, or 0.
__global__ void first_singular_kernel(int64_t batch, int nops_per, const int* inv_info, int* info) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < batch;
       b += (int64_t)gridDim.x * blockDim.x) {
    int first = 0;
    for (int j = 0; j < nops_per && first == 0; ++j)
      if (inv_info[b * nops_per + j] != 0) first = j + 1;
    info[b] = first;
  }
}

unsigned grid_for(int64_t total) {
  const int64_t want = (total + 255) / 256;
  return (unsigned)(want < 148 * 32 ? want : 148 * 32);
}

}  // namespace

size_t beyn_ws_bytes(int n, int64_t batch, int nq) {
  Workspace ws;
  ws.take((size_t)batch * 2 * nq * n * n * sizeof(z64));
  ws.take((size_t)batch * 2 * nq * sizeof(int));
  ws.take(zinv_scratch_bytes(n, batch * 2 * nq));
  return ws.off + 256;
}

int beyn_moments_run(int n, int64_t batch, MatRef aji, MatRef aii, MatRef aij, double r_o, double r_i, int nq,
                     MatRef q0, MatRef q1, int* info, Workspace& ws, cudaStream_t s) {
  const int64_t nops = batch * 2 * nq;
  z64* W = static_cast<z64*>(ws.take((size_t)nops * n * n * sizeof(z64)));
  int* inv_info = static_cast<int*>(ws.take((size_t)nops * sizeof(int)));
  const size_t scr_bytes = zinv_scratch_bytes(n, nops);
  void* scr = ws.take(scr_bytes);
  if (W == nullptr || ws.overflow) {
    set_error("qtx_beyn_moments: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  const int64_t per = (int64_t)n * n;
  {
    ProfScope prof(QTX_KERNEL_FORMAT, (double)nops * per * 16.0 + 3.0 * batch * per * 16.0, s);
    contour_operator_kernel<<<grid_for(per * nops), 256, 0, s>>>(n, batch, nq, r_o, r_i, aji, aii, aij, W);
    QTX_CHECK_LAUNCH();
  }
  QTX_CHECK_CUDA(cudaMemsetAsync(inv_info, 0, sizeof(int) * nops, s));
  MatRef Wm{W, n, per};
  QTX_TRY(zinv_ex(n, nops, Wm, Wm, inv_info, nullptr, scr, scr_bytes, s));
  {
    ProfScope prof(QTX_KERNEL_REDUCE, (double)nops * per * 16.0 + 2.0 * batch * per * 16.0, s);
    contour_moments_kernel<<<grid_for(per * batch), 256, 0, s>>>(n, batch, nq, r_o, r_i, W, q0, q1);
    QTX_CHECK_LAUNCH();
  }
  if (info != nullptr) {
    first_singular_kernel<<<grid_for(batch), 256, 0, s>>>(batch, 2 * nq, inv_info, info);
    QTX_CHECK_LAUNCH();
  }
  return QTX_OK;
}

}  // namespace qtx

using namespace qtx;

extern "C" size_t qtx_beyn_moments_workspace(int n, int64_t batch, int num_quad_points) {
  if (n <= 0 || batch <= 0 || num_quad_points <= 0) return 0;
  return beyn_ws_bytes(n, batch, num_quad_points);
}

extern "C" int qtx_beyn_moments(int n, int64_t batch, qtx_mat a_ji, qtx_mat a_ii, qtx_mat a_ij, double r_o,
                                double r_i, int num_quad_points, qtx_mat q0, qtx_mat q1, int* info,
                                void* workspace, size_t workspace_bytes, qtx_stream stream) {
  try {
    if (n <= 0 || batch <= 0) return QTX_OK;
    if (num_quad_points <= 0 || n > 1024 || a_ji.ptr == nullptr || a_ii.ptr == nullptr ||
        a_ij.ptr == nullptr || q0.ptr == nullptr || q1.ptr == nullptr || !(r_o > 0.0) || !(r_i > 0.0)) {
      set_error("qtx_beyn_moments: invalid arguments");
      return QTX_ERR_ARG;
    }
    const size_t need = beyn_ws_bytes(n, batch, num_quad_points);
    if (workspace == nullptr || workspace_bytes < need) {
      set_error("qtx_beyn_moments: workspace too small (" + std::to_string(workspace_bytes) + " < " +
                std::to_string(need) + " bytes)");
      return QTX_ERR_WORKSPACE;
    }
    Workspace ws;
    ws.base = static_cast<char*>(workspace);
    ws.cap = workspace_bytes;
    return beyn_moments_run(n, batch, from_abi(a_ji), from_abi(a_ii), from_abi(a_ij), r_o, r_i,
                            num_quad_points, from_abi(q0), from_abi(q1), info, ws, (cudaStream_t)stream);
  } catch (const std::exception& e) {
    set_error(std::string("qtx_beyn_moments: internal error: ") + e.what());
    return QTX_ERR_ARG;
  }
}
