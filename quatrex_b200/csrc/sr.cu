// Open-boundary conditions: Sancho-Rubio decimation, the OBCSystem
// fixed-point refinement, contact self-energies and the Caroli
// transmission.
//
// Sancho-Rubio (qttools boundary_conditions/obc/sancho_rubio.py:33-85):
//   inv = eps^-1;  eps -= alpha inv beta + beta inv alpha;
//   eps_s -= alpha inv beta;  alpha = alpha inv alpha;  beta = beta inv beta
// As written that is one inverse and ten products per step; here
// alpha inv and beta inv are formed once and reused (six products), the
// eps_s update is the second output of the alpha inv beta product, and the
// convergence measure ||(|alpha| + |beta|)||_F / 2 is one FP64 reduction
// per energy. Every loop is bounded by max_iterations.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace qtx {

namespace {

const z64 ONE{1.0, 0.0};
const z64 MONE{-1.0, 0.0};

__global__ void fill_int_kernel(int* p, int64_t n, int v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// lesser = -f (S - S^H), greater = -(f - 1) (S - S^H)   (i f Gamma with
// Gamma = i (S - S^H)); 32x32 tiles, S^H staged through shared memory.
__global__ void __launch_bounds__(256) gamma_scale_kernel(int n, int64_t batch, MatRef S,
                                                          const double* occ, MatRef L, MatRef G) {
  __shared__ z64 tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int64_t b = blockIdx.z; b < batch; b += gridDim.z) {
    const z64* s = at<const z64>(S, b);
    __syncthreads();
    for (int i = 0; i < 4; ++i) {
      const int sr = c0 + ty + i * 8, sc = r0 + tx;
      tile[ty + i * 8][tx] = (sr < n && sc < n) ? s[(int64_t)sr * S.ld + sc] : make_double2(0, 0);
    }
    __syncthreads();
    const double f = occ[b];
    for (int i = 0; i < 4; ++i) {
      const int r = r0 + ty + i * 8, c = c0 + tx;
      if (r >= n || c >= n) continue;
      const z64 v = s[(int64_t)r * S.ld + c];
      const z64 w = tile[tx][ty + i * 8];  // S[c][r]
      const z64 d = make_double2(v.x - w.x, v.y + w.y);  // S - S^H
      if (!L.null()) at<z64>(L, b)[(int64_t)r * L.ld + c] = make_double2(-f * d.x, -f * d.y);
      if (!G.null())
        at<z64>(G, b)[(int64_t)r * G.ld + c] = make_double2(-(f - 1.0) * d.x, -(f - 1.0) * d.y);
    }
  }
}

int fill_int(int* p, int64_t n, int v, cudaStream_t s) {
  if (n <= 0) return QTX_OK;
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4096);
  ProfScope prof(QTX_KERNEL_BLOCKOPS, 4.0 * (double)n, s);
  fill_int_kernel<<<blocks, 256, 0, s>>>(p, n, v);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

struct G {
  GemmDesc d;
  G(int M, int N, int K, int64_t batch, MatRef A, MatRef B, MatRef C, z64 alpha = ONE) {
    d.M = M;
    d.N = N;
    d.K = K;
    d.batch = batch;
    d.A = A;
    d.B = B;
    d.C = C;
    d.alpha = alpha;
  }
  G& plus(const MatRef& m, z64 c, int ct = 0) {
    if (!m.null()) d.add[d.nadd++] = Addend{m, c, ct};
    return *this;
  }
  G& second(const MatRef& c3, z64 scale) {
    d.C3 = c3;
    d.scale3 = scale;
    return *this;
  }
  G& plus3(const MatRef& m, z64 c) {
    if (!m.null()) d.add[d.nadd + d.nadd3++] = Addend{m, c, 0};
    return *this;
  }
  G& mask(const int* a) {
    d.active = a;
    return *this;
  }
  int run(cudaStream_t s) { return zgemm(d, s); }
};

}  // namespace

size_t sancho_rubio_ws(int n, int64_t batch) {
  Workspace ws;
  for (int k = 0; k < 10; ++k) ws.mat(n, n, batch);
  ws.take(sizeof(double) * batch);
  ws.take(sizeof(int) * batch);
  ws.take(zinv_scratch_bytes(n, batch));
  ws.take(oz_scratch_bytes(n, n, n, batch, gemm_slices()));
  return ws.off + 256;
}

namespace {

struct SRState {
  MatRef eps, eps_s, alpha[2], beta[2], inv_e, aI, bI, t1;
  double* delta;
  int* active;
  void* scr;  // scratch of the multi-CTA inverse
  size_t scr_bytes;
};

SRState sr_state(int n, int64_t batch, Workspace& ws) {
  SRState st;
  st.eps = ws.mat(n, n, batch);
  st.eps_s = ws.mat(n, n, batch);
  st.alpha[0] = ws.mat(n, n, batch);
  st.alpha[1] = ws.mat(n, n, batch);
  st.beta[0] = ws.mat(n, n, batch);
  st.beta[1] = ws.mat(n, n, batch);
  st.inv_e = ws.mat(n, n, batch);
  st.aI = ws.mat(n, n, batch);
  st.bI = ws.mat(n, n, batch);
  st.t1 = ws.mat(n, n, batch);
  st.delta = static_cast<double*>(ws.take(sizeof(double) * batch));
  st.active = static_cast<int*>(ws.take(sizeof(int) * batch));
  st.scr_bytes = zinv_scratch_bytes(n, batch);
  st.scr = ws.take(st.scr_bytes);
  return st;
}

MatRef offset(const MatRef& m, int64_t entries) {
  MatRef r = m;
  r.p = static_cast<z64*>(m.p) + entries * m.stride;
  return r;
}

// Copies one system's inputs into entries [off, off + batch) of the state.
int sr_load(int n, int64_t batch, int64_t off, const SRState& st, MatRef aii, MatRef aij,
            MatRef aji, cudaStream_t s) {
  Addend t{aii, ONE, 0};
  QTX_TRY(zcombine(n, n, batch, offset(st.eps, off), &t, 1, nullptr, s));
  QTX_TRY(zcombine(n, n, batch, offset(st.eps_s, off), &t, 1, nullptr, s));
  Addend u{aji, ONE, 0};
  QTX_TRY(zcombine(n, n, batch, offset(st.alpha[0], off), &u, 1, nullptr, s));
  Addend v{aij, ONE, 0};
  QTX_TRY(zcombine(n, n, batch, offset(st.beta[0], off), &v, 1, nullptr, s));
  return QTX_OK;
}

// The decimation loop on the whole state; eps_s holds the result.
int sr_iterate(int n, int64_t batch, const SRState& st, int max_iterations, double tol,
               int per_energy, int* iterations, int* converged, int* info, cudaStream_t s) {
  QTX_TRY(fill_int(st.active, batch, 1, s));
  std::vector<double> hdelta(batch);
  std::vector<int> hactive(batch, 1);
  int it = 0, cur = 0;
  bool done = false;
  const int* mask = per_energy ? st.active : nullptr;
  while (it < max_iterations && !done) {
    const int nx = cur ^ 1;
    QTX_TRY(zinv_ex(n, batch, st.eps, st.inv_e, info, mask, st.scr, st.scr_bytes, s));
    QTX_TRY(G(n, n, n, batch, st.alpha[cur], st.inv_e, st.aI).mask(mask).run(s));
    QTX_TRY(G(n, n, n, batch, st.beta[cur], st.inv_e, st.bI).mask(mask).run(s));
    // t1 = alpha inv beta;  eps_s <- eps_s - t1.
    QTX_TRY(G(n, n, n, batch, st.aI, st.beta[cur], st.t1)
                .second(st.eps_s, MONE)
                .plus3(st.eps_s, ONE)
                .mask(mask)
                .run(s));
    // eps <- eps - t1 - beta inv alpha.
    QTX_TRY(G(n, n, n, batch, st.bI, st.alpha[cur], st.eps, MONE)
                .plus(st.eps, ONE)
                .plus(st.t1, MONE)
                .mask(mask)
                .run(s));
    QTX_TRY(G(n, n, n, batch, st.aI, st.alpha[cur], st.alpha[nx]).mask(mask).run(s));
    QTX_TRY(G(n, n, n, batch, st.bI, st.beta[cur], st.beta[nx]).mask(mask).run(s));
    QTX_TRY(sr_delta(n, batch, st.alpha[nx], st.beta[nx], st.delta, mask, s));
    ++it;
    QTX_CHECK_CUDA(cudaMemcpyAsync(hdelta.data(), st.delta, sizeof(double) * batch,
                                   cudaMemcpyDeviceToHost, s));
    QTX_CHECK_CUDA(cudaStreamSynchronize(s));
    cur = nx;
    if (per_energy) {
      int remaining = 0;
      bool changed = false;
      for (int64_t b = 0; b < batch; ++b) {
        if (!hactive[b]) continue;
        if (hdelta[b] < tol) {
          hactive[b] = 0;
          changed = true;
        } else {
          ++remaining;
        }
      }
      if (remaining == 0) done = true;
      if (changed && !done) {
        QTX_CHECK_CUDA(cudaMemcpyAsync(st.active, hactive.data(), sizeof(int) * batch,
                                       cudaMemcpyHostToDevice, s));
        QTX_CHECK_CUDA(cudaStreamSynchronize(s));
      }
    } else {
      double mx = 0.0;
      for (int64_t b = 0; b < batch; ++b) mx = std::max(mx, hdelta[b]);
      if (mx < tol) done = true;
    }
  }
  if (iterations) *iterations = it;
  if (converged) *converged = done ? 1 : 0;
  return QTX_OK;
}

// Device-side convergence bookkeeping of one decimation step (one CTA):
// per-energy mode retires entries whose delta is below tol; batch-wide mode
// retires all once the largest active delta is below tol. Counts the step
// if any entry was still active and records whether all have converged.
__global__ void __launch_bounds__(256) sr_update_kernel(int64_t batch, const double* delta, int* active,
                                                         double tol, int per_energy, int* iters,
                                                         int* converged) {
  __shared__ double s_max[8];
  __shared__ int s_any[8], s_left[8];
  double mx = 0.0;
  int any = 0;
  for (int64_t b = threadIdx.x; b < batch; b += blockDim.x)
    if (active[b]) {
      any = 1;
      mx = fmax(mx, delta[b]);
    }
  for (int off = 16; off > 0; off >>= 1) {
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    any |= __shfl_xor_sync(0xffffffffu, any, off);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    s_max[w] = mx;
    s_any[w] = any;
  }
  __syncthreads();
  mx = 0.0;
  any = 0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
    mx = fmax(mx, s_max[k]);
    any |= s_any[k];
  }
  int left = 0;
  for (int64_t b = threadIdx.x; b < batch; b += blockDim.x) {
    if (!active[b]) continue;
    const bool done = per_energy ? (delta[b] < tol) : (mx < tol);
    if (done)
      active[b] = 0;
    else
      ++left;
  }
  for (int off = 16; off > 0; off >>= 1) left += __shfl_xor_sync(0xffffffffu, left, off);
  __syncthreads();
  if (l == 0) s_left[w] = left;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tot += s_left[k];
    if (any) *iters += 1;
    *converged = (tot == 0) ? 1 : 0;
  }
}

// Host-sync-free decimation: max_iterations steps are enqueued; once every
// entry has retired the remaining steps' kernels find no active entry and
// return at once. d_iters / d_converged are device ints.
int sr_iterate_async(int n, int64_t batch, const SRState& st, int max_iterations, double tol,
                     int per_energy, int* d_iters, int* d_converged, int* info, cudaStream_t s) {
  QTX_TRY(fill_int(st.active, batch, 1, s));
  QTX_TRY(fill_int(d_iters, 1, 0, s));
  QTX_TRY(fill_int(d_converged, 1, 0, s));
  int cur = 0;
  const int* mask = st.active;
  for (int it = 0; it < max_iterations; ++it) {
    const int nx = cur ^ 1;
    QTX_TRY(zinv_ex(n, batch, st.eps, st.inv_e, info, mask, st.scr, st.scr_bytes, s));
    QTX_TRY(G(n, n, n, batch, st.alpha[cur], st.inv_e, st.aI).mask(mask).run(s));
    QTX_TRY(G(n, n, n, batch, st.beta[cur], st.inv_e, st.bI).mask(mask).run(s));
    QTX_TRY(G(n, n, n, batch, st.aI, st.beta[cur], st.t1)
                .second(st.eps_s, MONE)
                .plus3(st.eps_s, ONE)
                .mask(mask)
                .run(s));
    QTX_TRY(G(n, n, n, batch, st.bI, st.alpha[cur], st.eps, MONE)
                .plus(st.eps, ONE)
                .plus(st.t1, MONE)
                .mask(mask)
                .run(s));
    QTX_TRY(G(n, n, n, batch, st.aI, st.alpha[cur], st.alpha[nx]).mask(mask).run(s));
    QTX_TRY(G(n, n, n, batch, st.bI, st.beta[cur], st.beta[nx]).mask(mask).run(s));
    QTX_TRY(sr_delta(n, batch, st.alpha[nx], st.beta[nx], st.delta, mask, s));
    {
      ProfScope prof(QTX_KERNEL_REDUCE, 12.0 * (double)batch, s);
      sr_update_kernel<<<1, 256, 0, s>>>(batch, st.delta, st.active, tol, per_energy, d_iters,
                                         d_converged);
      QTX_CHECK_LAUNCH();
    }
    cur = nx;
  }
  // Entries retired in different steps left their newest alpha/beta in
  // different buffers; eps_s (updated in place) is all that is read next.
  return QTX_OK;
}

}  // namespace

int sancho_rubio_multi_async_run(int n, int nsys, const int64_t* batches, const qtx_mat* aii,
                                 const qtx_mat* aij, const qtx_mat* aji, const qtx_mat* x,
                                 int max_iterations, double tol, int per_energy, int* d_iters,
                                 int* d_converged, int* info, Workspace& ws, cudaStream_t s) {
  int64_t total = 0;
  for (int k = 0; k < nsys; ++k) total += batches[k];
  SRState st = sr_state(n, total, ws);
  OzScope oz(ws, n, total);
  if (ws.overflow) {
    set_error("sancho_rubio_multi_async: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  int64_t off = 0;
  for (int k = 0; k < nsys; ++k) {
    QTX_TRY(sr_load(n, batches[k], off, st, from_abi(aii[k]), from_abi(aij[k]), from_abi(aji[k]), s));
    off += batches[k];
  }
  QTX_TRY(sr_iterate_async(n, total, st, max_iterations, tol, per_energy, d_iters, d_converged, info, s));
  off = 0;
  for (int k = 0; k < nsys; ++k) {
    QTX_TRY(zinv_ex(n, batches[k], offset(st.eps_s, off), from_abi(x[k]), info ? info + off : nullptr,
                    nullptr, st.scr, st.scr_bytes, s));
    off += batches[k];
  }
  return QTX_OK;
}

int sancho_rubio_run(int n, int64_t batch, MatRef aii, MatRef aij, MatRef aji, MatRef x,
                     int max_iterations, double tol, int per_energy, int* iterations,
                     int* converged, double* delta_out, int* info, Workspace& ws, cudaStream_t s) {
  SRState st = sr_state(n, batch, ws);
  OzScope oz(ws, n, batch);
  if (ws.overflow) {
    set_error("sancho_rubio: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  QTX_TRY(sr_load(n, batch, 0, st, aii, aij, aji, s));
  QTX_TRY(sr_iterate(n, batch, st, max_iterations, tol, per_energy, iterations, converged, info, s));
  if (delta_out)
    QTX_CHECK_CUDA(cudaMemcpyAsync(delta_out, st.delta, sizeof(double) * batch,
                                   cudaMemcpyDeviceToDevice, s));
  QTX_TRY(zinv_ex(n, batch, st.eps_s, x, info, nullptr, st.scr, st.scr_bytes, s));
  return QTX_OK;
}

int sancho_rubio_multi_run(int n, int nsys, const int64_t* batches, const qtx_mat* aii,
                           const qtx_mat* aij, const qtx_mat* aji, const qtx_mat* x,
                           int max_iterations, double tol, int per_energy, int* iterations,
                           int* converged, int* info, Workspace& ws, cudaStream_t s) {
  int64_t total = 0;
  for (int k = 0; k < nsys; ++k) total += batches[k];
  SRState st = sr_state(n, total, ws);
  OzScope oz(ws, n, total);
  if (ws.overflow) {
    set_error("sancho_rubio_multi: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  int64_t off = 0;
  for (int k = 0; k < nsys; ++k) {
    QTX_TRY(sr_load(n, batches[k], off, st, from_abi(aii[k]), from_abi(aij[k]), from_abi(aji[k]), s));
    off += batches[k];
  }
  QTX_TRY(sr_iterate(n, total, st, max_iterations, tol, per_energy, iterations, converged, info, s));
  off = 0;
  for (int k = 0; k < nsys; ++k) {
    QTX_TRY(zinv_ex(n, batches[k], offset(st.eps_s, off), from_abi(x[k]),
                    info ? info + off : nullptr, nullptr, st.scr, st.scr_bytes, s));
    off += batches[k];
  }
  return QTX_OK;
}

size_t obc_refine_ws(int n, int64_t batch) {
  Workspace ws;
  for (int k = 0; k < 2; ++k) ws.mat(n, n, batch);
  ws.take(zinv_scratch_bytes(n, batch));
  ws.take(oz_scratch_bytes(n, n, n, batch, gemm_slices()));
  return ws.off + 256;
}

int obc_refine_run(int n, int64_t batch, MatRef aii, MatRef aij, MatRef aji, MatRef x, MatRef xref,
                   double* rel, double* abs_res, int* info, Workspace& ws, cudaStream_t s) {
  MatRef T = ws.mat(n, n, batch), S = ws.mat(n, n, batch);
  const size_t scr_bytes = zinv_scratch_bytes(n, batch);
  void* scr = ws.take(scr_bytes);
  OzScope oz(ws, n, batch);
  if (ws.overflow) {
    set_error("obc_refine: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  QTX_TRY(G(n, n, n, batch, aji, x, T).run(s));
  QTX_TRY(G(n, n, n, batch, T, aij, S, MONE).plus(aii, ONE).run(s));
  QTX_TRY(zinv_ex(n, batch, S, S, info, nullptr, scr, scr_bytes, s));
  QTX_TRY(znorm_diff(n, batch, S, x, abs_res, nullptr, rel, s));
  Addend t{S, ONE, 0};
  QTX_TRY(zcombine(n, n, batch, xref, &t, 1, nullptr, s));
  return QTX_OK;
}

size_t contact_ws(int n, int64_t batch) {
  Workspace ws;
  ws.mat(n, n, batch);
  ws.mat(n, n, batch);
  ws.take(oz_scratch_bytes(n, n, n, batch, gemm_slices()));
  return ws.off + 256;
}

int contact_run(int n, int64_t batch, MatRef aij, MatRef aji, MatRef g, const double* occ,
                MatRef sigma, MatRef sl, MatRef sg, Workspace& ws, cudaStream_t s) {
  MatRef T = ws.mat(n, n, batch);
  MatRef Sg = sigma.null() ? ws.mat(n, n, batch) : sigma;
  OzScope oz(ws, n, batch);
  if (ws.overflow) {
    set_error("contact_self_energy: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  QTX_TRY(G(n, n, n, batch, aji, g, T).run(s));
  QTX_TRY(G(n, n, n, batch, T, aij, Sg).run(s));
  if (!sl.null() || !sg.null()) {
    if (occ == nullptr) {
      set_error("contact_self_energy: occupancies required for lesser/greater outputs");
      return QTX_ERR_ARG;
    }
    dim3 grid((n + 31) / 32, (n + 31) / 32, (unsigned)std::min<int64_t>(batch, 65535));
    ProfScope prof(QTX_KERNEL_BLOCKOPS, 48.0 * n * n * (double)batch, s);
    gamma_scale_kernel<<<grid, dim3(32, 8), 0, s>>>(n, batch, Sg, occ, sl, sg);
    QTX_CHECK_LAUNCH();
  }
  return QTX_OK;
}

size_t transmission_ws(int m, int n, int64_t batch) {
  Workspace ws;
  const int bm = std::max(m, n);
  for (int k = 0; k < 4; ++k) ws.mat(bm, bm, batch);
  return ws.off + 256;
}

int transmission_run(int m, int n, int64_t batch, MatRef g0n, MatRef sl, MatRef sr, double* T,
                     Workspace& ws, cudaStream_t s) {
  const int bm = std::max(m, n);
  MatRef GL = ws.mat(bm, bm, batch), GR = ws.mat(bm, bm, batch);
  MatRef P1 = ws.mat(bm, bm, batch), P2 = ws.mat(bm, bm, batch);
  if (ws.overflow) {
    set_error("transmission: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  GL.ld = m;
  GR.ld = n;
  P1.ld = n;
  P2.ld = n;
  const z64 I{0.0, 1.0}, MI{0.0, -1.0};
  Addend tl[2] = {Addend{sl, I, 0}, Addend{sl, MI, 1}};
  QTX_TRY(zcombine(m, m, batch, GL, tl, 2, nullptr, s));
  Addend tr[2] = {Addend{sr, I, 0}, Addend{sr, MI, 1}};
  QTX_TRY(zcombine(n, n, batch, GR, tr, 2, nullptr, s));
  QTX_TRY(G(m, n, m, batch, GL, g0n, P1).run(s));
  QTX_TRY(G(m, n, n, batch, P1, GR, P2).run(s));
  QTX_TRY(zre_inner(m, n, batch, P2, g0n, T, s));
  return QTX_OK;
}

}  // namespace qtx
