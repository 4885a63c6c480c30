// Memory-bound block kernels of the NEGF path: elementwise combinations
// with conjugate transposes, the anti-Hermitian projection of X^<, X^> with
// the density epilogue, traces of products (Meir-Wingreen current), the
// per-energy norms of the Sancho-Rubio convergence test and OBC residuals,
// and complex128 <-> complex64 conversion.
//
// The elementwise kernels and traces are templates over the stored element
// type (complex128 = double2 for the FP64 path, complex64 = float2 for the
// mixed path); arithmetic is done in double either way. Transposed operands
// are staged through a 32x32 shared-memory tile (one padding column) so
// global loads and stores stay coalesced. Reductions use warp shuffles and
// one shared-memory combine per CTA; one CTA reduces one stack entry, so
// results are deterministic.
#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace qtx {
namespace {

constexpr int TILE = 32;
constexpr int ROWS = 8;  // threads per tile column: block = 32 x 8

__device__ __forceinline__ z64 ld2(const double2& v) { return v; }
__device__ __forceinline__ z64 ld2(const float2& v) { return make_double2(v.x, v.y); }
template <typename T>
__device__ __forceinline__ T st2(z64 v);
template <>
__device__ __forceinline__ double2 st2<double2>(z64 v) {
  return v;
}
template <>
__device__ __forceinline__ float2 st2<float2>(z64 v) {
  return make_float2((float)v.x, (float)v.y);
}

struct CombineArgs {
  MatRef out;
  Addend t[kMaxAddends];
  int nterms;
  int m, n;
  int64_t batch;
  const int* active;
};

// out = sum_t coef_t op_t(X_t) on 32x32 tiles; grid (tiles_n, tiles_m, batch).
template <typename T>
__global__ void __launch_bounds__(TILE* ROWS) combine_kernel(const CombineArgs a) {
  __shared__ z64 tile[TILE][TILE + 1];
  const int c0 = blockIdx.x * TILE, r0 = blockIdx.y * TILE;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int64_t b = blockIdx.z; b < a.batch; b += gridDim.z) {
    if (a.active != nullptr && a.active[b] == 0) continue;
    z64 acc[TILE / ROWS];
#pragma unroll
    for (int i = 0; i < TILE / ROWS; ++i) acc[i] = make_double2(0.0, 0.0);
    for (int t = 0; t < a.nterms; ++t) {
      const Addend& ad = a.t[t];
      const T* p = at<const T>(ad.m, b);
      if (!ad.conj_trans) {
#pragma unroll
        for (int i = 0; i < TILE / ROWS; ++i) {
          const int r = r0 + ty + i * ROWS, c = c0 + tx;
          if (r < a.m && c < a.n) acc[i] = zfma(ad.coef, ld2(p[(int64_t)r * ad.m.ld + c]), acc[i]);
        }
      } else {
        // op(X)[r][c] = conj(X[c][r]): load the (c0, r0) tile of X coalesced.
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TILE / ROWS; ++i) {
          const int xr = c0 + ty + i * ROWS, xc = r0 + tx;  // X row = out col
          tile[ty + i * ROWS][tx] =
              (xr < a.n && xc < a.m) ? ld2(p[(int64_t)xr * ad.m.ld + xc]) : make_double2(0.0, 0.0);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TILE / ROWS; ++i) {
          const int r = r0 + ty + i * ROWS, c = c0 + tx;
          if (r < a.m && c < a.n) acc[i] = zfma(ad.coef, zconj(tile[tx][ty + i * ROWS]), acc[i]);
        }
      }
    }
    T* o = at<T>(a.out, b);
#pragma unroll
    for (int i = 0; i < TILE / ROWS; ++i) {
      const int r = r0 + ty + i * ROWS, c = c0 + tx;
      if (r < a.m && c < a.n) o[(int64_t)r * a.out.ld + c] = st2<T>(acc[i]);
    }
  }
}

// out = 0.5 (X - X^H); density[b * ds + off + r] = Im X[r][r].
template <typename T>
__global__ void __launch_bounds__(TILE* ROWS)
    antiherm_kernel(int n, int64_t batch, MatRef X, MatRef out, double* dens, int64_t ds,
                    int64_t doff) {
  __shared__ z64 tile[TILE][TILE + 1];
  const int c0 = blockIdx.x * TILE, r0 = blockIdx.y * TILE;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int64_t b = blockIdx.z; b < batch; b += gridDim.z) {
    const T* x = at<const T>(X, b);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < TILE / ROWS; ++i) {
      const int xr = c0 + ty + i * ROWS, xc = r0 + tx;
      tile[ty + i * ROWS][tx] = (xr < n && xc < n) ? ld2(x[(int64_t)xr * X.ld + xc]) : make_double2(0, 0);
    }
    __syncthreads();
    T* o = out.null() ? nullptr : at<T>(out, b);
#pragma unroll
    for (int i = 0; i < TILE / ROWS; ++i) {
      const int r = r0 + ty + i * ROWS, c = c0 + tx;
      if (r < n && c < n) {
        const z64 v = ld2(x[(int64_t)r * X.ld + c]);
        const z64 w = tile[tx][ty + i * ROWS];  // X[c][r]
        const z64 h = make_double2(0.5 * (v.x - w.x), 0.5 * (v.y + w.y));
        if (o != nullptr) o[(int64_t)r * out.ld + c] = st2<T>(h);
        if (dens != nullptr && r == c) dens[b * ds + doff + r] = h.y;
      }
    }
  }
}

template <typename V>
__device__ __forceinline__ V block_sum(V v, V* red) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  V s = 0;
  const int nw = blockDim.x >> 5;
  for (int w = 0; w < nw; ++w) s += red[w];
  return s;
}

// Tr(X Y) = sum_{r,c} X[r][c] Y[c][r], via 32x32 tiles (Y tile staged
// transposed). A stack entry is reduced by the S CTAs of one thread-block
// cluster (S = 1 for large batches): CTA s takes the row tiles s, s + S, ...
// and the S partial sums are added in rank order by rank 0 through
// distributed shared memory, so the result does not depend on timing.
template <typename T>
__global__ void __launch_bounds__(256) trace_kernel(int n, int64_t batch, MatRef X, MatRef Y, z64 coef,
                                                    z64* res, int64_t rs, int64_t roff, int accumulate) {
  __shared__ z64 tile[TILE][TILE + 1];
  __shared__ double red[8];
  __shared__ double part[2];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  cg::cluster_group cluster = cg::this_cluster();
  const int S = (int)cluster.num_blocks(), rank = (int)cluster.block_rank();
  const int64_t b = blockIdx.x / S;  // uniform within a cluster
  if (b < batch) {
    const T* x = at<const T>(X, b);
    const T* y = at<const T>(Y, b);
    double sre = 0.0, sim = 0.0;
    for (int r0 = rank * TILE; r0 < n; r0 += S * TILE)
      for (int c0 = 0; c0 < n; c0 += TILE) {
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TILE / ROWS; ++i) {
          const int yr = c0 + ty + i * ROWS, yc = r0 + tx;
          tile[ty + i * ROWS][tx] =
              (yr < n && yc < n) ? ld2(y[(int64_t)yr * Y.ld + yc]) : make_double2(0, 0);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < TILE / ROWS; ++i) {
          const int r = r0 + ty + i * ROWS, c = c0 + tx;
          if (r < n && c < n) {
            const z64 a = ld2(x[(int64_t)r * X.ld + c]);
            const z64 w = tile[tx][ty + i * ROWS];  // Y[c][r]
            sre += a.x * w.x - a.y * w.y;
            sim += a.x * w.y + a.y * w.x;
          }
        }
      }
    sre = block_sum(sre, red);
    sim = block_sum(sim, red);
    if (threadIdx.x == 0) {
      part[0] = sre;
      part[1] = sim;
    }
  }
  cluster.sync();
  if (b < batch && rank == 0 && threadIdx.x == 0) {
    double tre = 0.0, tim = 0.0;
    for (int q = 0; q < S; ++q) {
      const double* pq = cluster.map_shared_rank(part, q);
      tre += pq[0];
      tim += pq[1];
    }
    const z64 v = zmul(coef, make_double2(tre, tim));
    z64* o = res + b * rs + roff;
    *o = accumulate ? zadd(*o, v) : v;
  }
  cluster.sync();  // the partials stay readable until rank 0 has summed them
}

// delta[b] = sqrt(sum (|x| + |y|)^2) / 2.
__global__ void __launch_bounds__(256) sr_delta_kernel(int n, int64_t batch, MatRef X, MatRef Y,
                                                       double* delta, const int* active) {
  __shared__ double red[8];
  for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
    if (active != nullptr && active[b] == 0) continue;
    const z64* x = at<const z64>(X, b);
    const z64* y = at<const z64>(Y, b);
    double s = 0.0;
    for (int64_t idx = threadIdx.x; idx < (int64_t)n * n; idx += blockDim.x) {
      const int r = (int)(idx / n), c = (int)(idx % n);
      const z64 a = x[(int64_t)r * X.ld + c];
      const z64 w = y[(int64_t)r * Y.ld + c];
      const double v = hypot(a.x, a.y) + hypot(w.x, w.y);
      s += v * v;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) delta[b] = 0.5 * sqrt(s);
  }
}

__global__ void __launch_bounds__(256) znorm_diff_kernel(int n, int64_t batch, MatRef X, MatRef Y,
                                                         double* nd, double* nx, double* rel) {
  __shared__ double red[8];
  for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
    const z64* x = at<const z64>(X, b);
    const z64* y = at<const z64>(Y, b);
    double sd = 0.0, sx = 0.0;
    for (int64_t idx = threadIdx.x; idx < (int64_t)n * n; idx += blockDim.x) {
      const int r = (int)(idx / n), c = (int)(idx % n);
      const z64 a = x[(int64_t)r * X.ld + c];
      const z64 w = y[(int64_t)r * Y.ld + c];
      const double dr = a.x - w.x, di = a.y - w.y;
      sd += dr * dr + di * di;
      sx += a.x * a.x + a.y * a.y;
    }
    sd = block_sum(sd, red);
    sx = block_sum(sx, red);
    if (threadIdx.x == 0) {
      if (nd != nullptr) nd[b] = sqrt(sd);
      if (nx != nullptr) nx[b] = sqrt(sx);
      if (rel != nullptr) rel[b] = sqrt(sd) / sqrt(sx);
    }
  }
}

// out[b] = Re sum conj(G) .* P  (= Re Tr(P G^H)).
template <typename T>
__global__ void __launch_bounds__(256) re_inner_kernel(int m, int n, int64_t batch, MatRef P, MatRef G,
                                                       double* out) {
  __shared__ double red[8];
  for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
    const T* p = at<const T>(P, b);
    const T* g = at<const T>(G, b);
    double s = 0.0;
    for (int64_t idx = threadIdx.x; idx < (int64_t)m * n; idx += blockDim.x) {
      const int r = (int)(idx / n), c = (int)(idx % n);
      const z64 a = ld2(p[(int64_t)r * P.ld + c]);
      const z64 w = ld2(g[(int64_t)r * G.ld + c]);
      s += a.x * w.x + a.y * w.y;
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[b] = s;
  }
}

template <typename TI, typename TO>
__global__ void convert_kernel(int m, int n, int64_t batch, MatRef in, MatRef out) {
  const int64_t per = (int64_t)m * n, total = per * batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / per, e = i % per;
    const int r = (int)(e / n), c = (int)(e % n);
    at<TO>(out, b)[(int64_t)r * out.ld + c] = st2<TO>(ld2(at<const TI>(in, b)[(int64_t)r * in.ld + c]));
  }
}

unsigned grid_z(int64_t batch) { return (unsigned)(batch < 65535 ? batch : 65535); }
unsigned grid_x(int64_t batch) { return (unsigned)(batch < 1048576 ? batch : 1048576); }

template <typename T>
int combine_t(int m, int n, int64_t batch, MatRef out, const Addend* terms, int nterms,
              const int* active, cudaStream_t s) {
  if (m <= 0 || n <= 0 || batch <= 0) return QTX_OK;
  CombineArgs a{};
  a.out = out;
  a.m = m;
  a.n = n;
  a.batch = batch;
  a.active = active;
  a.nterms = 0;
  for (int t = 0; t < nterms; ++t) {
    if (terms[t].m.null()) continue;
    if (a.nterms >= kMaxAddends) {
      set_error("combine: too many terms");
      return QTX_ERR_ARG;
    }
    a.t[a.nterms++] = terms[t];
  }
  dim3 grid((n + TILE - 1) / TILE, (m + TILE - 1) / TILE, grid_z(batch));
  ProfScope prof(QTX_KERNEL_BLOCKOPS, (double)sizeof(T) * m * n * (double)batch * (a.nterms + 1), s);
  combine_kernel<T><<<grid, dim3(TILE, ROWS), 0, s>>>(a);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

template <typename T>
int antiherm_t(int n, int64_t batch, MatRef X, MatRef out, double* density, int64_t dens_stride,
               int64_t dens_off, cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  dim3 grid((n + TILE - 1) / TILE, (n + TILE - 1) / TILE, grid_z(batch));
  ProfScope prof(QTX_KERNEL_BLOCKOPS, 2.0 * sizeof(T) * n * n * (double)batch, s);
  antiherm_kernel<T><<<grid, dim3(TILE, ROWS), 0, s>>>(n, batch, X, out, density, dens_stride, dens_off);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

template <typename T>
int trace_t(int n, int64_t batch, MatRef X, MatRef Y, z64 coef, z64* result, int64_t rstride,
            int64_t roff, int accumulate, cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  ProfScope prof(QTX_KERNEL_REDUCE, 2.0 * sizeof(T) * n * n * (double)batch, s);
  // CTAs per stack entry: enough for two waves of the SMs, at most 8 (a
  // portable cluster) and at most one per 32-row tile.
  int S = 1;
  while (S < 8 && (int64_t)S * 2 * batch <= 2 * 148 && S * TILE < n) S *= 2;
  if ((int64_t)batch * S > 0x7fffffffll) S = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(batch * S), 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = S;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  QTX_CHECK_CUDA(cudaLaunchKernelEx(&cfg, trace_kernel<T>, n, batch, X, Y, coef, result, rstride, roff, accumulate));
  return QTX_OK;
}

template <typename T>
int re_inner_t(int m, int n, int64_t batch, MatRef P, MatRef G, double* out, cudaStream_t s) {
  if (m <= 0 || n <= 0 || batch <= 0) return QTX_OK;
  ProfScope prof(QTX_KERNEL_REDUCE, 2.0 * sizeof(T) * m * n * (double)batch, s);
  re_inner_kernel<T><<<grid_x(batch), 256, 0, s>>>(m, n, batch, P, G, out);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

template <typename TI, typename TO>
int convert_t(int m, int n, int64_t batch, MatRef in, MatRef out, cudaStream_t s) {
  if (m <= 0 || n <= 0 || batch <= 0) return QTX_OK;
  const int64_t total = (int64_t)m * n * batch;
  const int64_t want = (total + 255) / 256;
  const unsigned blocks = (unsigned)(want < 148 * 64 ? want : 148 * 64);
  ProfScope prof(QTX_KERNEL_FORMAT, (double)(sizeof(TI) + sizeof(TO)) * (double)total, s);
  convert_kernel<TI, TO><<<blocks, 256, 0, s>>>(m, n, batch, in, out);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

}  // namespace

int zcombine(int m, int n, int64_t batch, MatRef out, const Addend* terms, int nterms,
             const int* active, cudaStream_t s) {
  return combine_t<double2>(m, n, batch, out, terms, nterms, active, s);
}
int ccombine(int m, int n, int64_t batch, MatRef out, const Addend* terms, int nterms,
             const int* active, cudaStream_t s) {
  return combine_t<float2>(m, n, batch, out, terms, nterms, active, s);
}

int zantiherm(int n, int64_t batch, MatRef X, MatRef out, double* density, int64_t dens_stride,
              int64_t dens_off, cudaStream_t s) {
  return antiherm_t<double2>(n, batch, X, out, density, dens_stride, dens_off, s);
}
int cantiherm(int n, int64_t batch, MatRef X, MatRef out, double* density, int64_t dens_stride,
              int64_t dens_off, cudaStream_t s) {
  return antiherm_t<float2>(n, batch, X, out, density, dens_stride, dens_off, s);
}

int ztrace_prod(int n, int64_t batch, MatRef X, MatRef Y, z64 coef, z64* result, int64_t rstride,
                int64_t roff, int accumulate, cudaStream_t s) {
  return trace_t<double2>(n, batch, X, Y, coef, result, rstride, roff, accumulate, s);
}
int ctrace_prod(int n, int64_t batch, MatRef X, MatRef Y, z64 coef, z64* result, int64_t rstride,
                int64_t roff, int accumulate, cudaStream_t s) {
  return trace_t<float2>(n, batch, X, Y, coef, result, rstride, roff, accumulate, s);
}

int sr_delta(int n, int64_t batch, MatRef X, MatRef Y, double* delta, const int* active,
             cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  ProfScope prof(QTX_KERNEL_REDUCE, 32.0 * n * n * (double)batch, s);
  sr_delta_kernel<<<grid_x(batch), 256, 0, s>>>(n, batch, X, Y, delta, active);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

int znorm_diff(int n, int64_t batch, MatRef X, MatRef Y, double* nrm_diff, double* nrm,
               double* rel, cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  ProfScope prof(QTX_KERNEL_REDUCE, 32.0 * n * n * (double)batch, s);
  znorm_diff_kernel<<<grid_x(batch), 256, 0, s>>>(n, batch, X, Y, nrm_diff, nrm, rel);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

int zre_inner(int m, int n, int64_t batch, MatRef P, MatRef G, double* out, cudaStream_t s) {
  return re_inner_t<double2>(m, n, batch, P, G, out, s);
}
int cre_inner(int m, int n, int64_t batch, MatRef P, MatRef G, double* out, cudaStream_t s) {
  return re_inner_t<float2>(m, n, batch, P, G, out, s);
}

int convert_c64_to_c128(int m, int n, int64_t batch, MatRef in, MatRef out, cudaStream_t s) {
  return convert_t<float2, double2>(m, n, batch, in, out, s);
}
int convert_c128_to_c64(int m, int n, int64_t batch, MatRef in, MatRef out, cudaStream_t s) {
  return convert_t<double2, float2>(m, n, batch, in, out, s);
}

}  // namespace qtx
