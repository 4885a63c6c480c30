// Batched complex128 inverse with the whole matrix on chip: one thread-block
// cluster per matrix, Gauss-Jordan with partial pivoting in distributed
// shared memory.
//
// Replaces the same batched inverse of qttools kernels/linalg/inv.py:6-40 as
// zinv.cu (numpy.linalg.inv / cupy.linalg.solve(a, I)), with the same pivot
// rule (largest |Re| + |Im| at or below the diagonal, lowest row on ties) and
// the same info convention (1-based column of the first zero pivot).
//
// Why: the one-CTA kernel streams the n x n matrix through HBM once per
// 16-column panel (16 passes at n = 256) and takes ~1.7 ms per matrix; the
// multi-CTA path pays three launches per panel. For batches below a few
// times the number of clusters the device can hold, a cluster of
// C = ceil(n / 32) CTAs (8 at n = 256) holds the matrix entirely in shared
// memory -- 32 columns per CTA -- and runs every panel on chip:
//
//   load:   each CTA fetches its 32 columns with TMA (cp.async.bulk.tensor,
//           3-D tensor map over (re/im doubles, rows, batch), 128-byte
//           swizzle, no multicast) into four [rows][8 complex] chunks;
//   panel:  the CTA owning the 16 columns of panel K factors them in place
//           (pivot search, Smith reciprocal, elimination of every row), then
//           arrives on the cluster barrier;
//   update: every CTA reads the panel transform T = X[:, K] and the pivot
//           rows from the owner's shared memory (DSMEM), applies the row
//           interchanges to its own columns and updates them,
//             X[r, J] = (r in K ? 0 : X[r, J]) + T[r, :] X[K, J],
//           with FP64 tensor-core MMAs (mma.sync m16n8k4, 4M complex split);
//   store:  columns are gathered back through DSMEM in the inverse column
//           order of the pivoting and written with coalesced stores.
//
// HBM traffic is the algorithmic minimum (read and write the matrix once).
// One cluster barrier per panel; the owner of the next panel factors it as
// soon as its own update is done while the other CTAs finish theirs.
// Every wait on the TMA mbarrier is bounded: on a time-out the CTA records
// the error (qtx_zinv_cluster_status), keeps taking part in every cluster
// barrier so that no CTA of the cluster waits forever, and its results are
// not to be used.
#include <cooperative_groups.h>
#include <cuda.h>

#include <mutex>

#include "common.cuh"
#include "gj_panel.cuh"

namespace cg = cooperative_groups;

namespace qtx {

__device__ int g_zinv_cluster_error = 0;

namespace {

constexpr int CW = 32;          // columns per CTA
constexpr int CNB = 16;         // panel width
constexpr int CT = 512;         // threads per CTA
constexpr int CWARPS = CT / 32;
constexpr int YS = CW + 2;      // Y row stride (complex)
constexpr long long kWait = 1ll << 26;

__device__ __forceinline__ void mma_f64(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ uint32_t saddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// Element (r, j) of a CTA's 32 columns: four chunks of [npad rows][8
// complex], 16-byte unit swizzled with the row (the TMA SWIZZLE_128B layout).
__device__ __forceinline__ int xoff(int npad, int r, int j) {
  return (j >> 3) * (npad * 8) + r * 8 + ((j & 7) ^ (r & 7));
}

struct ClusterSmem {
  // byte offsets inside the dynamic shared memory (base aligned to 1024)
  int npad;
  size_t x, t, y, piv, colsrc, red_v, red_i, bar, total;
  __host__ __device__ explicit ClusterSmem(int n) {
    npad = (n + 15) & ~15;
    x = 0;                                                  // 4 chunks [npad][8]
    t = x + (size_t)4 * npad * 8 * sizeof(z64);             // 2 chunks [npad][8]
    y = t + (size_t)2 * npad * 8 * sizeof(z64);             // [CNB][YS]
    piv = y + (size_t)CNB * YS * sizeof(z64);               // npad ints
    colsrc = piv + (size_t)npad * sizeof(int);              // npad ints
    red_v = colsrc + (size_t)npad * sizeof(int);
    red_i = red_v + (size_t)CWARPS * sizeof(double);
    bar = (red_i + (size_t)CWARPS * sizeof(int) + 15) & ~(size_t)15;  // 2 mbarriers
    total = bar + 16 + 1024;  // + alignment slack of the base
  }
};

__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (long long it = 0; it < kWait; ++it) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(saddr(bar)), "r"(parity));
    if (done) return true;
  }
  return false;
}

template <int C>
__global__ void __launch_bounds__(CT, 1)
    zinv_cluster_kernel(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active,
                        const __grid_constant__ CUtensorMap tmap, int use_tma) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int64_t b = blockIdx.x / C;
  if (b >= batch) return;  // whole clusters only: blockIdx.x / C is uniform in a cluster
  if (active != nullptr && active[b] == 0) return;

  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const ClusterSmem L(n);
  const int npad = L.npad;
  z64* Xs = reinterpret_cast<z64*>(base + L.x);
  z64* Ts = reinterpret_cast<z64*>(base + L.t);
  z64* Ys = reinterpret_cast<z64*>(base + L.y);
  int* pivrow = reinterpret_cast<int*>(base + L.piv);
  int* colsrc = reinterpret_cast<int*>(base + L.colsrc);
  double* red_v = reinterpret_cast<double*>(base + L.red_v);
  int* red_i = reinterpret_cast<int*>(base + L.red_i);
  uint64_t* lbar = reinterpret_cast<uint64_t*>(base + L.bar);  // the load of A
  uint64_t* tbar = lbar + 1;                                    // the panel transforms
  __shared__ int s_sing, s_first;
  __shared__ z64 prow[CNB], rowk[CNB];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int col0 = rank * CW;  // first global column of this CTA
  const size_t chunk = (size_t)npad * 8;  // complex elements per 8-column chunk

  // ---- load this CTA's 32 columns --------------------------------------
  if (tid == 0) {
    s_sing = 0;
    s_first = 0x7fffffff;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(saddr(lbar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(saddr(tbar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  __syncthreads();
  if (use_tma) {
    if (tid == 0) {
      const uint32_t bytes = 4u * (uint32_t)n * 128u;
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(lbar)), "r"(bytes)
                   : "memory");
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int x = 2 * (col0 + 8 * i);  // in doubles: 16-byte aligned
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(saddr(Xs + i * chunk)),
            "l"(&tmap), "r"(x), "r"(0), "r"((int)b), "r"(saddr(lbar))
            : "memory");
      }
    }
    if (warp == 0 && !mbar_wait_bounded(lbar, 0) && lane == 0) atomicExch(&g_zinv_cluster_error, 1);
  } else {
    const z64* a = at<const z64>(A, b);
    for (int idx = tid; idx < n * CW; idx += CT) {
      const int r = idx / CW, j = idx % CW, c = col0 + j;
      Xs[xoff(npad, r, j)] = c < n ? a[(int64_t)r * A.ld + c] : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
  cluster.sync();  // every CTA resident and loaded before any DSMEM access

  // ---- panels -----------------------------------------------------------
  uint32_t tphase = 0;
  for (int k0 = 0; k0 < n; k0 += CNB) {
    const int owner = k0 / CW, kl = k0 - owner * CW;
    const int nbp = min(CNB, n - k0);
    const bool own = rank == owner;
    const uint32_t tbytes = (uint32_t)(2 * chunk * sizeof(z64)) + CNB * sizeof(int);

    if (own) {
      gj_factor_panel16(
          n, k0, nbp, [&](int r, int c) { return Xs[xoff(npad, r, kl + c)]; },
          [&](int r, int c, z64 v) { Xs[xoff(npad, r, kl + c)] = v; }, pivrow, prow, rowk, red_v, red_i,
          &s_sing);
      // the panel's stores must be visible to the bulk copies below
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    } else if (tid == 0) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(tbar)), "r"(tbytes)
                   : "memory");
    }
    // Every CTA has finished reading the previous transform and the owner
    // has factored this panel.
    cluster_arrive();
    cluster_wait();
    if (own && tid == 0) {
      // The transform (columns kl..kl+15: two whole chunks) and its pivots
      // to every other CTA of the cluster (bulk copies, no multicast).
      const uint32_t src_t = saddr(Xs + (size_t)(kl >> 3) * chunk);
      const uint32_t src_p = saddr(pivrow + k0);
      for (int r = 0; r < C; ++r) {
        if (r == rank) continue;
        const uint32_t mb = cluster_addr(saddr(tbar), r);
        asm volatile(
            "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                cluster_addr(saddr(Ts), r)),
            "r"(src_t), "r"((uint32_t)(2 * chunk * sizeof(z64))), "r"(mb)
            : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                cluster_addr(saddr(pivrow + k0), r)),
            "r"(src_p), "r"((uint32_t)(CNB * sizeof(int))), "r"(mb)
            : "memory");
      }
    }
    if (!own) {
      if (warp == 0 && !mbar_wait_bounded(tbar, tphase) && lane == 0) atomicExch(&g_zinv_cluster_error, 1);
      tphase ^= 1u;
      __syncthreads();
    }
    const z64* T = own ? Xs + (size_t)(kl >> 3) * chunk : Ts;

    // Row interchanges of this CTA's other columns (lane = column), then the
    // pivot rows Y.
    if (warp == 0) {
      const int j = lane;
      const bool panel = own && j >= kl && j < kl + CNB;
      if (!panel) {
        for (int kk = 0; kk < nbp; ++kk) {
          const int k = k0 + kk, p = pivrow[k];
          if (p != k) {
            const z64 a = Xs[xoff(npad, k, j)], c = Xs[xoff(npad, p, j)];
            Xs[xoff(npad, k, j)] = c;
            Xs[xoff(npad, p, j)] = a;
          }
        }
      }
#pragma unroll
      for (int kk = 0; kk < CNB; ++kk)
        Ys[kk * YS + j] = (kk < nbp && !panel) ? Xs[xoff(npad, k0 + kk, j)] : make_double2(0.0, 0.0);
    }
    __syncthreads();

    // Update: warp w takes rows [16 w, 16 w + 16) of a pair of 8-column
    // tiles at a time (four independent accumulator chains); the owner skips
    // the pair that holds the panel (kl is 0 or 16: exactly one pair).
    const int mtiles = (n + 15) >> 4;
    for (int mt = warp; mt < mtiles; mt += CWARPS) {
      const int r0 = mt * 16;
      const int ra = r0 + g;
#pragma unroll 1
      for (int jp = 0; jp < 2; ++jp) {
        if (own && jp * 16 == kl) continue;
        double cre[2][4], cim[2][4];
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = ra + ((q >> 1) << 3);
            const int j = jp * 16 + t * 8 + 2 * tq + (q & 1);
            z64 v = make_double2(0.0, 0.0);
            if (r < n && !(r >= k0 && r < k0 + nbp)) v = Xs[xoff(npad, r, j)];
            cre[t][q] = v.x;
            cim[t][q] = v.y;
          }
#pragma unroll
        for (int k4 = 0; k4 < CNB; k4 += 4) {
          const int ka = k4 + tq;
          const z64 v0 = T[(ka >> 3) * chunk + ra * 8 + ((ka & 7) ^ (ra & 7))];
          const z64 v1 = T[(ka >> 3) * chunk + (ra + 8) * 8 + ((ka & 7) ^ ((ra + 8) & 7))];
#pragma unroll
          for (int t = 0; t < 2; ++t) {
            const z64 bv = Ys[ka * YS + jp * 16 + t * 8 + g];
            mma_f64(cre[t], v0.x, v1.x, bv.x);
            mma_f64(cim[t], v0.x, v1.x, bv.y);
            mma_f64(cre[t], -v0.y, -v1.y, bv.y);
            mma_f64(cim[t], v0.y, v1.y, bv.x);
          }
        }
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = ra + ((q >> 1) << 3);
            const int j = jp * 16 + t * 8 + 2 * tq + (q & 1);
            if (r < n) Xs[xoff(npad, r, j)] = make_double2(cre[t][q], cim[t][q]);
          }
      }
    }
    __syncthreads();
  }

  // ---- column permutation and store --------------------------------------
  // Output column q is column colsrc[q] of the Gauss-Jordan result (the
  // panel interchanges undone from the last pivot back).
  if (tid == 0) {
    for (int c = 0; c < n; ++c) colsrc[c] = c;
    for (int k = n - 1; k >= 0; --k) {
      const int p = pivrow[k];
      if (p != k) {
        const int t = colsrc[k];
        colsrc[k] = colsrc[p];
        colsrc[p] = t;
      }
    }
    if (s_sing != 0) atomicMin(cluster.map_shared_rank(&s_first, 0), s_sing);
  }
  __syncthreads();
  cluster.sync();  // every update and every first-singular report done
  {
    z64* x = at<z64>(X, b);
    const int ncols = min(CW, n - col0);
    // a warp stores 32 consecutive output columns of one row (512 bytes)
    const int jj = tid % CW;
    const int src = jj < ncols ? colsrc[col0 + jj] : 0;
    const z64* rX = cluster.map_shared_rank(Xs, src / CW);
    const int sj = src % CW;
    for (int r0 = tid / CW; r0 < n; r0 += 4 * (CT / CW)) {
      z64 v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = r0 + u * (CT / CW);
        if (r < n && jj < ncols) v[u] = rX[xoff(npad, r, sj)];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int r = r0 + u * (CT / CW);
        if (r < n && jj < ncols) x[(int64_t)r * X.ld + col0 + jj] = v[u];
      }
    }
  }
  if (rank == 0 && tid == 0 && info != nullptr && s_first != 0x7fffffff && info[b] == 0) info[b] = s_first;
  cluster.sync();  // no CTA leaves while another still reads its shared memory
}

// ---- host side -----------------------------------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static std::once_flag once;
  static EncodeTiled fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

// 3-D tensor map (re/im doubles, rows, batch) of A with a 16 x n box, or
// false when the layout does not allow one (then plain loads are used).
bool make_map(CUtensorMap* map, int n, int64_t batch, const MatRef& A) {
  EncodeTiled enc = encode_fn();
  if (enc == nullptr) return false;
  const uintptr_t p = reinterpret_cast<uintptr_t>(A.p);
  if ((p & 15) != 0 || A.stride <= 0 || A.ld < n || batch > 0x7fffffff) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * n, (cuuint64_t)n, (cuuint64_t)batch};
  const cuuint64_t strides[2] = {(cuuint64_t)A.ld * sizeof(z64), (cuuint64_t)A.stride * sizeof(z64)};
  if (strides[0] >= (1ull << 40) || strides[1] >= (1ull << 40)) return false;
  const cuuint32_t box[3] = {16, (cuuint32_t)n, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, A.p, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int C>
int launch_cluster(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s) {
  const ClusterSmem L(n);
  const size_t smem = L.total;
  QTX_CHECK_CUDA(cudaFuncSetAttribute(zinv_cluster_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  CUtensorMap map;
  const int use_tma = make_map(&map, n, batch, A) ? 1 : 0;
  if (!use_tma) memset(&map, 0, sizeof(map));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(batch * C), 1, 1);
  cfg.blockDim = dim3(CT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  ProfScope prof(QTX_KERNEL_ZINV, 8.0 * (double)n * n * n * (double)batch, s);
  QTX_CHECK_CUDA(cudaLaunchKernelEx(&cfg, zinv_cluster_kernel<C>, n, batch, A, X, info, active, map, use_tma));
  return QTX_OK;
}

}  // namespace

size_t zinv_cluster_smem(int n) { return ClusterSmem(n).total; }

int zinv_cluster(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  if (n > 8 * CW || batch * ((n + CW - 1) / CW) > 0x7fffffffll) {
    set_error("zinv_cluster: block size above 256 or batch too large");
    return QTX_ERR_UNSUPPORTED;
  }
  switch ((n + CW - 1) / CW) {
    case 1: return launch_cluster<1>(n, batch, A, X, info, active, s);
    case 2: return launch_cluster<2>(n, batch, A, X, info, active, s);
    case 3: return launch_cluster<3>(n, batch, A, X, info, active, s);
    case 4: return launch_cluster<4>(n, batch, A, X, info, active, s);
    case 5: return launch_cluster<5>(n, batch, A, X, info, active, s);
    case 6: return launch_cluster<6>(n, batch, A, X, info, active, s);
    case 7: return launch_cluster<7>(n, batch, A, X, info, active, s);
    default: return launch_cluster<8>(n, batch, A, X, info, active, s);
  }
}

int zinv_cluster_status_take(int* flag) {
  int h = 0;
  QTX_CHECK_CUDA(cudaMemcpyFromSymbol(&h, g_zinv_cluster_error, sizeof(int)));
  if (h) {
    const int zero = 0;
    QTX_CHECK_CUDA(cudaMemcpyToSymbol(g_zinv_cluster_error, &zero, sizeof(int)));
  }
  *flag = h;
  return QTX_OK;
}

}  // namespace qtx
