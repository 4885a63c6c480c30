// Batched complex128 inverse for large blocks and small batches: blocked
// Gauss-Jordan with partial pivoting spread over the whole GPU.
//
// Same algorithm and pivot rule as the one-CTA-per-matrix kernel (zinv.cu),
// which keeps only `batch` SMs busy: a batch of 16 blocks of 768 x 768 uses
// 16 of 148 SMs. Here each panel of NB columns is processed by three kernels:
//
//   1. zw_panel    one CTA per matrix: the n x NB panel in shared memory,
//                  column by column pivot search (|Re| + |Im|, lowest index on
//                  ties), row interchange, scaling and elimination; writes the
//                  panel transform T back into X[:, K] and the pivot rows;
//   2. zw_swap     one thread per column outside the panel: applies the
//                  panel's interchanges, moves rows K into the scratch Y and
//                  zeroes them in X;
//   3. zgemm       X[:, J] += T Y[:, J] for the column ranges left and right
//                  of the panel (batched DMMA GEMM, every SM).
//
// After the last panel the column permutation is undone (zw_colsrc computes
// the source column of every column, zw_permute gathers each row).
//
// Scratch per matrix: Y (NB x n complex128), pivot rows and column sources
// (n ints each).
#include "common.cuh"

namespace qtx {
namespace {

constexpr int PT = 256;  // threads of the panel kernel
constexpr int PW = PT / 32;

__device__ __forceinline__ z64 zrecip_w(z64 z) {
  // Smith's algorithm; 1/0 returns 0 (the singular flag is raised separately).
  if (fabs(z.x) >= fabs(z.y)) {
    if (z.x == 0.0 && z.y == 0.0) return make_double2(0.0, 0.0);
    const double r = z.y / z.x;
    const double den = z.x + z.y * r;
    return make_double2(1.0 / den, -r / den);
  }
  const double r = z.x / z.y;
  const double den = z.x * r + z.y;
  return make_double2(r / den, -1.0 / den);
}

__device__ __forceinline__ double cabs1_w(z64 z) { return fabs(z.x) + fabs(z.y); }

__device__ __forceinline__ void argmax_merge(double& v, int& i, double ov, int oi) {
  if (ov > v || (ov == v && oi < i)) {
    v = ov;
    i = oi;
  }
}

struct Scratch {
  z64* Y;       // batch x NB x n
  int* piv;     // batch x n
  int* colsrc;  // batch x n
};

template <int NB>
__host__ __device__ constexpr int panel_stride() {
  return NB + 1;  // odd stride in 16-byte units: row-per-thread access is conflict-free
}

template <int NB>
size_t panel_smem(int n) {
  return (size_t)n * panel_stride<NB>() * sizeof(z64) + 2 * NB * sizeof(z64) +
         2 * PW * (sizeof(double) + sizeof(int)) + 16;
}

// One CTA per matrix: Gauss-Jordan factorisation of the panel X[:, k0:k0+nbp].
template <int NB>
__global__ void __launch_bounds__(PT, 1) zw_panel(int n, int k0, int64_t batch, MatRef X, Scratch sc,
                                                  int* info, const int* active) {
  constexpr int PS = panel_stride<NB>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  z64* P = reinterpret_cast<z64*>(smem_raw);
  z64* prow = P + (size_t)n * PS;
  z64* rowk = prow + NB;
  double* red_v = reinterpret_cast<double*>(rowk + NB);  // 2 x PW (double-buffered)
  int* red_i = reinterpret_cast<int*>(red_v + 2 * PW);

  const int64_t b = blockIdx.x;
  if (b >= batch || (active != nullptr && active[b] == 0)) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nbp = min(NB, n - k0);
  z64* x = at<z64>(X, b);
  int* piv = sc.piv + b * n;

  for (int idx = tid; idx < n * NB; idx += PT) {
    const int r = idx / NB, c = idx % NB;
    P[r * PS + c] = (c < nbp) ? x[(int64_t)r * X.ld + k0 + c] : make_double2(0.0, 0.0);
  }
  __syncthreads();

  // Pivot candidate of the panel's first column.
  double best = -1.0;
  int besti = k0;
  for (int r = k0 + tid; r < n; r += PT) argmax_merge(best, besti, cabs1_w(P[r * PS]), r);
  int singular_at = 0;
  for (int kk = 0; kk < nbp; ++kk) {
    const int k = k0 + kk;
    const int buf = kk & 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, besti, off);
      argmax_merge(best, besti, ov, oi);
    }
    if (lane == 0) {
      red_v[buf * PW + warp] = best;
      red_i[buf * PW + warp] = besti;
    }
    __syncthreads();
    best = red_v[buf * PW];
    besti = red_i[buf * PW];
#pragma unroll
    for (int w = 1; w < PW; ++w) argmax_merge(best, besti, red_v[buf * PW + w], red_i[buf * PW + w]);
    const int p = besti;
    if (best <= 0.0 && singular_at == 0) singular_at = k + 1;
    const z64 dpiv = zrecip_w(P[p * PS + kk]);
    if (tid < NB) {
      rowk[tid] = P[k * PS + tid];
      prow[tid] = (tid == kk) ? dpiv : zmul(P[p * PS + tid], dpiv);
    }
    if (tid == 0) piv[k] = p;
    __syncthreads();
    // Eliminate (rows k and p swapped on the fly) and find the next pivot.
    best = -1.0;
    besti = k + 1;
    for (int r = tid; r < n; r += PT) {
      if (r == k) {
#pragma unroll
        for (int c = 0; c < NB; ++c) P[r * PS + c] = prow[c];
        continue;
      }
      const z64* src = (r == p) ? rowk : P + r * PS;
      const z64 f = src[kk];
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        if (c == kk) continue;
        const z64 v = src[c];
        const z64 q = prow[c];
        P[r * PS + c] = make_double2(v.x - (f.x * q.x - f.y * q.y), v.y - (f.x * q.y + f.y * q.x));
      }
      const z64 m = zmul(f, dpiv);
      P[r * PS + kk] = make_double2(-m.x, -m.y);
      if (kk + 1 < nbp && r > k) argmax_merge(best, besti, cabs1_w(P[r * PS + kk + 1]), r);
    }
  }
  __syncthreads();
  for (int idx = tid; idx < n * nbp; idx += PT) {
    const int r = idx / nbp, c = idx % nbp;
    x[(int64_t)r * X.ld + k0 + c] = P[r * PS + c];
  }
  if (tid == 0 && info != nullptr && singular_at != 0 && info[b] == 0) info[b] = singular_at;
}

// Row interchanges of the panel on the other columns; rows K move to Y.
template <int NB>
__global__ void zw_swap(int n, int k0, int64_t batch, MatRef X, Scratch sc, const int* active) {
  const int64_t b = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch || c >= n || (active != nullptr && active[b] == 0)) return;
  const int nbp = min(NB, n - k0);
  z64* Y = sc.Y + b * (int64_t)NB * n;
  if (c >= k0 && c < k0 + nbp) {
    for (int kk = 0; kk < NB; ++kk) Y[(int64_t)kk * n + c] = make_double2(0.0, 0.0);
    return;
  }
  z64* x = at<z64>(X, b);
  const int* piv = sc.piv + b * n;
  for (int kk = 0; kk < nbp; ++kk) {
    const int k = k0 + kk, p = piv[k];
    if (p != k) {
      const z64 t = x[(int64_t)k * X.ld + c];
      x[(int64_t)k * X.ld + c] = x[(int64_t)p * X.ld + c];
      x[(int64_t)p * X.ld + c] = t;
    }
  }
  for (int kk = 0; kk < NB; ++kk) {
    z64 v = make_double2(0.0, 0.0);
    if (kk < nbp) {
      v = x[(int64_t)(k0 + kk) * X.ld + c];
      x[(int64_t)(k0 + kk) * X.ld + c] = make_double2(0.0, 0.0);
    }
    Y[(int64_t)kk * n + c] = v;
  }
}

// Source column of every column: the interchanges undone from the last.
__global__ void zw_colsrc(int n, int64_t batch, Scratch sc, const int* active) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch || (active != nullptr && active[b] == 0)) return;
  int* cs = sc.colsrc + b * n;
  const int* piv = sc.piv + b * n;
  for (int c = 0; c < n; ++c) cs[c] = c;
  for (int k = n - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k) {
      const int t = cs[k];
      cs[k] = cs[p];
      cs[p] = t;
    }
  }
}

// x[r][c] <- x[r][colsrc[c]], one row per CTA (staged in shared memory).
__global__ void zw_permute(int n, int64_t batch, MatRef X, Scratch sc, const int* active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  z64* row = reinterpret_cast<z64*>(smem_raw);
  const int r = blockIdx.x;
  const int64_t b = blockIdx.y;
  if (b >= batch || (active != nullptr && active[b] == 0)) return;
  z64* x = at<z64>(X, b) + (int64_t)r * X.ld;
  const int* cs = sc.colsrc + b * n;
  for (int c = threadIdx.x; c < n; c += blockDim.x) row[c] = x[c];
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x) x[c] = row[cs[c]];
}

__global__ void zw_copy(int n, int64_t batch, MatRef A, MatRef X, const int* active) {
  const int64_t b = blockIdx.y;
  if (b >= batch || (active != nullptr && active[b] == 0)) return;
  const z64* a = at<const z64>(A, b);
  z64* x = at<z64>(X, b);
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < (int64_t)n * n;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(idx / n), c = (int)(idx % n);
    x[(int64_t)r * X.ld + c] = a[(int64_t)r * A.ld + c];
  }
}

template <int NB>
int run_wide(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, Scratch sc,
             cudaStream_t s) {
  const size_t psm = panel_smem<NB>(n);
  QTX_CHECK_CUDA(cudaFuncSetAttribute(zw_panel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
  const int panels = (n + NB - 1) / NB;
  ProfScope prof(QTX_KERNEL_ZINV, 8.0 * (double)n * n * n * (double)batch, s, 4 * panels + 3);
  if (A.p != X.p || A.ld != X.ld || A.stride != X.stride) {
    zw_copy<<<dim3(64, (unsigned)batch), 256, 0, s>>>(n, batch, A, X, active);
    QTX_CHECK_LAUNCH();
  }
  for (int k0 = 0; k0 < n; k0 += NB) {
    const int nbp = n - k0 < NB ? n - k0 : NB;
    zw_panel<NB><<<(unsigned)batch, PT, psm, s>>>(n, k0, batch, X, sc, info, active);
    QTX_CHECK_LAUNCH();
    zw_swap<NB><<<dim3((n + 127) / 128, (unsigned)batch), 128, 0, s>>>(n, k0, batch, X, sc, active);
    QTX_CHECK_LAUNCH();
    // X[:, J] += T Y[:, J] for J left and right of the panel (the panel's own
    // columns, which hold T, are neither read as C nor written).
    for (int side = 0; side < 2; ++side) {
      const int c0 = side == 0 ? 0 : k0 + nbp;
      const int nc = side == 0 ? k0 : n - k0 - nbp;
      if (nc <= 0) continue;
      GemmDesc d;
      d.M = n;
      d.N = nc;
      d.K = nbp;
      d.batch = batch;
      d.A = MatRef{static_cast<z64*>(X.p) + k0, X.ld, X.stride};
      d.B = MatRef{sc.Y + c0, n, (int64_t)NB * n};
      d.C = MatRef{static_cast<z64*>(X.p) + c0, X.ld, X.stride};
      d.add[0] = Addend{d.C, make_double2(1.0, 0.0), 0};
      d.nadd = 1;
      d.active = active;
      QTX_TRY(zgemm(d, s));
    }
  }
  zw_colsrc<<<(unsigned)((batch + 63) / 64), 64, 0, s>>>(n, batch, sc, active);
  QTX_CHECK_LAUNCH();
  zw_permute<<<dim3((unsigned)n, (unsigned)batch), 256, (size_t)n * sizeof(z64), s>>>(n, batch, X, sc, active);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

int g_inverse_path = 0;  // 0 automatic, 1 one CTA per matrix, 2 multi-CTA, 3 cluster, 4 column split

}  // namespace

int num_sms() {
  static int sms = 0;
  if (sms == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 148;
  }
  return sms;
}

int inverse_path() { return g_inverse_path; }

namespace {

// Panel width: as wide as the n x NB panel fits in shared memory.
int panel_width(int n) { return n <= 416 ? 32 : (n <= 832 ? 16 : 8); }

}  // namespace

size_t zinv_scratch_bytes(int n, int64_t batch) {
  if (n <= 0 || batch <= 0) return 0;
  const int nb = panel_width(n);
  return (size_t)batch * ((size_t)nb * n * sizeof(z64) + 2 * (size_t)n * sizeof(int)) + 1024;
}

void set_inverse_path(int mode) { g_inverse_path = mode; }

bool zinv_prefers_cluster(int n, int64_t batch) {
  if (n > 256) return false;
  if (g_inverse_path == 3) return true;
  if (g_inverse_path != 0) return false;
  // A cluster per matrix (ceil(n / 32) CTAs, one per SM at n = 256) finishes
  // one matrix 2.2x sooner than one CTA streaming it through HBM (0.59 vs
  // 1.31 ms at n = 256), but holds C SMs for it, and the GPU co-schedules
  // only about half of the SM count in clusters of 8: measured on B200, it
  // wins while batch x C stays within half the SMs (n = 256: batch <= 9).
  const int c = (n + 31) / 32;
  return batch * c * 2 <= (int64_t)num_sms();
}

bool zinv_prefers_wide(int n, int64_t batch) {
  if (g_inverse_path == 1 || g_inverse_path == 3 || g_inverse_path == 4) return false;
  if (g_inverse_path == 2) return true;
  // One CTA per matrix leaves SMs idle when the batch is below the SM count;
  // the multi-CTA path pays n/NB launches and a pass over the matrix per
  // panel. Up to n = 400 the column-split clusters of the one-CTA kernel
  // (zinv.cu) use the idle SMs instead; above, the measured crossover on
  // B200 (TFLOP/s of both paths against the batch) is batch 64 at n = 512.
  const int sms = num_sms();
  return n > 400 && batch * 2 <= sms;
}

int zinv_ex(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, void* scratch,
            size_t scratch_bytes, cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  if (zinv_prefers_cluster(n, batch)) return zinv_cluster(n, batch, A, X, info, active, s);
  if (scratch == nullptr || scratch_bytes < zinv_scratch_bytes(n, batch) || !zinv_prefers_wide(n, batch) ||
      n > 1024 || batch > 65535)
    return zinv(n, batch, A, X, info, active, s);
  if (A.null() || X.null()) {
    set_error("zinv: null matrix");
    return QTX_ERR_ARG;
  }
  const int nb = panel_width(n);
  char* p = static_cast<char*>(scratch);
  p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255));
  Scratch sc;
  sc.Y = reinterpret_cast<z64*>(p);
  sc.piv = reinterpret_cast<int*>(sc.Y + (size_t)batch * nb * n);
  sc.colsrc = sc.piv + (size_t)batch * n;
  if (nb == 32) return run_wide<32>(n, batch, A, X, info, active, sc, s);
  if (nb == 16) return run_wide<16>(n, batch, A, X, info, active, sc, s);
  return run_wide<8>(n, batch, A, X, info, active, sc, s);
}

}  // namespace qtx
