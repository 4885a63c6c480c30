// Batched complex128 matrix inverse: blocked Gauss-Jordan with partial
// pivoting, one CTA per matrix.
//
// Replaces the batched inverse of qttools kernels/linalg/inv.py:6-40
// (numpy.linalg.inv on CPU; cupy.linalg.solve(a, I) -> cuBLAS batched
// getrf/getrs on NVIDIA GPUs). Every diagonal Schur-complement block of the
// RGF forward sweep and every Sancho-Rubio step inverts through here.
//
// Algorithm (in place in X, n x n, panel width NB):
//   for each panel K = [k0, k0 + NB):
//     1. stage the n x NB panel X[:, K] in shared memory;
//     2. factor it column by column: pivot = argmax_{r >= k} |Re|+|Im|
//        (LAPACK izamax measure), swap, scale the pivot row by 1/pivot
//        (Smith's complex division), eliminate every other row. Afterwards
//        the panel holds T[:, K], where T is the Gauss-Jordan transform of
//        this panel: T = [A_KK^-1 ; -A_RK A_KK^-1] in block form;
//     3. apply the panel's row swaps to all other columns (global memory);
//     4. update every other column tile J:
//          X[:, J] = [0 ; X[R, J]] + T[:, K] X[K, J]
//        a n x |J| x NB complex GEMM on the FP64 tensor pipe (DMMA);
//     5. write the panel back.
//   Finally undo the column permutation (pivots applied in reverse order).
// Total work n^3 complex multiply-adds = 8 n^3 real flops.
#include <cooperative_groups.h>

#include "common.cuh"
#include "gj_panel.cuh"

namespace cg = cooperative_groups;

namespace qtx {
namespace {

constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr int JW = 32;  // column-tile width of the trailing update

__device__ __forceinline__ void mma_f64(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// 1 / (a + ib) by Smith's algorithm (avoids overflow of a^2 + b^2).
__device__ __forceinline__ z64 zrecip(z64 z) {
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

__device__ __forceinline__ double cabs1(z64 z) { return fabs(z.x) + fabs(z.y); }

template <int NB>
struct Smem {
  static constexpr int PS = NB + 4;  // panel row stride (= 4 mod 8 in 16 B units)
  static constexpr int YS = JW + 2;  // Y row stride (= 2 mod 8)
  static constexpr int NA = 2 * NB;  // rows a panel's pivoting can touch
  static size_t bytes(int n) {
    size_t s = (size_t)n * PS * sizeof(z64);  // panel
    s += (size_t)NB * YS * sizeof(z64);       // Y tile
    s += (size_t)NA * JW * sizeof(z64);       // staged old values of the affected rows
    s += (size_t)2 * NB * sizeof(z64);        // scaled pivot row, old row k
    s += (size_t)WARPS * (sizeof(double) + sizeof(int));
    s += (size_t)3 * NA * sizeof(int);  // affected rows, their sources, source slots
    s += (size_t)3 * n * sizeof(int);   // pivot rows, column sources, row -> slot map
    return s + 64;
  }
};

template <int NB>
__global__ void __launch_bounds__(THREADS, 1) zinv_kernel(int n, int64_t batch, MatRef A, MatRef X,
                                                        int* info, const int* active) {
  using S = Smem<NB>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  z64* P = reinterpret_cast<z64*>(smem_raw);
  z64* Y = P + (size_t)n * S::PS;
  z64* stage = Y + NB * S::YS;
  z64* prow = stage + S::NA * JW;
  z64* rowk = prow + NB;
  double* red_v = reinterpret_cast<double*>(rowk + NB);
  int* red_i = reinterpret_cast<int*>(red_v + WARPS);
  int* aff_row = red_i + WARPS;      // affected row indices
  int* aff_src = aff_row + S::NA;    // row whose old value each affected row receives
  int* aff_sslot = aff_src + S::NA;  // slot of that source row in the stage
  int* pivrow = aff_sslot + S::NA;
  int* colsrc = pivrow + n;
  int* slot_of = colsrc + n;  // row -> stage slot, -1 if the row is not affected

  for (int r = threadIdx.x; r < n; r += THREADS) slot_of[r] = -1;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane >> 2;
  const int tq = lane & 3;

  for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
    if (active != nullptr && active[b] == 0) continue;
    const z64* a = at<const z64>(A, b);
    z64* x = at<z64>(X, b);
    const int64_t lda = A.ld, ldx = X.ld;
    if (a != x) {
      for (int64_t idx = tid; idx < (int64_t)n * n; idx += THREADS) {
        const int r = (int)(idx / n), c = (int)(idx % n);
        x[(int64_t)r * ldx + c] = a[(int64_t)r * lda + c];
      }
    }
    int singular_at = 0;
    __syncthreads();

    for (int k0 = 0; k0 < n; k0 += NB) {
      const int nbp = min(NB, n - k0);
      // 1. Stage the panel (zero-padded to NB columns).
      for (int idx = tid; idx < n * NB; idx += THREADS) {
        const int r = idx / NB, c = idx % NB;
        P[r * S::PS + c] = (c < nbp) ? x[(int64_t)r * ldx + k0 + c] : make_double2(0.0, 0.0);
      }
      __syncthreads();

      // 2. Factor the panel.
      for (int kk = 0; kk < nbp; ++kk) {
        const int k = k0 + kk;
        double best = -1.0;
        int besti = k;
        for (int r = k + tid; r < n; r += THREADS) {
          const double v = cabs1(P[r * S::PS + kk]);
          if (v > best) {
            best = v;
            besti = r;
          }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, best, off);
          const int oi = __shfl_xor_sync(0xffffffffu, besti, off);
          if (ov > best || (ov == best && oi < besti)) {
            best = ov;
            besti = oi;
          }
        }
        if (lane == 0) {
          red_v[warp] = best;
          red_i[warp] = besti;
        }
        __syncthreads();
        best = red_v[0];
        besti = red_i[0];
#pragma unroll
        for (int w = 1; w < WARPS; ++w) {
          const double ov = red_v[w];
          const int oi = red_i[w];
          if (ov > best || (ov == best && oi < besti)) {
            best = ov;
            besti = oi;
          }
        }
        const int p = besti;
        if (best == 0.0 && singular_at == 0) singular_at = k + 1;
        // Nobody writes P in this phase, so every thread can read the pivot.
        const z64 dpiv = zrecip(P[p * S::PS + kk]);
        if (tid < NB) {
          const int c = tid;
          rowk[c] = P[k * S::PS + c];
          prow[c] = (c == kk) ? dpiv : zmul(P[p * S::PS + c], dpiv);
        }
        if (tid == 0) pivrow[k] = p;
        __syncthreads();
        // Eliminate; rows k and p are swapped on the fly (row p receives the
        // old row k, row k becomes the scaled pivot row).
        for (int r = tid; r < n; r += THREADS) {
          if (r == k) {
            for (int c = 0; c < NB; ++c) P[r * S::PS + c] = prow[c];
            continue;
          }
          const z64* src = (r == p) ? rowk : P + r * S::PS;
          const z64 f = src[kk];
          for (int c = 0; c < NB; ++c) {
            if (c == kk) continue;
            const z64 v = src[c];
            P[r * S::PS + c] = make_double2(v.x - (f.x * prow[c].x - f.y * prow[c].y),
                                            v.y - (f.x * prow[c].y + f.y * prow[c].x));
          }
          const z64 m = zmul(f, dpiv);
          P[r * S::PS + kk] = make_double2(-m.x, -m.y);
        }
        __syncthreads();
      }

      // 3. The panel's row interchanges as a permutation of the (at most
      //    2 NB) rows they touch: affected row aff_row[a] receives the old
      //    content of row aff_src[a], staged in slot aff_sslot[a].
      __shared__ int s_na;
      if (tid == 0) {
        int na = 0;
        for (int kk = 0; kk < nbp; ++kk) {
          const int k = k0 + kk, p = pivrow[k];
          int ik = slot_of[k], ip = slot_of[p];
          if (ik < 0) {
            ik = na++;
            aff_row[ik] = k;
            aff_src[ik] = k;
            slot_of[k] = ik;
          }
          if (ip < 0) {
            ip = na++;
            aff_row[ip] = p;
            aff_src[ip] = p;
            slot_of[p] = ip;
          }
          const int t = aff_src[ik];
          aff_src[ik] = aff_src[ip];
          aff_src[ip] = t;
        }
        for (int a = 0; a < na; ++a) aff_sslot[a] = slot_of[aff_src[a]];
        s_na = na;
      }
      __syncthreads();
      const int na = s_na;

      // 4. Trailing update of every other column tile:
      //      X[:, J] <- [0 ; X[R, J]] + T[:, K] X[K, J]   (rows permuted).
      for (int j0 = 0; j0 < n; j0 += JW) {
        // Columns of the panel itself are computed but never stored.
        if (j0 >= k0 && j0 + JW <= k0 + nbp) continue;
        for (int idx = tid; idx < na * JW; idx += THREADS) {
          const int a = idx / JW, c = idx % JW;
          const int gc = j0 + c;
          stage[a * JW + c] = (gc < n && (gc < k0 || gc >= k0 + nbp))
                                  ? x[(int64_t)aff_row[a] * ldx + gc]
                                  : make_double2(0.0, 0.0);
        }
        __syncthreads();
        for (int idx = tid; idx < NB * JW; idx += THREADS) {
          const int kk = idx / JW, c = idx % JW;
          Y[kk * S::YS + c] =
              (kk < nbp) ? stage[aff_sslot[slot_of[k0 + kk]] * JW + c] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        const int mtiles = (n + 15) / 16;
        for (int base = warp; base < mtiles; base += 2 * WARPS) {
          double cre[2][JW / 8][4], cim[2][JW / 8][4];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r0 = (base + h * WARPS) * 16;
#pragma unroll
            for (int j = 0; j < JW / 8; ++j)
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const int r = r0 + g + ((q >> 1) << 3);
                const int cl = j * 8 + 2 * tq + (q & 1);
                const int c = j0 + cl;
                z64 v = make_double2(0.0, 0.0);
                if (r < n && c < n && !(r >= k0 && r < k0 + nbp) && (c < k0 || c >= k0 + nbp)) {
                  const int sl = slot_of[r];
                  v = (sl >= 0) ? stage[aff_sslot[sl] * JW + cl] : x[(int64_t)r * ldx + c];
                }
                cre[h][j][q] = v.x;
                cim[h][j][q] = v.y;
              }
          }
#pragma unroll
          for (int k4 = 0; k4 < NB; k4 += 4) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int ra = (base + h * WARPS) * 16 + g;
              const z64 v0 = (ra < n) ? P[ra * S::PS + k4 + tq] : make_double2(0, 0);
              const z64 v1 = (ra + 8 < n) ? P[(ra + 8) * S::PS + k4 + tq] : make_double2(0, 0);
              const double nai0 = -v0.y, nai1 = -v1.y;
#pragma unroll
              for (int j = 0; j < JW / 8; ++j) {
                const z64 bv = Y[(k4 + tq) * S::YS + j * 8 + g];
                mma_f64(cre[h][j], v0.x, v1.x, bv.x);
                mma_f64(cim[h][j], v0.x, v1.x, bv.y);
              }
#pragma unroll
              for (int j = 0; j < JW / 8; ++j) {
                const z64 bv = Y[(k4 + tq) * S::YS + j * 8 + g];
                mma_f64(cre[h][j], nai0, nai1, bv.y);
                mma_f64(cim[h][j], v0.y, v1.y, bv.x);
              }
            }
          }
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r0 = (base + h * WARPS) * 16;
#pragma unroll
            for (int j = 0; j < JW / 8; ++j)
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                const int r = r0 + g + ((q >> 1) << 3);
                const int c = j0 + j * 8 + 2 * tq + (q & 1);
                if (r < n && c < n && (c < k0 || c >= k0 + nbp))
                  x[(int64_t)r * ldx + c] = make_double2(cre[h][j][q], cim[h][j][q]);
              }
          }
        }
        __syncthreads();
      }
      if (tid == 0)
        for (int a = 0; a < na; ++a) slot_of[aff_row[a]] = -1;

      // 5. Write the panel back.
      for (int idx = tid; idx < n * nbp; idx += THREADS) {
        const int r = idx / nbp, c = idx % nbp;
        x[(int64_t)r * ldx + k0 + c] = P[r * S::PS + c];
      }
      __syncthreads();
    }

    // Undo the column permutation: swaps applied from the last pivot back.
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
    }
    __syncthreads();
    // Row-wise gather through the (now free) panel buffer, one warp per row.
    z64* rowbuf = P + (size_t)warp * n;
    for (int r = warp; r < n; r += WARPS) {
      for (int c = lane; c < n; c += 32) rowbuf[c] = x[(int64_t)r * ldx + colsrc[c]];
      __syncwarp();
      for (int c = lane; c < n; c += 32) x[(int64_t)r * ldx + c] = rowbuf[c];
      __syncwarp();
    }
    // Report the first singular block seen for this stack entry (callers
    // zero `info` once per entry point).
    if (tid == 0 && info != nullptr && singular_at != 0 && info[b] == 0) info[b] = singular_at;
    __syncthreads();
  }
}

template <int NB>
int launch(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s) {
  const size_t smem = Smem<NB>::bytes(n);
  if (smem > 227 * 1024) {
    set_error("zinv: block size too large for the shared-memory panel");
    return QTX_ERR_UNSUPPORTED;
  }
  QTX_CHECK_CUDA(
      cudaFuncSetAttribute(zinv_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const unsigned grid = (unsigned)(batch < 1048576 ? batch : 1048576);
  ProfScope prof(QTX_KERNEL_ZINV, 8.0 * (double)n * n * n * (double)batch, s);
  zinv_kernel<NB><<<grid, THREADS, smem, s>>>(n, batch, A, X, info, active);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

// ---------------------------------------------------------------------------
// Second generation (n <= 720): the same Gauss-Jordan with the same pivot
// rule, reorganised so that the trailing update runs without barriers.
// Per panel of NB columns:
//   1. stage the n x NB panel (odd row stride: row-per-thread access is
//      conflict-free) and factor it (one barrier pair per column, the next
//      column's pivot candidate found during the elimination);
//   2. apply the panel's row interchanges to the other columns in global
//      memory: the <= 2 NB affected rows are read into registers, then
//      written to their new places;
//   3. stage the pivot rows Y = X[K, :] (other columns) once;
//   4. every warp updates its 16-row slices over all column tiles:
//      X[r, J] = (r in K ? 0 : X[r, J]) + T[r, :] Y[:, J]  (DMMA), with no
//      barrier, so 16 warps overlap their loads and MMAs;
//   5. write the panel transform T back into X[:, K].
constexpr int T2 = 512;
constexpr int W2 = T2 / 32;
constexpr int JN = 2;    // n8 tiles per column tile of the trailing update
constexpr int PV = 8;  // elements per thread of one row-interchange block

template <int NB>
struct Smem2 {
  static constexpr int PS = NB + 1;
  // Y row stride: covers whole 16-column tiles, 2 mod 8 in 16-byte units.
  __host__ __device__ static int ys(int n) { return ((n + 15) / 16) * 16 + 2; }
  static size_t bytes(int n) {
    size_t s = (size_t)n * PS * sizeof(z64);          // panel
    s += (size_t)NB * ys(n) * sizeof(z64);            // pivot rows Y
    s += (size_t)2 * NB * sizeof(z64);                // scaled pivot row, old row k
    s += (size_t)2 * W2 * (sizeof(double) + sizeof(int));
    s += (size_t)2 * (2 * NB) * sizeof(int);          // affected rows and their sources
    s += (size_t)2 * n * sizeof(int) + 16;            // pivot rows, column sources
    return s + 64;
  }
};

// Column split (csplit = C > 1, launched as clusters of C CTAs, one matrix
// per cluster): every CTA of the cluster factors each panel itself (the
// same arithmetic on the same data, so the same transform and pivots) and
// applies it to its own range of whole panels' columns; the panel's columns
// are written back by the CTA that owns them. A cluster barrier after each
// panel orders the owner's writes before the next panel's loads (read
// through L2), and the final row gather is split by rows. The serial panel
// factorization stays, the update is divided by C: for small batches, C SMs
// per matrix instead of one.
template <int NB>
__global__ void __launch_bounds__(T2, 1) zinv2_kernel(int n, int64_t batch, MatRef A, MatRef X, int* info,
                                                      const int* active, int csplit) {
  using S = Smem2<NB>;
  // Column block of the row-interchange pass: all 2 NB affected rows of CW
  // columns fit T2 x PV registers.
  constexpr int CW = (T2 * PV) / (2 * NB);
  static_assert(NB % 4 == 0 && 2 * NB * CW <= T2 * PV, "panel width and interchange block");
  constexpr int PS = S::PS;
  const int YS = S::ys(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  z64* P = reinterpret_cast<z64*>(smem_raw);
  z64* Y = P + (size_t)n * PS;
  z64* prow = Y + (size_t)NB * YS;
  z64* rowk = prow + NB;
  double* red_v = reinterpret_cast<double*>(rowk + NB);  // 2 x W2
  int* red_i = reinterpret_cast<int*>(red_v + 2 * W2);   // 2 x W2
  int* aff_row = red_i + 2 * W2;                         // 2 NB
  int* aff_src = aff_row + 2 * NB;                       // 2 NB
  int* pivrow = aff_src + 2 * NB;                        // n
  int* colsrc = pivrow + n;                              // n
  __shared__ int s_na, s_sing;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int rank = (int)(blockIdx.x % csplit);
  // this CTA's columns [c_lo, c_hi): whole panels
  auto cbound = [&](int q) {
    const int v = (int)(((int64_t)n * q / csplit + NB - 1) / NB) * NB;
    return v < n ? v : n;
  };
  const int c_lo = cbound(rank), c_hi = cbound(rank + 1), cw = c_hi - c_lo;
  auto cluster_sync = [&]() {
    if (csplit > 1) cg::this_cluster().sync();
  };

  for (int64_t b = blockIdx.x / csplit; b < batch; b += gridDim.x / csplit) {
    if (active != nullptr && active[b] == 0) continue;
    const z64* a = at<const z64>(A, b);
    z64* x = at<z64>(X, b);
    const int64_t ldx = X.ld;
    if (a != x) {
      for (int64_t idx = tid; idx < (int64_t)n * cw; idx += T2) {
        const int r = (int)(idx / cw), c = c_lo + (int)(idx % cw);
        x[(int64_t)r * ldx + c] = a[(int64_t)r * A.ld + c];
      }
    }
    if (tid == 0) s_sing = 0;
    __syncthreads();
    cluster_sync();

    for (int k0 = 0; k0 < n; k0 += NB) {
      const int nbp = min(NB, n - k0);
      // 1. Stage the panel and factor it: in registers for 16-column panels
      //    of at most 256 rows (two lanes per row), through shared memory
      //    otherwise.
      if (NB == 16 && n <= 256) {
      for (int idx = tid; idx < n * NB; idx += T2) {
        const int r = idx / NB, c = idx % NB;
        P[r * PS + c] = (c < nbp) ? __ldcg(&x[(int64_t)r * ldx + k0 + c]) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      gj_factor_panel16(
          n, k0, nbp, [&](int r, int c) { return P[r * PS + c]; },
          [&](int r, int c, z64 v) { P[r * PS + c] = v; }, pivrow, prow, rowk, red_v, red_i, &s_sing);
      __syncthreads();
      } else {
      for (int idx = tid; idx < n * NB; idx += T2) {
        const int r = idx / NB, c = idx % NB;
        P[r * PS + c] = (c < nbp) ? __ldcg(&x[(int64_t)r * ldx + k0 + c]) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      double best = -1.0;
      int besti = k0;
      for (int r = k0 + tid; r < n; r += T2) {
        const double v = cabs1(P[r * PS]);
        if (v > best || (v == best && r < besti)) {
          best = v;
          besti = r;
        }
      }
      for (int kk = 0; kk < nbp; ++kk) {
        const int k = k0 + kk;
        const int buf = kk & 1;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, best, off);
          const int oi = __shfl_xor_sync(0xffffffffu, besti, off);
          if (ov > best || (ov == best && oi < besti)) {
            best = ov;
            besti = oi;
          }
        }
        if (lane == 0) {
          red_v[buf * W2 + warp] = best;
          red_i[buf * W2 + warp] = besti;
        }
        __syncthreads();
        best = red_v[buf * W2];
        besti = red_i[buf * W2];
#pragma unroll
        for (int w = 1; w < W2; ++w) {
          const double ov = red_v[buf * W2 + w];
          const int oi = red_i[buf * W2 + w];
          if (ov > best || (ov == best && oi < besti)) {
            best = ov;
            besti = oi;
          }
        }
        const int p = besti;
        if (best <= 0.0 && tid == 0 && s_sing == 0) s_sing = k + 1;
        const z64 dpiv = zrecip(P[p * PS + kk]);
        if (tid < NB) {
          rowk[tid] = P[k * PS + tid];
          prow[tid] = (tid == kk) ? dpiv : zmul(P[p * PS + tid], dpiv);
        }
        if (tid == 0) pivrow[k] = p;
        __syncthreads();
        best = -1.0;
        besti = k + 1;
        for (int r = tid; r < n; r += T2) {
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
          if (kk + 1 < nbp && r > k) {
            const double v = cabs1(P[r * PS + kk + 1]);
            if (v > best || (v == best && r < besti)) {
              best = v;
              besti = r;
            }
          }
        }
      }
      }
      // 2. The panel's interchanges as a permutation of the affected rows:
      //    row aff_row[a] receives the old content of row aff_src[a].
      if (tid == 0) {
        int na = 0;
        for (int kk = 0; kk < nbp; ++kk) {
          const int k = k0 + kk, p = pivrow[k];
          int ik = -1, ip = -1;
          for (int u = 0; u < na; ++u) {
            if (aff_row[u] == k) ik = u;
            if (aff_row[u] == p) ip = u;
          }
          if (ik < 0) {
            ik = na++;
            aff_row[ik] = k;
            aff_src[ik] = k;
          }
          if (ip < 0) {
            ip = na++;
            aff_row[ip] = p;
            aff_src[ip] = p;
          }
          const int t = aff_src[ik];
          aff_src[ik] = aff_src[ip];
          aff_src[ip] = t;
        }
        s_na = na;
      }
      __syncthreads();
      const int na = s_na;
      const bool pin = k0 >= c_lo && k0 < c_hi;  // the panel lies in this CTA's columns
      const int oc = cw - (pin ? nbp : 0);       // this CTA's columns outside the panel
      // In column blocks of CW: all affected rows of a column move within
      // one block (read all, barrier, write all).
      for (int cb = 0; cb < oc; cb += CW) {
        z64 v[PV];
#pragma unroll
        for (int u = 0; u < PV; ++u) {
          const int li = tid + u * T2;
          const int aa = li / CW, cc = cb + li % CW;
          if (aa < na && cc < oc) {
            const int c = c_lo + cc + ((pin && c_lo + cc >= k0) ? nbp : 0);
            v[u] = x[(int64_t)aff_src[aa] * ldx + c];
          }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < PV; ++u) {
          const int li = tid + u * T2;
          const int aa = li / CW, cc = cb + li % CW;
          if (aa < na && cc < oc) {
            const int c = c_lo + cc + ((pin && c_lo + cc >= k0) ? nbp : 0);
            x[(int64_t)aff_row[aa] * ldx + c] = v[u];
          }
        }
        __syncthreads();
      }
      // 3. Pivot rows (other columns) into Y.
      const int ny = YS - 2;  // columns of whole tiles; those >= n stay zero
      for (int idx = tid; idx < NB * ny; idx += T2) {
        const int kk = idx / ny, c = idx % ny;
        Y[kk * YS + c] = (kk < nbp && c >= c_lo && c < c_hi && (c < k0 || c >= k0 + nbp))
                             ? x[(int64_t)(k0 + kk) * ldx + c]
                             : make_double2(0.0, 0.0);
      }
      __syncthreads();
      // 4. Trailing update, one 16-row slice per warp at a time, no barriers.
      const int mtiles = (n + 15) / 16;
      for (int mt = warp; mt < mtiles; mt += W2) {
        const int r0 = mt * 16;
        // A fragments of this slice for all k (the panel transform rows).
        for (int j0 = c_lo; j0 < c_hi; j0 += 8 * JN) {
          if (j0 >= k0 && j0 + 8 * JN <= k0 + nbp) continue;  // inside the panel
          double cre[JN][4], cim[JN][4];
#pragma unroll
          for (int j = 0; j < JN; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int r = r0 + g + ((q >> 1) << 3);
              const int c = j0 + j * 8 + 2 * tq + (q & 1);
              z64 v = make_double2(0.0, 0.0);
              if (r < n && c < n && !(r >= k0 && r < k0 + nbp) && (c < k0 || c >= k0 + nbp))
                v = x[(int64_t)r * ldx + c];
              cre[j][q] = v.x;
              cim[j][q] = v.y;
            }
#pragma unroll
          for (int k4 = 0; k4 < NB; k4 += 4) {
            const int ra = r0 + g;
            const z64 v0 = (ra < n) ? P[ra * PS + k4 + tq] : make_double2(0.0, 0.0);
            const z64 v1 = (ra + 8 < n) ? P[(ra + 8) * PS + k4 + tq] : make_double2(0.0, 0.0);
            const double nai0 = -v0.y, nai1 = -v1.y;
            double br[JN], bi[JN];
#pragma unroll
            for (int j = 0; j < JN; ++j) {
              const z64 bv = Y[(k4 + tq) * YS + j0 + j * 8 + g];
              br[j] = bv.x;
              bi[j] = bv.y;
            }
#pragma unroll
            for (int j = 0; j < JN; ++j) {
              mma_f64(cre[j], v0.x, v1.x, br[j]);
              mma_f64(cim[j], v0.x, v1.x, bi[j]);
            }
#pragma unroll
            for (int j = 0; j < JN; ++j) {
              mma_f64(cre[j], nai0, nai1, bi[j]);
              mma_f64(cim[j], v0.y, v1.y, br[j]);
            }
          }
#pragma unroll
          for (int j = 0; j < JN; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int r = r0 + g + ((q >> 1) << 3);
              const int c = j0 + j * 8 + 2 * tq + (q & 1);
              if (r < n && c < n && (c < k0 || c >= k0 + nbp))
                x[(int64_t)r * ldx + c] = make_double2(cre[j][q], cim[j][q]);
            }
        }
      }
      __syncthreads();
      // 5. The panel transform back into X[:, K] (by the CTA owning K).
      if (pin) {
        for (int idx = tid; idx < n * nbp; idx += T2) {
          const int r = idx / nbp, c = idx % nbp;
          x[(int64_t)r * ldx + k0 + c] = P[r * PS + c];
        }
      }
      __syncthreads();
      cluster_sync();
    }

    // Undo the column permutation: swaps applied from the last pivot back.
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
    }
    __syncthreads();
    // Row-wise gather through the (now free) panel buffer: PS rows fit.
    // Rows rank, rank + C, ... of a column split (read through L2: the
    // other CTAs wrote their columns).
    const int nbufs = PS < W2 ? PS : W2;
    if (warp < nbufs) {
      z64* rowbuf = P + (size_t)warp * n;
      for (int r = rank + warp * csplit; r < n; r += nbufs * csplit) {
        for (int c = lane; c < n; c += 32) rowbuf[c] = __ldcg(&x[(int64_t)r * ldx + colsrc[c]]);
        __syncwarp();
        for (int c = lane; c < n; c += 32) x[(int64_t)r * ldx + c] = rowbuf[c];
        __syncwarp();
      }
    }
    if (tid == 0 && rank == 0 && info != nullptr && s_sing != 0 && info[b] == 0) info[b] = s_sing;
    __syncthreads();
    // the next matrix's copy must not overwrite rows still being gathered
    cluster_sync();
  }
}

template <int NB>
int launch2(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s,
            int csplit = 1) {
  const size_t smem = Smem2<NB>::bytes(n);
  if (smem > 227 * 1024) {
    set_error("zinv: block size too large for the shared-memory panel");
    return QTX_ERR_UNSUPPORTED;
  }
  QTX_CHECK_CUDA(
      cudaFuncSetAttribute(zinv2_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t mats = batch < 131072 ? batch : 131072;
  ProfScope prof(QTX_KERNEL_ZINV, 8.0 * (double)n * n * n * (double)batch, s);
  if (csplit <= 1) {
    zinv2_kernel<NB><<<(unsigned)mats, T2, smem, s>>>(n, batch, A, X, info, active, 1);
    QTX_CHECK_LAUNCH();
    return QTX_OK;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(mats * csplit), 1, 1);
  cfg.blockDim = dim3(T2, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)csplit;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  QTX_CHECK_CUDA(cudaLaunchKernelEx(&cfg, zinv2_kernel<NB>, n, batch, A, X, info, active, csplit));
  return QTX_OK;
}

// Column split for n <= 400 (16-column panels): the largest C in {1, 2, 4, 8}
// with batch x C within the SM count, at least 32 columns per CTA, and all
// batch clusters co-resident (cudaOccupancyMaxActiveClusters, cached per
// n and C). Inverse path 4 forces the largest C the block size allows.
int column_split(int n, int64_t batch) {
  const int path = inverse_path();
  if ((path != 0 && path != 4) || n > 400) return 1;
  int cmax = 1;
  while (cmax < 8 && n / (2 * cmax) >= 32) cmax *= 2;
  if (path == 4) return cmax;
  const int sms = num_sms();
  int c = 1;
  while (c < cmax && batch * (2 * c) <= sms) c *= 2;
  while (c > 1) {
    static thread_local std::vector<std::pair<int64_t, int>> cache;  // (n * 16 + c, active clusters)
    const int64_t key = (int64_t)n * 16 + c;
    int active = -1;
    for (auto& e : cache)
      if (e.first == key) active = e.second;
    if (active < 0) {
      const size_t smem = Smem2<16>::bytes(n);
      if (cudaFuncSetAttribute(zinv2_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
        return 1;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(c * batch), 1, 1);
      cfg.blockDim = dim3(T2, 1, 1);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)c;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int nc = 0;
      if (cudaOccupancyMaxActiveClusters(&nc, zinv2_kernel<16>, &cfg) != cudaSuccess) {
        cudaGetLastError();
        nc = 0;
      }
      active = nc;
      cache.emplace_back(key, active);
    }
    if (active >= batch) return c;
    c /= 2;
  }
  return 1;
}

}  // namespace

int zinv(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  if (A.null() || X.null()) {
    set_error("zinv: null matrix");
    return QTX_ERR_ARG;
  }
  if (zinv_prefers_cluster(n, batch)) return zinv_cluster(n, batch, A, X, info, active, s);
  if (n <= 400) return launch2<16>(n, batch, A, X, info, active, s, column_split(n, batch));
  if (n <= 720) return launch2<8>(n, batch, A, X, info, active, s);
  if (n <= 1024) return launch<8>(n, batch, A, X, info, active, s);
  set_error("zinv: block sizes above 1024 are not supported");
  return QTX_ERR_UNSUPPORTED;
}

}  // namespace qtx
