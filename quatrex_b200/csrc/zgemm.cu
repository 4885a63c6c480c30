// Batched complex128 GEMM on the sm_100a FP64 tensor pipe.
//
// Every block product of the RGF recursions (qttools
// greens_function_solver/rgf.py:71-110,234-428) and of the Sancho-Rubio
// decimation (boundary_conditions/obc/sancho_rubio.py:64-71) goes through
// this kernel. tcgen05 has no FP64 kind, so FP64 products are issued as
// warp-level DMMA (mma.sync m16n8k4 .f64) -- on B200 the FP64 tensor and
// vector rates are equal, and DMMA needs 8x fewer issue slots than DFMA.
//
// Complex arithmetic uses the 3M (Gauss) form on interleaved operands: one
// 16-byte shared-memory load yields the real and the imaginary fragment of an
// element, and the three real MMAs  Ar Br,  Ai Bi  and  (Ar + Ai)(Br + Bi)
// give  Re = p1 - p2  and  Im = p3 - p1 - p2  in the epilogue.
// Conjugate-transposed operands are staged k-major so every fragment load
// stays conflict-free (strides = 4 mod 8 or 2 mod 8 in 16-byte units), and
// conjugation is a compile-time sign flip.
//
// Tiles: CTA 64x64 complex, 4 warps of 32x32, BK = 8 complex per stage,
// 4-stage cp.async pipeline (zero-filled at the matrix edges). The epilogue
// fuses up to four scaled (optionally conjugate-transposed) addends, a
// conjugate-transposed second store and a second output with its own
// addends, so chains like  S = A_jj - Sigma - P A_ij  or
// X_ij = -X_ii A X_jj  with  X_ji = -X_ij^H  are one launch. It runs through
// a padded shared-memory tile: transposed operands are read and written with
// lanes along rows, the others with lanes along columns (coalesced both ways,
// many independent loads in flight).
#include "common.cuh"

namespace qtx {
namespace {

constexpr int BM = 64;
constexpr int BN = 64;
constexpr int BK = 8;
constexpr int STAGES = 4;
constexpr int THREADS = 128;
constexpr int WM = 32;
constexpr int WN = 32;
constexpr int MT = WM / 16;  // m16 tiles per warp
constexpr int NT = WN / 8;   // n8 tiles per warp

// Shared-memory strides (complex elements).
constexpr int S_MK = BK + 4;  // [row][k] layouts: stride = 4 mod 8
constexpr int S_KM = BM + 2;  // [k][row] layouts: stride = 2 mod 8
constexpr int A_MK_SIZE = BM * S_MK;
constexpr int A_KM_SIZE = BK * S_KM;
constexpr int B_NK_SIZE = BN * S_MK;
constexpr int B_KN_SIZE = BK * (BN + 2);
constexpr int TS = BN + 1;  // epilogue tile row stride (complex): 1 mod 8 in 16-byte units

__device__ __forceinline__ void mma_f64(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool pred) {
  const int bytes = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Loads one BK slice of op(A) (OPA = 0: A is M x K; 1: A is K x M) or of
// op(B) (OPB = 0: B is K x N; 1: B is N x K) into shared memory.
template <int OP, bool IS_A>
__device__ __forceinline__ void load_tile(z64* sm, const z64* g, int64_t ld, int rows_total,
                                          int cols_total, int r0, int k0, int tid) {
  // "rows" = M (for A) or N (for B); the tile spans 64 rows x BK k-values.
  if (OP == (IS_A ? 0 : 1)) {
    // Global rows are the M/N index, k contiguous: [row][k] layout.
#pragma unroll
    for (int it = 0; it < (64 * BK) / THREADS; ++it) {
      const int idx = tid + it * THREADS;
      const int r = idx / BK;
      const int k = idx % BK;
      const int gr = r0 + r, gk = k0 + k;
      const bool ok = (gr < rows_total) && (gk < cols_total);
      const z64* src = ok ? g + (int64_t)gr * ld + gk : g;
      cp_async16(sm + r * S_MK + k, src, ok);
    }
  } else {
    // Global rows are the k index, M/N contiguous: [k][row] layout.
#pragma unroll
    for (int it = 0; it < (64 * BK) / THREADS; ++it) {
      const int idx = tid + it * THREADS;
      const int k = idx / 64;
      const int r = idx % 64;
      const int gr = r0 + r, gk = k0 + k;
      const bool ok = (gr < rows_total) && (gk < cols_total);
      const z64* src = ok ? g + (int64_t)gk * ld + gr : g;
      cp_async16(sm + k * S_KM + r, src, ok);
    }
  }
}

struct KernelArgs {
  GemmDesc d;
};

template <int OPA, int OPB>
__global__ void __launch_bounds__(THREADS, 2) zgemm_kernel(const KernelArgs args) {
  const GemmDesc& d = args.d;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  z64* smem = reinterpret_cast<z64*>(smem_raw);
  constexpr int A_SIZE = (OPA == 0) ? A_MK_SIZE : A_KM_SIZE;
  constexpr int B_SIZE = (OPB == 1) ? B_NK_SIZE : B_KN_SIZE;
  z64* As = smem;
  z64* Bs = smem + STAGES * A_SIZE;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int g = lane >> 2;
  const int tq = lane & 3;
  const int wm0 = (warp >> 1) * WM;
  const int wn0 = (warp & 1) * WN;
  const int m0 = blockIdx.y * BM;
  const int n0 = blockIdx.x * BN;
  const int M = d.M, N = d.N, K = d.K;
  const int KT = (K + BK - 1) / BK;

  for (int64_t b = blockIdx.z; b < d.batch; b += gridDim.z) {
    if (d.active != nullptr && d.active[b] == 0) continue;
    const z64* Ag = d.a_ptrs ? d.a_ptrs[b] : at<const z64>(d.A, b);
    const z64* Bg = d.b_ptrs ? d.b_ptrs[b] : at<const z64>(d.B, b);

    // 3M (Gauss) products: p1 = sum ar br, p2 = sum ai bi,
    // p3 = sum (ar + ai)(br + bi); Re = p1 - p2, Im = p3 - p1 - p2.
    double p1[MT][NT][4], p2[MT][NT][4], p3[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          p1[i][j][q] = 0.0;
          p2[i][j][q] = 0.0;
          p3[i][j][q] = 0.0;
        }

    // Prologue.
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < KT) {
        load_tile<OPA, true>(As + s * A_SIZE, Ag, d.A.ld, M, K, m0, s * BK, tid);
        load_tile<OPB, false>(Bs + s * B_SIZE, Bg, d.B.ld, N, K, n0, s * BK, tid);
      }
      cp_async_commit();
    }

    for (int kt = 0; kt < KT; ++kt) {
      cp_async_wait<STAGES - 2>();
      __syncthreads();
      {
        const int nk = kt + STAGES - 1;
        if (nk < KT) {
          const int st = nk % STAGES;
          load_tile<OPA, true>(As + st * A_SIZE, Ag, d.A.ld, M, K, m0, nk * BK, tid);
          load_tile<OPB, false>(Bs + st * B_SIZE, Bg, d.B.ld, N, K, n0, nk * BK, tid);
        }
        cp_async_commit();
      }
      const z64* as = As + (kt % STAGES) * A_SIZE;
      const z64* bs = Bs + (kt % STAGES) * B_SIZE;
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double ar[MT][2], ai[MT][2], sa[MT][2];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
          const int r = wm0 + i * 16 + g;
          z64 v0, v1;
          if (OPA == 0) {
            v0 = as[r * S_MK + kk + tq];
            v1 = as[(r + 8) * S_MK + kk + tq];
          } else {
            v0 = as[(kk + tq) * S_KM + r];
            v1 = as[(kk + tq) * S_KM + r + 8];
          }
          ar[i][0] = v0.x;
          ar[i][1] = v1.x;
          ai[i][0] = (OPA == 1) ? -v0.y : v0.y;
          ai[i][1] = (OPA == 1) ? -v1.y : v1.y;
          sa[i][0] = ar[i][0] + ai[i][0];
          sa[i][1] = ar[i][1] + ai[i][1];
        }
        double br[NT], bi[NT], sb[NT];
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const int c = wn0 + j * 8 + g;
          z64 v;
          if (OPB == 1)
            v = bs[c * S_MK + kk + tq];
          else
            v = bs[(kk + tq) * (BN + 2) + c];
          br[j] = v.x;
          bi[j] = (OPB == 1) ? -v.y : v.y;
          sb[j] = br[j] + bi[j];
        }
        // Three passes over the 2x4 tiles: the products feeding one
        // accumulator are 8 independent MMAs apart.
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) mma_f64(p1[i][j], ar[i][0], ar[i][1], br[j]);
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) mma_f64(p2[i][j], ai[i][0], ai[i][1], bi[j]);
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) mma_f64(p3[i][j], sa[i][0], sa[i][1], sb[j]);
      }
    }
    cp_async_wait<0>();
    __syncthreads();

    // Epilogue through a padded shared-memory tile (it reuses the stage
    // buffers) so that global reads and writes are coalesced in either
    // orientation. Phase A (fragment layout, lanes mostly along rows):
    // alpha * acc + the conjugate-transposed addends -> tile.
    z64* tile = smem;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int rl = wm0 + i * 16 + g + ((q >> 1) << 3);
          const int cl = wn0 + j * 8 + 2 * tq + (q & 1);
          const double re = p1[i][j][q] - p2[i][j][q];
          const double im = p3[i][j][q] - (p1[i][j][q] + p2[i][j][q]);
          tile[rl * TS + cl] = zmul(d.alpha, make_double2(re, im));
        }
    for (int t = 0; t < d.nadd; ++t) {
      const Addend& ad = d.add[t];
      if (!ad.conj_trans) continue;
      const z64* p = (t == 0 && d.d_ptrs) ? d.d_ptrs[b] : at<const z64>(ad.m, b);
      z64 x[MT][NT][4];  // all loads first: many in flight, no aliasing stalls
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = m0 + wm0 + i * 16 + g + ((q >> 1) << 3);
            const int c = n0 + wn0 + j * 8 + 2 * tq + (q & 1);
            x[i][j][q] = (r < M && c < N) ? p[(int64_t)c * ad.m.ld + r] : make_double2(0.0, 0.0);
          }
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int rl = wm0 + i * 16 + g + ((q >> 1) << 3);
            const int cl = wn0 + j * 8 + 2 * tq + (q & 1);
            tile[rl * TS + cl] = zfma(ad.coef, zconj(x[i][j][q]), tile[rl * TS + cl]);
          }
    }
    __syncthreads();
    // Phase B (lanes along columns): the other addends, C3 and C.
    constexpr int PER = BM * BN / THREADS;  // elements per thread
    for (int t = 0; t < d.nadd; ++t) {
      const Addend& ad = d.add[t];
      if (ad.conj_trans) continue;
      const z64* p = (t == 0 && d.d_ptrs) ? d.d_ptrs[b] : at<const z64>(ad.m, b);
      z64 x[PER];  // all loads first: many in flight, no aliasing stalls
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int e = tid + k * THREADS;
        const int r = m0 + e / BN, c = n0 + e % BN;
        x[k] = (r < M && c < N) ? p[(int64_t)r * ad.m.ld + c] : make_double2(0.0, 0.0);
      }
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int e = tid + k * THREADS;
        const int rl = e / BN, cl = e % BN;
        tile[rl * TS + cl] = zfma(ad.coef, x[k], tile[rl * TS + cl]);
      }
    }
    if (!d.C3.null()) {
#pragma unroll 4
      for (int e = tid; e < BM * BN; e += THREADS) {
        const int rl = e / BN, cl = e % BN;
        const int r = m0 + rl, c = n0 + cl;
        if (r >= M || c >= N) continue;
        z64 v3 = zmul(d.scale3, tile[rl * TS + cl]);
        for (int t = d.nadd; t < d.nadd + d.nadd3; ++t) {
          const Addend& ad = d.add[t];
          const z64* p = at<const z64>(ad.m, b);
          const z64 x = ad.conj_trans ? zconj(p[(int64_t)c * ad.m.ld + r]) : p[(int64_t)r * ad.m.ld + c];
          v3 = zfma(ad.coef, x, v3);
        }
        at<z64>(d.C3, b)[(int64_t)r * d.C3.ld + c] = v3;
      }
    }
    if (!d.C.null()) {
      z64* out = d.c_ptrs ? d.c_ptrs[b] : at<z64>(d.C, b);
#pragma unroll 8
      for (int e = tid; e < BM * BN; e += THREADS) {
        const int rl = e / BN, cl = e % BN;
        const int r = m0 + rl, c = n0 + cl;
        if (r < M && c < N) out[(int64_t)r * d.C.ld + c] = tile[rl * TS + cl];
      }
    }
    // Phase C (lanes along rows): the conjugate-transposed second store,
    // after every thread's phase-B updates of the tile.
    if (!d.C2.null()) {
      __syncthreads();
      z64* out2 = at<z64>(d.C2, b);
#pragma unroll 8
      for (int e = tid; e < BM * BN; e += THREADS) {
        const int rl = e % BM, cl = e / BM;
        const int r = m0 + rl, c = n0 + cl;
        if (r < M && c < N) out2[(int64_t)c * d.C2.ld + r] = zmul(d.coef2, zconj(tile[rl * TS + cl]));
      }
    }
    __syncthreads();  // the tile aliases the stage buffers of the next entry
  }
}

template <int OPA, int OPB>
int launch(const GemmDesc& d, cudaStream_t s) {
  constexpr int A_SIZE = (OPA == 0) ? A_MK_SIZE : A_KM_SIZE;
  constexpr int B_SIZE = (OPB == 1) ? B_NK_SIZE : B_KN_SIZE;
  constexpr size_t stages = STAGES * (A_SIZE + B_SIZE) * sizeof(z64);
  constexpr size_t tile = (size_t)BM * TS * sizeof(z64);
  constexpr size_t smem = stages > tile ? stages : tile;
  QTX_CHECK_CUDA(cudaFuncSetAttribute(zgemm_kernel<OPA, OPB>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((d.N + BN - 1) / BN, (d.M + BM - 1) / BM,
            (unsigned)(d.batch < 65535 ? d.batch : 65535));
  KernelArgs args{d};
  ProfScope prof(QTX_KERNEL_ZGEMM, 8.0 * d.M * d.N * (double)d.K * (double)d.batch, s);
  zgemm_kernel<OPA, OPB><<<grid, THREADS, smem, s>>>(args);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

bool aligned16(const MatRef& m) { return (reinterpret_cast<uintptr_t>(m.p) & 15u) == 0; }

}  // namespace

int zgemm(const GemmDesc& d, cudaStream_t s) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return QTX_OK;
  if (d.K < 0 || d.nadd < 0 || d.nadd3 < 0 || d.nadd + d.nadd3 > kMaxAddends) {
    set_error("zgemm: invalid sizes or addend count");
    return QTX_ERR_ARG;
  }
  const bool grouped = d.a_ptrs || d.b_ptrs || d.c_ptrs || d.d_ptrs;
  if (grouped && (d.K <= 0 || !d.a_ptrs || !d.b_ptrs || !d.c_ptrs || d.nadd > 1 || d.nadd3 > 0 ||
                  (d.nadd == 1 && !d.d_ptrs) || !d.C2.null() || !d.C3.null())) {
    set_error("zgemm: the grouped form needs A, B and C tables, K > 0, at most one addend (with its table) "
              "and no second outputs");
    return QTX_ERR_ARG;
  }
  if (!grouped && d.K > 0 && (d.A.null() || d.B.null())) {
    // A zero operand: the product vanishes; only the addends remain.
    GemmDesc z = d;
    z.K = 0;
    z.A = d.C.null() ? d.C3 : d.C;
    z.B = z.A;
    return zgemm(z, s);
  }
  if ((d.K > 0 && (!aligned16(d.A) || !aligned16(d.B))) || !aligned16(d.C) || !aligned16(d.C2) ||
      !aligned16(d.C3)) {
    set_error("zgemm: complex128 operands must be 16-byte aligned");
    return QTX_ERR_ARG;
  }
  GemmDesc dd = d;
  for (int t = 0; !grouped && t < d.nadd + d.nadd3; ++t) {
    if (dd.add[t].m.null()) {  // drop zero addends
      for (int u = t; u + 1 < dd.nadd + dd.nadd3; ++u) dd.add[u] = dd.add[u + 1];
      if (t < dd.nadd)
        --dd.nadd;
      else
        --dd.nadd3;
      --t;
      if (dd.nadd + dd.nadd3 <= 0) break;
    }
  }
  if (dd.K == 0) {
    // Pure epilogue: the tile loop runs zero iterations.
    if (dd.A.null()) dd.A = dd.C.null() ? dd.C3 : dd.C;
    if (dd.B.null()) dd.B = dd.A;
  }
  if (!grouped && dd.K > 0 && gemm_slices() > 0 && oz_supported(dd.K, gemm_slices())) {
    size_t bytes = 0;
    void* scr = oz_bound(&bytes);
    if (scr != nullptr) return zgemm_oz(dd, gemm_slices(), scr, bytes, s);
  }
  const int key = dd.opA * 2 + dd.opB;
  switch (key) {
    case 0: return launch<0, 0>(dd, s);
    case 1: return launch<0, 1>(dd, s);
    case 2: return launch<1, 0>(dd, s);
    default: return launch<1, 1>(dd, s);
  }
}

}  // namespace qtx
