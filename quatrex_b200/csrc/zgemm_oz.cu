// Complex128 GEMM emulated on the int8 tensor cores (tcgen05.mma.kind::i8).
//
//   out = alpha op(A) op(B) + sum_t coef_t op_t(D_t)      (the zgemm contract)
//
// B200's FP64 tensor rate is a small fraction of its int8 rate, so the FP64
// products of the RGF and Sancho-Rubio recursions can instead be formed from
// exact integer products of short slices of the operands (the splitting idea
// of Ozaki, Ogita, Oishi and Rump, Numer. Algorithms 59 (2012), in its
// integer-tensor-core form):
//
// * Complex -> real. Rows of op(A) interleave (re, im) along k (A', M x 2K);
//   op(B) is expanded to B'' (2N x 2K) with rows 2j = (re, -im) and
//   2j+1 = (im, re) per k. The even / odd columns of A' B''^T are Re / Im C.
// * Split (oz_split_kernel, oz_split_strip_kernel). Every row of A' and every
//   row pair of B'' gets a power-of-two scale 2^e with all |x| < 2^e;
//   x 2^(L-e), L = 8S - 2, is rounded to an integer X (|X| <= 2^L) and written
//   as S balanced base-256 digits, X = sum_p D_p 256^(S-1-p), D_p in
//   [-128, 127] (the leading one in [-65, 65]): the bytes of
//   (X + 0x80..80) xor 0x80..80. Digit p of every element forms int8 plane p,
//   stored as the GEMM consumes it: one contiguous, already swizzled block per
//   (row tile, 64-byte K block), zero-padded to the tile grid.
// * Products (oz_gemm_kernel). sum_k X_ik Y_jk = sum_{p,q} 256^(2S-2-p-q)
//   (D_p E_q^T)_ij. The pairs with p + q = d < S are summed exactly into int32
//   TMEM accumulator d (|D E| <= 2^14; S * 2K * 2^14 < 2^31 is checked); the
//   pairs with p + q >= S fall below the rounding of X and are dropped. With
//   the accumulators side by side in TMEM, A plane p times the stacked B
//   planes 0..S-1-p is one MMA of M=128, N = 64 (S-p) (split at N = 256)
//   per 32-byte K step.
// * Epilogue. T = sum_d acc_d 256^(S-1-d) in FP64, times
//   2^(e_i + f_j - 2L + 8(S-1)), then zgemm's epilogue (alpha, addends, C,
//   the conjugate-transposed C2, C3).
//
// Error per element: below 2 S K 2^(4-8S) max_k|op(A)_ik| max_k|op(B)_kj|
// (rounding to L bits plus the dropped pairs); measured relative to
// (|A||B|)_ij it is ~3e-10 at S = 5, ~1e-12 at S = 6, ~7e-15 at S = 7.
// An element whose row of op(A) or column of op(B) holds an Inf or NaN is
// NaN (the digits of a non-finite value do not exist).
//
// CTA tile 128 x 64 real columns (32 complex); a 64-byte K stage holds the
// S A blocks and S B blocks (2S bulk copies, no multicast). One producer
// thread keeps 2-4 stages in flight on full/empty mbarriers; one thread
// issues the MMAs and commits each stage back to its empty barrier; all
// warps run the epilogue once the final commit lands. Every mbarrier wait
// is bounded; on a time-out the CTA records the error, lets its copies and
// MMAs in flight finish, skips its epilogue, frees its TMEM and returns.
#include <algorithm>

#include "common.cuh"

namespace qtx {

namespace {

constexpr int TM = 128;                // UMMA M: rows of op(A) per CTA
constexpr int KS = 64;                 // int8 K per pipeline stage (64-byte rows, two MMA K steps;
                                       // 32-byte stages measured slower)
constexpr int THREADS = 256;
constexpr int PLANE_A = TM * KS;       // 8 KB
constexpr int SPLIT_ROWS = 32;         // op-rows per split CTA
constexpr int SPLIT_K = 32;            // complex k per split tile (4 per thread)
constexpr long long kWaitLimit = 1ll << 26;

__device__ int g_oz_error = 0;

// Per plane count S: the CTA's real output columns TN (UMMA N of one digit
// group), CTAs per SM and the stage ring. The S int32 accumulator groups take
// S x TN TMEM columns; at most 256 lets two CTAs share an SM, so that one's
// loads, barrier round trips and epilogue overlap the other's MMAs (S <= 4 at
// TN = 64, S = 5 at TN = 48); S >= 6 keeps one CTA per SM with 64 columns.
template <int S>
struct Cfg {
  static constexpr int TN = S == 5 ? 48 : 64;
  static constexpr int TNC = TN / 2;         // complex output columns per CTA
  static constexpr int TILE_LD = TNC + 1;    // epilogue tile row (complex), padded
  static constexpr int PLANE_B = TN * KS;    // one B plane block
  static constexpr int CPS = S * TN <= 256 ? 2 : 1;
  static constexpr int STAGE = S * (PLANE_A + PLANE_B);
  static constexpr int BUDGET = CPS == 2 ? 110 * 1024 : 220 * 1024;
  static constexpr int NS = BUDGET / STAGE >= 4 ? 4 : BUDGET / STAGE;
  static constexpr int TMEM_COLS = S * TN <= 256 ? 256 : 512;
  static constexpr int L = 8 * S - 2;
  static constexpr int GROUPS_PER_MMA = 256 / TN;  // UMMA N <= 256
  static_assert(S >= 3 && S <= 8, "slice count");
  static_assert(NS >= 2, "at least two stages");
  static_assert(TM * TILE_LD * 16 <= NS * STAGE, "epilogue tile must fit the stages");
  static_assert(TN % 16 == 0 && TN % 8 == 0, "UMMA N granularity");
};

// Complex output columns per CTA for S planes (the padding unit of op(B)).
constexpr int tnc_for(int slices) { return slices == 5 ? 24 : 32; }

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Padded geometry of one call: rows of A', complex columns of op(B), K.
struct Geom {
  int Mp, Np, Kc, Kp;
  size_t item_bytes(int S) const {
    return sizeof(int) * (size_t)(Mp + Np) + (size_t)S * (size_t)(Mp + 2 * Np) * Kp;
  }
};
Geom geom(int M, int N, int K, int tnc) {
  Geom g;
  g.Mp = round_up(std::max(M, 1), TM);
  g.Np = round_up(std::max(N, 1), tnc);
  g.Kc = round_up(std::max(K, 1), KS / 2);
  g.Kp = 2 * g.Kc;
  return g;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of 16-byte chunk `ch` of `row` in a K-major tile of KS-byte
// rows, swizzled as the UMMA descriptor below declares: 8-row groups of
// 8 KS bytes; the chunk index XOR row bits above the 128-byte line
// (SWIZZLE_32B: chunk ^ (row / 4) % 2; SWIZZLE_64B: chunk ^ (row / 2) % 4).
__device__ __forceinline__ uint32_t swz_offset(int row, int ch) {
  const int x = KS == 64 ? ((row >> 1) & 3) : ((row >> 2) & 1);
  return (uint32_t)((row >> 3) * (8 * KS) + (row & 7) * KS + ((ch ^ x) << 4));
}

// UMMA shared-memory descriptor, K-major, SWIZZLE_32B (KS = 32) or
// SWIZZLE_64B (KS = 64), 8-row groups 8 KS bytes apart.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  static_assert(KS == 32 || KS == 64, "stage rows of 32 or 64 bytes");
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                   // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((8 * KS) >> 4) << 32;     // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;                   // descriptor version (sm_100)
  d |= (uint64_t)(KS == 64 ? 4 : 6) << 61;  // SWIZZLE_64B / SWIZZLE_32B
  return d;
}

// Instruction descriptor: D s32, A/B s8, K-major both, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

// 2^s as a double for -1022 <= s <= 1023 (exact).
__device__ __forceinline__ double pow2(int s) { return __longlong_as_double((long long)(s + 1023) << 52); }
// x 2^s, exactly as scalbn, with one multiply where 2^s and the result are normal.
__device__ __forceinline__ double ldexp_fast(double x, int s) {
  return (s >= -1000 && s <= 1000) ? x * pow2(s) : scalbn(x, s);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity));
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
      smem_addr(bar)));
}

// Bulk global -> shared copy completing on an mbarrier (no multicast).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Biased exponent field of |x| (0 for zero and subnormals).
__device__ __forceinline__ int exp_bits(double x) {
  return (int)((__double_as_longlong(x) >> 52) & 0x7FF);
}
// Scale exponent e with |x| < 2^e for every x of a row whose largest
// exponent field is eb.
__device__ __forceinline__ int scale_exp(int eb) { return eb > 0 ? eb - 1022 : -1022; }

// ---------------------------------------------------------------------------
// Split: one CTA per SPLIT_ROWS op-rows of one batch entry. Sweep 1 finds
// each row's scale exponent, sweep 2 (whose reads hit L2) writes the digit
// planes. STRIDED: consecutive op-rows are adjacent in memory (op-row r,
// index k at X[k ld + r]); otherwise k is contiguous (X[r ld + k]).
// ---------------------------------------------------------------------------
struct SplitArgs {
  MatRef X;
  int rows, K;  // logical op-rows and depth
  int conj;
  int rows_p, Kc, Kp;
  int64_t b0, bc;
  int* expo;       // [bc][rows_p] biased exponent fields
  int8_t* planes;  // [S][bc][prows][Kp], prows = rows_p (A) or 2 rows_p (B)
  const int* active;
};

__device__ __forceinline__ void cp_async16z(uint32_t dst, const void* src, bool pred) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(pred ? 16 : 0));
}

constexpr int SPLIT_LD = SPLIT_K + 1;                            // tile row (complex), padded
constexpr int SPLIT_TILE = SPLIT_ROWS * SPLIT_LD;                // complex elements per tile
constexpr size_t SPLIT_SMEM = 2 * SPLIT_TILE * sizeof(double2);  // two tiles (double buffer)

template <int S, bool ISB, bool STRIDED>
__global__ void __launch_bounds__(THREADS, 4) oz_split_kernel(const SplitArgs a) {
  constexpr int L = 8 * S - 2;
  extern __shared__ __align__(16) uint8_t split_smem[];
  double2* tiles = reinterpret_cast<double2*>(split_smem);  // [2][SPLIT_ROWS][SPLIT_LD]
  __shared__ int red[8][SPLIT_ROWS];
  __shared__ int rexp[SPLIT_ROWS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = blockIdx.x * SPLIT_ROWS;
  const int bl = blockIdx.y;
  const int64_t b = a.b0 + bl;
  if (a.active != nullptr && a.active[b] == 0) return;
  const double2* X = at<const double2>(a.X, b);
  const double sgn = a.conj ? -1.0 : 1.0;

  // K tile t of the strip -> shared buffer `buf` (cp.async, zero-filled
  // outside the matrix); column perm(k) = 8 (k % 4) + k / 4 within a row.
  auto load_tile = [&](int t, int buf) {
    double2* tl = tiles + buf * SPLIT_TILE;
    const int k0 = t * SPLIT_K;
    if (STRIDED) {
#pragma unroll
      for (int i = warp; i < SPLIT_K; i += 8) {
        const int k = k0 + i, r = r0 + lane;
        const bool ok = k < a.K && r < a.rows;
        cp_async16z(smem_addr(tl + lane * SPLIT_LD + 8 * (i & 3) + (i >> 2)),
                    ok ? X + (int64_t)k * a.X.ld + r : X, ok);
      }
    } else {
#pragma unroll
      for (int i = warp; i < SPLIT_ROWS; i += 8) {
        const int r = r0 + i;
#pragma unroll
        for (int j = lane; j < SPLIT_K; j += 32) {
          const int k = k0 + j;
          const bool ok = k < a.K && r < a.rows;
          cp_async16z(smem_addr(tl + i * SPLIT_LD + 8 * (j & 3) + (j >> 2)), ok ? X + (int64_t)r * a.X.ld + k : X,
                      ok);
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  const int ntiles = (a.Kc + SPLIT_K - 1) / SPLIT_K;
  load_tile(0, 0);  // in flight during sweep 1

  // Sweep 1: the largest exponent field of each op-row.
  if (STRIDED) {
    // lanes along rows, warps along k
    const int r = r0 + lane;
    int m = 0;
    if (r < a.rows) {
      // 8 independent loads in flight per lane
      int mm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      int k = warp;
      for (; k + 56 < a.K; k += 64) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const double2 v = X[(int64_t)(k + 8 * u) * a.X.ld + r];
          mm[u] = max(mm[u], max(exp_bits(v.x), exp_bits(v.y)));
        }
      }
      for (; k < a.K; k += 8) {
        const double2 v = X[(int64_t)k * a.X.ld + r];
        mm[0] = max(mm[0], max(exp_bits(v.x), exp_bits(v.y)));
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) m = max(m, mm[u]);
    }
    red[warp][lane] = m;
    __syncthreads();
    if (warp == 0) {
      int mm = red[0][lane];
#pragma unroll
      for (int w = 1; w < 8; ++w) mm = max(mm, red[w][lane]);
      rexp[lane] = mm;
    }
  } else {
    // one warp per row, lanes along k; the warp's 4 rows interleaved so that
    // 4 x 4 independent loads are in flight per lane
    int m4[4] = {0, 0, 0, 0};
    for (int k = lane; k < a.K; k += 128) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int r = r0 + warp + 8 * q, kk = k + 32 * u;
          if (r < a.rows && kk < a.K) {
            const double2 v = X[(int64_t)r * a.X.ld + kk];
            m4[q] = max(m4[q], max(exp_bits(v.x), exp_bits(v.y)));
          }
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int m = m4[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) rexp[warp + 8 * q] = m;
    }
  }
  __syncthreads();
  // the last CTA may reach past the padded row count (a multiple of the
  // GEMM's tile, not of SPLIT_ROWS): those rows are neither stored nor read
  if (tid < SPLIT_ROWS && r0 + tid < a.rows_p) a.expo[(int64_t)bl * a.rows_p + r0 + tid] = rexp[tid];

  // Sweep 2: digits, SPLIT_K complex k at a time through shared memory. The
  // tile stores k at column perm(k) = 8 (k % 4) + k / 4, so the 8 lanes that
  // read 4 consecutive k each hit distinct banks.
  const int rr = tid >> 3;       // op-row of this thread
  const int kc = (tid & 7) * 4;  // first of its 4 k in the tile
  const int e = scale_exp(rexp[rr]);
  const int sx = L - e;  // x 2^sx is the integer X before rounding
  const bool fast = sx >= -1000 && sx <= 1000;
  const double fx = fast ? pow2(sx) : 0.0;
  const int prows = ISB ? 2 * a.rows_p : a.rows_p;
  const size_t plane = (size_t)a.bc * prows * a.Kp;
  const int nkb = a.Kp / KS;
  for (int t = 0; t < ntiles; ++t) {
    const int k0 = t * SPLIT_K;
    if (t + 1 < ntiles) {
      load_tile(t + 1, (t + 1) & 1);  // its buffer was last read before the barrier ending t - 1
      asm volatile("cp.async.wait_group 1;\n" ::);
    } else {
      asm volatile("cp.async.wait_group 0;\n" ::);
    }
    __syncthreads();
    const double2* tl = tiles + (t & 1) * SPLIT_TILE;
    const int kb = k0 + kc;
    if (kb >= a.Kc || r0 + rr >= a.rows_p) {
      __syncthreads();
      continue;
    }
    // Balanced base-256 digits (each in [-128, 127]) of X are the bytes of
    // Z = (X + C) xor C, C = 0x80 in each of the S low bytes: adding C makes
    // every byte non-negative and xor 0x80 re-centres it. Digit p (most
    // significant first) is byte S-1-p. -X_im gets its own Z (its digits are
    // not the negated digits of X_im where one is -128).
    constexpr unsigned long long kC = 0x8080808080808080ull >> (8 * (8 - S));
    uint32_t zr[4][2], zi[4][2], zn[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double2 v = tl[rr * SPLIT_LD + 8 * j + (kc >> 2)];  // k = kc + j
      const long long xr = __double2ll_rn(fast ? v.x * fx : scalbn(v.x, sx));
      const long long xi = __double2ll_rn(fast ? sgn * v.y * fx : scalbn(sgn * v.y, sx));
      const unsigned long long ur = ((unsigned long long)xr + kC) ^ kC;
      const unsigned long long ui = ((unsigned long long)xi + kC) ^ kC;
      zr[j][0] = (uint32_t)ur, zr[j][1] = (uint32_t)(ur >> 32);
      zi[j][0] = (uint32_t)ui, zi[j][1] = (uint32_t)(ui >> 32);
      if (ISB) {
        const unsigned long long un = ((unsigned long long)(-xi) + kC) ^ kC;
        zn[j][0] = (uint32_t)un, zn[j][1] = (uint32_t)(un >> 32);
      }
    }
    const int row = r0 + rr;
#pragma unroll
    for (int p = 0; p < S; ++p) {
      const int bi = S - 1 - p;          // byte of Z holding digit p
      const int hw = bi >> 2;            // its 32-bit half
      const uint32_t sel = (uint32_t)(bi & 3);
      const uint32_t pair = sel | ((4u + sel) << 4);  // byte sel of x, byte sel of y
      uint32_t w0[2], w1[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int j0 = 2 * q, j1 = 2 * q + 1;
        if (ISB) {
          // row 2j: (re, -im); row 2j+1: (im, re)
          w0[q] = __byte_perm(__byte_perm(zr[j0][hw], zn[j0][hw], pair), __byte_perm(zr[j1][hw], zn[j1][hw], pair),
                              0x5410);
          w1[q] = __byte_perm(__byte_perm(zi[j0][hw], zr[j0][hw], pair), __byte_perm(zi[j1][hw], zr[j1][hw], pair),
                              0x5410);
        } else {
          w0[q] = __byte_perm(__byte_perm(zr[j0][hw], zi[j0][hw], pair), __byte_perm(zr[j1][hw], zi[j1][hw], pair),
                              0x5410);
          w1[q] = 0u;
        }
      }
      // plane block (p, entry, row tile, K block) as the GEMM stages load it:
      // 8 bytes = one half of a 16-byte swizzle chunk
      const int col = 2 * kb;  // byte column
      const size_t kblk = (size_t)(col / KS);
      const int ch = (col % KS) / 16, half = col & 15;
      int8_t* ptile = a.planes + (size_t)p * plane + (size_t)bl * prows * a.Kp;
      const uint2 v0 = make_uint2(w0[0], w0[1]);
      if (ISB) {
        const uint2 v1 = make_uint2(w1[0], w1[1]);
        const int r2 = 2 * row;
        constexpr int TNB = Cfg<S>::TN;
        int8_t* blk = ptile + ((size_t)(r2 / TNB) * nkb + kblk) * Cfg<S>::PLANE_B;
        *reinterpret_cast<uint2*>(blk + swz_offset(r2 % TNB, ch) + half) = v0;
        *reinterpret_cast<uint2*>(blk + swz_offset(r2 % TNB + 1, ch) + half) = v1;
      } else {
        int8_t* blk = ptile + ((size_t)(row / TM) * nkb + kblk) * PLANE_A;
        *reinterpret_cast<uint2*>(blk + swz_offset(row % TM, ch) + half) = v0;
      }
    }
    __syncthreads();  // buffer t & 1 is refilled at iteration t + 1
  }
}


// ---------------------------------------------------------------------------
// Split, strip form: one CTA per STRIP_ROWS op-rows of one batch entry with
// the whole K strip staged in shared memory by one wave of cp.async, so the
// operand is read from HBM once; exponents and digits come from the copy.
// Within a row, complex k sits at strip_pos(k): 256-element segments with
// k % 8 major, so the 32 lanes that each take 8 consecutive k read distinct
// banks. Used for padded K from 512 up to STRIP_MAX_KC.
// ---------------------------------------------------------------------------
constexpr int STRIP_ROWS = 8;
constexpr int STRIP_MAX_KC = 1792;  // 8 rows x 1792 x 16 B = 224 KB

__device__ __forceinline__ int strip_pos(int k) { return (k & ~255) | ((k & 7) << 5) | ((k >> 3) & 31); }

__host__ __device__ inline int strip_len(int Kc) { return (Kc + 255) / 256 * 256; }

template <int S, bool ISB, bool STRIDED>
__global__ void __launch_bounds__(THREADS, 2) oz_split_strip_kernel(const SplitArgs a) {
  constexpr int L = 8 * S - 2;
  extern __shared__ __align__(16) uint8_t split_smem[];
  double2* strip = reinterpret_cast<double2*>(split_smem);  // [STRIP_ROWS][KL]
  __shared__ int rexp[STRIP_ROWS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = blockIdx.x * STRIP_ROWS;
  const int bl = blockIdx.y;
  const int64_t b = a.b0 + bl;
  if (a.active != nullptr && a.active[b] == 0) return;
  const double2* X = at<const double2>(a.X, b);
  const double sgn = a.conj ? -1.0 : 1.0;
  const int KL = strip_len(a.Kc);  // padded row length (zero-filled past K)

  if (STRIDED) {
    // the 8 op-rows of one k are adjacent: 8 lanes per k, 32 k per pass
    const int i = tid & 7, r = r0 + i;
    for (int k = tid >> 3; k < KL; k += THREADS / 8) {
      const bool ok = k < a.K && r < a.rows;
      cp_async16z(smem_addr(strip + i * KL + strip_pos(k)), ok ? X + (int64_t)k * a.X.ld + r : X, ok);
    }
  } else {
    const int r = r0 + warp;  // warp w loads row w
    for (int k = lane; k < KL; k += 32) {
      const bool ok = k < a.K && r < a.rows;
      cp_async16z(smem_addr(strip + warp * KL + strip_pos(k)), ok ? X + (int64_t)r * a.X.ld + k : X, ok);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();

  // Row scale exponent: warp w reduces row w.
  const double2* row_s = strip + warp * KL;
  {
    int m = 0;
    for (int q = lane; q < KL; q += 32) {
      const double2 v = row_s[q];
      m = max(m, max(exp_bits(v.x), exp_bits(v.y)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) {
      rexp[warp] = m;
      a.expo[(int64_t)bl * a.rows_p + r0 + warp] = m;
    }
  }
  __syncwarp();
  const int e = scale_exp(rexp[warp]);
  const int sx = L - e;
  const bool fast = sx >= -1000 && sx <= 1000;
  const double fx = fast ? pow2(sx) : 0.0;
  const int prows = ISB ? 2 * a.rows_p : a.rows_p;
  const size_t plane = (size_t)a.bc * prows * a.Kp;
  const int nkb = a.Kp / KS;
  const int row = r0 + warp;
  constexpr unsigned long long kC = 0x8080808080808080ull >> (8 * (8 - S));

  // Digits: lane l takes chunks c = l, l + 32, ... of 8 consecutive k.
  for (int c = lane; c < a.Kc / 8; c += 32) {
    uint32_t zr[8][2], zi[8][2], zn[8][2];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double2 v = row_s[(c >> 5) * 256 + 32 * j + (c & 31)];  // k = 8c + j
      const long long xr = __double2ll_rn(fast ? v.x * fx : scalbn(v.x, sx));
      const long long xi = __double2ll_rn(fast ? sgn * v.y * fx : scalbn(sgn * v.y, sx));
      const unsigned long long ur = ((unsigned long long)xr + kC) ^ kC;
      const unsigned long long ui = ((unsigned long long)xi + kC) ^ kC;
      zr[j][0] = (uint32_t)ur, zr[j][1] = (uint32_t)(ur >> 32);
      zi[j][0] = (uint32_t)ui, zi[j][1] = (uint32_t)(ui >> 32);
      if (ISB) {
        const unsigned long long un = ((unsigned long long)(-xi) + kC) ^ kC;
        zn[j][0] = (uint32_t)un, zn[j][1] = (uint32_t)(un >> 32);
      }
    }
    const int col = 16 * c;  // byte column of the chunk: one 16-byte swizzle chunk
    const size_t kblk = (size_t)(col / KS);
    const int ch = (col % KS) / 16;
#pragma unroll
    for (int p = 0; p < S; ++p) {
      const int bi = S - 1 - p;
      const int hw = bi >> 2;
      const uint32_t sel = (uint32_t)(bi & 3);
      const uint32_t pair = sel | ((4u + sel) << 4);
      uint32_t w0[4], w1[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j0 = 2 * q, j1 = 2 * q + 1;
        if (ISB) {
          w0[q] = __byte_perm(__byte_perm(zr[j0][hw], zn[j0][hw], pair), __byte_perm(zr[j1][hw], zn[j1][hw], pair),
                              0x5410);
          w1[q] = __byte_perm(__byte_perm(zi[j0][hw], zr[j0][hw], pair), __byte_perm(zi[j1][hw], zr[j1][hw], pair),
                              0x5410);
        } else {
          w0[q] = __byte_perm(__byte_perm(zr[j0][hw], zi[j0][hw], pair), __byte_perm(zr[j1][hw], zi[j1][hw], pair),
                              0x5410);
          w1[q] = 0u;
        }
      }
      int8_t* ptile = a.planes + (size_t)p * plane + (size_t)bl * prows * a.Kp;
      const uint4 v0 = make_uint4(w0[0], w0[1], w0[2], w0[3]);
      if (ISB) {
        const uint4 v1 = make_uint4(w1[0], w1[1], w1[2], w1[3]);
        const int r2 = 2 * row;
        constexpr int TNB = Cfg<S>::TN;
        int8_t* blk = ptile + ((size_t)(r2 / TNB) * nkb + kblk) * Cfg<S>::PLANE_B;
        *reinterpret_cast<uint4*>(blk + swz_offset(r2 % TNB, ch)) = v0;
        *reinterpret_cast<uint4*>(blk + swz_offset(r2 % TNB + 1, ch)) = v1;
      } else {
        int8_t* blk = ptile + ((size_t)(row / TM) * nkb + kblk) * PLANE_A;
        *reinterpret_cast<uint4*>(blk + swz_offset(row % TM, ch)) = v0;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Products and epilogue.
// ---------------------------------------------------------------------------
struct GArgs {
  int M, N, Mp, Np, Kp;
  int64_t b0, bc;
  int na, nb;  // plane batch entries of A / B: bc, or 1 for an operand broadcast over the batch
  const int8_t* pa;  // [S][bc][Mp][Kp]
  const int8_t* pb;  // [S][bc][2 Np][Kp]
  const int* ea;     // [bc][Mp]
  const int* eb;     // [bc][Np]
  z64 alpha;
  Addend add[kMaxAddends];
  int nadd, nadd3;
  MatRef C, C2, C3;
  z64 coef2, scale3;
  const int* active;
};

__device__ __forceinline__ z64 addend_at(const GArgs& a, int t, int64_t b, int r, int c) {
  const Addend& ad = a.add[t];
  const z64* p = at<const z64>(ad.m, b);
  const z64 x = ad.conj_trans ? zconj(p[(int64_t)c * ad.m.ld + r]) : p[(int64_t)r * ad.m.ld + c];
  return zmul(ad.coef, x);
}

// The MMAs of one 64-byte K stage. The S group accumulators lie side by side
// in TMEM (group d in columns [64 d, 64 d + 64)) and the B slices side by
// side in shared memory, so A slice p times the stack of B slices
// 0..S-1-p lands on groups p..S-1 in one instruction of N = 64 (S - p),
// split at N = 256: each pair (p, q) with p + q < S is formed exactly once.
template <int S>
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t sa, uint32_t sb, bool first) {
  using C = Cfg<S>;
#pragma unroll
  for (int kk = 0; kk < KS / 32; ++kk) {
#pragma unroll
    for (int p = 0; p < S; ++p) {
      const uint64_t da = make_desc(sa + p * PLANE_A + kk * 32);
#pragma unroll
      for (int g0 = 0; g0 < S - p; g0 += C::GROUPS_PER_MMA) {
        const int ng = (S - p - g0) < C::GROUPS_PER_MMA ? (S - p - g0) : C::GROUPS_PER_MMA;
        const uint64_t db = make_desc(sb + g0 * C::PLANE_B + kk * 32);
        mma_i8(tmem + (uint32_t)((p + g0) * C::TN), da, db, idesc_i8(ng * C::TN),
               (first && kk == 0 && p == 0) ? 0u : 1u);
      }
    }
  }
}

// Epilogue, part 1 (lane = tile row rl = 32 wl + lane; TMEM lane quarter
// wl): real columns [c_lo, c_hi) of the S digit-group accumulators are
// combined in FP64, scaled by 2^(e_r + f_c - 2L + 8(S-1)), multiplied by
// alpha, the conjugate-transposed addends added, and the complex results
// written to the shared tile.
template <int S>
__device__ __forceinline__ void epilogue_tmem(const GArgs& a, uint32_t tmem, z64* tile, const int* s_ea,
                                              const int* s_eb, int64_t b, int m0, int nr0, int wl, int lane,
                                              int c_lo, int c_hi) {
  constexpr int L = 8 * S - 2;
  constexpr int TN = Cfg<S>::TN, TILE_LD = Cfg<S>::TILE_LD;
  const int rl = wl * 32 + lane;
  const int r = m0 + rl;
  const uint32_t lane_base = tmem + ((uint32_t)(wl * 32) << 16);
  const int er = scale_exp(s_ea[rl]) - 2 * L + 8 * (S - 1);
  int n_ct = 0;
  for (int t = 0; t < a.nadd; ++t) n_ct += a.add[t].conj_trans;
#pragma unroll 1
  for (int c0 = c_lo; c0 < c_hi; c0 += 8) {
    uint32_t v[S][8];
#pragma unroll
    for (int d = 0; d < S; ++d)
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
          : "=r"(v[d][0]), "=r"(v[d][1]), "=r"(v[d][2]), "=r"(v[d][3]), "=r"(v[d][4]), "=r"(v[d][5]),
            "=r"(v[d][6]), "=r"(v[d][7])
          : "r"(lane_base + (uint32_t)(d * TN + c0)));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
    double T[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      T[j] = (double)(int)v[0][j];
#pragma unroll
      for (int d = 1; d < S; ++d) T[j] = fma(T[j], 256.0, (double)(int)v[d][j]);
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int cl = c0 / 2 + jj;
      const int c = nr0 / 2 + cl;
      const int sh = er + scale_exp(s_eb[cl]);
      z64 z = zmul(a.alpha, make_double2(ldexp_fast(T[2 * jj], sh), ldexp_fast(T[2 * jj + 1], sh)));
      if (s_ea[rl] == 0x7FF || s_eb[cl] == 0x7FF)  // Inf or NaN in the row / column: no digits
        z = make_double2(__longlong_as_double(0x7FF8000000000000ll), __longlong_as_double(0x7FF8000000000000ll));
      if (n_ct > 0 && r < a.M && c < a.N)
        for (int t = 0; t < a.nadd; ++t)
          if (a.add[t].conj_trans) z = zadd(z, addend_at(a, t, b, r, c));
      tile[rl * TILE_LD + cl] = z;
    }
  }
}

// Epilogue, part 2 (lane = tile column, threads t0.. of nt): the other
// addends, C3 and C; the tile keeps the primary result for C2.
template <int S>
__device__ __forceinline__ void epilogue_rows(const GArgs& a, z64* tile, int64_t b, int m0, int n0, int t0,
                                              int nt) {
  constexpr int TNC = Cfg<S>::TNC, TILE_LD = Cfg<S>::TILE_LD;
#pragma unroll 1
  for (int e = t0; e < TM * TNC; e += nt) {
    const int rl = e / TNC, cl = e % TNC;
    const int rr = m0 + rl, c = n0 + cl;
    if (rr >= a.M || c >= a.N) continue;
    z64 v = tile[rl * TILE_LD + cl];
    for (int t = 0; t < a.nadd; ++t)
      if (!a.add[t].conj_trans) v = zadd(v, addend_at(a, t, b, rr, c));
    if (!a.C3.null()) {
      z64 v3 = zmul(a.scale3, v);
      for (int t = a.nadd; t < a.nadd + a.nadd3; ++t) v3 = zadd(v3, addend_at(a, t, b, rr, c));
      at<z64>(a.C3, b)[(int64_t)rr * a.C3.ld + c] = v3;
    }
    if (!a.C.null()) at<z64>(a.C, b)[(int64_t)rr * a.C.ld + c] = v;
    if (!a.C2.null()) tile[rl * TILE_LD + cl] = v;
  }
}

// Epilogue, part 3 (lane = tile row): the conjugate-transposed store C2.
template <int S>
__device__ __forceinline__ void epilogue_c2(const GArgs& a, const z64* tile, int64_t b, int m0, int n0, int t0,
                                            int nt) {
  constexpr int TNC = Cfg<S>::TNC, TILE_LD = Cfg<S>::TILE_LD;
#pragma unroll 1
  for (int e = t0; e < TM * TNC; e += nt) {
    const int rl = e % TM, cl = e / TM;
    const int rr = m0 + rl, c = n0 + cl;
    if (rr >= a.M || c >= a.N) continue;
    at<z64>(a.C2, b)[(int64_t)c * a.C2.ld + rr] = zmul(a.coef2, zconj(tile[rl * TILE_LD + cl]));
  }
}

template <int S>
__global__ void __launch_bounds__(THREADS, Cfg<S>::CPS) oz_gemm_kernel(const GArgs a) {
  using C = Cfg<S>;
  constexpr int TN = C::TN, TNC = C::TNC, PLANE_B = C::PLANE_B;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::NS * C::STAGE);  // stage loaded
  uint64_t* empty = full + C::NS;                                             // stage consumed by the MMAs
  uint64_t* done = empty + C::NS;                                             // all MMAs complete
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  int* s_ea = reinterpret_cast<int*>(tmem_slot + 4);  // [TM] row scale exponents (biased)
  int* s_eb = s_ea + TM;                              // [TNC] column scale exponents
  z64* tile = reinterpret_cast<z64*>(smem);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nr0 = blockIdx.x * TN;  // first B'' row (real output column)
  const int m0 = blockIdx.y * TM;
  const int bl = blockIdx.z;
  const int64_t b = a.b0 + bl;
  if (a.active != nullptr && a.active[b] == 0) return;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 32) {
    for (int i = 0; i < C::NS; ++i) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  const int ba = a.na > 1 ? bl : 0, bb = a.nb > 1 ? bl : 0;  // plane entries of this batch entry
  if (tid < TM) s_ea[tid] = a.ea[(int64_t)ba * a.Mp + m0 + tid];
  else if (tid < TM + TNC) s_eb[tid - TM] = a.eb[(int64_t)bb * a.Np + nr0 / 2 + tid - TM];
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;

  // Plane block (p, entry, tile, K block) is contiguous and pre-swizzled.
  const int nkb = a.Kp / KS;
  const int MT = a.Mp / TM, NT = 2 * a.Np / TN;
  const int8_t* ga = a.pa + ((size_t)ba * MT + blockIdx.y) * nkb * PLANE_A;
  const int8_t* gb = a.pb + ((size_t)bb * NT + blockIdx.x) * nkb * PLANE_B;
  const size_t sliceA = (size_t)a.na * MT * nkb * PLANE_A;
  const size_t sliceB = (size_t)a.nb * NT * nkb * PLANE_B;

  bool ok = true;
  if (warp == 1 && lane == 0) {
    // Producer: 2S bulk copies per stage onto full[buf], once the MMAs of the
    // stage that used the buffer before have released it (empty[buf]).
    int issued = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      const int buf = kb % C::NS;
      const uint32_t u = (uint32_t)(kb / C::NS);
      if (kb >= C::NS && !mbar_wait(&empty[buf], (u - 1u) & 1u)) {
        ok = false;
        break;
      }
      const uint32_t st = smem_addr(smem + buf * C::STAGE);
      expect_tx(&full[buf], (uint32_t)C::STAGE);
#pragma unroll
      for (int p = 0; p < S; ++p)
        bulk_g2s(st + p * PLANE_A, ga + p * sliceA + (size_t)kb * PLANE_A, PLANE_A, &full[buf]);
#pragma unroll
      for (int q = 0; q < S; ++q)
        bulk_g2s(st + S * PLANE_A + q * PLANE_B, gb + q * sliceB + (size_t)kb * PLANE_B, PLANE_B, &full[buf]);
      issued = kb + 1;
    }
    if (!ok)  // let the copies in flight land before the CTA exits
      for (int kb = issued > C::NS ? issued - C::NS : 0; kb < issued; ++kb)
        mbar_wait(&full[kb % C::NS], (uint32_t)(kb / C::NS) & 1u);
  } else if (warp == 0 && lane == 0) {
    // MMA issuer: consumes the stages in order; tcgen05.commit releases each.
    for (int kb = 0; kb < nkb; ++kb) {
      const int buf = kb % C::NS;
      if (!mbar_wait(&full[buf], (uint32_t)(kb / C::NS) & 1u)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const uint32_t sa = smem_addr(smem + buf * C::STAGE);
      issue_stage<S>(tmem, sa, sa + S * PLANE_A, kb == 0);
      mma_commit(&empty[buf]);
    }
    mma_commit(done);  // tracks every MMA issued above, on either path
    if (!mbar_wait(done, 0)) ok = false;
  }
  ok = __syncthreads_and(ok);

  if (ok) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    // Phase A: lane = tile row (TMEM lane quarter of warp w is w % 4), warps
    // 0-3 / 4-7 take real columns 0-31 / 32-63.
    epilogue_tmem<S>(a, tmem, tile, s_ea, s_eb, b, m0, nr0, warp & 3, lane, (warp >> 2) * (TN / 2),
                     (warp >> 2) * (TN / 2) + TN / 2);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    epilogue_rows<S>(a, tile, b, m0, nr0 / 2, tid, THREADS);
    if (!a.C2.null()) {
      __syncthreads();
      epilogue_c2<S>(a, tile, b, m0, nr0 / 2, tid, THREADS);
    }
  } else if (tid == 0) {
    atomicExch(&g_oz_error, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(C::TMEM_COLS));
}

// Thread-local GEMM path and bound scratch.
thread_local int t_slices = 0;
thread_local void* t_scratch = nullptr;
thread_local size_t t_scratch_bytes = 0;

template <int S>
int run_split(const MatRef& X, int rows, int K, int conj, bool isb, bool strided, const Geom& g,
              int rows_p, int64_t b0, int64_t bc, int* expo, int8_t* planes, const int* active,
              cudaStream_t s) {
  SplitArgs a{};
  a.X = X;
  a.rows = rows;
  a.K = K;
  a.conj = conj;
  a.rows_p = rows_p;
  a.Kc = g.Kc;
  a.Kp = g.Kp;
  a.b0 = b0;
  a.bc = bc;
  a.expo = expo;
  a.planes = planes;
  a.active = active;
  if (strip_len(g.Kc) >= 512 && strip_len(g.Kc) <= STRIP_MAX_KC) {
    // whole K strips in shared memory: one HBM read of the operand (measured
    // faster than the two-sweep form from K = 512 on, slower below)
    const size_t smem = (size_t)STRIP_ROWS * strip_len(g.Kc) * sizeof(double2);
    dim3 grid(rows_p / STRIP_ROWS, (unsigned)bc);
    auto launch = [&](auto kern) -> int {
      QTX_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kern<<<grid, THREADS, smem, s>>>(a);
      return QTX_OK;
    };
    if (isb) {
      QTX_TRY(strided ? launch(oz_split_strip_kernel<S, true, true>) : launch(oz_split_strip_kernel<S, true, false>));
    } else {
      QTX_TRY(strided ? launch(oz_split_strip_kernel<S, false, true>)
                      : launch(oz_split_strip_kernel<S, false, false>));
    }
    QTX_CHECK_LAUNCH();
    return QTX_OK;
  }
  dim3 grid((rows_p + SPLIT_ROWS - 1) / SPLIT_ROWS, (unsigned)bc);
  auto launch = [&](auto kern) -> int {
    QTX_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SPLIT_SMEM));
    kern<<<grid, THREADS, SPLIT_SMEM, s>>>(a);
    return QTX_OK;
  };
  if (isb) {
    QTX_TRY(strided ? launch(oz_split_kernel<S, true, true>) : launch(oz_split_kernel<S, true, false>));
  } else {
    QTX_TRY(strided ? launch(oz_split_kernel<S, false, true>) : launch(oz_split_kernel<S, false, false>));
  }
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

// Digit planes of the batch chunk [b0, b0 + n): [ea][eb] exponents, then the
// A and B planes. An operand with batch stride 0 (one matrix for every
// entry, e.g. the coupling blocks) is split once per chunk.
template <int S>
int run(const GemmDesc& d, void* scratch, size_t bytes, cudaStream_t s) {
  using C = Cfg<S>;
  static_assert(C::TNC == tnc_for(S), "padding unit of op(B) matches the tile");
  const Geom g = geom(d.M, d.N, d.K, C::TNC);
  const bool bca = d.A.stride == 0, bcb = d.B.stride == 0;
  const size_t a_item = sizeof(int) * (size_t)g.Mp + (size_t)S * g.Mp * g.Kp;
  const size_t b_item = sizeof(int) * (size_t)g.Np + (size_t)S * 2 * g.Np * g.Kp;
  const size_t fixed = (bca ? a_item : 0) + (bcb ? b_item : 0) + 1024;
  const size_t per = (bca ? 0 : a_item) + (bcb ? 0 : b_item);
  int64_t bc = std::min<int64_t>(d.batch, 65535);
  if (per > 0 && bytes < fixed + per * (size_t)bc) bc = bytes > fixed ? (int64_t)((bytes - fixed) / per) : 0;
  if (bc <= 0 || bytes < fixed) {
    set_error("zgemm (int8 emulation): scratch too small for one batch entry");
    return QTX_ERR_WORKSPACE;
  }
  const size_t smem = (size_t)C::NS * C::STAGE + 1024 + 256 + sizeof(int) * (TM + C::TNC);
  QTX_CHECK_CUDA(cudaFuncSetAttribute(oz_gemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (int64_t b0 = 0; b0 < d.batch; b0 += bc) {
    const int64_t n = std::min<int64_t>(bc, d.batch - b0);
    const int64_t na = bca ? 1 : n, nb = bcb ? 1 : n;
    char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(scratch) + 255) & ~uintptr_t(255));
    int* ea = reinterpret_cast<int*>(base);
    int* eb = ea + (size_t)na * g.Mp;
    int8_t* pa = reinterpret_cast<int8_t*>(base + ((sizeof(int) * ((size_t)na * g.Mp + (size_t)nb * g.Np) + 255) & ~size_t(255)));
    int8_t* pb = pa + (size_t)S * na * g.Mp * g.Kp;
    {
      ProfScope prof(QTX_KERNEL_SPLIT, 16.0 * ((double)d.M * na + (double)d.N * nb) * d.K, s, 2);
      QTX_TRY(run_split<S>(d.A, d.M, d.K, d.opA, false, d.opA == 1, g, g.Mp, bca ? 0 : b0, na, ea, pa,
                           bca ? nullptr : d.active, s));
      QTX_TRY(run_split<S>(d.B, d.N, d.K, d.opB, true, d.opB == 0, g, g.Np, bcb ? 0 : b0, nb, eb, pb,
                           bcb ? nullptr : d.active, s));
    }
    GArgs a{};
    a.M = d.M;
    a.N = d.N;
    a.Mp = g.Mp;
    a.Np = g.Np;
    a.Kp = g.Kp;
    a.b0 = b0;
    a.bc = n;
    a.na = (int)na;
    a.nb = (int)nb;
    a.pa = pa;
    a.pb = pb;
    a.ea = ea;
    a.eb = eb;
    a.alpha = d.alpha;
    for (int t = 0; t < kMaxAddends; ++t) a.add[t] = d.add[t];
    a.nadd = d.nadd;
    a.nadd3 = d.nadd3;
    a.C = d.C;
    a.C2 = d.C2;
    a.C3 = d.C3;
    a.coef2 = d.coef2;
    a.scale3 = d.scale3;
    a.active = d.active;
    ProfScope prof(QTX_KERNEL_ZGEMM_EMU, 8.0 * d.M * d.N * (double)d.K * (double)n, s);
    dim3 grid(2 * g.Np / C::TN, g.Mp / TM, (unsigned)n);
    oz_gemm_kernel<S><<<grid, THREADS, smem, s>>>(a);
    QTX_CHECK_LAUNCH();
  }
  return QTX_OK;
}

}  // namespace

size_t oz_scratch_bytes(int M, int N, int K, int64_t batch, int slices) {
  if (slices <= 0 || batch <= 0) return 0;
  const Geom g = geom(M, N, K, tnc_for(slices));
  return g.item_bytes(slices) * (size_t)std::min<int64_t>(batch, 65535) + 1024;
}

bool oz_supported(int K, int slices) {
  // S digit pairs of |D E| <= 2^14 summed over 2K must stay inside int32.
  return slices >= 3 && slices <= 8 && (double)slices * 2.0 * K * 16384.0 < 2147483648.0;
}

int zgemm_oz(const GemmDesc& d, int slices, void* scratch, size_t bytes, cudaStream_t s) {
  if (!oz_supported(d.K, slices)) {
    set_error("zgemm (int8 emulation): slice count outside 3-8 or K too large for int32 sums");
    return QTX_ERR_ARG;
  }
  switch (slices) {
    case 3: return run<3>(d, scratch, bytes, s);
    case 4: return run<4>(d, scratch, bytes, s);
    case 5: return run<5>(d, scratch, bytes, s);
    case 6: return run<6>(d, scratch, bytes, s);
    case 7: return run<7>(d, scratch, bytes, s);
    default: return run<8>(d, scratch, bytes, s);
  }
}

void set_gemm_slices(int slices) { t_slices = slices; }
int gemm_slices() { return t_slices; }

void* oz_bound(size_t* bytes) {
  if (bytes) *bytes = t_scratch_bytes;
  return t_scratch;
}

OzScope::OzScope(Workspace& ws, int n, int64_t batch) {
  prev_p = t_scratch;
  prev_bytes = t_scratch_bytes;
  if (t_slices > 0 && n > 0) {
    const size_t bytes = oz_scratch_bytes(n, n, n, batch, t_slices);
    void* p = ws.take(bytes);
    t_scratch = p;
    t_scratch_bytes = p ? bytes : 0;
  }
}
OzScope::~OzScope() {
  t_scratch = prev_p;
  t_scratch_bytes = prev_bytes;
}

int oz_status_take(int* flag) {
  int h = 0;
  QTX_CHECK_CUDA(cudaMemcpyFromSymbol(&h, g_oz_error, sizeof(int)));
  if (h) {
    const int zero = 0;
    QTX_CHECK_CUDA(cudaMemcpyToSymbol(g_oz_error, &zero, sizeof(int)));
  }
  *flag = h;
  return QTX_OK;
}

}  // namespace qtx
