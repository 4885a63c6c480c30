// Batched complex64 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a)
// with split-TF32 products accumulated in FP32 (the mixed-precision path).
//
//   out = alpha op(A) op(B) + sum_t coef_t op_t(D_t)     (complex64 in / out)
//
// Each FP32 operand x is split into x_hi = tf32(x) and x_lo = tf32(x - x_hi);
// a real product is a_hi b_hi + a_hi b_lo + a_lo b_hi (the lo*lo term is
// below FP32 rounding). A complex product is the 4M combination of real
// products, with the subtraction folded into the instruction descriptor's
// negate bit: 12 tcgen05.mma.kind::tf32 per K step of 8.
//
// CTA tile 128 x 64 (one UMMA M=128, N=64), K block 32 FP32 (128-byte rows,
// SWIZZLE_128B K-major), eight warps, one buffer of split planes (96 KB) so
// that two CTAs share an SM and one's prologue/epilogue overlaps the other's
// MMAs. While the tensor cores run the MMAs of block kb (issued by one
// thread), all warps load block kb+1 from global memory into registers, wait
// for the MMAs (tcgen05.commit -> mbarrier), then split and store the planes.
// Accumulators live in TMEM (Re in columns 0-63, Im in 64-127) and are read
// back with tcgen05.ld. The epilogue goes through a padded shared-memory tile
// so that global reads and writes are coalesced in either orientation:
// row-per-lane for conjugate-transposed addends and the transposed store,
// column-per-lane for everything else. Every mbarrier wait is bounded; on a
// time-out the CTA raises the error flag, skips its epilogue, frees its TMEM
// and returns.
#include "common.cuh"

namespace qtx {
namespace {

constexpr int TM = 128;       // UMMA M
constexpr int TN = 64;        // UMMA N
constexpr int TK = 32;        // fp32 elements per K block (128 B rows)
constexpr int THREADS = 256;  // eight warps
constexpr int PLANE_A = TM * TK * 4;  // bytes of one A plane (16 KB)
constexpr int PLANE_B = TN * TK * 4;  // bytes of one B plane (8 KB)
constexpr int PLANES_BYTES = 4 * PLANE_A + 4 * PLANE_B;  // re/im x hi/lo for A and B
constexpr int CTAS_PER_SM = 2;                               // one plane buffer each
constexpr int S_LD = TN + 1;                                 // padded epilogue tile row (float2)
constexpr int A_TASKS = TM * (TK / 4) / THREADS;             // 4 row-chunks of op(A) per thread
constexpr int B_TASKS = TN * (TK / 4) / THREADS;             // 2 row-chunks of op(B) per thread
constexpr int TMEM_COLS = 128;
constexpr long long kWaitLimit = 1ll << 26;  // bounded mbarrier polls

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_trunc(float x) {
  return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
}

// Byte offset of the 16-byte chunk holding (row, k4-chunk) in a SWIZZLE_128B
// K-major tile: 8-row groups of 1024 B, chunk index XOR (row % 8).
__device__ __forceinline__ uint32_t sw128_offset(int row, int chunk) {
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4));
}

// UMMA shared-memory descriptor, K-major SWIZZLE_128B, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)(1) << 16;             // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;     // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;               // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;               // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D f32, A/B tf32, K-major both, N = 64, M = 128.
__host__ __device__ constexpr uint32_t make_idesc(bool neg_a) {
  return (1u << 4)                  // D format f32
         | (2u << 7)                // A tf32
         | (2u << 10)               // B tf32
         | ((neg_a ? 1u : 0u) << 13)
         | ((uint32_t)(TN >> 3) << 17)
         | ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
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

// Bounded wait; returns false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < kWaitLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
      smem_addr(bar)));
}

__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::);
}

struct Args {
  int M, N, K;
  int64_t batch;
  MatRef A, B;
  int opA, opB;
  float2 alpha;
  struct Add {
    MatRef m;
    float2 coef;
    int ct;
  } add[kMaxAddends];
  int nadd, nadd3;
  MatRef C, C2, C3;
  float2 coef2, scale3;
  int* err;
};

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

struct Regs {
  float2 a[A_TASKS][4];
  float2 b[B_TASKS][4];
};

// Task t of op(A): (row, chunk of 4 k). Lanes walk the memory-contiguous index.
template <int OPA>
__device__ __forceinline__ void a_task(int t, int& row, int& chunk) {
  if (OPA == 0) {
    row = t >> 3;
    chunk = t & 7;
  } else {
    row = t & (TM - 1);
    chunk = t >> 7;
  }
}
template <int OPB>
__device__ __forceinline__ void b_task(int t, int& row, int& chunk) {
  if (OPB == 1) {
    row = t >> 3;
    chunk = t & 7;
  } else {
    row = t & (TN - 1);
    chunk = t >> 6;
  }
}

// Global -> registers for one K block (all loads issued back to back). With
// VEC (operands 16-byte aligned, even leading dimensions) the K-contiguous
// operands are read two complex numbers per 16-byte load.
template <int OPA, int OPB, bool VEC>
__device__ __forceinline__ void load_regs(const Args& a, const c32* Ag, const c32* Bg, Regs& R, int m0,
                                          int n0, int k0, int tid) {
#pragma unroll
  for (int i = 0; i < A_TASKS; ++i) {
    int row, chunk;
    a_task<OPA>(tid + i * THREADS, row, chunk);
    const int gr = m0 + row;
    if (OPA == 0 && VEC) {
#pragma unroll
      for (int e = 0; e < 4; e += 2) {
        const int gk = k0 + chunk * 4 + e;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gr < a.M && gk + 1 < a.K) {
          v = *reinterpret_cast<const float4*>(Ag + (int64_t)gr * a.A.ld + gk);
        } else if (gr < a.M && gk < a.K) {
          const float2 w = Ag[(int64_t)gr * a.A.ld + gk];
          v = make_float4(w.x, w.y, 0.f, 0.f);
        }
        R.a[i][e] = make_float2(v.x, v.y);
        R.a[i][e + 1] = make_float2(v.z, v.w);
      }
      continue;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gk = k0 + chunk * 4 + e;
      float2 v = make_float2(0.f, 0.f);
      if (gr < a.M && gk < a.K) {
        if (OPA == 0) {
          v = Ag[(int64_t)gr * a.A.ld + gk];
        } else {
          v = Ag[(int64_t)gk * a.A.ld + gr];
          v.y = -v.y;
        }
      }
      R.a[i][e] = v;
    }
  }
#pragma unroll
  for (int i = 0; i < B_TASKS; ++i) {
    int row, chunk;
    b_task<OPB>(tid + i * THREADS, row, chunk);
    const int gn = n0 + row;
    if (OPB == 1 && VEC) {
#pragma unroll
      for (int e = 0; e < 4; e += 2) {
        const int gk = k0 + chunk * 4 + e;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gn < a.N && gk + 1 < a.K) {
          v = *reinterpret_cast<const float4*>(Bg + (int64_t)gn * a.B.ld + gk);
        } else if (gn < a.N && gk < a.K) {
          const float2 w = Bg[(int64_t)gn * a.B.ld + gk];
          v = make_float4(w.x, w.y, 0.f, 0.f);
        }
        R.b[i][e] = make_float2(v.x, -v.y);
        R.b[i][e + 1] = make_float2(v.z, -v.w);
      }
      continue;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int gk = k0 + chunk * 4 + e;
      float2 v = make_float2(0.f, 0.f);
      if (gn < a.N && gk < a.K) {
        if (OPB == 0) {
          v = Bg[(int64_t)gk * a.B.ld + gn];
        } else {
          v = Bg[(int64_t)gn * a.B.ld + gk];
          v.y = -v.y;
        }
      }
      R.b[i][e] = v;
    }
  }
}

__device__ __forceinline__ void split4(const float2 (&v)[4], float4& hr, float4& lr, float4& hi, float4& li) {
  float* phr = &hr.x;
  float* plr = &lr.x;
  float* phi = &hi.x;
  float* pli = &li.x;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float rh = tf32_trunc(v[e].x), ih = tf32_trunc(v[e].y);
    phr[e] = rh;
    plr[e] = tf32_trunc(v[e].x - rh);
    phi[e] = ih;
    pli[e] = tf32_trunc(v[e].y - ih);
  }
}

// Registers -> the eight split planes (SWIZZLE_128B K-major).
template <int OPA, int OPB>
__device__ __forceinline__ void store_planes(const Regs& R, uint8_t* planes, int tid) {
  uint8_t* pb = planes + 4 * PLANE_A;
#pragma unroll
  for (int i = 0; i < A_TASKS; ++i) {
    int row, chunk;
    a_task<OPA>(tid + i * THREADS, row, chunk);
    float4 hr, lr, hi, li;
    split4(R.a[i], hr, lr, hi, li);
    const uint32_t off = sw128_offset(row, chunk);
    *reinterpret_cast<float4*>(planes + off) = hr;
    *reinterpret_cast<float4*>(planes + PLANE_A + off) = lr;
    *reinterpret_cast<float4*>(planes + 2 * PLANE_A + off) = hi;
    *reinterpret_cast<float4*>(planes + 3 * PLANE_A + off) = li;
  }
#pragma unroll
  for (int i = 0; i < B_TASKS; ++i) {
    int row, chunk;
    b_task<OPB>(tid + i * THREADS, row, chunk);
    float4 hr, lr, hi, li;
    split4(R.b[i], hr, lr, hi, li);
    const uint32_t off = sw128_offset(row, chunk);
    *reinterpret_cast<float4*>(pb + off) = hr;
    *reinterpret_cast<float4*>(pb + PLANE_B + off) = lr;
    *reinterpret_cast<float4*>(pb + 2 * PLANE_B + off) = hi;
    *reinterpret_cast<float4*>(pb + 3 * PLANE_B + off) = li;
  }
}

// The 12 MMAs of one K step (8 fp32) on stage base addresses.
__device__ __forceinline__ void issue_kstep(uint32_t tmem, uint32_t sa, uint32_t sb, int kk,
                                            bool first) {
  const uint32_t koff = (uint32_t)kk * 32;  // bytes along the 128-byte row
  const uint64_t arh = make_desc(sa + 0 * PLANE_A + koff), arl = make_desc(sa + 1 * PLANE_A + koff);
  const uint64_t aih = make_desc(sa + 2 * PLANE_A + koff), ail = make_desc(sa + 3 * PLANE_A + koff);
  const uint64_t brh = make_desc(sb + 0 * PLANE_B + koff), brl = make_desc(sb + 1 * PLANE_B + koff);
  const uint64_t bih = make_desc(sb + 2 * PLANE_B + koff), bil = make_desc(sb + 3 * PLANE_B + koff);
  constexpr uint32_t ID = make_idesc(false), IDN = make_idesc(true);
  const uint32_t re = tmem, im = tmem + TN;
  // Re += Ar Br - Ai Bi  (small terms first)
  mma_tf32(re, arl, brh, ID, first ? 0u : 1u);
  mma_tf32(re, arh, brl, ID, 1u);
  mma_tf32(re, arh, brh, ID, 1u);
  mma_tf32(re, ail, bih, IDN, 1u);
  mma_tf32(re, aih, bil, IDN, 1u);
  mma_tf32(re, aih, bih, IDN, 1u);
  // Im += Ar Bi + Ai Br
  mma_tf32(im, arl, bih, ID, first ? 0u : 1u);
  mma_tf32(im, arh, bil, ID, 1u);
  mma_tf32(im, arh, bih, ID, 1u);
  mma_tf32(im, ail, brh, ID, 1u);
  mma_tf32(im, aih, brl, ID, 1u);
  mma_tf32(im, aih, brh, ID, 1u);
}

__device__ __forceinline__ float2 addend_at(const Args& a, int t, int64_t b, int r, int c) {
  const auto& ad = a.add[t];
  const c32* p = at<const c32>(ad.m, b);
  float2 x = ad.ct ? p[(int64_t)c * ad.m.ld + r] : p[(int64_t)r * ad.m.ld + c];
  if (ad.ct) x.y = -x.y;
  return cmulf(ad.coef, x);
}

template <int OPA, int OPB, bool VEC>
__global__ void __launch_bounds__(THREADS, CTAS_PER_SM) cgemm_tc_kernel(const Args a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment for the SWIZZLE_128B atoms.
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* planes = smem;
  float2* tile = reinterpret_cast<float2*>(smem);  // epilogue tile [TM][S_LD], reuses the planes
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + PLANES_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int m0 = blockIdx.y * TM;
  const int n0 = blockIdx.x * TN;
  const int KB = (a.K + TK - 1) / TK;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  uint32_t phase = 0;
  bool ok = true;
  Regs R;
  // Addends split by orientation: conjugate-transposed ones are read with
  // lanes along rows (phase A), the others with lanes along columns (phase B).
  int n_ct = 0;
  for (int t = 0; t < a.nadd; ++t) n_ct += a.add[t].ct;

  for (int64_t b = blockIdx.z; b < a.batch && ok; b += gridDim.z) {
    const c32* Ag = at<const c32>(a.A, b);
    const c32* Bg = at<const c32>(a.B, b);
    if (KB > 0) {
      load_regs<OPA, OPB, VEC>(a, Ag, Bg, R, m0, n0, 0, tid);
      store_planes<OPA, OPB>(R, planes, tid);
      fence_async_smem();
      __syncthreads();
    }
    for (int kb = 0; kb < KB; ++kb) {
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
        const uint32_t sa = smem_addr(planes);
        const uint32_t sb = sa + 4 * PLANE_A;
#pragma unroll
        for (int kk = 0; kk < TK / 8; ++kk) issue_kstep(tmem, sa, sb, kk, kb == 0 && kk == 0);
        mma_commit(bar);
      }
      const bool more = kb + 1 < KB;
      if (more) load_regs<OPA, OPB, VEC>(a, Ag, Bg, R, m0, n0, (kb + 1) * TK, tid);
      // One thread polls the MMA-completion barrier; the others wait at the
      // block barrier instead of spinning on shared memory.
      if (tid == 0 && !mbar_wait(bar, phase)) ok = false;
      phase ^= 1u;
      ok = __syncthreads_and(ok);
      if (more && ok) {
        store_planes<OPA, OPB>(R, planes, tid);
        fence_async_smem();
      }
      if (!__syncthreads_and(ok)) {
        ok = false;
        break;
      }
    }
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);

    // Phase A (warps 0-3 and 4-7 split the columns; lane = tile row, the
    // TMEM lane quarter of warp w is w % 4): alpha * acc + ct addends -> tile.
    {
      const int wl = warp & 3;
      const int rl = wl * 32 + lane;
      const int r = m0 + rl;
      const uint32_t lane_base = tmem + ((uint32_t)(wl * 32) << 16);
      const int cbeg = (warp >> 2) * (TN / 2);
#pragma unroll 1
      for (int c0 = cbeg; c0 < cbeg + TN / 2; c0 += 16) {
        uint32_t vr[16], vi[16];
        if (KB > 0) {
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
              : "=r"(vr[0]), "=r"(vr[1]), "=r"(vr[2]), "=r"(vr[3]), "=r"(vr[4]), "=r"(vr[5]),
                "=r"(vr[6]), "=r"(vr[7]), "=r"(vr[8]), "=r"(vr[9]), "=r"(vr[10]), "=r"(vr[11]),
                "=r"(vr[12]), "=r"(vr[13]), "=r"(vr[14]), "=r"(vr[15])
              : "r"(lane_base + (uint32_t)c0));
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
              : "=r"(vi[0]), "=r"(vi[1]), "=r"(vi[2]), "=r"(vi[3]), "=r"(vi[4]), "=r"(vi[5]),
                "=r"(vi[6]), "=r"(vi[7]), "=r"(vi[8]), "=r"(vi[9]), "=r"(vi[10]), "=r"(vi[11]),
                "=r"(vi[12]), "=r"(vi[13]), "=r"(vi[14]), "=r"(vi[15])
              : "r"(lane_base + (uint32_t)(TN + c0)));
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0u;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int c = n0 + c0 + j;
          float2 v = cmulf(a.alpha, make_float2(__uint_as_float(vr[j]), __uint_as_float(vi[j])));
          if (n_ct > 0 && r < a.M && c < a.N) {
            for (int t = 0; t < a.nadd; ++t) {
              if (!a.add[t].ct) continue;
              const float2 y = addend_at(a, t, b, r, c);
              v.x += y.x;
              v.y += y.y;
            }
          }
          tile[rl * S_LD + c0 + j] = v;
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();

    // Phase B (lane = tile column): remaining addends, C3 and C.
#pragma unroll 1
    for (int e = tid; e < TM * TN; e += THREADS) {
      const int rl = e / TN, cl = e % TN;
      const int r = m0 + rl, c = n0 + cl;
      if (r >= a.M || c >= a.N) continue;
      float2 v = tile[rl * S_LD + cl];
      for (int t = 0; t < a.nadd; ++t) {
        if (a.add[t].ct) continue;
        const float2 y = addend_at(a, t, b, r, c);
        v.x += y.x;
        v.y += y.y;
      }
      if (!a.C3.null()) {
        float2 v3 = cmulf(a.scale3, v);
        for (int t = a.nadd; t < a.nadd + a.nadd3; ++t) {
          const float2 y = addend_at(a, t, b, r, c);
          v3.x += y.x;
          v3.y += y.y;
        }
        at<c32>(a.C3, b)[(int64_t)r * a.C3.ld + c] = v3;
      }
      if (!a.C.null()) at<c32>(a.C, b)[(int64_t)r * a.C.ld + c] = v;
      if (!a.C2.null()) tile[rl * S_LD + cl] = v;
    }

    // Phase C (lane = tile row): the conjugate-transposed store C2.
    if (!a.C2.null()) {
      __syncthreads();
#pragma unroll 1
      for (int e = tid; e < TM * TN; e += THREADS) {
        const int rl = e % TM, cl = e / TM;
        const int r = m0 + rl, c = n0 + cl;
        if (r >= a.M || c >= a.N) continue;
        const float2 v = tile[rl * S_LD + cl];
        at<c32>(a.C2, b)[(int64_t)c * a.C2.ld + r] = cmulf(a.coef2, make_float2(v.x, -v.y));
      }
    }
    __syncthreads();
  }
  if (!ok && tid == 0 && a.err != nullptr) atomicExch(a.err, 1);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
}

template <int OPA, int OPB, bool VEC>
int launch_v(const Args& a, cudaStream_t s) {
  static_assert(TM * S_LD * (int)sizeof(float2) <= PLANES_BYTES, "epilogue tile must fit the planes");
  const size_t smem = (size_t)PLANES_BYTES + 64 + 1024;
  QTX_CHECK_CUDA(cudaFuncSetAttribute(cgemm_tc_kernel<OPA, OPB, VEC>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((a.N + TN - 1) / TN, (a.M + TM - 1) / TM, (unsigned)(a.batch < 65535 ? a.batch : 65535));
  ProfScope prof(QTX_KERNEL_CGEMM, 8.0 * a.M * a.N * (double)a.K * (double)a.batch, s);
  cgemm_tc_kernel<OPA, OPB, VEC><<<grid, THREADS, smem, s>>>(a);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

bool vec_ok(const MatRef& m) {
  return (reinterpret_cast<uintptr_t>(m.p) & 15u) == 0 && (m.ld % 2) == 0 && (m.stride % 2) == 0;
}

template <int OPA, int OPB>
int launch(const Args& a, cudaStream_t s) {
  // The 16-byte path reads the K-contiguous operands; both must allow it.
  const bool va = OPA != 0 || vec_ok(a.A);
  const bool vb = OPB != 1 || vec_ok(a.B);
  if (va && vb) return launch_v<OPA, OPB, true>(a, s);
  return launch_v<OPA, OPB, false>(a, s);
}

}  // namespace

int cgemm_tc(const CGemmDesc& d, cudaStream_t s) {
  if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return QTX_OK;
  if (d.nadd < 0 || d.nadd3 < 0 || d.nadd + d.nadd3 > kMaxAddends ||
      (d.K > 0 && (d.A.null() || d.B.null())) || (d.C.null() && d.C3.null())) {
    set_error("cgemm_tc: invalid arguments (null operand or output, or too many addends)");
    return QTX_ERR_ARG;
  }
  Args a{};
  a.M = d.M;
  a.N = d.N;
  a.K = d.K;
  a.batch = d.batch;
  a.A = d.A;
  a.B = d.B;
  a.opA = d.opA;
  a.opB = d.opB;
  a.alpha = d.alpha;
  a.nadd = 0;
  a.nadd3 = 0;
  for (int t = 0; t < d.nadd + d.nadd3; ++t) {
    if (d.add[t].m.null()) continue;
    const int k = a.nadd + a.nadd3;
    a.add[k].m = d.add[t].m;
    a.add[k].coef = d.add[t].coef;
    a.add[k].ct = d.add[t].conj_trans;
    if (t < d.nadd)
      ++a.nadd;
    else
      ++a.nadd3;
  }
  a.C = d.C;
  a.C2 = d.C2;
  a.C3 = d.C3;
  a.coef2 = d.coef2;
  a.scale3 = d.scale3;
  a.err = d.err;
  switch (d.opA * 2 + d.opB) {
    case 0: return launch<0, 0>(a, s);
    case 1: return launch<0, 1>(a, s);
    case 2: return launch<1, 0>(a, s);
    default: return launch<1, 1>(a, s);
  }
}

}  // namespace qtx
