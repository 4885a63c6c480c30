// Register-resident factorization of one Gauss-Jordan panel (n rows x NB
// columns), shared by the one-CTA (zinv.cu) and the cluster
// (zinv_cluster.cu) batched inverses.
//
// The panel stays in registers for all of its columns, so one column step
// touches shared memory only for the pivot search partials and the
// broadcast pivot row. Per column k:
//   pivot  p = argmax_{r >= k} |Re| + |Im| of column k (lowest row on ties,
//          the izamax measure of LAPACK that numpy.linalg.inv uses);
//   the threads of row p publish 1 / x_pk and the scaled pivot row, the
//   threads of row k the old row k;
//   row k <- scaled pivot row; row p <- old row k; every row r != k is
//   eliminated: x_rc -= x_rk * prow_c (c != k), x_rk <- -x_rk / x_pk.
// Afterwards the panel holds the transform T of the panel (T = [A_KK^-1 ;
// -A_RK A_KK^-1] in block form) and pivrow[k0 .. k0 + nbp) the pivot rows.
// Two CTA barriers per column; every thread of the CTA must call it.
#pragma once

#include "common.cuh"

namespace qtx {

// 1 / z for a complex z. z is scaled by the power of two 2^-e that brings its
// larger part into [0.5, 1) (exact), so that m = |z'|^2 lies in [0.25, 2);
// 1 / m comes from the hardware reciprocal estimate (PTX rcp.approx.ftz.f64)
// refined by three Newton-Raphson steps y <- y + y (1 - m y), each of which
// doubles the number of correct bits; then 1 / z = conj(z') (1 / m) 2^-e.
// A few ulps from the correctly rounded quotient, like Smith's algorithm,
// with one short dependency chain instead of three divisions.
// gj_recip_scaled: the same with frexp / ldexp (any exponent, zero, subnormals).
__device__ __forceinline__ z64 gj_recip_scaled(z64 z) {
  const double mx = fmax(fabs(z.x), fabs(z.y));
  if (mx == 0.0) return make_double2(0.0, 0.0);
  int e;
  frexp(mx, &e);
  const double xs = ldexp(z.x, -e), ys = ldexp(z.y, -e);
  const double m = fma(xs, xs, ys * ys);
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(m));
#pragma unroll
  for (int it = 0; it < 3; ++it) y = fma(y, fma(-m, y, 1.0), y);
  return make_double2(ldexp(xs * y, -e), ldexp(-ys * y, -e));
}

// gj_recip: for exponents away from the ends of the range the scale 2^-e is
// built from the exponent field and applied by multiplication (exact, and
// the final product rounds like ldexp), which keeps frexp / ldexp off the
// pivot row's critical path; bit-identical to gj_recip_scaled.
__device__ __forceinline__ z64 gj_recip(z64 z) {
  const double mx = fmax(fabs(z.x), fabs(z.y));
  const int eb = (int)((__double_as_longlong(mx) >> 52) & 0x7FF);  // biased exponent field
  if (eb < 24 || eb > 2000) return gj_recip_scaled(z);             // zero, subnormal or extreme
  const int e = eb - 1022;                                         // frexp's exponent of mx
  const double s = __longlong_as_double((long long)(1023 - e) << 52);  // 2^-e
  const double xs = z.x * s, ys = z.y * s;
  const double m = fma(xs, xs, ys * ys);
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(m));
#pragma unroll
  for (int it = 0; it < 3; ++it) y = fma(y, fma(-m, y, 1.0), y);
  return make_double2((xs * y) * s, (-ys * y) * s);
}

__device__ __forceinline__ double gj_abs1(z64 z) { return fabs(z.x) + fabs(z.y); }

// Panel of 16 columns, n <= 256, 512 threads: the two lanes 2i and 2i + 1
// of warp w hold row 16 w + i, columns 0-7 and 8-15 respectively, so a row's
// value in the pivot column reaches its partner lane with one shuffle.
// load(r, c) / store(r, c, v): panel element access (r < n, c < nbp).
// prow_s, rowk_s: 16 shared complex each; red_v / red_i: 16 shared entries
// each; sing: shared int, set to k + 1 at the first zero pivot if still 0.
template <class Load, class Store>
__device__ __forceinline__ void gj_factor_panel16(int n, int k0, int nbp, Load load, Store store, int* pivrow,
                                                  z64* prow_s, z64* rowk_s, double* red_v, int* red_i,
                                                  int* sing) {
  constexpr int NB = 16, H = 8, W = 16;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int h = lane & 1;                       // which 8 columns
  const int r = warp * 16 + (lane >> 1);        // which row
  const bool live = r < n;
  z64 v[H];
#pragma unroll
  for (int c = 0; c < H; ++c) v[c] = (live && h * H + c < nbp) ? load(r, h * H + c) : make_double2(0.0, 0.0);
#pragma unroll
  for (int kk = 0; kk < NB; ++kk) {
    if (kk >= nbp) break;
    const int k = k0 + kk;
    const int hk = kk / H, ck = kk % H;  // compile-time after unrolling
    // this row's value in column kk (held by the lane with h == hk)
    const z64 mine = (h == hk) ? v[ck] : make_double2(0.0, 0.0);
    z64 xk;
    xk.x = __shfl_xor_sync(0xffffffffu, mine.x, 1);
    xk.y = __shfl_xor_sync(0xffffffffu, mine.y, 1);
    if (h == hk) xk = mine;
    double best = -1.0;
    int besti = k;
    if (live && r >= k && h == hk) {
      best = gj_abs1(xk);
      besti = r;
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
    // every warp reduces the W partials with shuffles (lanes >= W repeat them)
    best = red_v[lane & (W - 1)];
    besti = red_i[lane & (W - 1)];
#pragma unroll
    for (int off = W / 2; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, besti, off);
      if (ov > best || (ov == best && oi < besti)) {
        best = ov;
        besti = oi;
      }
    }
    const int p = besti;
    if (r == p) {
      const z64 d = gj_recip(xk);
#pragma unroll
      for (int c = 0; c < H; ++c) prow_s[h * H + c] = (h * H + c == kk) ? d : zmul(v[c], d);
    }
    if (r == k) {
#pragma unroll
      for (int c = 0; c < H; ++c) rowk_s[h * H + c] = v[c];
    }
    if (tid == 0) {
      pivrow[k] = p;
      if (best <= 0.0 && *sing == 0) *sing = k + 1;
    }
    __syncthreads();
    // (the next column's partials, prow_s and rowk_s are written after its
    // first barrier, when every thread has read these)
    if (!live) continue;
    if (r == k) {
#pragma unroll
      for (int c = 0; c < H; ++c) v[c] = prow_s[h * H + c];
      continue;
    }
    z64 f = xk;
    if (r == p) {  // row p receives the old row k
#pragma unroll
      for (int c = 0; c < H; ++c) v[c] = rowk_s[h * H + c];
      f = rowk_s[kk];
    }
    const z64 dpiv = prow_s[kk];
#pragma unroll
    for (int c = 0; c < H; ++c) {
      if (h * H + c == kk) continue;
      const z64 qc = prow_s[h * H + c];
      v[c] = make_double2(v[c].x - (f.x * qc.x - f.y * qc.y), v[c].y - (f.x * qc.y + f.y * qc.x));
    }
    if (h == hk) {
      const z64 m = zmul(f, dpiv);
      v[ck] = make_double2(-m.x, -m.y);
    }
  }
  if (live) {
#pragma unroll
    for (int c = 0; c < H; ++c)
      if (h * H + c < nbp) store(r, h * H + c, v[c]);
  }
}

}  // namespace qtx
