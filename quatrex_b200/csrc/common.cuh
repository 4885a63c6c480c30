// Shared definitions for the quatrex_b200 CUDA library (sm_100a).
//
// Complex numbers are stored interleaved (re, im), exactly like numpy's
// complex128 / complex64, so DSDBSparse data buffers can be used in place.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <vector>

#include "qtx_b200.h"

namespace qtx {

using z64 = double2;  // complex128
using c32 = float2;   // complex64

// A strided stack of dense row-major complex matrices.
struct MatRef {
  void* p = nullptr;
  int64_t ld = 0;      // row stride in complex elements
  int64_t stride = 0;  // stack stride in complex elements
  __host__ __device__ bool null() const { return p == nullptr; }
};

inline MatRef from_abi(const qtx_mat& m) { return MatRef{m.ptr, m.ld, m.stride}; }

template <typename T>
__host__ __device__ inline T* at(const MatRef& m, int64_t batch) {
  return reinterpret_cast<T*>(m.p) + batch * m.stride;
}

__host__ __device__ inline z64 zmul(z64 a, z64 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline z64 zconj(z64 a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline z64 zadd(z64 a, z64 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline z64 zsub(z64 a, z64 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline z64 zscale(z64 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ inline z64 zfma(z64 a, z64 b, z64 c) {  // a*b + c
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

// Thread-local error message set by the host-side entry points.
void set_error(const std::string& msg);
const char* get_error();

#define QTX_CHECK_CUDA(call)                                                        \
  do {                                                                              \
    cudaError_t _e = (call);                                                        \
    if (_e != cudaSuccess) {                                                        \
      ::qtx::set_error(std::string(#call) + ": " + cudaGetErrorString(_e));         \
      return (int)QTX_ERR_CUDA;                                                     \
    }                                                                               \
  } while (0)

#define QTX_CHECK_LAUNCH()                                                          \
  do {                                                                              \
    cudaError_t _e = cudaGetLastError();                                            \
    if (_e != cudaSuccess) {                                                        \
      ::qtx::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e));    \
      return (int)QTX_ERR_CUDA;                                                     \
    }                                                                               \
  } while (0)

#define QTX_TRY(expr)             \
  do {                            \
    int _s = (expr);              \
    if (_s != QTX_OK) return _s;  \
  } while (0)

// ---------------------------------------------------------------------------
// Batched complex GEMM with a fused epilogue (zgemm.cu).
//
//   out  = alpha * op(A) op(B) + sum_t coef_t * op_t(D_t)        (t < nadd)
//   C    = out                                                   (if C)
//   C2   = coef2 * out^H            (transposed store, if C2)
//   C3   = scale3 * out + sum_t coef_t * op_t(D_t)  (nadd <= t < nadd+nadd3)
//
// op(X) is X or X^H. Addends may alias C only when not transposed (each
// element is read and written by the same thread). C must not alias A or B.
// ---------------------------------------------------------------------------
constexpr int kMaxAddends = 4;

struct Addend {
  MatRef m;
  z64 coef;
  int conj_trans;
};

struct GemmDesc {
  int M = 0, N = 0, K = 0;
  int64_t batch = 0;
  MatRef A, B;
  int opA = 0, opB = 0;  // 0: N, 1: conjugate transpose
  z64 alpha{1.0, 0.0};
  Addend add[kMaxAddends];
  int nadd = 0;   // addends of the primary output
  int nadd3 = 0;  // addends of C3 (stored after the primary ones)
  MatRef C;
  MatRef C2;
  z64 coef2{1.0, 0.0};
  MatRef C3;
  z64 scale3{1.0, 0.0};
  const int* active = nullptr;  // optional per-batch mask (0 = skip entry)
  // Grouped form (DMMA path only): device tables of per-entry pointers that
  // replace base + b * stride of A, B, the first addend and C (row strides
  // from the MatRefs); no C2 / C3.
  const z64* const* a_ptrs = nullptr;
  const z64* const* b_ptrs = nullptr;
  const z64* const* d_ptrs = nullptr;
  z64* const* c_ptrs = nullptr;
};

int zgemm(const GemmDesc& d, cudaStream_t s);

// The same GEMM emulated on the int8 tensor cores with `slices` digit planes
// per operand (zgemm_oz.cu); `scratch` holds the planes of a batch chunk.
size_t oz_scratch_bytes(int M, int N, int K, int64_t batch, int slices);
bool oz_supported(int K, int slices);
int zgemm_oz(const GemmDesc& d, int slices, void* scratch, size_t bytes, cudaStream_t s);
// GEMM path of the calling thread: 0 = FP64 DMMA, 3-8 = int8 emulation with
// that many slices (used where a driver bound scratch for it).
void set_gemm_slices(int slices);
int gemm_slices();
void* oz_bound(size_t* bytes);
// Reads and clears the device flag of timed-out waits in the emulated GEMM.
int oz_status_take(int* flag);

// Complex64 GEMM on tcgen05 with split-TF32 products (cgemm_tc.cu):
//   C = alpha op(A) op(B) + sum_t coef_t op_t(D_t);  C2 = coef2 C^H (optional).
struct CAddend {
  MatRef m;
  float2 coef;
  int conj_trans;
};
struct CGemmDesc {
  int M = 0, N = 0, K = 0;
  int64_t batch = 0;
  MatRef A, B;
  int opA = 0, opB = 0;
  float2 alpha{1.f, 0.f};
  CAddend add[kMaxAddends];
  int nadd = 0;
  int nadd3 = 0;  // addends of C3, stored after the primary ones
  MatRef C, C2, C3;
  float2 coef2{1.f, 0.f};
  float2 scale3{1.f, 0.f};
  int* err = nullptr;  // set to 1 if an mbarrier wait timed out
};
int cgemm_tc(const CGemmDesc& d, cudaStream_t s);

// Batched in-place Gauss-Jordan inversion with partial pivoting (zinv.cu).
// X <- A^{-1} for each of `batch` n x n matrices; X may alias A. `info[b]`
// (device, optional) receives 0 or the 1-based column of a zero pivot.
int zinv(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s);
// Inverse with optional scratch (zinv_wide.cu): for large blocks and small
// batches, a multi-CTA blocked Gauss-Jordan over the whole GPU when
// `scratch` holds zinv_scratch_bytes(n, batch); otherwise zinv().
size_t zinv_scratch_bytes(int n, int64_t batch);
int zinv_ex(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, void* scratch,
            size_t scratch_bytes, cudaStream_t s);
bool zinv_prefers_wide(int n, int64_t batch);
void set_inverse_path(int mode);
int inverse_path();
int num_sms();
// One thread-block cluster of ceil(n / 32) CTAs per matrix with the matrix in
// distributed shared memory (zinv_cluster.cu); n <= 256, no scratch.
int zinv_cluster(int n, int64_t batch, MatRef A, MatRef X, int* info, const int* active, cudaStream_t s);
bool zinv_prefers_cluster(int n, int64_t batch);
// Reads and clears the device flag of timed-out waits in zinv_cluster.
int zinv_cluster_status_take(int* flag);

// Elementwise combination (blockops.cu):
//   out = sum_t coef_t * op_t(X_t)   for up to 4 terms, over an m x n stack.
int zcombine(int m, int n, int64_t batch, MatRef out, const Addend* terms, int nterms,
             const int* active, cudaStream_t s);

// complex64 twin of zcombine (arithmetic in double).
int ccombine(int m, int n, int64_t batch, MatRef out, const Addend* terms, int nterms,
             const int* active, cudaStream_t s);

// out = 0.5 (X - X^H); optional density[b, off + r] = Im X[r, r].
int zantiherm(int n, int64_t batch, MatRef X, MatRef out, double* density, int64_t dens_stride,
              int64_t dens_off, cudaStream_t s);
int cantiherm(int n, int64_t batch, MatRef X, MatRef out, double* density, int64_t dens_stride,
              int64_t dens_off, cudaStream_t s);

// Element-type conversion of an m x n stack.
int convert_c64_to_c128(int m, int n, int64_t batch, MatRef in, MatRef out, cudaStream_t s);
int convert_c128_to_c64(int m, int n, int64_t batch, MatRef in, MatRef out, cudaStream_t s);

// result[b * rstride + roff] (+)= sign * Tr(X_b Y_b)  (complex, n x n).
int ztrace_prod(int n, int64_t batch, MatRef X, MatRef Y, z64 coef, z64* result, int64_t rstride,
                int64_t roff, int accumulate, cudaStream_t s);

int ctrace_prod(int n, int64_t batch, MatRef X, MatRef Y, z64 coef, z64* result, int64_t rstride,
                int64_t roff, int accumulate, cudaStream_t s);

// delta[b] = || |X_b| + |Y_b| ||_F / 2   (Sancho-Rubio convergence measure).
int sr_delta(int n, int64_t batch, MatRef X, MatRef Y, double* delta, const int* active,
             cudaStream_t s);

// Frobenius norms: nrm_diff[b] = ||X_b - Y_b||_F, nrm[b] = ||X_b||_F.
// rel (optional) = nrm_diff / nrm.
int znorm_diff(int n, int64_t batch, MatRef X, MatRef Y, double* nrm_diff, double* nrm,
               double* rel, cudaStream_t s);

// T[b] = Re Tr(GamL G GamR G^H) given P = GamL G GamR: Re sum conj(G) .* P.
int zre_inner(int m, int n, int64_t batch, MatRef P, MatRef G, double* out, cudaStream_t s);
int cre_inner(int m, int n, int64_t batch, MatRef P, MatRef G, double* out, cudaStream_t s);

// Launch profiler (profile.cu): RAII bracket of one kernel launch.
// Scopes nest: only the outermost scope of a thread records, with `launches`
// kernel launches attributed to it.
class ProfScope {
 public:
  ProfScope(int kind, double work, cudaStream_t s, int launches = 1);
  ~ProfScope();
  ProfScope(const ProfScope&) = delete;
  ProfScope& operator=(const ProfScope&) = delete;

 private:
  int idx_;
  cudaStream_t s_;
};

// Bump allocator over a caller-provided workspace. With base == nullptr it
// only measures the bytes a call sequence needs.
struct Workspace {
  char* base = nullptr;
  size_t cap = 0;
  size_t off = 0;
  bool overflow = false;
  void* take(size_t bytes) {
    off = (off + 255) & ~size_t(255);
    void* p = base ? base + off : nullptr;
    off += bytes;
    if (base && off > cap) overflow = true;
    return p;
  }
  MatRef mat(int rows, int cols, int64_t batch, size_t elem = sizeof(z64)) {
    const int64_t stride = (int64_t)rows * cols;
    MatRef m;
    m.p = take((size_t)stride * batch * elem);
    m.ld = cols;
    m.stride = stride;
    return m;
  }
};

// Reserves the emulated-GEMM scratch for n x n x n products over `batch`
// from a driver's workspace when the calling thread selected the int8 path,
// and binds it to the thread for the scope (restoring the previous binding).
struct OzScope {
  OzScope(Workspace& ws, int n, int64_t batch);
  ~OzScope();
  OzScope(const OzScope&) = delete;
  OzScope& operator=(const OzScope&) = delete;
  void* prev_p;
  size_t prev_bytes;
};

// A temporary reshaped to rows x cols inside a larger slot.
inline MatRef shaped(const MatRef& slot, int cols) {
  MatRef m = slot;
  m.ld = cols;
  return m;
}

// Block-tridiagonal stack view (host-side copy of a qtx_bt).
struct BTRef {
  int n = 0;
  std::vector<int> bs;
  std::vector<MatRef> diag, upper, lower;
};
BTRef bt_from_abi(const qtx_bt* t);

// Arguments of the selected-solve driver (rgf.cu).
struct SolveIO {
  BTRef a, sl, sg, xl, xg, xr;
  const MatRef* obc_r = nullptr;
  const MatRef* obc_l = nullptr;
  const MatRef* obc_g = nullptr;
  z64* current = nullptr;
  MatRef g0n;
  double* density = nullptr;
  int symmetric = 0;
};

}  // namespace qtx
