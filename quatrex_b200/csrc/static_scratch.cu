// qtx_selected_inv_static: RGF selected inversion that allocates nothing.
//
// Who needs it: callers that must not call cudaMalloc / cudaFree from the
// solve. cudaMalloc and cudaFree synchronise the whole device, and they
// fail or fragment memory once another allocator (a PyTorch or CuPy caching
// pool, or a solver framework that reserves the GPU up front) owns the
// device memory. Latency-bound loops that re-enter the solver per energy
// batch, and host codes whose memory is fully pre-reserved, therefore cannot
// hand the library a freshly allocated workspace. This entry point takes its
// scratch from a fixed file-scope device array instead.
//
// Limits and sharing:
//  * The array holds kStaticScratchBytes = 64 MiB on every GPU that loads the
//    library, for the lifetime of the process. Requests that need more
//    (sum_i b_i^2 + 6 b_max^2 complex128 elements per energy, 256-byte
//    aligned per buffer) are rejected with QTX_ERR_WORKSPACE before any
//    work is enqueued: split the energy batch.
//  * All calls on a device share the one array and it keeps whatever the
//    last call left in it. Every buffer of this path is fully written before
//    it is read, so nothing has to be cleared between calls. Two calls whose
//    work overlaps on the GPU (different streams without ordering) race on
//    the array and corrupt each other's results; order them on one stream.
//  * The array's host-side symbol is not a device address. On a device's
//    first call the entry point resolves the address with
//    cudaGetSymbolAddress (with that device current) and caches it; make
//    that first call on each device before any stream capture begins.
//  * With the launch profiler off (the default) the call performs no device
//    or host allocation.
//  * Arithmetic: always the FP64 DMMA products and the one-CTA-per-block
//    Gauss-Jordan inverse. The calling thread's GEMM path (qtx_set_gemm_path)
//    and the inverse-path knob are ignored: the int8-emulated products and
//    the multi-CTA inverse need scratch that is not part of the array.
#include <mutex>

#include "common.cuh"

namespace qtx {

constexpr size_t kStaticScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

int scratch_address(void** out) {
  int dev = 0;
  QTX_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("qtx_selected_inv_static: device ordinal out of range");
    return QTX_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("qtx_selected_inv_static: cudaGetSymbolAddress failed: ") +
                cudaGetErrorString(e));
      return QTX_ERR_CUDA;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return QTX_OK;
}

MatRef mref(const qtx_mat& m) { return from_abi(m); }

// Scratch views without any container: buffer k of the layout
//   g[0..N-1] (b_i x b_i each), then 6 temporaries of b_max x b_max.
struct Layout {
  const int32_t* bs;
  int n;
  int bm;
  int64_t batch;
  char* base;
  MatRef at(int k) const {  // k < n: g[k]; k >= n: temporary k - n
    Workspace w;
    w.base = base;
    w.cap = kStaticScratchBytes;
    MatRef m;
    for (int i = 0; i <= k; ++i) {
      const int r = i < n ? bs[i] : bm;
      m = w.mat(r, r, batch);
    }
    return m;
  }
  size_t bytes() const {
    Workspace w;
    for (int i = 0; i < n; ++i) w.mat(bs[i], bs[i], batch);
    for (int k = 0; k < 6; ++k) w.mat(bm, bm, batch);
    return w.off;
  }
};

GemmDesc gemm(int M, int N, int K, int64_t batch, MatRef A, MatRef B, MatRef C, z64 alpha) {
  GemmDesc d;
  d.M = M;
  d.N = N;
  d.K = K;
  d.batch = batch;
  d.A = A;
  d.B = B;
  d.C = C;
  d.alpha = alpha;
  return d;
}

void plus(GemmDesc& d, const MatRef& m, z64 coef) {
  if (!m.null()) d.add[d.nadd++] = Addend{m, coef, 0};
}

// Selects the FP64 DMMA products for the scope and restores the calling
// thread's GEMM path afterwards.
struct Fp64Products {
  int prev;
  Fp64Products() : prev(gemm_slices()) { set_gemm_slices(0); }
  ~Fp64Products() { set_gemm_slices(prev); }
};

int selected_inv_static(const qtx_bt* a, const qtx_mat* obc_retarded, const qtx_bt* x,
                        int64_t batch, int* info, cudaStream_t s);

}  // namespace
}  // namespace qtx

using namespace qtx;

extern "C" int qtx_selected_inv_static(const qtx_bt* a, const qtx_mat* obc_retarded,
                                       const qtx_bt* x, int64_t batch, int* info,
                                       qtx_stream stream) {
  // No C++ exception may cross the C ABI.
  try {
    Fp64Products fp64;
    return selected_inv_static(a, obc_retarded, x, batch, info, (cudaStream_t)stream);
  } catch (const std::exception& e) {
    set_error(std::string("qtx_selected_inv_static: internal error: ") + e.what());
    return QTX_ERR_ARG;
  } catch (...) {
    set_error("qtx_selected_inv_static: internal error");
    return QTX_ERR_ARG;
  }
}

namespace qtx {
namespace {

int selected_inv_static(const qtx_bt* a, const qtx_mat* obc_retarded, const qtx_bt* x,
                        int64_t batch, int* info, cudaStream_t s) {
  if (a == nullptr || x == nullptr || batch <= 0 || a->num_blocks <= 0 ||
      a->block_sizes == nullptr || a->diag == nullptr || x->num_blocks != a->num_blocks ||
      x->block_sizes == nullptr || x->diag == nullptr ||
      (a->num_blocks > 1 && (a->upper == nullptr || a->lower == nullptr || x->upper == nullptr ||
                             x->lower == nullptr))) {
    set_error("qtx_selected_inv_static: invalid block-tridiagonal arguments");
    return QTX_ERR_ARG;
  }
  const int N = a->num_blocks;
  const int32_t* bs = a->block_sizes;
  int bm = 0;
  for (int i = 0; i < N; ++i) {
    if (bs[i] <= 0 || bs[i] > 1024 || x->block_sizes[i] != bs[i]) {
      set_error("qtx_selected_inv_static: block sizes must match and lie in [1, 1024]");
      return QTX_ERR_ARG;
    }
    bm = bs[i] > bm ? bs[i] : bm;
  }
  Layout L{bs, N, bm, batch, nullptr};
  const size_t need = L.bytes();
  if (need > kStaticScratchBytes) {
    set_error("qtx_selected_inv_static: needs " + std::to_string(need) +
              " bytes of scratch, the static scratch holds " + std::to_string(kStaticScratchBytes) +
              " bytes; split the energy batch");
    return QTX_ERR_WORKSPACE;
  }
  void* base = nullptr;
  QTX_TRY(scratch_address(&base));
  L.base = static_cast<char*>(base);
  if (info) QTX_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, s));
  const z64 one{1.0, 0.0}, mone{-1.0, 0.0};
  auto obc = [&](int i) { return obc_retarded ? mref(obc_retarded[i]) : MatRef{}; };
  auto shaped_tmp = [&](int k, int cols) { return shaped(L.at(N + k), cols); };

  // Forward sweep (rgf.py:71-92).
  {
    const MatRef g0 = L.at(0);
    Addend t[2] = {Addend{mref(a->diag[0]), one, 0}, Addend{obc(0), mone, 0}};
    QTX_TRY(zcombine(bs[0], bs[0], batch, g0, t, 2, nullptr, s));
    QTX_TRY(zinv(bs[0], batch, g0, g0, info, nullptr, s));
  }
  for (int j = 1; j < N; ++j) {
    const int i = j - 1;
    const MatRef gi = L.at(i), gj = L.at(j);
    const MatRef P = shaped_tmp(0, bs[i]);
    QTX_TRY(zgemm(gemm(bs[j], bs[i], bs[i], batch, mref(a->lower[i]), gi, P, one), s));
    GemmDesc d = gemm(bs[j], bs[j], bs[i], batch, P, mref(a->upper[i]), gj, mone);
    plus(d, mref(a->diag[j]), one);
    plus(d, obc(j), mone);
    QTX_TRY(zgemm(d, s));
    QTX_TRY(zinv(bs[j], batch, gj, gj, info, nullptr, s));
  }
  if (x->diag[N - 1].ptr != nullptr) {
    Addend t{L.at(N - 1), one, 0};
    QTX_TRY(zcombine(bs[N - 1], bs[N - 1], batch, mref(x->diag[N - 1]), &t, 1, nullptr, s));
  }

  // Backward sweep (rgf.py:98-110).
  MatRef Gj = L.at(N - 1);
  for (int i = N - 2; i >= 0; --i) {
    const int j = i + 1;
    const MatRef gi = L.at(i);
    const MatRef T1 = shaped_tmp(2, bs[i]);
    QTX_TRY(zgemm(gemm(bs[j], bs[i], bs[j], batch, Gj, mref(a->lower[i]), T1, one), s));
    const MatRef xji = x->lower[i].ptr == nullptr ? shaped_tmp(3, bs[i]) : mref(x->lower[i]);
    QTX_TRY(zgemm(gemm(bs[j], bs[i], bs[i], batch, T1, gi, xji, mone), s));
    const MatRef U = shaped_tmp(1, bs[j]);
    QTX_TRY(zgemm(gemm(bs[i], bs[j], bs[i], batch, gi, mref(a->upper[i]), U, one), s));
    if (x->upper[i].ptr != nullptr)
      QTX_TRY(zgemm(gemm(bs[i], bs[j], bs[j], batch, U, Gj, mref(x->upper[i]), mone), s));
    const MatRef Gi = x->diag[i].ptr == nullptr ? shaped_tmp(4 + (i & 1), bs[i]) : mref(x->diag[i]);
    GemmDesc d = gemm(bs[i], bs[i], bs[j], batch, U, xji, Gi, mone);
    plus(d, gi, one);
    QTX_TRY(zgemm(d, s));
    Gj = Gi;
  }
  return QTX_OK;
}

}  // namespace
}  // namespace qtx
