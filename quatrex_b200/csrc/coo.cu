// DSDBCOO <-> dense block conversion on the device.
//
// qttools stores a DSDBSparse stack as data[stack, nnz] with block-sorted
// COO indices (datastructures/dsdbcoo.py:297-331, 886-977); reading a block
// densifies it (dsdbcoo.py:333-412, kernels/datastructure/*/dsdbcoo.py
// densify_block) and writing sparsifies it (dsdbcoo.py:466-521). Blocks
// whose nnz equals b_i * b_j in row-major order need neither: the solver
// reads and writes them in place. The kernels below handle all other
// blocks: one thread per (stack entry, nonzero), grid-strided.
#include "common.cuh"

namespace qtx {
namespace {

__global__ void zero_kernel(MatRef out, int m, int n, int64_t batch) {
  const int64_t per = (int64_t)m * n;
  const int64_t total = per * batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / per, e = i % per;
    const int r = (int)(e / n), c = (int)(e % n);
    at<z64>(out, b)[(int64_t)r * out.ld + c] = make_double2(0.0, 0.0);
  }
}

__global__ void densify_kernel(int64_t batch, const z64* data, int64_t dstride, int64_t nnz,
                               const int32_t* rows, const int32_t* cols, MatRef out, int m, int n) {
  const int64_t total = nnz * batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / nnz, k = i % nnz;
    const int r = rows[k], c = cols[k];
    if (r < 0 || r >= m || c < 0 || c >= n) continue;
    at<z64>(out, b)[(int64_t)r * out.ld + c] = data[b * dstride + k];
  }
}

__global__ void sparsify_kernel(int64_t batch, MatRef in, int64_t nnz, const int32_t* rows,
                                const int32_t* cols, z64* data, int64_t dstride) {
  const int64_t total = nnz * batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / nnz, k = i % nnz;
    data[b * dstride + k] = at<const z64>(in, b)[(int64_t)rows[k] * in.ld + cols[k]];
  }
}

unsigned blocks_for(int64_t total) {
  const int64_t b = (total + 255) / 256;
  return (unsigned)(b < 148 * 64 ? (b > 0 ? b : 1) : 148 * 64);
}

}  // namespace
}  // namespace qtx

using namespace qtx;

extern "C" int qtx_coo_densify(int64_t batch, const void* data, int64_t data_stride, int64_t nnz,
                               const int32_t* rows, const int32_t* cols, qtx_mat out, int m, int n,
                               qtx_stream stream) {
  if (batch < 0 || nnz < 0 || m < 0 || n < 0 || out.ptr == nullptr ||
      (nnz > 0 && (data == nullptr || rows == nullptr || cols == nullptr))) {
    set_error("qtx_coo_densify: invalid arguments");
    return QTX_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const MatRef o = from_abi(out);
  if ((int64_t)m * n * batch > 0) {
    ProfScope prof(QTX_KERNEL_FORMAT, 16.0 * m * n * (double)batch, s);
    zero_kernel<<<blocks_for((int64_t)m * n * batch), 256, 0, s>>>(o, m, n, batch);
    QTX_CHECK_LAUNCH();
  }
  if (nnz * batch > 0) {
    ProfScope prof(QTX_KERNEL_FORMAT, 32.0 * nnz * (double)batch, s);
    densify_kernel<<<blocks_for(nnz * batch), 256, 0, s>>>(
        batch, static_cast<const z64*>(data), data_stride, nnz, rows, cols, o, m, n);
    QTX_CHECK_LAUNCH();
  }
  return QTX_OK;
}

extern "C" int qtx_coo_sparsify(int64_t batch, qtx_mat in, int64_t nnz, const int32_t* rows,
                                const int32_t* cols, void* data, int64_t data_stride,
                                qtx_stream stream) {
  if (batch < 0 || nnz < 0 || in.ptr == nullptr ||
      (nnz > 0 && (data == nullptr || rows == nullptr || cols == nullptr))) {
    set_error("qtx_coo_sparsify: invalid arguments");
    return QTX_ERR_ARG;
  }
  if (nnz * batch == 0) return QTX_OK;
  ProfScope prof(QTX_KERNEL_FORMAT, 32.0 * nnz * (double)batch, (cudaStream_t)stream);
  sparsify_kernel<<<blocks_for(nnz * batch), 256, 0, (cudaStream_t)stream>>>(
      batch, from_abi(in), nnz, rows, cols, static_cast<z64*>(data), data_stride);
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

// ---------------------------------------------------------------------------
// System-matrix diagonal blocks A_ii(E) = z I - H_ii (quatrex
// electron/solver.py:668-709 with zero potential and scattering
// self-energy). h may have stack stride 0 (one Hamiltonian block shared by
// every energy).
// ---------------------------------------------------------------------------
namespace qtx {
namespace {
__global__ void assemble_diag_kernel(int n, int64_t batch, MatRef h, const z64* z, MatRef out) {
  const int64_t per = (int64_t)n * n;
  const int64_t total = per * batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / per, e = i % per;
    const int r = (int)(e / n), c = (int)(e % n);
    const z64 v = at<const z64>(h, b)[(int64_t)r * h.ld + c];
    z64 o = make_double2(-v.x, -v.y);
    if (r == c) o = zadd(o, z[b]);
    at<z64>(out, b)[(int64_t)r * out.ld + c] = o;
  }
}
}  // namespace
}  // namespace qtx

extern "C" int qtx_assemble_diag(int n, int64_t batch, qtx_mat h, const void* z, qtx_mat out,
                                 qtx_stream stream) {
  if (n <= 0 || batch <= 0) return QTX_OK;
  if (h.ptr == nullptr || z == nullptr || out.ptr == nullptr) {
    set_error("qtx_assemble_diag: null argument");
    return QTX_ERR_ARG;
  }
  const int64_t total = (int64_t)n * n * batch;
  ProfScope prof(QTX_KERNEL_FORMAT, 32.0 * (double)total, (cudaStream_t)stream);
  assemble_diag_kernel<<<blocks_for(total), 256, 0, (cudaStream_t)stream>>>(
      n, batch, from_abi(h), static_cast<const z64*>(z), from_abi(out));
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

// z[b] = E[b] + i eta: the complex energies of one batch.
namespace qtx {
namespace {
__global__ void energies_kernel(int64_t batch, const double* E, double eta, z64* z) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < batch;
       b += (int64_t)gridDim.x * blockDim.x)
    z[b] = make_double2(E[b], eta);
}
}  // namespace
}  // namespace qtx

extern "C" int qtx_assemble_energies(int64_t batch, const double* energies, double eta, void* z,
                                     qtx_stream stream) {
  if (batch <= 0) return QTX_OK;
  if (energies == nullptr || z == nullptr) {
    set_error("qtx_assemble_energies: null argument");
    return QTX_ERR_ARG;
  }
  ProfScope prof(QTX_KERNEL_FORMAT, 24.0 * (double)batch, (cudaStream_t)stream);
  energies_kernel<<<blocks_for(batch), 256, 0, (cudaStream_t)stream>>>(batch, energies, eta,
                                                                        static_cast<z64*>(z));
  QTX_CHECK_LAUNCH();
  return QTX_OK;
}

// Copies the byte ranges [offsets[r], offsets[r] + lengths[r]) of every row
// of a row-strided stack from src to dst (any direction; one 2D copy per
// range on the stream). For a DSDBCOO data[stack, nnz] buffer the ranges
// are the nonzero slices of the blocks one call reads or writes
// (dsdbcoo.py:297-331): moving only those between host and device replaces
// the reference's per-block host views (`stack[...]`, `.blocks[i, j]`).
extern "C" int qtx_copy_ranges(void* dst, int64_t dst_row_bytes, const void* src,
                               int64_t src_row_bytes, int64_t rows, const int64_t* offsets,
                               const int64_t* lengths, int num_ranges, qtx_stream stream) {
  if (rows <= 0 || num_ranges <= 0) return QTX_OK;
  if (dst == nullptr || src == nullptr || offsets == nullptr || lengths == nullptr ||
      dst_row_bytes <= 0 || src_row_bytes <= 0) {
    set_error("qtx_copy_ranges: invalid arguments");
    return QTX_ERR_ARG;
  }
  for (int r = 0; r < num_ranges; ++r) {
    if (offsets[r] < 0 || lengths[r] < 0 || offsets[r] + lengths[r] > dst_row_bytes ||
        offsets[r] + lengths[r] > src_row_bytes) {
      set_error("qtx_copy_ranges: range " + std::to_string(r) + " outside the rows");
      return QTX_ERR_ARG;
    }
  }
  for (int r = 0; r < num_ranges; ++r) {
    if (lengths[r] == 0) continue;
    QTX_CHECK_CUDA(cudaMemcpy2DAsync(static_cast<char*>(dst) + offsets[r], (size_t)dst_row_bytes,
                                     static_cast<const char*>(src) + offsets[r], (size_t)src_row_bytes,
                                     (size_t)lengths[r], (size_t)rows, cudaMemcpyDefault,
                                     (cudaStream_t)stream));
  }
  return QTX_OK;
}

// System-matrix assembly in one pass (quatrex electron/solver.py:668-709
// with _subtract_hamiltonian_and_self_energy, :611-665, no overlap):
//   A_ij = delta_ij (z_b I - diag(V_i)) - H_ij - Sigma^R_ij
//          - 1/2 (Sigma^>_ij - Sigma^<_ij)
// for every tridiagonal block (i, j) of a batch. The reference builds the
// same matrix in five passes over the DSDBCOO data (zero, unit diagonal,
// energy scale, potential, self-energy and Hamiltonian subtraction); here
// each output block is written once from one read of each input.
namespace qtx {
namespace {
struct AsmArgs {
  MatRef out, h, sr, sl, sg;
  const double* v;  // potential of the block's rows (diagonal blocks), or null
  const z64* z;     // complex energies (diagonal blocks), or null
  int m, n;
  int64_t batch;
};

__global__ void assemble_block_kernel(const AsmArgs a) {
  const int64_t per = (int64_t)a.m * a.n;
  const int64_t total = per * a.batch;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / per, e = i % per;
    const int r = (int)(e / a.n), c = (int)(e % a.n);
    z64 o = make_double2(0.0, 0.0);
    if (a.z != nullptr && r == c) {
      o = a.z[b];
      if (a.v != nullptr) o.x -= a.v[r];
    }
    if (!a.h.null()) o = zsub(o, at<const z64>(a.h, b)[(int64_t)r * a.h.ld + c]);
    if (!a.sr.null()) o = zsub(o, at<const z64>(a.sr, b)[(int64_t)r * a.sr.ld + c]);
    if (!a.sg.null()) {
      const z64 g = at<const z64>(a.sg, b)[(int64_t)r * a.sg.ld + c];
      o = make_double2(o.x - 0.5 * g.x, o.y - 0.5 * g.y);
    }
    if (!a.sl.null()) {
      const z64 l = at<const z64>(a.sl, b)[(int64_t)r * a.sl.ld + c];
      o = make_double2(o.x + 0.5 * l.x, o.y + 0.5 * l.y);
    }
    at<z64>(a.out, b)[(int64_t)r * a.out.ld + c] = o;
  }
}
}  // namespace
}  // namespace qtx

extern "C" int qtx_assemble_system(const qtx_bt* h, const double* potential, const void* z,
                                   const qtx_bt* sigma_retarded, const qtx_bt* sigma_lesser,
                                   const qtx_bt* sigma_greater, const qtx_bt* a, int64_t batch,
                                   qtx_stream stream) {
  try {
    if (batch <= 0) return QTX_OK;
    if (h == nullptr || a == nullptr || z == nullptr || h->num_blocks <= 0 || a->num_blocks != h->num_blocks ||
        h->block_sizes == nullptr || a->block_sizes == nullptr) {
      set_error("qtx_assemble_system: invalid arguments");
      return QTX_ERR_ARG;
    }
    const int N = h->num_blocks;
    for (const qtx_bt* t : {sigma_retarded, sigma_lesser, sigma_greater}) {
      if (t != nullptr && (t->num_blocks != N || t->block_sizes == nullptr)) {
        set_error("qtx_assemble_system: self-energy layout differs from the Hamiltonian");
        return QTX_ERR_ARG;
      }
    }
    std::vector<int64_t> off(N + 1, 0);
    for (int i = 0; i < N; ++i) {
      if (h->block_sizes[i] <= 0 || a->block_sizes[i] != h->block_sizes[i]) {
        set_error("qtx_assemble_system: block sizes differ");
        return QTX_ERR_ARG;
      }
      off[i + 1] = off[i] + h->block_sizes[i];
    }
    auto pick = [](const qtx_bt* t, int which, int k) -> MatRef {
      if (t == nullptr) return MatRef{};
      const qtx_mat* arr = which == 0 ? t->diag : (which == 1 ? t->upper : t->lower);
      return arr == nullptr ? MatRef{} : from_abi(arr[k]);
    };
    cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < N; ++i) {
      for (int which = 0; which < 3; ++which) {
        if (which > 0 && i + 1 >= N) continue;
        AsmArgs g;
        g.out = pick(a, which, i);
        if (g.out.null()) continue;  // block not wanted
        g.h = pick(h, which, i);
        g.sr = pick(sigma_retarded, which, i);
        g.sl = pick(sigma_lesser, which, i);
        g.sg = pick(sigma_greater, which, i);
        g.m = which == 2 ? h->block_sizes[i + 1] : h->block_sizes[i];
        g.n = which == 1 ? h->block_sizes[i + 1] : h->block_sizes[i];
        g.z = which == 0 ? static_cast<const z64*>(z) : nullptr;
        g.v = which == 0 && potential != nullptr ? potential + off[i] : nullptr;
        g.batch = batch;
        const int64_t total = (int64_t)g.m * g.n * batch;
        const int ins = 1 + !g.h.null() + !g.sr.null() + !g.sl.null() + !g.sg.null();
        ProfScope prof(QTX_KERNEL_FORMAT, 16.0 * ins * (double)total, s);
        assemble_block_kernel<<<blocks_for(total), 256, 0, s>>>(g);
        QTX_CHECK_LAUNCH();
      }
    }
    return QTX_OK;
  } catch (const std::exception& e) {
    set_error(std::string("qtx_assemble_system: internal error: ") + e.what());
    return QTX_ERR_ARG;
  }
}
