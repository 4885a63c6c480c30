// Host-side drivers of the block-tridiagonal RGF recursions.
//
// The reference (qttools greens_function_solver/rgf.py) walks the block
// chain in Python and densifies every block it touches. Here the chain is a
// fixed sequence of batched kernels over the whole energy batch, enqueued on
// one stream (capturable in a CUDA graph): fused GEMMs (zgemm.cu), in-place
// block inverses (zinv.cu) and memory-bound epilogues (blockops.cu). Left-
// connected Green's functions g_i stay resident in a caller-provided
// workspace; results go straight to the caller's output block views.
//
// In the forward sweep of selected_solve the retarded chain (Schur
// complement, inverse) runs on a high-priority helper stream while the
// lesser/greater products of the previous block run on the caller's stream:
// at small batches the inverse is latency-bound on a few SMs and the
// products fill the rest of the GPU beside it.
//
// Products that the reference evaluates twice are evaluated once (e.g.
// x_ii @ a_ij in rgf.py:107,110 and xr_ii @ sigma_ij in rgf.py:346,354), and
// the Meir-Wingreen current reuses the forward-sweep Sigma-tilde instead of
// recomputing it (rgf.py:388-402 repeats rgf.py:272-301): the same
// algebra with fewer products.
#include <algorithm>
#include <map>
#include <vector>

#include "common.cuh"

namespace qtx {

BTRef bt_from_abi(const qtx_bt* t) {
  BTRef r;
  if (t == nullptr) return r;
  r.n = t->num_blocks;
  r.bs.assign(t->block_sizes, t->block_sizes + r.n);
  r.diag.resize(r.n);
  r.upper.resize(r.n > 0 ? r.n - 1 : 0);
  r.lower.resize(r.n > 0 ? r.n - 1 : 0);
  for (int i = 0; i < r.n; ++i) {
    r.diag[i] = t->diag ? from_abi(t->diag[i]) : MatRef{};
    if (i + 1 < r.n) {
      r.upper[i] = t->upper ? from_abi(t->upper[i]) : MatRef{};
      r.lower[i] = t->lower ? from_abi(t->lower[i]) : MatRef{};
    }
  }
  return r;
}

namespace {

inline Addend add(const MatRef& m, z64 coef, int ct = 0) { return Addend{m, coef, ct}; }
const z64 ONE{1.0, 0.0};
const z64 MONE{-1.0, 0.0};

struct Gemm {
  GemmDesc d;
  Gemm(int M, int N, int K, int64_t batch, MatRef A, int opA, MatRef B, int opB, MatRef C,
       z64 alpha = ONE) {
    d.M = M;
    d.N = N;
    d.K = K;
    d.batch = batch;
    d.A = A;
    d.B = B;
    d.opA = opA;
    d.opB = opB;
    d.alpha = alpha;
    d.C = C;
  }
  Gemm& plus(const MatRef& m, z64 coef, int ct = 0) {
    if (!m.null()) d.add[d.nadd++] = add(m, coef, ct);
    return *this;
  }
  Gemm& store_h(const MatRef& c2, z64 coef) {
    d.C2 = c2;
    d.coef2 = coef;
    return *this;
  }
  Gemm& second(const MatRef& c3, z64 scale) {
    d.C3 = c3;
    d.scale3 = scale;
    return *this;
  }
  Gemm& plus3(const MatRef& m, z64 coef, int ct = 0) {
    if (!m.null()) d.add[d.nadd + d.nadd3++] = add(m, coef, ct);
    return *this;
  }
  int run(cudaStream_t s) { return zgemm(d, s); }
};

int copy_block(int m, int n, int64_t batch, MatRef dst, MatRef src, cudaStream_t s) {
  if (dst.null()) return QTX_OK;
  Addend t = add(src, ONE);
  return zcombine(m, n, batch, dst, &t, 1, nullptr, s);
}

int max_block(const std::vector<int>& bs) {
  int m = 0;
  for (int b : bs) m = std::max(m, b);
  return m;
}

}  // namespace

// ---------------------------------------------------------------------------
// selected_inv (rgf.py:25-113)
// ---------------------------------------------------------------------------
int selected_inv_run(const BTRef& a, const MatRef* obc_r, const BTRef& x, int64_t batch, int* info,
                     Workspace& ws, cudaStream_t s) {
  const int N = a.n;
  const std::vector<int>& bs = a.bs;
  const int bm = max_block(bs);
  std::vector<MatRef> g(N);
  for (int i = 0; i < N; ++i) g[i] = ws.mat(bs[i], bs[i], batch);
  MatRef tP = ws.mat(bm, bm, batch), tU = ws.mat(bm, bm, batch), tT = ws.mat(bm, bm, batch);
  MatRef tXji = ws.mat(bm, bm, batch);
  MatRef tG[2] = {ws.mat(bm, bm, batch), ws.mat(bm, bm, batch)};
  const size_t scr_bytes = zinv_scratch_bytes(bm, batch);
  void* scr = ws.take(scr_bytes);
  OzScope oz(ws, bm, batch);
  if (ws.base == nullptr) return QTX_OK;
  if (ws.overflow) {
    set_error("selected_inv: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  auto obc = [&](int i) { return obc_r ? obc_r[i] : MatRef{}; };

  // Forward sweep (rgf.py:71-92).
  {
    Addend t[2] = {add(a.diag[0], ONE), add(obc(0), MONE)};
    QTX_TRY(zcombine(bs[0], bs[0], batch, g[0], t, 2, nullptr, s));
    QTX_TRY(zinv_ex(bs[0], batch, g[0], g[0], info, nullptr, scr, scr_bytes, s));
  }
  for (int j = 1; j < N; ++j) {
    const int i = j - 1;
    MatRef P = shaped(tP, bs[i]);
    QTX_TRY(Gemm(bs[j], bs[i], bs[i], batch, a.lower[i], 0, g[i], 0, P).run(s));
    QTX_TRY(Gemm(bs[j], bs[j], bs[i], batch, P, 0, a.upper[i], 0, g[j], MONE)
                .plus(a.diag[j], ONE)
                .plus(obc(j), MONE)
                .run(s));
    QTX_TRY(zinv_ex(bs[j], batch, g[j], g[j], info, nullptr, scr, scr_bytes, s));
  }
  QTX_TRY(copy_block(bs[N - 1], bs[N - 1], batch, x.diag[N - 1], g[N - 1], s));

  // Backward sweep (rgf.py:98-110).
  MatRef Gj = g[N - 1];
  for (int i = N - 2; i >= 0; --i) {
    const int j = i + 1;
    MatRef T1 = shaped(tT, bs[i]);
    QTX_TRY(Gemm(bs[j], bs[i], bs[j], batch, Gj, 0, a.lower[i], 0, T1).run(s));
    MatRef xji = x.lower[i].null() ? shaped(tXji, bs[i]) : x.lower[i];
    QTX_TRY(Gemm(bs[j], bs[i], bs[i], batch, T1, 0, g[i], 0, xji, MONE).run(s));
    MatRef U = shaped(tU, bs[j]);
    QTX_TRY(Gemm(bs[i], bs[j], bs[i], batch, g[i], 0, a.upper[i], 0, U).run(s));
    if (!x.upper[i].null())
      QTX_TRY(Gemm(bs[i], bs[j], bs[j], batch, U, 0, Gj, 0, x.upper[i], MONE).run(s));
    MatRef Gi = x.diag[i].null() ? shaped(tG[i & 1], bs[i]) : x.diag[i];
    QTX_TRY(Gemm(bs[i], bs[i], bs[j], batch, U, 0, xji, 0, Gi, MONE).plus(g[i], ONE).run(s));
    Gj = Gi;
  }
  return QTX_OK;
}

// ---------------------------------------------------------------------------
// selected_solve (rgf.py:115-438), generic over the arithmetic:
//   Fp64  -- complex128 blocks, DMMA products, FP64 inverses;
//   Mixed -- complex64 blocks, tcgen05 split-TF32 products with FP32
//            accumulation, FP64 Gauss-Jordan inverses of the Schur
//            complements (upcast, invert, round back).
// ---------------------------------------------------------------------------
namespace {

struct Fp64 {
  static constexpr size_t E = sizeof(z64);
  static constexpr bool kInvTmp = false;
  using G = Gemm;
  static int combine(int m, int n, int64_t b, MatRef out, const Addend* t, int nt, cudaStream_t s) {
    return zcombine(m, n, b, out, t, nt, nullptr, s);
  }
  static int antiherm(int n, int64_t b, MatRef X, MatRef out, double* d, int64_t ds, int64_t doff,
                      cudaStream_t s) {
    return zantiherm(n, b, X, out, d, ds, doff, s);
  }
  static int trace(int n, int64_t b, MatRef X, MatRef Y, z64 coef, z64* r, int64_t rs, int64_t ro,
                   int acc, cudaStream_t s) {
    return ztrace_prod(n, b, X, Y, coef, r, rs, ro, acc, s);
  }
  static int inv(int n, int64_t b, MatRef X, int* info, MatRef, void* scr, size_t scr_bytes, cudaStream_t s) {
    return zinv_ex(n, b, X, X, info, nullptr, scr, scr_bytes, s);
  }
};

inline float2 f2(z64 v) { return make_float2((float)v.x, (float)v.y); }

struct MixedGemm {
  CGemmDesc d;
  MixedGemm(int M, int N, int K, int64_t batch, MatRef A, int opA, MatRef B, int opB, MatRef C,
            z64 alpha = ONE) {
    d.M = M;
    d.N = N;
    d.K = K;
    d.batch = batch;
    d.A = A;
    d.B = B;
    d.opA = opA;
    d.opB = opB;
    d.alpha = f2(alpha);
    d.C = C;
  }
  MixedGemm& plus(const MatRef& m, z64 coef, int ct = 0) {
    if (!m.null()) d.add[d.nadd++] = CAddend{m, f2(coef), ct};
    return *this;
  }
  MixedGemm& store_h(const MatRef& c2, z64 coef) {
    d.C2 = c2;
    d.coef2 = f2(coef);
    return *this;
  }
  MixedGemm& second(const MatRef& c3, z64 scale) {
    d.C3 = c3;
    d.scale3 = f2(scale);
    return *this;
  }
  MixedGemm& plus3(const MatRef& m, z64 coef, int ct = 0) {
    if (!m.null()) d.add[d.nadd + d.nadd3++] = CAddend{m, f2(coef), ct};
    return *this;
  }
  int run(cudaStream_t s) {
    if (d.K > 0 && (d.A.null() || d.B.null())) {
      // A zero operand: only the addends remain (a combine).
      Addend t[kMaxAddends];
      int nt = 0;
      for (int k = 0; k < d.nadd; ++k)
        t[nt++] = Addend{d.add[k].m, make_double2(d.add[k].coef.x, d.add[k].coef.y), d.add[k].conj_trans};
      if (!d.C.null()) QTX_TRY(ccombine(d.M, d.N, d.batch, d.C, t, nt, nullptr, s));
      if (!d.C3.null() || !d.C2.null()) {
        set_error("mixed gemm: zero operand with a second output is not supported");
        return QTX_ERR_UNSUPPORTED;
      }
      return QTX_OK;
    }
    return cgemm_tc(d, s);
  }
};

struct Mixed {
  static constexpr size_t E = sizeof(c32);
  static constexpr bool kInvTmp = true;
  using G = MixedGemm;
  static int combine(int m, int n, int64_t b, MatRef out, const Addend* t, int nt, cudaStream_t s) {
    return ccombine(m, n, b, out, t, nt, nullptr, s);
  }
  static int antiherm(int n, int64_t b, MatRef X, MatRef out, double* d, int64_t ds, int64_t doff,
                      cudaStream_t s) {
    return cantiherm(n, b, X, out, d, ds, doff, s);
  }
  static int trace(int n, int64_t b, MatRef X, MatRef Y, z64 coef, z64* r, int64_t rs, int64_t ro,
                   int acc, cudaStream_t s) {
    return ctrace_prod(n, b, X, Y, coef, r, rs, ro, acc, s);
  }
  // The Schur complement is inverted in FP64: upcast, Gauss-Jordan, round back.
  static int inv(int n, int64_t b, MatRef X, int* info, MatRef tmp, void* scr, size_t scr_bytes,
                 cudaStream_t s) {
    MatRef t = shaped(tmp, n);
    QTX_TRY(convert_c64_to_c128(n, n, b, X, t, s));
    QTX_TRY(zinv_ex(n, b, t, t, info, nullptr, scr, scr_bytes, s));
    return convert_c128_to_c64(n, n, b, t, X, s);
  }
};

template <class P>
int copy_block_t(int m, int n, int64_t batch, MatRef dst, MatRef src, cudaStream_t s) {
  if (dst.null()) return QTX_OK;
  Addend t = add(src, ONE);
  return P::combine(m, n, batch, dst, &t, 1, s);
}

// A helper stream per (device, caller stream) of the calling thread, at the
// device's highest priority, with the events that order it against the
// caller's stream; created on first use, kept for the thread's lifetime.
struct SideStream {
  cudaStream_t s = nullptr;
  cudaEvent_t fork = nullptr, inv = nullptr, xdone[2] = {nullptr, nullptr};
};

int side_stream(cudaStream_t s, SideStream** out) {
  thread_local std::map<std::pair<int, cudaStream_t>, SideStream> reg;
  int dev = 0;
  QTX_CHECK_CUDA(cudaGetDevice(&dev));
  SideStream& e = reg[{dev, s}];
  if (e.s == nullptr) {
    int least = 0, greatest = 0;
    QTX_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    QTX_CHECK_CUDA(cudaEventCreateWithFlags(&e.fork, cudaEventDisableTiming));
    QTX_CHECK_CUDA(cudaEventCreateWithFlags(&e.inv, cudaEventDisableTiming));
    QTX_CHECK_CUDA(cudaEventCreateWithFlags(&e.xdone[0], cudaEventDisableTiming));
    QTX_CHECK_CUDA(cudaEventCreateWithFlags(&e.xdone[1], cudaEventDisableTiming));
    QTX_CHECK_CUDA(cudaStreamCreateWithPriority(&e.s, cudaStreamNonBlocking, greatest));
  }
  *out = &e;
  return QTX_OK;
}

}  // namespace

template <class Prec>
int solve_impl(const SolveIO& io, int64_t batch, int* info, Workspace& ws, cudaStream_t s) {
  using Gemm = typename Prec::G;
  const BTRef& a = io.a;
  const int N = a.n;
  const std::vector<int>& bs = a.bs;
  const int bm = max_block(bs);
  const bool want_current = io.current != nullptr;
  std::vector<MatRef> gR(N), gX[2], st[2];
  for (int i = 0; i < N; ++i) gR[i] = ws.mat(bs[i], bs[i], batch, Prec::E);
  for (int x = 0; x < 2; ++x) {
    gX[x].resize(N);
    for (int i = 0; i < N; ++i) gX[x][i] = ws.mat(bs[i], bs[i], batch, Prec::E);
  }
  if (want_current)
    for (int x = 0; x < 2; ++x) {
      st[x].resize(N);
      for (int i = 0; i < N; ++i) st[x][i] = ws.mat(bs[i], bs[i], batch, Prec::E);
    }
  enum { P_, P2_, M_, T_, Q_, T2_, U_, V_, W_, Z_, R1_, TT_, T1X_, T2X_, Y_, XIJ_, GA_, GB_, CA_, CB_, NT_ };
  MatRef tmp[NT_];
  for (int k = 0; k < NT_; ++k) tmp[k] = ws.mat(bm, bm, batch, Prec::E);
  MatRef inv_tmp = Prec::kInvTmp ? ws.mat(bm, bm, batch, sizeof(z64)) : MatRef{};
  const size_t inv_scr_bytes = zinv_scratch_bytes(bm, batch);
  void* inv_scr = ws.take(inv_scr_bytes);
  OzScope oz(ws, Prec::E == sizeof(z64) ? bm : 0, batch);  // complex128 products only
  if (ws.base == nullptr) return QTX_OK;
  if (ws.overflow) {
    set_error("selected_solve: workspace too small");
    return QTX_ERR_WORKSPACE;
  }
  auto obc = [&](const MatRef* o, int i) { return o ? o[i] : MatRef{}; };
  const BTRef* sig[2] = {&io.sl, &io.sg};
  const MatRef* obx[2] = {io.obc_l, io.obc_g};
  const BTRef* out[2] = {&io.xl, &io.xg};
  auto sdiag = [&](int x, int i) { return sig[x]->n ? sig[x]->diag[i] : MatRef{}; };
  auto supper = [&](int x, int i) { return sig[x]->n ? sig[x]->upper[i] : MatRef{}; };
  auto odiag = [&](int x, int i) { return out[x]->n ? out[x]->diag[i] : MatRef{}; };
  auto oupper = [&](int x, int i) { return out[x]->n ? out[x]->upper[i] : MatRef{}; };
  auto olower = [&](int x, int i) { return out[x]->n ? out[x]->lower[i] : MatRef{}; };
  int64_t dens_stride = 0;
  std::vector<int64_t> offs(N + 1, 0);
  for (int i = 0; i < N; ++i) offs[i + 1] = offs[i] + bs[i];
  dens_stride = offs[N];
  const int64_t cur_stride = N + 1;

  // First layer (rgf.py:214-238).
  {
    Addend t[2] = {add(a.diag[0], ONE), add(obc(io.obc_r, 0), MONE)};
    QTX_TRY(Prec::combine(bs[0], bs[0], batch, gR[0], t, 2, s));
    QTX_TRY(Prec::inv(bs[0], batch, gR[0], info, inv_tmp, inv_scr, inv_scr_bytes, s));
    for (int x = 0; x < 2; ++x) {
      MatRef M = shaped(tmp[M_], bs[0]);
      Addend u[2] = {add(sdiag(x, 0), ONE), add(obc(obx[x], 0), ONE)};
      QTX_TRY(Prec::combine(bs[0], bs[0], batch, M, u, 2, s));
      MatRef T2 = shaped(tmp[T2_], bs[0]);
      QTX_TRY(Gemm(bs[0], bs[0], bs[0], batch, gR[0], 0, M, 0, T2).run(s));
      QTX_TRY(Gemm(bs[0], bs[0], bs[0], batch, T2, 0, gR[0], 1, gX[x][0]).run(s));
    }
  }
  // Forward sweep (rgf.py:241-302). The retarded chain runs on the helper
  // stream `sr`; the lesser/greater products of block j wait for the inverse
  // of block j, and the helper reuses the buffer of P (double-buffered by the
  // parity of j) only after the products of block j - 2 are done. Only for
  // batches below the SM count (at full batches the inverse occupies every
  // SM and the products would only share SMs with it), and not with the
  // int8-emulated products, whose digit-plane scratch is shared.
  const bool use_side =
      N > 1 && batch < (int64_t)num_sms() && !(gemm_slices() > 0 && oz_bound(nullptr) != nullptr);
  SideStream* ss = nullptr;
  cudaStream_t sr = s;
  if (use_side) {
    QTX_TRY(side_stream(s, &ss));
    sr = ss->s;
    QTX_CHECK_CUDA(cudaEventRecord(ss->fork, s));
    QTX_CHECK_CUDA(cudaStreamWaitEvent(sr, ss->fork, 0));
  }
  for (int j = 1; j < N; ++j) {
    const int i = j - 1;
    MatRef P = shaped(tmp[(j & 1) ? P2_ : P_], bs[i]);
    if (use_side && j >= 3) QTX_CHECK_CUDA(cudaStreamWaitEvent(sr, ss->xdone[j & 1], 0));
    QTX_TRY(Gemm(bs[j], bs[i], bs[i], batch, a.lower[i], 0, gR[i], 0, P).run(sr));
    QTX_TRY(Gemm(bs[j], bs[j], bs[i], batch, P, 0, a.upper[i], 0, gR[j], MONE)
                .plus(a.diag[j], ONE)
                .plus(obc(io.obc_r, j), MONE)
                .run(sr));
    QTX_TRY(Prec::inv(bs[j], batch, gR[j], info, inv_tmp, inv_scr, inv_scr_bytes, sr));
    if (use_side) {
      QTX_CHECK_CUDA(cudaEventRecord(ss->inv, sr));
      QTX_CHECK_CUDA(cudaStreamWaitEvent(s, ss->inv, 0));
    }
    for (int x = 0; x < 2; ++x) {
      MatRef Q{};
      if (!supper(x, i).null()) {
        Q = shaped(tmp[Q_], bs[j]);
        QTX_TRY(Gemm(bs[j], bs[j], bs[i], batch, P, 0, supper(x, i), 0, Q).run(s));
      }
      MatRef T = shaped(tmp[T_], bs[i]);
      QTX_TRY(Gemm(bs[j], bs[i], bs[i], batch, a.lower[i], 0, gX[x][i], 0, T).run(s));
      MatRef M = shaped(tmp[M_], bs[j]);
      if (want_current) {
        // Sigma-tilde (rgf.py:392-402) kept for the current; M = it + Sigma_jj.
        QTX_TRY(Gemm(bs[j], bs[j], bs[i], batch, T, 0, a.lower[i], 1, st[x][j])
                    .plus(Q, ONE, 1)
                    .plus(Q, MONE)
                    .second(M, ONE)
                    .plus3(sdiag(x, j), ONE)
                    .plus3(obc(obx[x], j), ONE)
                    .run(s));
      } else {
        QTX_TRY(Gemm(bs[j], bs[j], bs[i], batch, T, 0, a.lower[i], 1, M)
                    .plus(Q, ONE, 1)
                    .plus(Q, MONE)
                    .plus(sdiag(x, j), ONE)
                    .plus(obc(obx[x], j), ONE)
                    .run(s));
      }
      MatRef T2 = shaped(tmp[T2_], bs[j]);
      QTX_TRY(Gemm(bs[j], bs[j], bs[j], batch, gR[j], 0, M, 0, T2).run(s));
      QTX_TRY(Gemm(bs[j], bs[j], bs[j], batch, T2, 0, gR[j], 1, gX[x][j]).run(s));
    }
    if (use_side) QTX_CHECK_CUDA(cudaEventRecord(ss->xdone[j & 1], s));
  }
  // (The caller's stream has waited for the last inverse: every helper-stream
  // launch is ordered before what follows.)
  // Last diagonal blocks (rgf.py:305-312).
  for (int x = 0; x < 2; ++x)
    QTX_TRY(Prec::antiherm(bs[N - 1], batch, gX[x][N - 1], odiag(x, N - 1),
                      x == 0 ? io.density : nullptr, dens_stride, offs[N - 1], s));
  if (io.xr.n) QTX_TRY(copy_block_t<Prec>(bs[N - 1], bs[N - 1], batch, io.xr.diag[N - 1], gR[N - 1], s));

  // Backward sweep (rgf.py:315-412).
  MatRef GRj = gR[N - 1];
  MatRef col = gR[N - 1];  // G_{j, N-1}, j = N-1
  const bool want_g0n = !io.g0n.null();
  for (int i = N - 2; i >= 0; --i) {
    const int j = i + 1;
    MatRef U = shaped(tmp[U_], bs[j]);   // xr_ii a_ij
    MatRef V = shaped(tmp[V_], bs[i]);   // xr_jj a_ji
    MatRef W = shaped(tmp[W_], bs[j]);   // xr_ii a_ij xr_jj
    MatRef Z = shaped(tmp[Z_], bs[i]);   // xr_ii a_ij xr_jj a_ji
    QTX_TRY(Gemm(bs[i], bs[j], bs[i], batch, gR[i], 0, a.upper[i], 0, U).run(s));
    QTX_TRY(Gemm(bs[j], bs[i], bs[j], batch, GRj, 0, a.lower[i], 0, V).run(s));
    QTX_TRY(Gemm(bs[i], bs[j], bs[j], batch, U, 0, GRj, 0, W).run(s));
    QTX_TRY(Gemm(bs[i], bs[i], bs[j], batch, U, 0, V, 0, Z).run(s));
    for (int x = 0; x < 2; ++x) {
      const MatRef sx = supper(x, i);
      MatRef R1{}, TT{};
      if (!sx.null()) {
        R1 = shaped(tmp[R1_], bs[j]);
        TT = shaped(tmp[TT_], bs[i]);
        QTX_TRY(Gemm(bs[i], bs[j], bs[i], batch, gR[i], 0, sx, 0, R1).run(s));
        QTX_TRY(Gemm(bs[i], bs[i], bs[j], batch, R1, 0, W, 1, TT).run(s));
      }
      MatRef t1 = shaped(tmp[T1X_], bs[i]);
      QTX_TRY(Gemm(bs[i], bs[i], bs[i], batch, Z, 0, gX[x][i], 0, t1).plus(TT, MONE).run(s));
      MatRef t2 = shaped(tmp[T2X_], bs[j]);
      QTX_TRY(Gemm(bs[i], bs[j], bs[j], batch, U, 0, gX[x][j], 0, t2).run(s));
      MatRef xij = oupper(x, i).null() ? shaped(tmp[XIJ_], bs[j]) : oupper(x, i);
      MatRef xji = io.symmetric ? MatRef{} : olower(x, i);
      if (!sx.null()) {
        MatRef Y = shaped(tmp[Y_], bs[j]);
        QTX_TRY(Gemm(bs[i], bs[j], bs[j], batch, R1, 0, GRj, 1, Y).plus(t2, MONE).run(s));
        QTX_TRY(Gemm(bs[i], bs[j], bs[i], batch, gX[x][i], 0, V, 1, xij, MONE)
                    .plus(Y, ONE)
                    .store_h(xji, MONE)
                    .run(s));
      } else {
        QTX_TRY(Gemm(bs[i], bs[j], bs[i], batch, gX[x][i], 0, V, 1, xij, MONE)
                    .plus(t2, MONE)
                    .store_h(xji, MONE)
                    .run(s));
      }
      // X_ii = x_ii + temp_2x a_ij^H xr_ii^H + temp_1x - temp_1x^H (in place).
      QTX_TRY(Gemm(bs[i], bs[i], bs[j], batch, t2, 0, U, 1, gX[x][i])
                  .plus(gX[x][i], ONE)
                  .plus(t1, ONE)
                  .plus(t1, MONE, 1)
                  .run(s));
      QTX_TRY(Prec::antiherm(bs[i], batch, gX[x][i], odiag(x, i), x == 0 ? io.density : nullptr,
                        dens_stride, offs[i], s));
    }
    if (want_current) {
      // I_j = Tr(Sigma~^>_j X^<_jj - X^>_jj Sigma~^<_j)  (rgf.py:403-408).
      QTX_TRY(Prec::trace(bs[j], batch, st[1][j], gX[0][j], ONE, io.current, cur_stride, j, 0, s));
      QTX_TRY(Prec::trace(bs[j], batch, gX[1][j], st[0][j], MONE, io.current, cur_stride, j, 1, s));
    }
    if (want_g0n) {
      MatRef nc = shaped(tmp[(i & 1) ? CA_ : CB_], bs[N - 1]);
      if (i == 0) nc = io.g0n;
      QTX_TRY(Gemm(bs[i], bs[N - 1], bs[j], batch, U, 0, col, 0, nc, MONE).run(s));
      col = nc;
    }
    // xr_ii <- xr_ii + xr_ii a_ij xr_jj a_ji xr_ii  (rgf.py:410).
    MatRef Gi = (io.xr.n && !io.xr.diag[i].null()) ? io.xr.diag[i] : shaped(tmp[(i & 1) ? GA_ : GB_], bs[i]);
    QTX_TRY(Gemm(bs[i], bs[i], bs[i], batch, Z, 0, gR[i], 0, Gi).plus(gR[i], ONE).run(s));
    GRj = Gi;
  }
  if (want_g0n && N == 1) QTX_TRY(copy_block_t<Prec>(bs[0], bs[0], batch, io.g0n, gR[0], s));
  if (want_current) {
    // Boundary currents (rgf.py:414-428).
    const MatRef l0 = obc(io.obc_l, 0), g0 = obc(io.obc_g, 0);
    const MatRef ln = obc(io.obc_l, N - 1), gn = obc(io.obc_g, N - 1);
    // Slots 0 and N start from the caller's zero initialisation; a missing
    // OBC block contributes nothing.
    if (!g0.null())
      QTX_TRY(Prec::trace(bs[0], batch, g0, gX[0][0], ONE, io.current, cur_stride, 0, 0, s));
    if (!l0.null())
      QTX_TRY(Prec::trace(bs[0], batch, gX[1][0], l0, MONE, io.current, cur_stride, 0, g0.null() ? 0 : 1, s));
    if (!gn.null())
      QTX_TRY(Prec::trace(bs[N - 1], batch, gn, gX[0][N - 1], MONE, io.current, cur_stride, N, 0, s));
    if (!ln.null())
      QTX_TRY(Prec::trace(bs[N - 1], batch, gX[1][N - 1], ln, ONE, io.current, cur_stride, N,
                          gn.null() ? 0 : 1, s));
  }
  return QTX_OK;
}

int selected_solve_run(const SolveIO& io, int64_t batch, int* info, Workspace& ws, cudaStream_t s) {
  return solve_impl<Fp64>(io, batch, info, ws, s);
}

int selected_solve_mixed_run(const SolveIO& io, int64_t batch, int* info, Workspace& ws,
                             cudaStream_t s) {
  return solve_impl<Mixed>(io, batch, info, ws, s);
}

}  // namespace qtx
