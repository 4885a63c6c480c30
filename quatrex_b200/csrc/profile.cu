// Optional launch profiler: when enabled, every kernel launch of the
// library is bracketed by a pair of CUDA events on its stream, tagged with
// the kernel class and its algorithmic work (flops or bytes). Reading the
// profile synchronizes the recorded events and sums durations per class.
// Launches during CUDA-graph capture are not recorded.
#include <mutex>
#include <vector>

#include "common.cuh"

namespace qtx {
namespace {

struct Rec {
  cudaEvent_t a, b;
  int kind;
  double work;
  int launches;
};

thread_local int t_depth = 0;

std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

}  // namespace

ProfScope::ProfScope(int kind, double work, cudaStream_t s, int launches) : idx_(-1), s_(s) {
  if (t_depth++ > 0) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_on) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;
  Rec r{take_event(), take_event(), kind, work, launches};
  cudaEventRecord(r.a, s);
  idx_ = (int)g_recs.size();
  g_recs.push_back(r);
}

ProfScope::~ProfScope() {
  --t_depth;
  if (idx_ < 0) return;
  std::lock_guard<std::mutex> lk(g_mu);
  if (idx_ < (int)g_recs.size()) cudaEventRecord(g_recs[idx_].b, s_);
}

}  // namespace qtx

using namespace qtx;

extern "C" int qtx_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_on = on != 0;
  return QTX_OK;
}

extern "C" int qtx_profile_reset(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& r : g_recs) {
    g_pool.push_back(r.a);
    g_pool.push_back(r.b);
  }
  g_recs.clear();
  return QTX_OK;
}

extern "C" int qtx_profile_read(int kind, double* total_ms, double* total_work, int64_t* launches) {
  std::lock_guard<std::mutex> lk(g_mu);
  double ms = 0.0, work = 0.0;
  int64_t n = 0;
  for (auto& r : g_recs) {
    if (kind >= 0 && r.kind != kind) continue;
    if (cudaEventSynchronize(r.b) != cudaSuccess) {
      set_error("qtx_profile_read: event synchronisation failed");
      return QTX_ERR_CUDA;
    }
    float t = 0.f;
    if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) {
      set_error("qtx_profile_read: elapsed time unavailable");
      return QTX_ERR_CUDA;
    }
    ms += t;
    work += r.work;
    n += r.launches;
  }
  if (total_ms) *total_ms = ms;
  if (total_work) *total_work = work;
  if (launches) *launches = n;
  return QTX_OK;
}
