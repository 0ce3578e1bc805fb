// Ensemble of independent realisations (no reference counterpart; the
// reference's caller for many runs is a Python loop over Simulator.run_step).
//
// Each member keeps its own model and AMG hierarchy, so its numerics are
// exactly those of a single-grid run.  Members run concurrently: a pool of
// host threads, each with its own non-blocking CUDA stream, takes members
// largest-first (longest-processing-time order) and steps each to the end.
// Small members' kernels then overlap on the SMs instead of running one grid
// at a time, and each FGMRES host loop waits only on its own stream.
#include "common.cuh"
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

extern "C" int impes_ensemble_run(impes_model** models, impes_amg** amgs, double** p, double** sw,
                                  double** sg, double** so, const int* cells, int members,
                                  int steps, double dt, const impes_krylov_params* kp, int workers,
                                  impes_ensemble_member_stats* stats, double* span_ms) {
  using namespace impes;
  if (!models || !amgs || !p || !sw || !sg || !so || !cells || !kp || !stats || members < 0 ||
      steps < 1 || !(dt > 0)) {
    set_last_error("impes_ensemble_run: bad argument");
    return IMPES_ERR_ARG;
  }
  if (span_ms) *span_ms = 0.0;
  if (members == 0) return IMPES_OK;
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 != cudaSuccess) {
    set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e0));
    return IMPES_ERR_CUDA;
  }
  std::vector<int> order(members);
  for (int i = 0; i < members; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells[a] > cells[b]; });
  for (int i = 0; i < members; ++i) stats[i] = impes_ensemble_member_stats{};
  const int nw = std::max(1, std::min(workers, members));
  std::atomic<int> next{0};
  std::vector<std::string> errors(members);
  // device span of the whole run: every worker stream waits on `t_start`
  // (recorded on `span_s`) before its first member and records its own done
  // event; `span_s` waits on all of them and records `t_end`
  cudaStream_t span_s = nullptr;
  cudaEvent_t t_start = nullptr, t_end = nullptr;
  std::vector<cudaEvent_t> done(nw, nullptr);
  bool span_ok = cudaStreamCreateWithFlags(&span_s, cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreate(&t_start) == cudaSuccess && cudaEventCreate(&t_end) == cudaSuccess;
  for (int w = 0; w < nw && span_ok; ++w) span_ok = cudaEventCreate(&done[w]) == cudaSuccess;
  if (span_ok) span_ok = cudaEventRecord(t_start, span_s) == cudaSuccess;
  auto worker = [&](int wid) {
    cudaSetDevice(dev);
    cudaStream_t s = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    bool ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess;
    if (ok && span_ok) ok = cudaStreamWaitEvent(s, t_start, 0) == cudaSuccess;
    for (int q = next.fetch_add(1); q < members; q = next.fetch_add(1)) {
      const int m = order[q];
      impes_ensemble_member_stats& st = stats[m];
      st.worker = wid;
      if (!ok) {
        st.status = IMPES_ERR_CUDA;
        errors[m] = "stream or event creation failed";
        continue;
      }
      cudaEventRecord(a, s);
      for (int t = 0; t < steps; ++t) {
        impes_krylov_stats ks{};
        const int rc = impes_step(models[m], amgs[m], p[m], sw[m], sg[m], so[m], dt, 1, kp, 0, &ks,
                                  nullptr, s);
        st.iterations += ks.iterations;
        if (rc != IMPES_OK) {
          st.status = rc;
          errors[m] = impes_last_error();
          break;
        }
        st.steps_done = t + 1;
      }
      cudaEventRecord(b, s);
      float ms = 0.f;
      if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
        st.device_ms = ms;
    }
    if (span_ok && s) cudaEventRecord(done[wid], s);
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s) cudaStreamDestroy(s);
  };
  std::vector<std::thread> pool;
  pool.reserve(nw);
  for (int w = 0; w < nw; ++w) pool.emplace_back(worker, w);
  for (auto& t : pool) t.join();
  if (span_ok) {
    for (int w = 0; w < nw; ++w) cudaStreamWaitEvent(span_s, done[w], 0);
    cudaEventRecord(t_end, span_s);
    float ms = 0.f;
    if (span_ms && cudaEventSynchronize(t_end) == cudaSuccess &&
        cudaEventElapsedTime(&ms, t_start, t_end) == cudaSuccess)
      *span_ms = ms;
  }
  for (cudaEvent_t ev : done)
    if (ev) cudaEventDestroy(ev);
  if (t_start) cudaEventDestroy(t_start);
  if (t_end) cudaEventDestroy(t_end);
  if (span_s) cudaStreamDestroy(span_s);
  for (int m = 0; m < members; ++m)
    if (stats[m].status != IMPES_OK) {
      set_last_error("member " + std::to_string(m) + ": " + errors[m]);
      return stats[m].status;
    }
  return IMPES_OK;
}
