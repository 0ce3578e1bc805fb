// Shared device/host utilities for the IMPES + AMG library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>
#include <stdexcept>
#include <utility>

#include "../../include/impes_b200.h"

namespace impes {

// ------------------------------------------------------------------ errors
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

// Number of kernel launches issued by this library (every launch site calls it;
// graph replays add the kernels they hold).
void count_launch();
void count_launches(long long n);
unsigned long long launches();
unsigned long long thread_launches();   // launches issued by the calling host thread
// Raise a kernel's dynamic shared-memory limit to at least `bytes`; never
// lowers it, so host threads launching the same kernel with different sizes
// do not undo each other's setting.
void raise_smem_limit(const void* kernel, size_t bytes);

#define IMPES_CUDA(call)                                                        \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess)                                                      \
      throw ::impes::Error(IMPES_ERR_CUDA, std::string(#call) + ": " +          \
                                               cudaGetErrorString(e_));         \
  } while (0)

#define IMPES_CHECK_LAUNCH() IMPES_CUDA(cudaGetLastError())

#define IMPES_REQUIRE(cond, code, msg)                                          \
  do {                                                                          \
    if (!(cond)) throw ::impes::Error((code), (msg));                           \
  } while (0)

// ------------------------------------------------------------ device buffer
// Owning device allocation (library workspace; callers own their own I/O).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      cudaError_t e = cudaMalloc(&p, count * sizeof(T));
      if (e != cudaSuccess) {
        p = nullptr; n = 0;
        throw Error(IMPES_ERR_OOM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes: " +
                                       cudaGetErrorString(e));
      }
    }
  }
  void ensure(size_t count) { if (count > n) alloc(count); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr; n = 0;
  }
  T* get() const { return p; }
  size_t bytes() const { return n * sizeof(T); }
};

// Small pinned host scratch for device->host scalars.
template <typename T>
struct HostPinned {
  T* p = nullptr;
  size_t n = 0;
  explicit HostPinned(size_t count = 1) {
    n = count;
    if (cudaMallocHost(&p, count * sizeof(T)) != cudaSuccess) {
      p = nullptr;
      throw Error(IMPES_ERR_OOM, "cudaMallocHost failed");
    }
  }
  ~HostPinned() { if (p) cudaFreeHost(p); }
  HostPinned(const HostPinned&) = delete;
  HostPinned& operator=(const HostPinned&) = delete;
};

inline int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

inline unsigned grid_for(size_t n, int block, int max_per_sm = 8) {
  size_t g = (n + block - 1) / block;
  size_t cap = (size_t)num_sms() * max_per_sm * 8;
  if (g > cap) g = cap;
  return (unsigned)(g ? g : 1);
}

// ------------------------------------------- programmatic dependent launch
// Kernels of the solver chains (V-cycle, FGMRES) start with pdl_wait_release():
// griddepcontrol.wait holds the kernel until the grid it depends on has
// completed and its memory is visible (a no-op when the kernel was launched
// without the programmatic attribute), then launch_dependents lets the next
// kernel of the stream launch at once, so its blocks are scheduled while this
// grid runs and wait on the device instead of after a launch gap.  Only kernels
// that begin with this call may be launched through launch_pdl.
__device__ __forceinline__ void pdl_wait_release() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
// false when the environment sets IMPES_NO_PDL=1 (plain stream order)
bool pdl_enabled();
template <typename... P, typename... A>
void launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  IMPES_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
  count_launch();
}

// --------------------------------------------------------- device helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_sum_int(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum in a fixed tree order (deterministic for a fixed block size).
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double* smem /*>= BLOCK/32*/) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) smem[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < BLOCK / 32) ? smem[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// ------------------------------------------------------------ phase timers
// CUDA-event pairs around phases of the step; global, enabled on demand.
struct PhaseTimers {
  struct Rec { int phase; cudaEvent_t a, b; double bytes; };
  bool on = false;
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  // During stream capture, records become external event nodes of the graph,
  // collected in `capture`; after a replay has completed, harvest() adds them.
  std::vector<Rec>* capture = nullptr;
  const std::vector<Rec>* pending = nullptr;
  long long acc_n[16] = {};
  double acc_ms[16] = {}, acc_bytes[16] = {};
  void harvest() {
    if (!pending) return;
    for (const Rec& r : *pending) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess && r.phase >= 0 && r.phase < 16) {
        acc_n[r.phase] += 1;
        acc_ms[r.phase] += ms;
        acc_bytes[r.phase] += r.bytes;
      }
    }
    pending = nullptr;
  }
  cudaEvent_t take() {
    if (pool.empty()) {
      cudaEvent_t e;
      IMPES_CUDA(cudaEventCreate(&e));
      return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  int begin(int phase, cudaStream_t s) {
    if (!on) return -1;
    Rec r{phase, take(), take(), 0.0};
    if (capture) {
      IMPES_CUDA(cudaEventRecordWithFlags(r.a, s, cudaEventRecordExternal));
      capture->push_back(r);
      return -2 - (int)(capture->size() - 1);
    }
    IMPES_CUDA(cudaEventRecord(r.a, s));
    recs.push_back(r);
    return (int)recs.size() - 1;
  }
  void end(int idx, cudaStream_t s, double bytes) {
    if (idx == -1) return;
    if (idx <= -2) {
      Rec& r = (*capture)[-2 - idx];
      r.bytes = bytes;
      IMPES_CUDA(cudaEventRecordWithFlags(r.b, s, cudaEventRecordExternal));
      return;
    }
    recs[idx].bytes = bytes;
    IMPES_CUDA(cudaEventRecord(recs[idx].b, s));
  }
};
PhaseTimers& timers();

// ------------------------------------------------------------- host helpers
// Exclusive scan of int32 counts into int32 offsets (returns total).  Runs a
// three-phase block scan on `stream`; `total_host` is filled after a sync.
int exclusive_scan_i32(const int* d_in, int* d_out, int n, cudaStream_t stream);
// Same, result left on the device in d_out[n] (no host sync).
void exclusive_scan_i32_dev(const int* d_in, int* d_out, int n, cudaStream_t stream);

}  // namespace impes
