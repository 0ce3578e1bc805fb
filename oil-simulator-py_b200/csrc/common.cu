// Shared host utilities: thread-local error text and a device exclusive scan.
#include "common.cuh"
#include <atomic>
#include <cstdlib>
#include <map>
#include <mutex>

namespace impes {

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<unsigned long long> g_launches{0};
static thread_local unsigned long long t_launches = 0;   // this host thread's launches
void count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
void count_launches(long long n) {
  g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed);
  t_launches += (unsigned long long)n;
}
unsigned long long launches() { return g_launches.load(std::memory_order_relaxed); }
unsigned long long thread_launches() { return t_launches; }

void raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<const void*, size_t> current;
  std::lock_guard<std::mutex> lock(mu);
  size_t& c = current[kernel];
  if (bytes > c) {
    IMPES_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    c = bytes;
  }
}
const char* last_error_cstr() { return g_last_error.c_str(); }

bool pdl_enabled() {
  static const bool on = [] {
    const char* ev = getenv("IMPES_NO_PDL");
    return !(ev && ev[0] == '1');
  }();
  return on;
}

PhaseTimers& timers() {
  static PhaseTimers t;
  return t;
}

namespace {
constexpr int kScanBlock = 1024;

// Phase 1: per-block inclusive scan in shared memory; block totals to `sums`.
__global__ void k_scan_block(const int* __restrict__ in, int* __restrict__ out, int n,
                             int* __restrict__ sums) {
  __shared__ int s[kScanBlock];
  int i = blockIdx.x * kScanBlock + threadIdx.x;
  int v = (i < n) ? in[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < kScanBlock; o <<= 1) {
    int t = (threadIdx.x >= (unsigned)o) ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = s[threadIdx.x] - v;  // exclusive
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = s[threadIdx.x];
}

// Phase 2: add the scanned block offsets; last element gets the total.
__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ offs) {
  int i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += offs[blockIdx.x];
}
__global__ void k_scan_total(const int* __restrict__ in, int* __restrict__ out, int n) {
  out[n] = (n > 0) ? out[n - 1] + in[n - 1] : 0;
}
}  // namespace

void exclusive_scan_i32_dev(const int* d_in, int* d_out, int n, cudaStream_t stream) {
  if (n <= 0) {
    IMPES_CUDA(cudaMemsetAsync(d_out, 0, sizeof(int), stream));
    return;
  }
  int nb = (n + kScanBlock - 1) / kScanBlock;
  DBuf<int> sums(nb), offs(nb + 1);
  k_scan_block<<<nb, kScanBlock, 0, stream>>>(d_in, d_out, n, sums.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  if (nb > 1) {
    exclusive_scan_i32_dev(sums.p, offs.p, nb, stream);
    k_scan_add<<<nb, kScanBlock, 0, stream>>>(d_out, n, offs.p); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
  }
  k_scan_total<<<1, 1, 0, stream>>>(d_in, d_out, n); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  // temporaries are freed at scope exit: make sure the kernels using them ran
  IMPES_CUDA(cudaStreamSynchronize(stream));
}

int exclusive_scan_i32(const int* d_in, int* d_out, int n, cudaStream_t stream) {
  exclusive_scan_i32_dev(d_in, d_out, n, stream);
  int total = 0;
  IMPES_CUDA(cudaMemcpyAsync(&total, d_out + n, sizeof(int), cudaMemcpyDeviceToHost, stream));
  IMPES_CUDA(cudaStreamSynchronize(stream));
  return total;
}

}  // namespace impes
