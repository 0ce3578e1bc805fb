// AMG cycling: CSR kernels, l1-Jacobi smoothing, V-cycle, coarsest solve,
// stand-alone V-cycle solve, apply, and flexible GMRES.
//
// Reference: researchim-ai/oil-simulator-py src/solver/classical_amg.py
//   _spmv_csr :976-1009, _smooth :1016-1035, _v_cycle :1037-1106,
//   solve :1108-1155, apply :1157-1180.  FGMRES has no reference counterpart.
//
// Kernels are templated on the value type (double for the FP64 path, float for
// the FP32 V-cycle of the mixed path) and on the number of lanes that share a
// row (1 for the 7-point level, up to 32 for wide coarse rows).
#include "amg.cuh"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

// handle accessors (abi.cu)
bool impes_amg_handle_built(impes_amg* h);
impes::AMG* impes_amg_handle_core(impes_amg* h);

namespace impes {
namespace {

constexpr int TB = 256;
constexpr double kOmega = 0.7;  // classical_amg.py:1022

enum CsrMode { Y_AX = 0, Y_B_MINUS_AX = 1, Y_SMOOTH = 2, Y_ADD_AX = 3, Y_SMOOTH0 = 4, Y_W_AX = 5 };

// One group of LPR lanes per row.  MODE selects the fused epilogue:
//  Y_AX: y = A x;  Y_B_MINUS_AX: y = b - A x;  Y_SMOOTH: y = x + w*inv*(b - A x);
//  Y_ADD_AX: y += A x (prolongation);  Y_SMOOTH0: y = w*inv*b (x = 0);
//  Y_W_AX: y = wt .* (A x) (weighted operator of FGMRES, wt passed as inv).
// CT is int, or unsigned short with the column of entry k at
// col[k] + (rel ? row - 32768 : 0): plain 16-bit indices on levels of at most
// 65536 rows, row-relative ones on larger levels whose bandwidth fits.
template <typename CT>
__device__ __forceinline__ int col_base(long long row, int rel) {
  return (sizeof(CT) == 2 && rel) ? (int)row - 32768 : 0;
}

// sum_k val[k] * x[cb + col[k]] over k = a0, a0 + S, ... < e, added in that
// order; four entries' loads are issued before their products are added, so
// each thread keeps four gathers of x in flight (the rows of the coarse levels
// are latency-bound on the column -> x chain).  Same result bits as the plain
// loop.
template <typename T, typename CT, typename XT>
__device__ __forceinline__ T row_dot(int a0, int e, int S, const T* __restrict__ val, const CT* __restrict__ col,
                                     const XT* __restrict__ x, int cb, T acc) {
  int k = a0;
  for (; k + 3 * S < e; k += 4 * S) {
    const T v0 = val[k], v1 = val[k + S], v2 = val[k + 2 * S], v3 = val[k + 3 * S];
    const int c0 = (int)col[k], c1 = (int)col[k + S], c2 = (int)col[k + 2 * S], c3 = (int)col[k + 3 * S];
    const T x0 = x[cb + c0], x1 = x[cb + c1], x2 = x[cb + c2], x3 = x[cb + c3];
    acc += v0 * x0;
    acc += v1 * x1;
    acc += v2 * x2;
    acc += v3 * x3;
  }
  for (; k < e; k += S) acc += val[k] * x[cb + (int)col[k]];
  return acc;
}

// row_dot with eight entries' loads issued before their products (then four,
// then one): the SELL kernels, whose value and column loads are coalesced and
// cheap to issue, keep twice the gathers of x in flight.  Same summation order.
template <typename T, typename CT, typename XT>
__device__ __forceinline__ T row_dot8(int a0, int e, int S, const T* __restrict__ val, const CT* __restrict__ col,
                                      const XT* __restrict__ x, int cb, T acc) {
  int k = a0;
  for (; k + 7 * S < e; k += 8 * S) {
    T v[8];
    int c[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      v[u] = val[k + u * S];
      c[u] = (int)col[k + u * S];
    }
    T xv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) xv[u] = x[cb + c[u]];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc += v[u] * xv[u];
  }
  return row_dot(k, e, S, val, col, x, cb, acc);
}

template <typename T, typename CT, int LPR, int MODE>
__global__ void __launch_bounds__(TB) k_csr(int n, const int* __restrict__ rowptr,
                                            const CT* __restrict__ col, const T* __restrict__ val,
                                            const T* __restrict__ x, const T* __restrict__ b,
                                            const T* __restrict__ inv, T* __restrict__ y, int rel) {
  pdl_wait_release();
  const int g = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  const int rows_per_block = TB / LPR;
  for (long long row = (long long)blockIdx.x * rows_per_block + g; row < n;
       row += (long long)gridDim.x * rows_per_block) {
    T acc = T(0);
    if (MODE != Y_SMOOTH0) {
      const int a = rowptr[row], e = rowptr[row + 1];
      const int cb = col_base<CT>(row, rel);
      acc = row_dot(a + lane, e, LPR, val, col, x, cb, acc);
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
    }
    if (lane == 0) {
      if (MODE == Y_AX) y[row] = acc;
      else if (MODE == Y_B_MINUS_AX) y[row] = b[row] - acc;
      else if (MODE == Y_SMOOTH) y[row] = x[row] + T(kOmega) * inv[row] * (b[row] - acc);
      else if (MODE == Y_ADD_AX) y[row] = y[row] + acc;
      else if (MODE == Y_SMOOTH0) y[row] = T(kOmega) * inv[row] * b[row];
      else if (MODE == Y_W_AX) y[row] = inv[row] * acc;
    }
  }
}

// Wide rows (coarse Galerkin levels, hundreds to thousands of entries per row):
// WPR warps per row, chosen by the mean row length.  Thread t of the row group
// takes entries a+t, a+t+G, ... (G = 32*WPR), so each warp's value and column
// loads are coalesced and its gathers of x hit adjacent columns.  CT and rel as
// in k_csr (16-bit columns: 6 bytes per fp32 entry instead of 8).  With WPR > 1
// the row's first warp adds the group's partial sums in a fixed order.  Same
// epilogues as k_csr.
template <typename T, typename CT, int MODE, int WPR>
__global__ void __launch_bounds__(TB) k_csr_rows(int n, const int* __restrict__ rowptr,
                                                 const CT* __restrict__ col, const T* __restrict__ val,
                                                 const T* __restrict__ x, const T* __restrict__ b,
                                                 const T* __restrict__ inv, T* __restrict__ y, int rel) {
  pdl_wait_release();
  constexpr int kWarps = TB / 32, kRows = kWarps / WPR, G = 32 * WPR;
  __shared__ T part[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int grp = warp / WPR, sub = warp % WPR;
  const int tid = sub * 32 + lane;
  for (long long base = (long long)blockIdx.x * kRows; base < n; base += (long long)gridDim.x * kRows) {
    const long long row = base + grp;
    T acc = T(0);
    if (row < n) {
      const int a = rowptr[row], e = rowptr[row + 1];
      const int cb = col_base<CT>(row, rel);
      acc = row_dot(a + tid, e, G, val, col, x, cb, acc);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    }
    if (WPR == 1) {
      if (lane == 0 && row < n) {
        if (MODE == Y_AX) y[row] = acc;
        else if (MODE == Y_B_MINUS_AX) y[row] = b[row] - acc;
        else if (MODE == Y_SMOOTH) y[row] = x[row] + T(kOmega) * inv[row] * (b[row] - acc);
        else if (MODE == Y_ADD_AX) y[row] = y[row] + acc;
        else if (MODE == Y_W_AX) y[row] = inv[row] * acc;
      }
      continue;
    }
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (sub == 0 && lane == 0 && row < n) {
      T t = part[warp];
#pragma unroll
      for (int w = 1; w < WPR; ++w) t += part[warp + w];
      if (MODE == Y_AX) y[row] = t;
      else if (MODE == Y_B_MINUS_AX) y[row] = b[row] - t;
      else if (MODE == Y_SMOOTH) y[row] = x[row] + T(kOmega) * inv[row] * (b[row] - t);
      else if (MODE == Y_ADD_AX) y[row] = y[row] + t;
      else if (MODE == Y_W_AX) y[row] = inv[row] * t;
    }
    __syncthreads();
  }
}

// 16-byte asynchronous global -> shared copy; src_bytes < 16 zero-fills the rest
// (only src_bytes are read from global memory).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned saddr = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// Wide rows, streamed: each warp walks its rows in chunks of kCh entries that
// cp.async brings into shared memory (two stages, the next chunk -- of this row
// or of the warp's next row -- in flight while the current one is consumed), so
// HBM sees many outstanding 16-byte requests per warp instead of one load per
// lane per step.  Chunks start at 8-entry boundaries (16-byte aligned for fp32
// values and 16-bit columns); the last piece of a row is clamped to the row end,
// so nothing past it is read.  Entries of a chunk outside the row are skipped.
// fp32 values only (the mixed V-cycle).  CT and rel as in k_csr; same epilogues.
// Chunks are 512 entries with 16-bit columns and 384 with int columns.
template <typename CT, int MODE>
__global__ void __launch_bounds__(TB) k_csr_stream(int n, const int* __restrict__ rowptr,
                                                   const CT* __restrict__ col, const float* __restrict__ val,
                                                   const float* __restrict__ x, const float* __restrict__ b,
                                                   const float* __restrict__ inv, float* __restrict__ y,
                                                   int rel) {
  pdl_wait_release();
  constexpr int kWarps = TB / 32;
  constexpr int kCh = sizeof(CT) == 2 ? 512 : 384;   // 48 KB of stages per block
  __shared__ __align__(16) float s_val[kWarps][2][kCh];
  __shared__ __align__(16) CT s_col[kWarps][2][kCh];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long stride = (long long)gridDim.x * kWarps;
  long long row = (long long)blockIdx.x * kWarps + warp;
  if (row >= n) return;                       // warp-uniform
  constexpr int VP = 16 / sizeof(float);      // values per 16-byte piece
  constexpr int CP = 16 / sizeof(CT);         // columns per piece
  // issue the copies of chunk [g0, g0 + kCh) of a row ending at e into stage st
  auto fetch = [&](int g0, int e, int st) {
    for (int q = lane; q < kCh / VP; q += 32) {
      const int gi = g0 + q * VP;
      const int valid = e - gi;
      if (valid > 0) cp_async16(&s_val[warp][st][q * VP], val + gi, (valid >= VP ? VP : valid) * 4);
    }
    for (int q = lane; q < kCh / CP; q += 32) {
      const int gi = g0 + q * CP;
      const int valid = e - gi;
      if (valid > 0)
        cp_async16(&s_col[warp][st][q * CP], col + gi, (valid >= CP ? CP : valid) * (int)sizeof(CT));
    }
  };
  int a = rowptr[row], e = rowptr[row + 1];
  int g = a & ~7;                             // current chunk start
  int st = 0;
  fetch(g, e, st);
  cp_async_commit();
  float acc = 0.0f;
  while (true) {
    // the task after this chunk: the next chunk of this row, or the next row
    long long nrow = row;
    int na = a, ne = e, ng = g + kCh;
    if (ng >= e) {
      nrow = row + stride;
      if (nrow < n) { na = rowptr[nrow]; ne = rowptr[nrow + 1]; ng = na & ~7; }
    }
    if (nrow < n) fetch(ng, ne, st ^ 1);
    cp_async_commit();
    cp_async_wait1();
    __syncwarp();
    const int lo = a > g ? a - g : 0;
    const int hi = e - g < kCh ? e - g : kCh;
    const int cb = col_base<CT>(row, rel);
    for (int j = lo + lane; j < hi; j += 32) acc += s_val[warp][st][j] * x[cb + (int)s_col[warp][st][j]];
    __syncwarp();                             // stage st is refilled two chunks on
    if (g + kCh >= e) {                       // row done
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0) {
        if (MODE == Y_AX) y[row] = acc;
        else if (MODE == Y_B_MINUS_AX) y[row] = b[row] - acc;
        else if (MODE == Y_SMOOTH) y[row] = x[row] + float(kOmega) * inv[row] * (b[row] - acc);
        else if (MODE == Y_ADD_AX) y[row] = y[row] + acc;
        else if (MODE == Y_W_AX) y[row] = inv[row] * acc;
      }
      acc = 0.0f;
    }
    if (nrow >= n) break;
    row = nrow; a = na; e = ne; g = ng;
    st ^= 1;
  }
}

template <typename T, typename CT, int MODE>
void launch_wide(int n, int avg, const int* rowptr, const CT* col, const T* val, const T* x,
                 const T* b, const T* inv, T* y, int rel, cudaStream_t s) {
  auto grid = [&](int rows_per_block) {
    return grid_for(((size_t)(n + rows_per_block - 1) / rows_per_block) * TB, TB, 16);
  };
  // fp32 rows longer than 512 entries on levels of 48 MB or more: streamed
  // through shared memory (A/B on the 1e6-cell case, ~100 MB levels: 28 us
  // against 30 us per wide sweep).  Shorter rows are faster with the direct
  // kernel, and so are levels that stay in L2: on 64 models of <= 262,144 cells
  // stepped concurrently, streaming their <= 30 MB levels cost 20-35 % of the
  // run (the 48 KB of shared memory per block crowds out the other models).
  if constexpr (sizeof(T) == 4) {
    constexpr double kStreamMinBytes = 48.0 * (1 << 20);
    if (avg > 512 && (double)n * avg * (sizeof(T) + sizeof(CT)) >= kStreamMinBytes) {
      launch_pdl(k_csr_stream<CT, MODE>, grid(8), TB, 0, s, n, rowptr, col, (const float*)val, (const float*)x,
                                                    (const float*)b, (const float*)inv, (float*)y, rel);
      return;
    }
  }
  if (avg <= 512) {
    launch_pdl(k_csr_rows<T, CT, MODE, 1>, grid(8), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel);
  } else if (avg <= 1536) {
    launch_pdl(k_csr_rows<T, CT, MODE, 2>, grid(4), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel);
  } else {
    launch_pdl(k_csr_rows<T, CT, MODE, 4>, grid(2), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel);
  }
}

template <typename T, typename CT, int MODE>
void launch_lanes(int lpr, int n, const int* rowptr, const CT* col, const T* val, const T* x,
                  const T* b, const T* inv, T* y, int rel, cudaStream_t s) {
  auto grid = [&](int l) { return grid_for(((size_t)n * l + TB - 1) / TB * TB, TB, 16); };
  switch (lpr) {
    case 1: launch_pdl(k_csr<T, CT, 1, MODE>, grid(1), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel); break;
    case 2: launch_pdl(k_csr<T, CT, 2, MODE>, grid(2), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel); break;
    case 4: launch_pdl(k_csr<T, CT, 4, MODE>, grid(4), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel); break;
    case 8: launch_pdl(k_csr<T, CT, 8, MODE>, grid(8), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel); break;
    case 16: launch_pdl(k_csr<T, CT, 16, MODE>, grid(16), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel); break;
    default: launch_pdl(k_csr<T, CT, 32, MODE>, grid(32), TB, 0, s, n, rowptr, col, val, x, b, inv, y, rel); break;
  }
}

// Lanes per row by mean row length (the rule used until a level is autotuned).
inline int default_lpr(int avg) { return avg <= 8 ? 1 : avg <= 16 ? 4 : avg <= 48 ? 8 : avg <= 96 ? 16 : 32; }

// col16 / rel: the level's columns as 16-bit indices (absolute when rel is 0,
// row - 32768 + col16 when rel is 1), or null for the int columns.  lpr > 0
// (an autotuned choice, rows of at most 96 entries on average) overrides the
// lanes per row.
template <typename T, int MODE>
void launch_csr(int n, int avg, const int* rowptr, const int* col, const T* val, const T* x,
                const T* b, const T* inv, T* y, cudaStream_t s,
                const unsigned short* col16 = nullptr, int rel = 0, int lpr_tuned = 0) {
  if (n <= 0) return;
  int lpr = default_lpr(avg);
  if (lpr_tuned > 0 && avg <= 96) lpr = lpr_tuned;
  if (MODE == Y_SMOOTH0) lpr = 1;
  if (lpr < 32 || (lpr_tuned == 32 && avg <= 96)) {
    if (col16) launch_lanes<T, unsigned short, MODE>(lpr, n, rowptr, col16, val, x, b, inv, y, rel, s);
    else launch_lanes<T, int, MODE>(lpr, n, rowptr, col, val, x, b, inv, y, 0, s);
  } else {
    if (col16) launch_wide<T, unsigned short, MODE>(n, avg, rowptr, col16, val, x, b, inv, y, rel, s);
    else launch_wide<T, int, MODE>(n, avg, rowptr, col, val, x, b, inv, y, 0, s);
  }
  IMPES_CHECK_LAUNCH();
}

// Restriction fused with the coarse level's first l1-Jacobi sweep from zero:
// bc = R r (as k_csr Y_AX with LPR lanes per row) and xc = w inv_c bc (as
// Y_SMOOTH0), so the coarse level starts with two sweeps left.
template <typename T, int LPR>
__global__ void __launch_bounds__(TB) k_restrict_s0(int nc, const int* __restrict__ rowptr,
                                                    const int* __restrict__ col, const T* __restrict__ val,
                                                    const T* __restrict__ r, const T* __restrict__ inv_c,
                                                    T* __restrict__ bc, T* __restrict__ xc) {
  pdl_wait_release();
  const int g = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  const int rows_per_block = TB / LPR;
  for (long long row = (long long)blockIdx.x * rows_per_block + g; row < nc;
       row += (long long)gridDim.x * rows_per_block) {
    T acc = row_dot(rowptr[row] + lane, rowptr[row + 1], LPR, val, col, r, 0, T(0));
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
    if (lane == 0) {
      bc[row] = acc;
      xc[row] = T(kOmega) * inv_c[row] * acc;
    }
  }
}

template <typename T>
void launch_restrict_s0(const Level& L, int lpr, const T* rval, const T* r, const T* inv_c, T* bc, T* xc,
                        cudaStream_t s) {
  const int n = L.nc;
  auto grid = [&](int l) { return grid_for(((size_t)n * l + TB - 1) / TB * TB, TB, 16); };
  switch (lpr) {
    case 1: launch_pdl(k_restrict_s0<T, 1>, grid(1), TB, 0, s, n, (const int*)L.rrow.p, (const int*)L.rcol.p, rval, r, inv_c, bc, xc); break;
    case 2: launch_pdl(k_restrict_s0<T, 2>, grid(2), TB, 0, s, n, (const int*)L.rrow.p, (const int*)L.rcol.p, rval, r, inv_c, bc, xc); break;
    case 4: launch_pdl(k_restrict_s0<T, 4>, grid(4), TB, 0, s, n, (const int*)L.rrow.p, (const int*)L.rcol.p, rval, r, inv_c, bc, xc); break;
    case 8: launch_pdl(k_restrict_s0<T, 8>, grid(8), TB, 0, s, n, (const int*)L.rrow.p, (const int*)L.rcol.p, rval, r, inv_c, bc, xc); break;
    case 16: launch_pdl(k_restrict_s0<T, 16>, grid(16), TB, 0, s, n, (const int*)L.rrow.p, (const int*)L.rcol.p, rval, r, inv_c, bc, xc); break;
    default: launch_pdl(k_restrict_s0<T, 32>, grid(32), TB, 0, s, n, (const int*)L.rrow.p, (const int*)L.rcol.p, rval, r, inv_c, bc, xc); break;
  }
  IMPES_CHECK_LAUNCH();
}

// ------------------------------------------------------ SELL-32 sweeps
// Sliced ELLPACK with slices of one warp (C = 32) and rows sorted by length
// inside windows (Kreutzer et al., "A unified sparse matrix data format for
// efficient general sparse matrix-vector multiplication on modern processors
// with wide SIMD units", SIAM J. Sci. Comput. 36(5), 2014), with LPR lanes per
// row: a slice holds 32 / LPR rows, and entry j of its row q sits at
// sptr[s] + 32 (j / LPR) + q LPR + j % LPR.  At each step the warp's value and
// column loads are one contiguous segment, where the CSR kernels' loads touch
// up to 32 / LPR segments.  Lane l of a row adds entries l, l + LPR, ... and
// the lanes are reduced as in k_csr with the same LPR, so a row sums in the
// same order (padding adds +0).  CT and rel as in k_csr; same epilogues.
template <typename T, typename CT, int LPR, int MODE>
__global__ void __launch_bounds__(TB) k_sell(int n, int nslices, const int* __restrict__ sptr,
                                             const int* __restrict__ perm, const CT* __restrict__ col,
                                             const T* __restrict__ val, const T* __restrict__ x,
                                             const T* __restrict__ b, const T* __restrict__ inv,
                                             T* __restrict__ y, int rel) {
  pdl_wait_release();
  constexpr int R = 32 / LPR;   // rows per slice
  const int lane = threadIdx.x & 31;
  const int warps = (int)((gridDim.x * (unsigned)TB) >> 5);
  for (int s = (int)((blockIdx.x * (unsigned)TB + threadIdx.x) >> 5); s < nslices; s += warps) {
    const int r = s * R + lane / LPR;
    const int row = perm[r < n ? r : n - 1];
    const int cb = col_base<CT>(row, rel);
    T acc = row_dot8(sptr[s] + lane, sptr[s + 1], 32, val, col, x, cb, T(0));
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
    if (r < n && lane % LPR == 0) {
      if (MODE == Y_AX) y[row] = acc;
      else if (MODE == Y_B_MINUS_AX) y[row] = b[row] - acc;
      else if (MODE == Y_SMOOTH) y[row] = x[row] + T(kOmega) * inv[row] * (b[row] - acc);
      else if (MODE == Y_ADD_AX) y[row] = y[row] + acc;
      else if (MODE == Y_W_AX) y[row] = inv[row] * acc;
    }
  }
}

template <typename T> const T* sell_values(const Level& L);
template <> inline const double* sell_values<double>(const Level& L) { return L.sell_val.p; }
template <> inline const float* sell_values<float>(const Level& L) { return L.sell_valf.p; }

template <typename T, typename CT, int MODE>
void launch_sell_ct(const Level& L, const CT* col, int rel, const T* x, const T* b, const T* inv, T* y,
                    cudaStream_t s) {
  const unsigned grid = grid_for((size_t)L.sell_slices * 32, TB, 16);
  const int* sp = L.sell_ptr.p;
  const int* pm = L.sell_perm.p;
  const T* v = sell_values<T>(L);
  switch (L.sell_lpr) {
    case 1: launch_pdl(k_sell<T, CT, 1, MODE>, grid, TB, 0, s, L.n, L.sell_slices, sp, pm, col, v, x, b, inv, y, rel); break;
    case 2: launch_pdl(k_sell<T, CT, 2, MODE>, grid, TB, 0, s, L.n, L.sell_slices, sp, pm, col, v, x, b, inv, y, rel); break;
    case 4: launch_pdl(k_sell<T, CT, 4, MODE>, grid, TB, 0, s, L.n, L.sell_slices, sp, pm, col, v, x, b, inv, y, rel); break;
    default: launch_pdl(k_sell<T, CT, 8, MODE>, grid, TB, 0, s, L.n, L.sell_slices, sp, pm, col, v, x, b, inv, y, rel); break;
  }
  IMPES_CHECK_LAUNCH();
}

template <typename T, int MODE>
void launch_sell(const Level& L, const T* x, const T* b, const T* inv, T* y, cudaStream_t s) {
  if (L.sell_col16.p)
    launch_sell_ct<T, unsigned short, MODE>(L, (const unsigned short*)L.sell_col16.p, L.col16_rel, x, b, inv, y, s);
  else
    launch_sell_ct<T, int, MODE>(L, (const int*)L.sell_col.p, 0, x, b, inv, y, s);
}

// ------------------------------------------------------ DIA sweeps
// A level whose entries lie on at most Level::kDiaMax diagonals (the 7-point
// stencil of a structured grid) as one value array per diagonal: one thread per
// row, every value load and every x load of a warp contiguous, no column
// indices.  The diagonals are added in ascending offset, the row's CSR order,
// skipping offsets that leave the matrix (entries the pattern lacks hold 0).
struct DiaOffsets {
  int off[Level::kDiaMax];
};
template <typename T, int MODE>
__global__ void __launch_bounds__(TB) k_dia(int n, int nd, DiaOffsets o, const T* __restrict__ val,
                                            const T* __restrict__ x, const T* __restrict__ b,
                                            const T* __restrict__ inv, T* __restrict__ y) {
  pdl_wait_release();
  for (int i = blockIdx.x * TB + threadIdx.x; i < n; i += gridDim.x * TB) {
    T acc = T(0);
#pragma unroll
    for (int d = 0; d < Level::kDiaMax; ++d) {
      if (d < nd) {
        const int j = i + o.off[d];
        if (j >= 0 && j < n) acc += val[(long long)d * n + i] * x[j];
      }
    }
    if (MODE == Y_AX) y[i] = acc;
    else if (MODE == Y_B_MINUS_AX) y[i] = b[i] - acc;
    else if (MODE == Y_SMOOTH) y[i] = x[i] + T(kOmega) * inv[i] * (b[i] - acc);
    else if (MODE == Y_ADD_AX) y[i] = y[i] + acc;
    else if (MODE == Y_W_AX) y[i] = inv[i] * acc;
  }
}
// ND diagonals known at compile time (the 7-point stencil): every value and x
// load of a row is issued before the first product, with the x index clamped
// into the matrix -- where the pattern has no entry the value is 0, so the
// product adds +-0 and the sum is the same as skipping it.
// RPT rows per thread (rows i and i + TB of a block's tile of RPT * TB rows),
// so a thread has RPT * 2 * ND loads in flight.
template <typename T, int ND, int MODE, int RPT>
__global__ void __launch_bounds__(TB) k_dia_n(int n, DiaOffsets o, const T* __restrict__ val,
                                              const T* __restrict__ x, const T* __restrict__ b,
                                              const T* __restrict__ inv, T* __restrict__ y) {
  pdl_wait_release();
  for (int base = blockIdx.x * TB * RPT; base < n; base += gridDim.x * TB * RPT) {
    T v[RPT][ND], xv[RPT][ND];
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int i = base + q * TB + threadIdx.x;
      const int ic = i < n ? i : n - 1;
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        int j = ic + o.off[d];
        j = j < 0 ? 0 : (j >= n ? n - 1 : j);
        v[q][d] = val[(long long)d * n + ic];
        xv[q][d] = x[j];
      }
    }
#pragma unroll
    for (int q = 0; q < RPT; ++q) {
      const int i = base + q * TB + threadIdx.x;
      if (i >= n) continue;
      T acc = T(0);
#pragma unroll
      for (int d = 0; d < ND; ++d) acc += v[q][d] * xv[q][d];
      if (MODE == Y_AX) y[i] = acc;
      else if (MODE == Y_B_MINUS_AX) y[i] = b[i] - acc;
      else if (MODE == Y_SMOOTH) y[i] = x[i] + T(kOmega) * inv[i] * (b[i] - acc);
      else if (MODE == Y_ADD_AX) y[i] = y[i] + acc;
      else if (MODE == Y_W_AX) y[i] = inv[i] * acc;
    }
  }
}

template <typename T> const T* dia_values(const Level& L);
template <> inline const double* dia_values<double>(const Level& L) { return L.dia_val.p; }
template <> inline const float* dia_values<float>(const Level& L) { return L.dia_valf.p; }

template <typename T, int MODE>
void launch_dia(const Level& L, const T* x, const T* b, const T* inv, T* y, cudaStream_t s) {
  DiaOffsets o{};
  for (int d = 0; d < Level::kDiaMax; ++d) o.off[d] = L.dia_off[d];
  if (L.dia_nd == 7 && L.dia_rpt == 2)
    launch_pdl(k_dia_n<T, 7, MODE, 2>, grid_for((L.n + 1) / 2, TB, 16), TB, 0, s, L.n, o, dia_values<T>(L), x, b,
               inv, y);
  else if (L.dia_nd == 7)
    launch_pdl(k_dia_n<T, 7, MODE, 1>, grid_for(L.n, TB, 16), TB, 0, s, L.n, o, dia_values<T>(L), x, b, inv, y);
  else
    launch_pdl(k_dia<T, MODE>, grid_for(L.n, TB, 16), TB, 0, s, L.n, L.dia_nd, o, dia_values<T>(L), x, b, inv, y);
  IMPES_CHECK_LAUNCH();
}

// ------------------------------------------- grid-tile sweeps (level 0)
// When a level's DIA pattern is the 7-point stencil of a grid (Level::grid_*),
// two l1-Jacobi sweeps -- and, before the coarse correction, the residual after
// them -- run in ONE launch instead of two or three.  A block owns a tile of
// kTileX x kTileY (x, y) columns with all nz cells of each (two blocks per SM).  The first sweep is
// computed on the tile and a halo of H - 1 columns into shared memory (H = 3
// with the residual, 2 without), the second on the tile and a halo of H - 2
// (shared memory when the residual follows, else straight to the output), the
// residual on the tile.  Every pass over the tile needs the previous one only
// within one column of it, so the matrix, b and the l1 weights stream from HBM
// once per launch; the halo columns read them again, mostly from L2 (1.4x the
// tile's rows with the residual, 1.2x without).  Each row is the expression of
// k_dia_n (dia_dot, then x + w inv (b - acc) or b - acc), so the results are the
// per-pass kernels' to the last bit but for the sign of a zero: a neighbour
// outside the grid, or across a line's end, enters as 0 * 0 where k_dia_n adds
// 0 * x of a clamped index.
// Opt-in (IMPES_DIA_TILE=1, read at setup): on the 1e6-cell case a launch takes
// ~24 us against ~12 us for one streaming DIA pass, so the fused pre-smoothing
// (three passes) gains what the fused post-smoothing (two passes) loses, and
// the step is no faster; the halo passes repeat ~3x the loads per tile and the
// cells of a thread are dependent rounds through L2.
constexpr int kTileX = 16, kTileY = 10, kTileThreads = 512;

struct DiaGrid {
  int nx, ny, nz;
  int tiles_y;    // tiles along y (blockIdx.x = tile_x * tiles_y + tile_y)
  int per_pass;   // columns a pass of the block covers: kTileThreads / nz
};

template <typename T, int ND>
__device__ __forceinline__ T dia_dot(const T (&v)[ND], const T (&xv)[ND]) {
  T acc = T(0);
#pragma unroll
  for (int d = 0; d < ND; ++d) acc += v[d] * xv[d];
  return acc;
}

// One pass over the columns of halo HALO around the tile (clipped to the grid):
// a sweep (RES false) or the residual (RES true) of every cell.  Neighbour
// values come from the global vector when SRC_HALO < 0, else from the shared-
// memory region of halo SRC_HALO; out_s (shared memory, region of halo HALO)
// and/or out_g (global, tile columns only) receive the result.  A thread takes
// kTileU columns per trip (its z cell of each) and issues all their loads
// before the first product, so each thread has kTileU rows' loads in flight.
constexpr int kTileU = 2;
template <typename T, int HALO, int SRC_HALO, bool RES>
__device__ __forceinline__ void tile_pass(const DiaGrid& g, int n, int X0, int Y0, const T* __restrict__ val,
                                          const T* src, const T* __restrict__ b, const T* __restrict__ inv,
                                          T* out_s, T* __restrict__ out_g) {
  constexpr int RX = kTileX + 2 * HALO, RY = kTileY + 2 * HALO;
  constexpr int SH = SRC_HALO > 0 ? SRC_HALO - HALO : 0;   // this region inside the source region
  constexpr int SRY = kTileY + 2 * (SRC_HALO > 0 ? SRC_HALO : 0);
  if (threadIdx.x >= g.per_pass * g.nz) return;   // past the last whole group of nz threads
  const int iz = threadIdx.x % g.nz;
  const int a = g.ny * g.nz;
  for (int col0 = threadIdx.x / g.nz; col0 < RX * RY; col0 += kTileU * g.per_pass) {
    T v[kTileU][7], xv[kTileU][7], bi[kTileU], wi[kTileU];
    int idx[kTileU];
    bool live[kTileU];
#pragma unroll
    for (int u = 0; u < kTileU; ++u) {
      const int col = col0 + u * g.per_pass;
      const int cx = col / RY, cy = col - cx * RY;
      const int ix = X0 - HALO + cx, iy = Y0 - HALO + cy;
      live[u] = col < RX * RY && ix >= 0 && ix < g.nx && iy >= 0 && iy < g.ny;
      const int i = live[u] ? (ix * g.ny + iy) * g.nz + iz : 0;
      idx[u] = i;
      const bool ok[7] = {live[u] && ix > 0, live[u] && iy > 0, live[u] && iz > 0, live[u],
                          live[u] && iz < g.nz - 1, live[u] && iy < g.ny - 1, live[u] && ix < g.nx - 1};
#pragma unroll
      for (int d = 0; d < 7; ++d) v[u][d] = val[(long long)d * n + i];
      bi[u] = b[i];
      wi[u] = RES ? T(0) : inv[i];
      if constexpr (SRC_HALO < 0) {
        const int off[7] = {-a, -g.nz, -1, 0, 1, g.nz, a};
#pragma unroll
        for (int d = 0; d < 7; ++d) xv[u][d] = ok[d] ? src[i + off[d]] : T(0);
      } else {
        const int c = ((cx + SH) * SRY + (cy + SH)) * g.nz + iz;
        const int off[7] = {-SRY * g.nz, -g.nz, -1, 0, 1, g.nz, SRY * g.nz};
#pragma unroll
        for (int d = 0; d < 7; ++d) xv[u][d] = ok[d] ? src[c + off[d]] : T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < kTileU; ++u) {
      if (!live[u]) continue;
      const int col = col0 + u * g.per_pass;
      const int cx = col / RY, cy = col - cx * RY;
      const T acc = dia_dot<T, 7>(v[u], xv[u]);
      T y;
      if constexpr (RES) y = bi[u] - acc;
      else y = xv[u][3] + T(kOmega) * wi[u] * (bi[u] - acc);
      if (out_s) out_s[col * g.nz + iz] = y;
      if (out_g && cx >= HALO && cx < HALO + kTileX && cy >= HALO && cy < HALO + kTileY) out_g[idx[u]] = y;
    }
  }
}

// Two sweeps from x0 into xout; with RES also r = b - A xout.  x0 must not
// alias xout (neighbouring tiles read x0 while this one writes).
template <typename T, bool RES>
__global__ void __launch_bounds__(kTileThreads, 2) k_dia_tile(DiaGrid g, const T* __restrict__ val,
                                                           const T* __restrict__ x0, const T* __restrict__ b,
                                                           const T* __restrict__ inv, T* __restrict__ xout,
                                                           T* __restrict__ r) {
  extern __shared__ __align__(16) unsigned char tile_smem[];
  pdl_wait_release();
  constexpr int H = RES ? 3 : 2;
  const int n = g.nx * g.ny * g.nz;
  const int X0 = (blockIdx.x / g.tiles_y) * kTileX, Y0 = (blockIdx.x % g.tiles_y) * kTileY;
  T* s1 = reinterpret_cast<T*>(tile_smem);
  // every thread reaches every barrier (threads past per_pass * nz only skip
  // the passes' work)
  tile_pass<T, H - 1, -1, false>(g, n, X0, Y0, val, x0, b, inv, s1, nullptr);
  __syncthreads();
  if constexpr (RES) {
    T* s2 = s1 + (kTileX + 2 * (H - 1)) * (kTileY + 2 * (H - 1)) * g.nz;
    tile_pass<T, 1, H - 1, false>(g, n, X0, Y0, val, s1, b, inv, s2, xout);
    __syncthreads();
    tile_pass<T, 0, 1, true>(g, n, X0, Y0, val, s2, b, inv, nullptr, r);
  } else {
    tile_pass<T, 0, H - 1, false>(g, n, X0, Y0, val, s1, b, inv, nullptr, xout);
  }
}

template <typename T, bool RES>
size_t dia_tile_smem(const Level& L) {
  constexpr int H = RES ? 3 : 2;
  size_t cols = (size_t)(kTileX + 2 * (H - 1)) * (kTileY + 2 * (H - 1));
  if (RES) cols += (size_t)(kTileX + 2) * (kTileY + 2);
  return cols * L.grid_nz * sizeof(T);
}
constexpr size_t kTileSmemMax = 200 * 1024;

// The level's sweeps may run on grid tiles in precision T.
template <typename T>
bool dia_tile_ok(const AMG& h, const Level& L, int slot) {
  return h.use_dia_tile && L.grid_nz > 0 && L.grid_nz <= kTileThreads && L.dia_on[slot] &&
         dia_values<T>(L) != nullptr && h.prm.smoother == IMPES_SMOOTHER_L1_JACOBI &&
         dia_tile_smem<T, true>(L) <= kTileSmemMax;
}

template <typename T, bool RES>
void launch_dia_tile(const Level& L, const T* x0, const T* b, const T* inv, T* xout, T* r, cudaStream_t s) {
  const size_t smem = dia_tile_smem<T, RES>(L);
  // raise the dynamic shared-memory limit once per instantiation (thread-safe
  // initialisation: ensemble workers launch concurrently)
  static const cudaError_t attr = cudaFuncSetAttribute((const void*)k_dia_tile<T, RES>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       (int)kTileSmemMax);
  IMPES_CUDA(attr);
  DiaGrid g{L.grid_nx, L.grid_ny, L.grid_nz, (L.grid_ny + kTileY - 1) / kTileY, kTileThreads / L.grid_nz};
  const int tiles = ((L.grid_nx + kTileX - 1) / kTileX) * g.tiles_y;
  launch_pdl(k_dia_tile<T, RES>, tiles, kTileThreads, smem, s, g, dia_values<T>(L), x0, b, inv, xout, r);
  IMPES_CHECK_LAUNCH();
}


// A product of a level's A with the layout chosen for this precision (DIA,
// SELL or the CSR kernels with the tuned lanes per row).
template <typename T, int MODE>
void launch_a(const Level& L, int slot, const T* x, const T* b, const T* inv, T* y, cudaStream_t s) {
  if (L.dia_on[slot] && dia_values<T>(L))
    launch_dia<T, MODE>(L, x, b, inv, y, s);
  else if (L.sell_on[slot] && sell_values<T>(L))
    launch_sell<T, MODE>(L, x, b, inv, y, s);
  else
    launch_csr<T, MODE>(L.n, L.avg_row, L.rowptr.p, L.col.p, (const T*)(sizeof(T) == 8 ? (const void*)L.val.p
                                                                                        : (const void*)L.valf.p),
                        x, b, inv, y, s, L.col16.p, L.col16_rel, L.lpr_a[slot]);
}

// ------------------------------------------------------ Chebyshev smoother
// The Chebyshev iteration for diag(inv) A on [lower * lmax, lmax] (Saad,
// Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 12.1), an option of
// this library (the reference smooths with l1-Jacobi): r = inv (b - A x),
// d_0 = r / theta, then per step x += d_k, r -= inv A d_k,
// d_{k+1} = rho_{k+1} rho_k d_k + (2 rho_{k+1} / delta) r, with
// rho_0 = delta / theta and rho_{k+1} = 1 / (2 theta / delta - rho_k).  The last
// product's step also adds d_{k+1} to x, so nu updates of x take nu - 1 products
// after the initial residual.  lmax is the level's Gershgorin bound, read from
// device memory (the bits of a double), so a captured graph follows updates.
struct ChebArgs {
  const unsigned long long* lmax;
  double lower;
  int k;        // index of the direction this step multiplies
  int last;     // last product: x also takes the next direction
  int zero_x;   // x starts at zero (not read)
};
__device__ __forceinline__ void cheb_coeffs(const ChebArgs& ca, double& theta, double& c1, double& c2) {
  const double lm = __longlong_as_double((long long)*ca.lmax);
  const double lo = __dmul_rn(ca.lower, lm);
  theta = __dmul_rn(0.5, __dadd_rn(lm, lo));
  const double delta = __dmul_rn(0.5, __dsub_rn(lm, lo));
  const double sigma = __ddiv_rn(theta, delta);
  double rho = __ddiv_rn(1.0, sigma);
  for (int q = 0; q < ca.k; ++q) rho = __ddiv_rn(1.0, __dsub_rn(__dmul_rn(2.0, sigma), rho));
  const double rn = __ddiv_rn(1.0, __dsub_rn(__dmul_rn(2.0, sigma), rho));
  c1 = __dmul_rn(rn, rho);
  c2 = __ddiv_rn(__dmul_rn(2.0, rn), delta);
}
enum ChebMode { CH_INIT = 0, CH_STEP = 1 };
// LPR lanes per row (1..32).  CH_INIT gathers v = x: r = inv (b - A x),
// dnext = r / theta.  CH_STEP gathers v = d_k: r -= inv A d_k, x += d_k
// (+ d_{k+1} on the last step), dnext = d_{k+1}.  CT and rel as in k_csr.
template <typename T, typename CT, int LPR, int MODE>
__global__ void __launch_bounds__(TB) k_cheb(int n, const int* __restrict__ rowptr,
                                             const CT* __restrict__ col, const T* __restrict__ val,
                                             const T* __restrict__ v, const T* __restrict__ b,
                                             const T* __restrict__ inv, T* __restrict__ r,
                                             T* __restrict__ x, T* __restrict__ dnext, int rel,
                                             ChebArgs ca) {
  pdl_wait_release();
  double theta, c1, c2;
  cheb_coeffs(ca, theta, c1, c2);
  const int g = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  const int rows_per_block = TB / LPR;
  for (long long row = (long long)blockIdx.x * rows_per_block + g; row < n;
       row += (long long)gridDim.x * rows_per_block) {
    T acc = T(0);
    const int a = rowptr[row], e = rowptr[row + 1];
    const int cb = col_base<CT>(row, rel);
    acc = row_dot(a + lane, e, LPR, val, col, v, cb, acc);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
    if (lane == 0) {
      if (MODE == CH_INIT) {
        const T ri = inv[row] * (b[row] - acc);
        r[row] = ri;
        dnext[row] = ri / T(theta);
      } else {
        const T ri = r[row] - inv[row] * acc;
        const T di = v[row];
        const T dn = T(c1) * di + T(c2) * ri;
        T xi = ca.zero_x ? T(0) : x[row];
        xi = xi + di;
        if (ca.last) xi = xi + dn;
        x[row] = xi;
        r[row] = ri;
        if (!ca.last) dnext[row] = dn;
      }
    }
  }
}
// x = 0: r = inv b, d_0 = r / theta (no product); with nu == 1, x = d_0 too
template <typename T>
__global__ void k_cheb_init0(int n, const T* __restrict__ b, const T* __restrict__ inv, T* __restrict__ r,
                             T* __restrict__ d, T* __restrict__ x, ChebArgs ca) {
  pdl_wait_release();
  double theta, c1, c2;
  cheb_coeffs(ca, theta, c1, c2);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const T ri = inv[i] * b[i];
    r[i] = ri;
    d[i] = ri / T(theta);
    if (x) x[i] = d[i];
  }
}
template <typename T>
__global__ void k_cheb_add(int n, const T* __restrict__ d, T* __restrict__ x) {
  pdl_wait_release();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = x[i] + d[i];
}

template <typename T, typename CT, int MODE>
void launch_cheb_ct(int n, int avg, const int* rowptr, const CT* col, const T* val, const T* v, const T* b,
                    const T* inv, T* r, T* x, T* dnext, int rel, const ChebArgs& ca, cudaStream_t s,
                    int lpr_tuned = 0) {
  const int lpr = (lpr_tuned > 0 && avg <= 96) ? lpr_tuned
                  : (avg <= 8 ? 1 : avg <= 16 ? 4 : avg <= 48 ? 8 : avg <= 96 ? 16 : 32);
  auto grid = [&](int l) { return grid_for(((size_t)n * l + TB - 1) / TB * TB, TB, 16); };
  switch (lpr) {
    case 1: launch_pdl(k_cheb<T, CT, 1, MODE>, grid(1), TB, 0, s, n, rowptr, col, val, v, b, inv, r, x, dnext, rel, ca); break;
    case 2: launch_pdl(k_cheb<T, CT, 2, MODE>, grid(2), TB, 0, s, n, rowptr, col, val, v, b, inv, r, x, dnext, rel, ca); break;
    case 4: launch_pdl(k_cheb<T, CT, 4, MODE>, grid(4), TB, 0, s, n, rowptr, col, val, v, b, inv, r, x, dnext, rel, ca); break;
    case 8: launch_pdl(k_cheb<T, CT, 8, MODE>, grid(8), TB, 0, s, n, rowptr, col, val, v, b, inv, r, x, dnext, rel, ca); break;
    case 16: launch_pdl(k_cheb<T, CT, 16, MODE>, grid(16), TB, 0, s, n, rowptr, col, val, v, b, inv, r, x, dnext, rel, ca); break;
    default: launch_pdl(k_cheb<T, CT, 32, MODE>, grid(32), TB, 0, s, n, rowptr, col, val, v, b, inv, r, x, dnext, rel, ca); break;
  }
  IMPES_CHECK_LAUNCH();
}

#define GRID_LOOP(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

template <typename A, typename B>
__global__ void k_convert(long long n, const A* in, B* out) {
  pdl_wait_release(); GRID_LOOP(i, n) out[i] = (B)in[i]; }
template <typename A, typename B>
__global__ void k_div_convert(long long n, const A* in, const double* w, B* out) {
  pdl_wait_release();
  GRID_LOOP(i, n) out[i] = (B)(in[i] / w[i]);
}
__global__ void k_mul(long long n, const double* a, const double* b, double* out) {
  pdl_wait_release();
  GRID_LOOP(i, n) out[i] = a[i] * b[i];
}
__global__ void k_mul_inplace(long long n, double* a, const double* b) {
  pdl_wait_release(); GRID_LOOP(i, n) a[i] *= b[i]; }
__global__ void k_zero(long long n, double* a) {
  pdl_wait_release(); GRID_LOOP(i, n) a[i] = 0.0; }

// v - sum_{q<k} h[q] * V[q*ld + i] (or v + ..., sign = -1 / +1) with the q
// terms added one after another as in the plain loop, but with the loads of up
// to eight vectors issued together so that each thread keeps several HBM
// requests in flight.
template <int SIGN>
__device__ __forceinline__ double axpy_rows(double v, const double* __restrict__ h, int k,
                                            const double* __restrict__ V, long long ld, long long i) {
  int q = 0;
  for (; q + 8 <= k; q += 8) {
    double a[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) a[u] = V[(q + u) * ld + i];
#pragma unroll
    for (int u = 0; u < 8; ++u) v = SIGN > 0 ? v + h[q + u] * a[u] : v - h[q + u] * a[u];
  }
  for (; q < k; ++q) v = SIGN > 0 ? v + h[q] * V[q * ld + i] : v - h[q] * V[q * ld + i];
  return v;
}

// ---------------------------------------------------- deterministic dots
constexpr int kDotBlocks = 592;   // 4 x 148 SMs, fixed so partials have a fixed order
constexpr int kMD = 8;            // vectors per multi-dot launch

// partial[q * kDotBlocks + block] = sum over the block of V[q] . w   (q < k)
__global__ void __launch_bounds__(TB) k_multidot(long long n, const double* __restrict__ Vbase,
                                                 long long ldv, int k, const double* __restrict__ w,
                                                 double* __restrict__ partial) {
  pdl_wait_release();
  __shared__ double s[kMD][TB / 32];
  double acc[kMD];
#pragma unroll
  for (int q = 0; q < kMD; ++q) acc[q] = 0.0;
  GRID_LOOP(i, n) {
    const double wi = w[i];
#pragma unroll
    for (int q = 0; q < kMD; ++q)
      if (q < k) acc[q] += Vbase[q * ldv + i] * wi;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kMD; ++q) {
    double v = warp_sum(acc[q]);
    if (lane == 0) s[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kMD && threadIdx.x < k) {
    double t = 0.0;
    for (int u = 0; u < TB / 32; ++u) t += s[threadIdx.x][u];
    partial[threadIdx.x * kDotBlocks + blockIdx.x] = t;
  }
}
// Gram-Schmidt dot accumulation over this thread's elements (grid stride),
// two elements per trip so that each thread has the loads of 2 x 8 vectors in
// flight; every accumulator adds its elements in index order, as a one-element
// loop would.
__device__ __forceinline__ void multidot_acc(double* acc, long long n, const double* __restrict__ V,
                                             long long ldv, int q0, int k, int self,
                                             const double* __restrict__ w) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i + stride < n; i += 2 * stride) {
    const double w0 = w[i], w1 = w[i + stride];
    double a0[kMD], a1[kMD];
#pragma unroll
    for (int u = 0; u < kMD; ++u) {
      const int q = q0 + u;
      a0[u] = q < k ? V[q * ldv + i] : w0;
      a1[u] = q < k ? V[q * ldv + i + stride] : w1;
    }
#pragma unroll
    for (int u = 0; u < kMD; ++u) {
      const int q = q0 + u;
      if (q < k || (q == k && self)) {
        acc[u] += a0[u] * w0;
        acc[u] += a1[u] * w1;
      }
    }
  }
  for (; i < n; i += stride) {
    const double wi = w[i];
#pragma unroll
    for (int u = 0; u < kMD; ++u) {
      const int q = q0 + u;
      if (q < k) acc[u] += V[q * ldv + i] * wi;
      else if (q == k && self) acc[u] += wi * wi;
    }
  }
}
// w -= sum_q h[q] V[q] over this thread's elements, two per trip; returns the
// partial sum of squares of the new w in index order.
__device__ __forceinline__ double update_rows(long long n, const double* __restrict__ V, long long ldv,
                                              const double* __restrict__ h, int k, double* __restrict__ w) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double acc = 0.0;
  for (; i + stride < n; i += 2 * stride) {
    const double v0 = axpy_rows<-1>(w[i], h, k, V, ldv, i);
    const double v1 = axpy_rows<-1>(w[i + stride], h, k, V, ldv, i + stride);
    w[i] = v0;
    w[i + stride] = v1;
    acc += v0 * v0;
    acc += v1 * v1;
  }
  for (; i < n; i += stride) {
    const double v = axpy_rows<-1>(w[i], h, k, V, ldv, i);
    w[i] = v;
    acc += v * v;
  }
  return acc;
}

// Gram-Schmidt dots of FGMRES in one launch: block (x, g) sums, over its slice
// of rows, V[q] . w for the 8 vectors q = 8g .. 8g+7 below k, and w . w as
// vector q = k when self is set; partial[q * kDotBlocks + x].  With pred set
// the launch does nothing unless *pred is non-zero (the optional second
// Gram-Schmidt pass, decided on the device).
__global__ void __launch_bounds__(TB, 4) k_multidot_g(long long n, const double* __restrict__ Vbase,
                                                   long long ldv, int k, int self,
                                                   const double* __restrict__ w,
                                                   double* __restrict__ partial, const int* pred) {
  pdl_wait_release();
  if (pred && *pred == 0) return;
  __shared__ double s[kMD][TB / 32];
  const int q0 = blockIdx.y * kMD;
  const int kk = k + (self ? 1 : 0);
  double acc[kMD];
#pragma unroll
  for (int u = 0; u < kMD; ++u) acc[u] = 0.0;
  multidot_acc(acc, n, Vbase, ldv, q0, k, self, w);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int u = 0; u < kMD; ++u) {
    double v = warp_sum(acc[u]);
    if (lane == 0) s[u][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kMD && q0 + (int)threadIdx.x < kk) {
    double t = 0.0;
    for (int u = 0; u < TB / 32; ++u) t += s[threadIdx.x][u];
    partial[(q0 + threadIdx.x) * kDotBlocks + blockIdx.x] = t;
  }
}
// Second Gram-Schmidt pass wanted when the first pass left less than 0.7 of the
// vector's norm ("twice is enough", Giraud, Langou & Rozloznik 2005):
// flag = ||w'||^2 < 0.49 ||w||^2.
__global__ void k_reorth_flag(const double* nrm2_after, const double* nrm2_before, int* flag) {
  pdl_wait_release();
  *flag = (*nrm2_after < 0.49 * *nrm2_before) ? 1 : 0;
}
// out[q] (+)= sum of partials, fixed order
__global__ void k_dot_finalize(int k, const double* partial, double* out, int accumulate,
                               const int* pred = nullptr) {
  pdl_wait_release();
  if (pred && *pred == 0) return;
  const int q = blockIdx.x;
  double t = 0.0;
  for (int b = threadIdx.x; b < kDotBlocks; b += 32) t += partial[q * kDotBlocks + b];
  t = warp_sum(t);
  if (threadIdx.x == 0) out[q] = accumulate ? out[q] + t : t;
  (void)k;
}
// w -= sum_q h[q] V[q]; optionally partial norms of the result
__global__ void __launch_bounds__(TB) k_update(long long n, const double* __restrict__ Vbase,
                                               long long ldv, int k, const double* __restrict__ h,
                                               double* __restrict__ w, double* __restrict__ partial,
                                               const int* pred = nullptr) {
  pdl_wait_release();
  if (pred && *pred == 0) return;
  __shared__ double sh[128];
  __shared__ double s[TB / 32];
  for (int q = threadIdx.x; q < k; q += blockDim.x) sh[q] = h[q];
  __syncthreads();
  const double acc = update_rows(n, Vbase, ldv, sh, k, w);
  if (partial) {
    double t = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double u = 0.0;
      for (int q = 0; q < TB / 32; ++q) u += s[q];
      partial[blockIdx.x] = u;
    }
  }
}
__global__ void k_scale_by_inv_sqrt(long long n, const double* in, double* out, const double* nrm2) {
  pdl_wait_release();
  const double inv = 1.0 / sqrt(*nrm2);
  GRID_LOOP(i, n) out[i] = in[i] * inv;
}

// --------------------------------------------------- coarsest dense solve
// Dense copy of the coarsest matrix with DOF 0 pinned (classical_amg.py:1045-1055).
__global__ void k_dense_pinned(int n, const int* rowptr, const int* col, const double* val, double* M) {
  GRID_LOOP(t, (long long)n * n) M[t] = 0.0;
}
template <typename TV>
__global__ void k_dense_fill(int n, const int* rowptr, const int* col, const TV* val, double* M,
                             int pin) {
  GRID_LOOP(i, n) {
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      int j = col[e];
      if (pin && (i == 0 || j == 0)) continue;
      M[(long long)i * n + j] = val[e];
    }
    if (pin && i == 0) M[0] = 1.0;
  }
}
// In-place Gauss-Jordan inversion with partial pivoting: block b inverts M[b]
// (the pinned and the unpinned coarsest matrix in one launch).  With SMEM the
// n x n matrix lives in shared memory for the whole elimination (n <= 168 in
// 227 KB); otherwise it stays in global memory.  Pivot ties go to the lower row.
constexpr int kGJ = 1024;
struct GJArgs {
  double* M[2];
  int* perm[2];
  int* singular[2];
};
template <bool SMEM, int NT = kGJ>
__global__ void __launch_bounds__(NT) k_gauss_jordan(int n, GJArgs args) {
  __shared__ double s_val[NT / 32];
  __shared__ int s_idx[NT / 32];
  __shared__ int s_p;
  __shared__ double s_inv;
  __shared__ int s_perm[512];        // row interchanges (n <= 500), kept on chip
  extern __shared__ double s_dyn[];
  double* s_row = s_dyn;             // n (pivot row)
  double* s_col = s_row + n;         // n (pivot column)
  double* G = args.M[blockIdx.x];
  int* perm = args.perm[blockIdx.x];
  double* M = SMEM ? s_col + n : G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (SMEM) {
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) M[t] = G[t];
    __syncthreads();
  }
  for (int k = 0; k < n; ++k) {
    double best = -1.0;
    int bi = k;
    for (int i = k + threadIdx.x; i < n; i += blockDim.x) {
      const double v = fabs(M[i * n + k]);
      if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    if (lane == 0) { s_val[warp] = best; s_idx[warp] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double bv = -1.0;
      int b = k;
      for (int w = 0; w < nw; ++w)
        if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < b)) { bv = s_val[w]; b = s_idx[w]; }
      s_p = b;
      s_perm[k] = b;
      if (!(bv > 0.0)) *args.singular[blockIdx.x] = 1;
      const double piv = M[b * n + k];
      s_inv = piv != 0.0 ? 1.0 / piv : 0.0;
    }
    __syncthreads();
    const int p = s_p;
    const double inv = s_inv;
    // swap rows k and p, scale the pivot row, keep it and the pivot column
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      const double rk = M[k * n + j], rp = M[p * n + j];
      if (p != k) M[p * n + j] = rk;
      const double v = (j == k) ? inv : rp * inv;
      M[k * n + j] = v;
      s_row[j] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_col[i] = M[i * n + k];
    __syncthreads();
    for (int i = warp; i < n; i += nw) {
      if (i == k) continue;
      const double f = s_col[i];
      for (int j = lane; j < n; j += 32) {
        if (j == k) M[i * n + j] = -f * s_row[k];
        else M[i * n + j] -= f * s_row[j];
      }
    }
    __syncthreads();
  }
  // undo the row interchanges as column interchanges, last first
  for (int k = threadIdx.x; k < n; k += blockDim.x) perm[k] = s_perm[k];
  for (int k = n - 1; k >= 0; --k) {
    const int p = s_perm[k];
    if (p != k)
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = M[i * n + k];
        M[i * n + k] = M[i * n + p];
        M[i * n + p] = a;
      }
    __syncthreads();
  }
  if (SMEM)
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) G[t] = M[t];
}
// k_gauss_jordan for n <= kGJPingPong with one block barrier per pivot step:
// every warp finds the pivot itself (column k of the previous matrix, same rule:
// largest |value|, ties to the lower row) and step k writes a second copy of
// the matrix from the first (rows k and p swapped, the pivot row scaled, the
// others updated), so no row is read after it is rewritten.  Each element gets
// the same operations in the same order as in k_gauss_jordan.
constexpr int kGJPingPong = 64;
__global__ void __launch_bounds__(256) k_gauss_jordan_pp(int n, GJArgs args) {
  extern __shared__ double s_dyn[];
  __shared__ int s_perm[kGJPingPong];
  double* A = s_dyn;                 // n x n, even steps read here
  double* B = A + (size_t)n * n;     // n x n, odd steps read here
  double* G = args.M[blockIdx.x];
  int* perm = args.perm[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) A[t] = G[t];
  __syncthreads();
  bool singular = false;
  for (int k = 0; k < n; ++k) {
    const double* M = (k & 1) ? B : A;
    double* W = (k & 1) ? A : B;
    double best = -1.0;
    int bi = k;
    for (int i = k + lane; i < n; i += 32) {
      const double v = fabs(M[i * n + k]);
      if (v > best) { best = v; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, best, o);
      const int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
    }
    const int p = __shfl_sync(0xffffffffu, bi, 0);
    best = __shfl_sync(0xffffffffu, best, 0);
    if (!(best > 0.0)) singular = true;
    if (threadIdx.x == 0) s_perm[k] = p;
    const double piv = M[p * n + k];
    const double inv = piv != 0.0 ? 1.0 / piv : 0.0;
    for (int i = warp; i < n; i += nw) {
      // row i of the swapped matrix: old row p at k, old row k at p
      const int src = (i == k) ? p : (i == p ? k : i);
      if (i == k) {
        for (int j = lane; j < n; j += 32) W[k * n + j] = (j == k) ? inv : M[p * n + j] * inv;
      } else {
        const double f = M[src * n + k];
        for (int j = lane; j < n; j += 32) {
          const double sr = (j == k) ? inv : M[p * n + j] * inv;
          W[i * n + j] = (j == k) ? -f * sr : M[src * n + j] - f * sr;
        }
      }
    }
    __syncthreads();
  }
  if (singular && threadIdx.x == 0) *args.singular[blockIdx.x] = 1;
  double* M = (n & 1) ? B : A;       // the last step wrote here
  for (int k = threadIdx.x; k < n; k += blockDim.x) perm[k] = s_perm[k];
  for (int k = n - 1; k >= 0; --k) {
    const int p = s_perm[k];
    if (p != k)
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = M[i * n + k];
        M[i * n + k] = M[i * n + p];
        M[i * n + p] = a;
      }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) G[t] = M[t];
}
// x = Ainv * b with b[0] pinned to 0 (the reference's coarsest solve), or, in
// Krylov mode while the unpinned matrix was invertible, x = Afree^-1 * b.
template <typename T>
__global__ void k_coarse_apply(int n, const double* __restrict__ Apin, const double* __restrict__ Afree,
                               const int* __restrict__ free_singular, int krylov,
                               const T* __restrict__ b, T* __restrict__ x) {
  pdl_wait_release();
  extern __shared__ double s_b[];
  const bool use_free = krylov && Afree != nullptr && *free_singular == 0;
  const double* Ainv = use_free ? Afree : Apin;
  const int pin = use_free ? 0 : 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_b[i] = (pin && i == 0) ? 0.0 : (double)b[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int i = blockIdx.x * nw + warp; i < n; i += gridDim.x * nw) {
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc += Ainv[(long long)i * n + j] * s_b[j];
    acc = warp_sum(acc);
    if (lane == 0) x[i] = (T)acc;
  }
}
template <typename T>
__global__ void k_pin_copy(int n, const T* b, T* out) {
  pdl_wait_release(); GRID_LOOP(i, n) out[i] = (i == 0) ? T(0) : b[i]; }

}  // namespace

bool amg_level_tiled(const AMG& h, int l, int slot) {
  const Level& L = *h.levels[l];
  if (L.coarsest || L.n <= h.prm.light_sweep_rows) return false;
  return slot == 0 ? dia_tile_ok<double>(h, L, 0) : dia_tile_ok<float>(h, L, 1);
}

// =================================================================== host
void coarse_factor(AMG& h, Level& L, cudaStream_t s, bool from_fp32) {
  if (L.n > 500 || L.n == 0) return;
  const int n = L.n;
  // the reference's pinned matrix (row/column 0 replaced by e_0) and the
  // unpinned one used inside FGMRES (the pinned solve would freeze x[0] there)
  L.lu.ensure((size_t)n * n);
  L.lu_free.ensure((size_t)n * n);
  L.piv.ensure(2 * (size_t)n);
  double* mats[2] = {L.lu.p, L.lu_free.p};
  for (int q = 0; q < 2; ++q) {
    k_dense_pinned<<<grid_for((size_t)n * n, TB), TB, 0, s>>>(n, L.rowptr.p, L.col.p, L.val.p, mats[q]); ::impes::count_launch();
    if (from_fp32) {
      k_dense_fill<float><<<grid_for(n, TB), TB, 0, s>>>(n, L.rowptr.p, L.col.p, L.valf.p, mats[q], q == 0 ? 1 : 0); ::impes::count_launch();
    } else {
      k_dense_fill<double><<<grid_for(n, TB), TB, 0, s>>>(n, L.rowptr.p, L.col.p, L.val.p, mats[q], q == 0 ? 1 : 0); ::impes::count_launch();
    }
  }
  IMPES_CHECK_LAUNCH();
  IMPES_CUDA(cudaMemsetAsync(h.iflag.p + 2, 0, 2 * sizeof(int), s));
  GJArgs args{{L.lu.p, L.lu_free.p}, {L.piv.p, L.piv.p + n}, {h.iflag.p + 2, h.iflag.p + 3}};
  const size_t smem_full = sizeof(double) * ((size_t)n * n + 2 * (size_t)n);
  if (n <= kGJPingPong) {
    const size_t smem_pp = sizeof(double) * 2 * (size_t)n * n;
    raise_smem_limit((const void*)k_gauss_jordan_pp, smem_pp);
    k_gauss_jordan_pp<<<2, 256, smem_pp, s>>>(n, args); ::impes::count_launch();
  } else if (n <= 128) {
    // small coarsest matrices: 8 warps keep each of the n pivot steps' block
    // barriers short (the elimination has at most 128 rows to share out)
    raise_smem_limit((const void*)k_gauss_jordan<true, 256>, smem_full);
    k_gauss_jordan<true, 256><<<2, 256, smem_full, s>>>(n, args); ::impes::count_launch();
  } else if (smem_full <= (size_t)(224u << 10)) {
    raise_smem_limit((const void*)k_gauss_jordan<true>, smem_full);
    k_gauss_jordan<true><<<2, kGJ, smem_full, s>>>(n, args); ::impes::count_launch();
  } else {
    k_gauss_jordan<false><<<2, kGJ, 2 * n * sizeof(double), s>>>(n, args); ::impes::count_launch();
  }
  IMPES_CHECK_LAUNCH();
}

void spmv(const Level& L, const double* x, double* y, cudaStream_t s) {
  launch_csr<double, Y_AX>(L.n, L.avg_row, L.rowptr.p, L.col.p, L.val.p, x, nullptr, nullptr, y, s);
}

double dot_host(AMG& h, const double* a, const double* b, int n, cudaStream_t s) {
  h.red.ensure((size_t)kMD * kDotBlocks);
  launch_pdl(k_multidot, kDotBlocks, TB, 0, s, n, a, 0, 1, b, h.red.p);
  launch_pdl(k_dot_finalize, 1, 32, 0, s, 1, (const double*)h.red.p, h.scal.p, 0, (const int*)nullptr);
  IMPES_CHECK_LAUNCH();
  IMPES_CUDA(cudaMemcpyAsync(h.hbuf.p, h.scal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  timers().harvest();
  return h.hbuf.p[0];
}

namespace {

template <typename T> struct LV;
template <> struct LV<double> {
  static constexpr int slot = 0;
  static double* u(Level& L) { return L.u.p; }
  static const double* val(const Level& L) { return L.val.p; }
  static const double* inv(const Level& L) { return L.inv_relax.p; }
  static const double* pval(const Level& L) { return L.pval.p; }
  static const double* rval(const Level& L) { return L.rval.p; }
  static double* x(Level& L) { return L.x.p; }
  static double* b(Level& L) { return L.b.p; }
  static double* r(Level& L) { return L.r.p; }
  static double* t(Level& L) { return L.t.p; }
};
template <> struct LV<float> {
  static constexpr int slot = 1;
  static float* u(Level& L) { return L.uf.p; }
  static const float* val(const Level& L) { return L.valf.p; }
  static const float* inv(const Level& L) { return L.inv_relaxf.p; }
  static const float* pval(const Level& L) { return L.pvalf.p; }
  static const float* rval(const Level& L) { return L.rvalf.p; }
  static float* x(Level& L) { return L.xf.p; }
  static float* b(Level& L) { return L.bf.p; }
  static float* r(Level& L) { return L.rf.p; }
  static float* t(Level& L) { return L.tf.p; }
};

// Algorithmic bytes of CSR products (value size sv, vector size sx).
inline double spmv_bytes(double sv, double sx, double nnz, double rows, double cols, double si = 4.0) {
  return (sv + si) * nnz + 4.0 * (rows + 1) + sx * cols + sx * rows;
}
// l1-Jacobi sweep: values, column indices (si bytes each), row pointers, x, b, inv, y.
inline double sweep_bytes(double s, double nnz, double n, double si = 4.0) {
  return (s + si) * nnz + 4.0 * n + 4.0 * s * n;
}
// Bytes one sweep of level L moves in the layout it runs in: the CSR formula
// above; a DIA copy's diagonals (zeros included) and x, b, inv, y; a SELL
// copy's padded values and columns, its row permutation and slice pointers.
template <typename T>
double layout_sweep_bytes(const Level& L, int slot) {
  const double s = sizeof(T), n = L.n;
  if (L.dia_on[slot]) return s * (double)L.dia_nd * n + 4.0 * s * n;
  if (L.sell_on[slot])
    return (s + (L.sell_col16.p ? 2.0 : 4.0)) * (double)L.sell_len + 4.0 * n + 4.0 * (L.sell_slices + 1.0) +
           4.0 * s * n;
  return sweep_bytes(s, L.nnz, n, L.col16.p ? 2.0 : 4.0);
}

// Algorithmic bytes of one Chebyshev step: values, columns, row pointers, the
// gathered direction, r and x read and written, inv, the next direction.
inline double cheb_bytes(double s, double nnz, double n, double si) {
  return (s + si) * nnz + 4.0 * n + 7.0 * s * n;
}

// nu Chebyshev updates of x (see ChebArgs); x stays in its buffer (LV<T>::x),
// r, t and u hold the scaled residual and the two directions.
template <typename T>
T* smooth_cheb(const AMG& h, Level& L, T* x, const T* b, int nu, bool zero_x, cudaStream_t s, bool top) {
  T* r = LV<T>::r(L);
  T* dc = LV<T>::t(L);
  T* dn = LV<T>::u(L);
  ChebArgs ca{L.cheb_lmax.p + LV<T>::slot, h.prm.cheb_lower, 0, 0, 0};
  const double si = L.col16.p ? 2.0 : 4.0;
  const bool wide = L.avg_row > 96;
  if (zero_x) {
    launch_pdl(k_cheb_init0<T>, grid_for(L.n, TB), TB, 0, s, L.n, b, LV<T>::inv(L), r, dc, nu == 1 ? x : nullptr, ca);
    IMPES_CHECK_LAUNCH();
  } else {
    const int tid = top ? timers().begin(IMPES_PH_SMOOTH_L0, s) : (wide ? timers().begin(IMPES_PH_SMOOTH_WIDE, s) : -1);
    if (L.col16.p)
      launch_cheb_ct<T, unsigned short, CH_INIT>(L.n, L.avg_row, L.rowptr.p, L.col16.p, LV<T>::val(L), x, b,
                                                 LV<T>::inv(L), r, x, dc, L.col16_rel, ca, s, L.lpr_a[LV<T>::slot]);
    else
      launch_cheb_ct<T, int, CH_INIT>(L.n, L.avg_row, L.rowptr.p, L.col.p, LV<T>::val(L), x, b, LV<T>::inv(L),
                                      r, x, dc, 0, ca, s, L.lpr_a[LV<T>::slot]);
    timers().end(tid, s, sweep_bytes(sizeof(T), L.nnz, L.n, si));
    if (nu == 1) {
      launch_pdl(k_cheb_add<T>, grid_for(L.n, TB), TB, 0, s, L.n, dc, x);
      IMPES_CHECK_LAUNCH();
    }
  }
  for (int k = 0; k + 1 < nu; ++k) {
    ca.k = k;
    ca.last = (k + 2 == nu);
    ca.zero_x = (zero_x && k == 0);
    const int tid = top ? timers().begin(IMPES_PH_SMOOTH_L0, s) : (wide ? timers().begin(IMPES_PH_SMOOTH_WIDE, s) : -1);
    if (L.col16.p)
      launch_cheb_ct<T, unsigned short, CH_STEP>(L.n, L.avg_row, L.rowptr.p, L.col16.p, LV<T>::val(L), dc,
                                                 nullptr, LV<T>::inv(L), r, x, dn, L.col16_rel, ca, s,
                                                 L.lpr_a[LV<T>::slot]);
    else
      launch_cheb_ct<T, int, CH_STEP>(L.n, L.avg_row, L.rowptr.p, L.col.p, LV<T>::val(L), dc, nullptr,
                                      LV<T>::inv(L), r, x, dn, 0, ca, s, L.lpr_a[LV<T>::slot]);
    timers().end(tid, s, cheb_bytes(sizeof(T), L.nnz, L.n, si));
    std::swap(dc, dn);
  }
  return x;
}

// nu l1-Jacobi sweeps (classical_amg.py:1016-1035), or nu Chebyshev updates
// when the hierarchy selects that smoother (jacobi_only: the coarsest level's
// 50 sweeps stay l1-Jacobi); returns the buffer holding x.  Level-0 sweeps with
// a non-zero iterate are timed as IMPES_PH_SMOOTH_L0.
template <typename T>
T* smooth(const AMG& h, Level& L, T* x, T* spare, const T* b, int nu, bool zero_x, cudaStream_t s,
          bool top = false, bool jacobi_only = false) {
  if (!jacobi_only && h.prm.smoother == IMPES_SMOOTHER_CHEBYSHEV && L.cheb_lmax.p && x == LV<T>::x(L))
    return smooth_cheb<T>(h, L, x, b, nu, zero_x, s, top);
  for (int it = 0; it < nu; ++it) {
    if (zero_x && it == 0) {
      launch_csr<T, Y_SMOOTH0>(L.n, L.avg_row, L.rowptr.p, L.col.p, LV<T>::val(L), nullptr, b,
                               LV<T>::inv(L), x, s);
      continue;
    }
    const bool wide = L.avg_row > 96;   // the warp-per-row instance of k_csr
    const int tid = top ? timers().begin(IMPES_PH_SMOOTH_L0, s)
                        : (wide ? timers().begin(IMPES_PH_SMOOTH_WIDE, s) : -1);
    launch_a<T, Y_SMOOTH>(L, LV<T>::slot, x, b, LV<T>::inv(L), spare, s);
    timers().end(tid, s, layout_sweep_bytes<T>(L, LV<T>::slot));
    std::swap(x, spare);
  }
  return x;
}

// Algorithmic bytes of one V-cycle from level l down, started from zero (5
// sweeps, residual, restriction, prolongation, vector updates; dense coarsest
// apply).
template <typename T>
double vcycle_bytes(const AMG& h, int l) {
  const double sz = sizeof(T);
  double tot = 0.0;
  for (size_t q = l; q < h.levels.size(); ++q) {
    const Level& L = *h.levels[q];
    if (L.coarsest) {
      tot += L.n <= 500 ? 8.0 * L.n * (double)L.n + 2.0 * sz * L.n : 50.0 * sweep_bytes(sz, L.nnz, L.n);
      break;
    }
    // first sweep from zero (b, inv, y), four full sweeps (one on a light
    // level), the residual
    const double si = L.col16.p ? 2.0 : 4.0;
    const double full = L.n <= h.prm.light_sweep_rows ? 1.0 : 4.0;
    tot += 3.0 * sz * L.n + full * sweep_bytes(sz, L.nnz, L.n, si) + spmv_bytes(sz, sz, L.nnz, L.n, L.n, si) +
           spmv_bytes(sz, sz, L.pnnz, L.nc, L.n) + spmv_bytes(sz, sz, L.pnnz, L.n, L.nc) + 2.0 * sz * L.n;
  }
  return tot;
}

// ------------------------------------------------- fused V-cycle tail
// The levels of at most kTailRows rows (and the dense coarsest solve) cost a
// few microseconds per kernel whatever their size: each does 8 launches per
// V-cycle.  k_vcycle_tail runs the whole V-cycle of those levels in ONE launch
// of a thread-block cluster, with a hardware cluster barrier (barrier.cluster
// arrive.release / wait.acquire) between the phases: the same sequence as
// vcycle() -- first sweep from zero, two sweeps, residual, restriction, the
// next level, prolongation, two sweeps; the dense coarsest apply -- with
// kTailLanes lanes per row.  Vectors that change between phases are read past
// L1 (ld.global.cg).  Chebyshev hierarchies keep the per-level kernels.
//
// Opt-in (IMPES_TAIL=1): on the 1e6-cell hierarchy one phase of the cluster
// kernel costs ~2.5 us per pass over its rows, no less than a programmatic-
// dependent launch of the per-level kernel on all 148 SMs, and a 16-CTA cluster
// needs several passes per phase on levels of more than a few thousand rows
// (fusing the levels of <= 24,576 rows made the step 15.4 ms against 11.7).
constexpr int kTailRows = 4096;
constexpr int kTailLanes = 4;
constexpr int kTailThreads = 1024;
constexpr int kTailMaxLevels = 16;

template <typename T>
struct TailLevel {
  int n, nc, coarsest, rel;
  const int* rowptr;
  const unsigned short* col16;   // or null: col
  const int* col;
  const T* val;
  const T* inv;
  const int *prow, *pcol, *rrow, *rcol;
  const T *pval, *rval;
  T *x, *t, *b, *r;
  const double *lu, *lu_free;    // coarsest: pinned / unpinned inverses
};
template <typename T>
struct TailArgs {
  TailLevel<T> lv[kTailMaxLevels];
  int nlev;
  const int* free_singular;
  int krylov;
};

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
  return r;
}
template <typename T> __device__ __forceinline__ T ldcg(const T* p) { return __ldcg(p); }

// y = f(A x) over the rows of one CSR block (kTailLanes lanes per row)
// Rows are dealt out a warp (32 / kTailLanes rows) at a time, so every lane of
// a warp runs the same number of loop trips and takes part in each shuffle.
template <typename T, int MODE>
__device__ void tail_csr(int n, const int* __restrict__ rowptr, const unsigned short* __restrict__ col16,
                         const int* __restrict__ col, int rel, const T* __restrict__ val, const T* x, const T* b,
                         const T* __restrict__ inv, T* y, unsigned gtid, unsigned gthreads) {
  const int lane = gtid % kTailLanes;
  constexpr int kRowsPerWarp = 32 / kTailLanes;
  const long long warp = gtid >> 5, nwarps = gthreads >> 5;
  for (long long base = warp * kRowsPerWarp; base < n; base += nwarps * kRowsPerWarp) {
    const long long row = base + (int)((gtid & 31) / kTailLanes);
    const bool valid = row < n;
    T acc = T(0);
    if (MODE != Y_SMOOTH0 && valid) {
      const int a = rowptr[row], e = rowptr[row + 1];
      if (col16) {
        const int cb = rel ? (int)row - 32768 : 0;
        for (int k = a + lane; k < e; k += kTailLanes) acc += val[k] * ldcg(x + cb + (int)col16[k]);
      } else {
        for (int k = a + lane; k < e; k += kTailLanes) acc += val[k] * ldcg(x + col[k]);
      }
    }
#pragma unroll
    for (int o = kTailLanes / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, kTailLanes);
    if (lane == 0 && valid) {
      if (MODE == Y_AX) y[row] = acc;
      else if (MODE == Y_B_MINUS_AX) y[row] = ldcg(b + row) - acc;
      else if (MODE == Y_SMOOTH) y[row] = ldcg(x + row) + T(kOmega) * inv[row] * (ldcg(b + row) - acc);
      else if (MODE == Y_ADD_AX) y[row] = ldcg(y + row) + acc;
      else if (MODE == Y_SMOOTH0) y[row] = T(kOmega) * inv[row] * ldcg(b + row);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads) k_vcycle_tail(const __grid_constant__ TailArgs<T> A) {
  pdl_wait_release();
  const unsigned gthreads = cluster_size() * blockDim.x;
  const unsigned gtid = cluster_rank() * blockDim.x + threadIdx.x;
  // down: pre-smoothing, residual, restriction
  int l = 0;
  for (; l < A.nlev && !A.lv[l].coarsest; ++l) {
    const TailLevel<T>& L = A.lv[l];
    tail_csr<T, Y_SMOOTH0>(L.n, L.rowptr, L.col16, L.col, L.rel, L.val, nullptr, L.b, L.inv, L.x, gtid, gthreads);
    cluster_barrier();
    tail_csr<T, Y_SMOOTH>(L.n, L.rowptr, L.col16, L.col, L.rel, L.val, L.x, L.b, L.inv, L.t, gtid, gthreads);
    cluster_barrier();
    tail_csr<T, Y_SMOOTH>(L.n, L.rowptr, L.col16, L.col, L.rel, L.val, L.t, L.b, L.inv, L.x, gtid, gthreads);
    cluster_barrier();
    tail_csr<T, Y_B_MINUS_AX>(L.n, L.rowptr, L.col16, L.col, L.rel, L.val, L.x, L.b, nullptr, L.r, gtid,
                              gthreads);
    cluster_barrier();
    const TailLevel<T>& N = A.lv[l + 1];
    tail_csr<T, Y_AX>(L.nc, L.rrow, nullptr, L.rcol, 0, L.rval, L.r, nullptr, nullptr, N.b, gtid, gthreads);
    cluster_barrier();
  }
  // coarsest: x = Ainv b, pinned (b[0] = 0) unless Krylov mode uses the
  // invertible unpinned matrix (k_coarse_apply)
  {
    const TailLevel<T>& C = A.lv[l];
    const bool use_free = A.krylov && C.lu_free != nullptr && ldcg(A.free_singular) == 0;
    const double* Ainv = use_free ? C.lu_free : C.lu;
    const int pin = use_free ? 0 : 1;
    const int warp = gtid >> 5, lane = gtid & 31, nw = gthreads >> 5;
    for (int i = warp; i < C.n; i += nw) {
      double acc = 0.0;
      for (int j = lane; j < C.n; j += 32)
        acc += Ainv[(long long)i * C.n + j] * ((pin && j == 0) ? 0.0 : (double)ldcg(C.b + j));
      acc = warp_sum(acc);
      if (lane == 0) C.x[i] = (T)acc;
    }
    cluster_barrier();
  }
  // up: prolongation and post-smoothing
  for (--l; l >= 0; --l) {
    const TailLevel<T>& L = A.lv[l];
    const TailLevel<T>& N = A.lv[l + 1];
    tail_csr<T, Y_ADD_AX>(L.n, L.prow, nullptr, L.pcol, 0, L.pval, N.x, nullptr, nullptr, L.x, gtid, gthreads);
    cluster_barrier();
    tail_csr<T, Y_SMOOTH>(L.n, L.rowptr, L.col16, L.col, L.rel, L.val, L.x, L.b, L.inv, L.t, gtid, gthreads);
    cluster_barrier();
    tail_csr<T, Y_SMOOTH>(L.n, L.rowptr, L.col16, L.col, L.rel, L.val, L.t, L.b, L.inv, L.x, gtid, gthreads);
    cluster_barrier();
  }
}

// Whether levels l.. qualify for the fused tail: at most kTailRows rows each,
// rows of at most 96 entries, at most kTailMaxLevels levels, a dense coarsest
// level (n <= 500) and the l1-Jacobi smoother.
bool tail_eligible(const AMG& h, int l) {
  if (h.prm.smoother != IMPES_SMOOTHER_L1_JACOBI || !h.use_tail || h.prm.light_sweep_rows > 0) return false;
  if ((int)h.levels.size() - l > kTailMaxLevels) return false;
  for (size_t q = l; q < h.levels.size(); ++q) {
    const Level& L = *h.levels[q];
    if (L.n > kTailRows) return false;
    if (L.coarsest) return L.n <= 500 && L.lu.p != nullptr;
    if (L.avg_row > 96) return false;
  }
  return false;
}

template <typename T>
void launch_tail(AMG& h, int l, cudaStream_t s) {
  TailArgs<T> A{};
  A.nlev = (int)h.levels.size() - l;
  A.free_singular = h.iflag.p + 3;
  A.krylov = h.krylov_mode ? 1 : 0;
  for (int q = 0; q < A.nlev; ++q) {
    Level& L = *h.levels[l + q];
    TailLevel<T>& d = A.lv[q];
    d.n = L.n; d.nc = L.nc; d.coarsest = L.coarsest ? 1 : 0; d.rel = L.col16_rel;
    d.rowptr = L.rowptr.p; d.col16 = L.col16.p; d.col = L.col.p;
    d.val = LV<T>::val(L); d.inv = LV<T>::inv(L);
    d.prow = L.prow.p; d.pcol = L.pcol.p; d.rrow = L.rrow.p; d.rcol = L.rcol.p;
    d.pval = LV<T>::pval(L); d.rval = LV<T>::rval(L);
    d.x = LV<T>::x(L); d.t = LV<T>::t(L); d.b = LV<T>::b(L); d.r = LV<T>::r(L);
    d.lu = L.lu.p; d.lu_free = L.lu_free.p;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(h.tail_cluster);
  cfg.blockDim = dim3(kTailThreads);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cfg.gridDim.x;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  IMPES_CUDA(cudaLaunchKernelEx(&cfg, k_vcycle_tail<T>, A));
  count_launch();
}

// ------------------------------------------------ shared-memory V-cycle tail
// The fp32 V-cycle of the smallest levels (those that fit together in one
// CTA's shared memory with the dense coarsest inverse read from L2) in ONE
// launch of one 1024-thread CTA: each level's matrix, transfer operators and
// work vectors are staged into shared memory, then the same phase sequence as
// vcycle() runs with block barriers in between -- first sweep from zero, two
// sweeps, residual, restriction, the next level, prolongation, two sweeps; the
// dense coarsest apply.  A phase then costs a shared-memory pass instead of a
// dependent chain of L2 round trips and a kernel boundary.  Four lanes per row.
constexpr int kSTailThreads = 1024;
constexpr int kSTailMaxLevels = 8;
constexpr size_t kSTailSmem = 200u << 10;

struct STailLevel {
  int n, nc, nnz, pnnz, coarsest, rel;
  const int* rowptr;
  const unsigned short* col16;      // or null: col
  const int* col;
  const float* val;
  const float* inv;
  const int *prow, *pcol, *rrow, *rcol;
  const float *pval, *rval;
  // byte offsets of the staged copies in shared memory
  int o_rowptr, o_col, o_val, o_inv, o_prow, o_pcol, o_pval, o_rrow, o_rcol, o_rval, o_x, o_t, o_b, o_r;
  const double *lu, *lu_free;       // coarsest: pinned / unpinned inverses (global)
};
struct STailArgs {
  STailLevel lv[kSTailMaxLevels];
  int nlev;
  int col_bytes;                    // 2 or 4 (all levels alike)
  const float* b_in;                // the first level's right-hand side (global)
  float* x_out;                     // and its result
  const int* free_singular;
  int krylov;
};

// count elements of src into shared memory at byte offset off: the 16-byte
// pieces with cp.async (no register round trip; the caller waits for all of a
// stage's copies at once), the last partial piece element by element.  The
// sources are cudaMalloc'd arrays and the offsets 16-byte aligned.
template <typename E>
__device__ __forceinline__ void stail_copy(unsigned char* smem, int off, const E* src, int count) {
  const int bytes = count * (int)sizeof(E);
  const int n16 = bytes >> 4;
  const unsigned char* s8 = reinterpret_cast<const unsigned char*>(src);
  for (int i = threadIdx.x; i < n16; i += blockDim.x) cp_async16(smem + off + 16 * i, s8 + 16 * i, 16);
  E* dst = reinterpret_cast<E*>(smem + off);
  for (int e = (n16 << 4) / (int)sizeof(E) + threadIdx.x; e < count; e += blockDim.x) dst[e] = src[e];
}
__device__ __forceinline__ void stail_copy_wait() {
  cp_async_commit();
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// y = f(A x) over rows of a CSR block in shared memory, kTailLanes lanes per row
template <int MODE>
__device__ void stail_csr(int n, const int* rowptr, const unsigned short* col16, const int* col, int rel,
                          const float* val, const float* x, const float* b, const float* inv, float* y) {
  const int lane = threadIdx.x % kTailLanes;
  constexpr int kRowsPerPass = kSTailThreads / kTailLanes;
  for (int base = 0; base < n; base += kRowsPerPass) {
    const int row = base + (int)threadIdx.x / kTailLanes;
    const bool valid = row < n;
    float acc = 0.f;
    if (MODE != Y_SMOOTH0 && valid) {
      const int a = rowptr[row], e = rowptr[row + 1];
      if (col16) {
        const int cb = rel ? row - 32768 : 0;
        for (int k = a + lane; k < e; k += kTailLanes) acc += val[k] * x[cb + (int)col16[k]];
      } else {
        for (int k = a + lane; k < e; k += kTailLanes) acc += val[k] * x[col[k]];
      }
    }
#pragma unroll
    for (int o = kTailLanes / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, kTailLanes);
    if (lane == 0 && valid) {
      if (MODE == Y_AX) y[row] = acc;
      else if (MODE == Y_B_MINUS_AX) y[row] = b[row] - acc;
      else if (MODE == Y_SMOOTH) y[row] = x[row] + kOmega * inv[row] * (b[row] - acc);
      else if (MODE == Y_ADD_AX) y[row] = y[row] + acc;
      else if (MODE == Y_SMOOTH0) y[row] = kOmega * inv[row] * b[row];
    }
  }
}

__global__ void __launch_bounds__(kSTailThreads) k_vcycle_stail(const __grid_constant__ STailArgs A) {
  pdl_wait_release();
  extern __shared__ __align__(16) unsigned char smem[];
  // stage every level (the coarsest only its vectors)
  for (int l = 0; l < A.nlev; ++l) {
    const STailLevel& L = A.lv[l];
    if (!L.coarsest) {
      stail_copy(smem, L.o_rowptr, L.rowptr, L.n + 1);
      if (A.col_bytes == 2) stail_copy(smem, L.o_col, L.col16, L.nnz);
      else stail_copy(smem, L.o_col, L.col, L.nnz);
      stail_copy(smem, L.o_val, L.val, L.nnz);
      stail_copy(smem, L.o_inv, L.inv, L.n);
      stail_copy(smem, L.o_prow, L.prow, L.n + 1);
      stail_copy(smem, L.o_pcol, L.pcol, L.pnnz);
      stail_copy(smem, L.o_pval, L.pval, L.pnnz);
      stail_copy(smem, L.o_rrow, L.rrow, L.nc + 1);
      stail_copy(smem, L.o_rcol, L.rcol, L.pnnz);
      stail_copy(smem, L.o_rval, L.rval, L.pnnz);
    }
  }
  stail_copy(smem, A.lv[0].o_b, A.b_in, A.lv[0].n);
  stail_copy_wait();
  __syncthreads();
  auto F = [&](int off) { return reinterpret_cast<float*>(smem + off); };
  auto I = [&](int off) { return reinterpret_cast<const int*>(smem + off); };
  auto colp16 = [&](const STailLevel& L) {
    return A.col_bytes == 2 ? reinterpret_cast<const unsigned short*>(smem + L.o_col) : nullptr;
  };
  auto colp32 = [&](const STailLevel& L) {
    return A.col_bytes == 4 ? reinterpret_cast<const int*>(smem + L.o_col) : nullptr;
  };
  int l = 0;
  for (; l < A.nlev && !A.lv[l].coarsest; ++l) {
    const STailLevel& L = A.lv[l];
    const int* rp = I(L.o_rowptr);
    stail_csr<Y_SMOOTH0>(L.n, rp, colp16(L), colp32(L), L.rel, F(L.o_val), nullptr, F(L.o_b), F(L.o_inv), F(L.o_x));
    __syncthreads();
    stail_csr<Y_SMOOTH>(L.n, rp, colp16(L), colp32(L), L.rel, F(L.o_val), F(L.o_x), F(L.o_b), F(L.o_inv), F(L.o_t));
    __syncthreads();
    stail_csr<Y_SMOOTH>(L.n, rp, colp16(L), colp32(L), L.rel, F(L.o_val), F(L.o_t), F(L.o_b), F(L.o_inv), F(L.o_x));
    __syncthreads();
    stail_csr<Y_B_MINUS_AX>(L.n, rp, colp16(L), colp32(L), L.rel, F(L.o_val), F(L.o_x), F(L.o_b), nullptr,
                            F(L.o_r));
    __syncthreads();
    const STailLevel& N = A.lv[l + 1];
    stail_csr<Y_AX>(L.nc, I(L.o_rrow), nullptr, I(L.o_rcol), 0, F(L.o_rval), F(L.o_r), nullptr, nullptr, F(N.o_b));
    __syncthreads();
  }
  {  // coarsest: x = Ainv b, pinned (b[0] = 0) unless Krylov mode uses the unpinned inverse
    const STailLevel& C = A.lv[l];
    const bool use_free = A.krylov && C.lu_free != nullptr && *A.free_singular == 0;
    const double* Ainv = use_free ? C.lu_free : C.lu;
    const int pin = use_free ? 0 : 1;
    const float* cb = F(C.o_b);
    float* cx = F(C.o_x);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = warp; i < C.n; i += nw) {
      double acc = 0.0;
      for (int j = lane; j < C.n; j += 32) acc += Ainv[(long long)i * C.n + j] * ((pin && j == 0) ? 0.0 : (double)cb[j]);
      acc = warp_sum(acc);
      if (lane == 0) cx[i] = (float)acc;
    }
    __syncthreads();
  }
  for (--l; l >= 0; --l) {
    const STailLevel& L = A.lv[l];
    const STailLevel& N = A.lv[l + 1];
    const int* rp = I(L.o_rowptr);
    stail_csr<Y_ADD_AX>(L.n, I(L.o_prow), nullptr, I(L.o_pcol), 0, F(L.o_pval), F(N.o_x), nullptr, nullptr,
                        F(L.o_x));
    __syncthreads();
    stail_csr<Y_SMOOTH>(L.n, rp, colp16(L), colp32(L), L.rel, F(L.o_val), F(L.o_x), F(L.o_b), F(L.o_inv), F(L.o_t));
    __syncthreads();
    stail_csr<Y_SMOOTH>(L.n, rp, colp16(L), colp32(L), L.rel, F(L.o_val), F(L.o_t), F(L.o_b), F(L.o_inv), F(L.o_x));
    __syncthreads();
  }
  const float* x0 = F(A.lv[0].o_x);
  for (int i = threadIdx.x; i < A.lv[0].n; i += blockDim.x) A.x_out[i] = x0[i];
}

// Shared-memory layout of levels l.. (16-byte aligned arrays); returns the
// bytes, or 0 when the levels do not qualify (rows of more than 96 entries, a
// coarsest level without its dense inverses, too many levels, mixed column
// widths).
size_t stail_layout(const AMG& h, int l, STailArgs* A) {
  if ((int)h.levels.size() - l > kSTailMaxLevels) return 0;
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 15) & ~(size_t)15; return (int)o; };
  int col_bytes = 0;
  for (size_t q = l; q < h.levels.size(); ++q) {
    const Level& L = *h.levels[q];
    STailLevel d{};
    d.n = L.n; d.nc = L.nc; d.nnz = L.nnz; d.pnnz = L.pnnz; d.coarsest = L.coarsest ? 1 : 0;
    if (L.coarsest) {
      if (L.n > 500 || !L.lu.p) return 0;
      d.lu = L.lu.p; d.lu_free = L.lu_free.p;
      d.o_x = take(4 * (size_t)L.n);
      d.o_b = take(4 * (size_t)L.n);
      if (A) A->lv[q - l] = d;
      break;
    }
    if (L.avg_row > 96 || !L.valf.p || !L.inv_relaxf.p || !L.pvalf.p || !L.rvalf.p) return 0;
    const int cb = L.col16.p ? 2 : 4;
    if (col_bytes && cb != col_bytes) return 0;
    col_bytes = cb;
    d.rel = L.col16.p ? L.col16_rel : 0;
    d.rowptr = L.rowptr.p; d.col16 = L.col16.p; d.col = L.col.p; d.val = L.valf.p; d.inv = L.inv_relaxf.p;
    d.prow = L.prow.p; d.pcol = L.pcol.p; d.pval = L.pvalf.p;
    d.rrow = L.rrow.p; d.rcol = L.rcol.p; d.rval = L.rvalf.p;
    d.o_rowptr = take(4 * ((size_t)L.n + 1));
    d.o_col = take((size_t)cb * L.nnz);
    d.o_val = take(4 * (size_t)L.nnz);
    d.o_inv = take(4 * (size_t)L.n);
    d.o_prow = take(4 * ((size_t)L.n + 1));
    d.o_pcol = take(4 * (size_t)L.pnnz);
    d.o_pval = take(4 * (size_t)L.pnnz);
    d.o_rrow = take(4 * ((size_t)L.nc + 1));
    d.o_rcol = take(4 * (size_t)L.pnnz);
    d.o_rval = take(4 * (size_t)L.pnnz);
    d.o_x = take(4 * (size_t)L.n);
    d.o_t = take(4 * (size_t)L.n);
    d.o_b = take(4 * (size_t)L.n);
    d.o_r = take(4 * (size_t)L.n);
    if (A) A->lv[q - l] = d;
  }
  if (A) {
    A->nlev = (int)h.levels.size() - l;
    A->col_bytes = col_bytes ? col_bytes : 2;
  }
  return off;
}

// First level of the shared-memory tail: the coarsest-most levels whose
// staged copies fit in kSTailSmem, at least one level above the coarsest; -1
// when none, or a Chebyshev hierarchy, or no fp32 chain.  Opt-in
// (IMPES_STAIL=1, read at setup): on the 1e6-cell hierarchy (levels of 758,
// 208 and 55 rows in the tail) the step is 1.8 % slower than with the
// per-level kernels -- sixteen dependent phases on one SM cost more than
// sixteen programmatic-dependent launches on all of them.
int amg_stail_level(AMG& h) {
  const char* ev = getenv("IMPES_STAIL");
  if (!(ev && ev[0] == '1')) return -1;
  if (!h.prm.mixed_precision || h.prm.smoother != IMPES_SMOOTHER_L1_JACOBI || h.levels.size() < 2 ||
      h.prm.light_sweep_rows > 0)
    return -1;
  int best = -1;
  for (int l = (int)h.levels.size() - 2; l >= 1; --l) {
    const size_t bytes = stail_layout(h, l, nullptr);
    if (bytes == 0 || bytes > kSTailSmem) break;
    best = l;
  }
  if (best >= 0) {
    h.stail_smem = stail_layout(h, best, nullptr);
    if (cudaFuncSetAttribute((const void*)k_vcycle_stail, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)h.stail_smem) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
  }
  return best;
}

void launch_stail(AMG& h, int l, cudaStream_t s) {
  STailArgs A{};
  stail_layout(h, l, &A);
  A.b_in = LV<float>::b(*h.levels[l]);
  A.x_out = LV<float>::x(*h.levels[l]);
  A.free_singular = h.iflag.p + 3;
  A.krylov = h.krylov_mode ? 1 : 0;
  launch_pdl(k_vcycle_stail, 1, kSTailThreads, h.stail_smem, s, A);
  IMPES_CHECK_LAUNCH();
}

// _v_cycle (classical_amg.py:1037-1106) on level l: input b in LV<T>::b(L),
// initial x in LV<T>::x(L) (ignored when zero_x); returns the buffer with x.
template <typename T>
T* vcycle(AMG& h, int l, bool zero_x, cudaStream_t s, bool first_sweep_done = false) {
  Level& L = *h.levels[l];
  if (l > 0 && zero_x && l == h.tail_level && !L.coarsest) {
    launch_tail<T>(h, l, s);
    return LV<T>::x(L);
  }
  if constexpr (sizeof(T) == 4) {
    if (l > 0 && zero_x && l == h.stail_level && !L.coarsest) {
      launch_stail(h, l, s);
      return LV<T>::x(L);
    }
  }
  if (L.coarsest) {
    if (L.n <= 500) {
      const int n = L.n;
      launch_pdl(k_coarse_apply<T>, std::max(1, (n + 7) / 8), 256, n * sizeof(double), s, 
          n, L.lu.p, L.lu_free.p, h.iflag.p + 3, h.krylov_mode ? 1 : 0, LV<T>::b(L), LV<T>::x(L));
      IMPES_CHECK_LAUNCH();
      return LV<T>::x(L);
    }
    // n > 500: 50 l1-Jacobi sweeps from zero on the pinned right-hand side
    T* bp = LV<T>::r(L);
    launch_pdl(k_pin_copy<T>, grid_for(L.n, TB), TB, 0, s, L.n, LV<T>::b(L), bp);
    return smooth<T>(h, L, LV<T>::x(L), LV<T>::t(L), bp, 50, true, s, false, true);
  }
  const int tid = (l == 0) ? timers().begin(IMPES_PH_VCYCLE, s) : -1;
  // three sweeps before the coarse correction and two after, one and one on
  // the levels that light_sweep_rows selects
  const bool light = L.n <= h.prm.light_sweep_rows;
  const int pre = light ? 1 : 3, post = light ? 1 : 2;
  // the last two pre-sweeps with the residual, and the two post-sweeps, as
  // single grid-tile launches where the level is a grid's 7-point DIA
  const bool tiled = !light && dia_tile_ok<T>(h, L, LV<T>::slot);
  // first_sweep_done: the caller has already formed x = w inv b in x (the
  // first l1-Jacobi sweep from zero), so pre - 1 sweeps remain
  T* x = LV<T>::x(L);
  if (tiled) {
    int rem = first_sweep_done ? pre - 1 : pre;
    if (!first_sweep_done && zero_x) {
      x = smooth<T>(h, L, x, LV<T>::t(L), LV<T>::b(L), 1, true, s, l == 0);
      --rem;
    }
    if (rem > 2) x = smooth<T>(h, L, x, LV<T>::t(L), LV<T>::b(L), rem - 2, false, s, l == 0);
    T* o = (x == LV<T>::x(L)) ? LV<T>::t(L) : LV<T>::x(L);
    const int tt = timers().begin(IMPES_PH_TILE_L0, s);
    launch_dia_tile<T, true>(L, x, LV<T>::b(L), LV<T>::inv(L), o, LV<T>::r(L), s);
    timers().end(tt, s, 12.0 * sizeof(T) * L.n);
    x = o;
  } else if (!first_sweep_done) {
    x = smooth<T>(h, L, x, LV<T>::t(L), LV<T>::b(L), pre, zero_x, s, l == 0);
  } else if (pre > 1) {
    x = smooth<T>(h, L, x, LV<T>::t(L), LV<T>::b(L), pre - 1, false, s, l == 0);
  }
  T* spare = (x == LV<T>::x(L)) ? LV<T>::t(L) : LV<T>::x(L);
  Level& Nc = *h.levels[l + 1];
  if (!tiled) launch_a<T, Y_B_MINUS_AX>(L, LV<T>::slot, x, LV<T>::b(L), nullptr, LV<T>::r(L), s);
  // the restriction also takes the coarse level's first sweep from zero when
  // that level smooths with l1-Jacobi through the per-level kernels
  const bool fuse_s0 = !Nc.coarsest && L.r_avg <= 96 && !(l + 1 == h.tail_level) &&
                       !(sizeof(T) == 4 && l + 1 == h.stail_level) &&
                       !(h.prm.smoother == IMPES_SMOOTHER_CHEBYSHEV && Nc.cheb_lmax.p);
  if (fuse_s0) {
    const int lpr_r = L.lpr_r[LV<T>::slot] > 0 ? L.lpr_r[LV<T>::slot] : default_lpr(L.r_avg);
    launch_restrict_s0<T>(L, lpr_r, LV<T>::rval(L), LV<T>::r(L), LV<T>::inv(Nc), LV<T>::b(Nc), LV<T>::x(Nc), s);
  } else {
    launch_csr<T, Y_AX>(L.nc, L.r_avg, L.rrow.p, L.rcol.p, LV<T>::rval(L), LV<T>::r(L), nullptr,
                        nullptr, LV<T>::b(Nc), s, nullptr, 0, L.lpr_r[LV<T>::slot]);
  }
  T* ec = vcycle<T>(h, l + 1, true, s, fuse_s0);
  launch_csr<T, Y_ADD_AX>(L.n, L.p_avg, L.prow.p, L.pcol.p, LV<T>::pval(L), ec, nullptr, nullptr, x, s,
                          nullptr, 0, L.lpr_p[LV<T>::slot]);
  T* out = spare;
  if (tiled) {
    const int tt = timers().begin(IMPES_PH_TILE_L0, s);
    launch_dia_tile<T, false>(L, x, LV<T>::b(L), LV<T>::inv(L), spare, nullptr, s);
    timers().end(tt, s, 11.0 * sizeof(T) * L.n);
  } else {
    out = smooth<T>(h, L, x, spare, LV<T>::b(L), post, false, s, l == 0);
  }
  timers().end(tid, s, vcycle_bytes<T>(h, l));
  return out;
}

// One V-cycle from level 0 (input in LV<T>::b(L0), initial iterate in
// LV<T>::x(L0) unless zero_x), replayed from a CUDA graph captured on first use.
template <typename T>
T* vcycle_top(AMG& h, bool zero_x, cudaStream_t s) {
  if (!h.use_graphs) return vcycle<T>(h, 0, zero_x, s);
  PhaseTimers& tm = timers();
  AMG::VGraph& g = h.vgraph[sizeof(T) == 4][zero_x][h.krylov_mode][tm.on];
  if (!g.exec) {
    if (!h.cap_stream) IMPES_CUDA(cudaStreamCreateWithFlags(&h.cap_stream, cudaStreamNonBlocking));
    const unsigned long long before = thread_launches();
    if (tm.on) tm.capture = &g.timers;   // timer nodes only in the timed variant
    IMPES_CUDA(cudaStreamBeginCapture(h.cap_stream, cudaStreamCaptureModeThreadLocal));
    T* out = nullptr;
    cudaGraph_t graph = nullptr;
    try {
      out = vcycle<T>(h, 0, zero_x, h.cap_stream);
    } catch (...) {
      tm.capture = nullptr;
      cudaStreamEndCapture(h.cap_stream, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    tm.capture = nullptr;
    IMPES_CUDA(cudaStreamEndCapture(h.cap_stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    IMPES_CUDA(e);
    g.out = out;
    g.kernels = (long long)(thread_launches() - before);
    count_launches(-g.kernels);
  }
  IMPES_CUDA(cudaGraphLaunch(g.exec, s));
  count_launches(g.kernels);
  if (tm.on && !g.timers.empty()) tm.pending = &g.timers;
  return (T*)g.out;
}

}  // namespace

// ------------------------------------------------------------- autotuner
// Lanes per row of the CSR kernels, picked from timed trials per level: the
// l1-Jacobi sweep stands for the kernels on A (sweeps, residuals, Chebyshev
// steps, the FGMRES operator), Y_AX on R for the restriction and Y_ADD_AX on P
// for the prolongation.  Each candidate (1, 2, 4, 8, 16, 32 lanes, at most four
// times the mean row length) runs twice untimed and then in three batches of
// eight between CUDA events on the level's own work vectors (the fastest batch
// counts; large levels are timed from a cold L2, below), and the fewest lanes
// within 3 % of the fastest is kept.  The first choice made for a shape
// (precision, operator, log2 of the rows in halves, mean row length) is kept
// for the whole process, so hierarchies of the same shape -- a rebuilt one, or
// ensemble members alike in size -- launch the same kernels and sum in the same
// order.  Levels with more than 96 entries per row keep the warps-per-row
// kernels.  IMPES_NO_TUNE=1 keeps the mean-row-length rule.
//
// IMPES_TUNE_CACHE=<file> makes the choices persistent: the file's entries
// (one "precision operator rows avg choice" line each) are loaded before a
// hierarchy is tuned and the process's choices are written back after, so a
// later process -- another run, or one under a profiler whose serialised
// launches would time differently -- launches the same kernels.
namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune_cache;

const char* tune_cache_path() {
  const char* ev = getenv("IMPES_TUNE_CACHE");
  return (ev && ev[0]) ? ev : nullptr;
}
void tune_cache_load() {
  const char* path = tune_cache_path();
  if (!path) return;
  FILE* f = fopen(path, "r");
  if (!f) return;
  int a, b, c, d, v;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  while (fscanf(f, "%d %d %d %d %d", &a, &b, &c, &d, &v) == 5) g_tune_cache.emplace(std::make_tuple(a, b, c, d), v);
  fclose(f);
}
void tune_cache_save() {
  const char* path = tune_cache_path();
  if (!path) return;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  FILE* f = fopen(path, "w");
  if (!f) return;
  for (const auto& e : g_tune_cache)
    fprintf(f, "%d %d %d %d %d\n", std::get<0>(e.first), std::get<1>(e.first), std::get<2>(e.first),
            std::get<3>(e.first), e.second);
  fclose(f);
}

// Cold-cache trials: a level whose sweep streams more than kColdBytes is timed
// one launch at a time after g_flush (allocated while a hierarchy is tuned) is
// overwritten, as a V-cycle sees it -- the other levels' data passes through
// L2 between two sweeps of a large level.  Smaller levels run back to back
// (on the 1e6-cell hierarchy a 24 MB threshold timed its 34 MB level 2 cold
// and picked a kernel 1.5x slower in the V-cycle).
constexpr double kColdBytes = 40.0 * (1 << 20);
constexpr size_t kFlushBytes = 192u << 20;
thread_local void* g_flush = nullptr;   // per tuning thread (ensembles tune on several)

template <typename F>
float time_trials(F launch, double bytes, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
  for (int w = 0; w < 2; ++w) launch();
  float total = 0.f, ms = 0.f;
  if (g_flush && bytes > kColdBytes) {
    for (int w = 0; w < 8; ++w) {
      IMPES_CUDA(cudaMemsetAsync(g_flush, w, kFlushBytes, s));
      IMPES_CUDA(cudaEventRecord(e0, s));
      launch();
      IMPES_CUDA(cudaEventRecord(e1, s));
      IMPES_CUDA(cudaEventSynchronize(e1));
      IMPES_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      total += ms;
    }
    return total;
  }
  // warm: the fastest of three batches of eight back-to-back launches (a batch
  // that another process or a clock change slowed is not the one kept)
  float best = 0.f;
  for (int rep = 0; rep < 3; ++rep) {
    IMPES_CUDA(cudaEventRecord(e0, s));
    for (int w = 0; w < 8; ++w) launch();
    IMPES_CUDA(cudaEventRecord(e1, s));
    IMPES_CUDA(cudaEventSynchronize(e1));
    IMPES_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = rep == 0 ? ms : std::min(best, ms);
  }
  return best;
}
inline double level_bytes(size_t value_bytes, int n, double avg, bool col16) {
  return (double)n * avg * (value_bytes + (col16 ? 2.0 : 4.0)) + (double)n * (4.0 + 4.0 * value_bytes);
}

template <typename T, int MODE>
float time_lpr(int lpr, int n, int avg, const int* rowptr, const int* col, const T* val, const T* x,
               const T* b, const T* inv, T* y, const unsigned short* col16, int rel, cudaStream_t s,
               cudaEvent_t e0, cudaEvent_t e1) {
  return time_trials([&] { launch_csr<T, MODE>(n, avg, rowptr, col, val, x, b, inv, y, s, col16, rel, lpr); },
                     level_bytes(sizeof(T), n, avg, col16 != nullptr), s, e0, e1);
}

template <typename T, int MODE>
int tune_one(int slot, int kind, int n, int avg, const int* rowptr, const int* col, const T* val, const T* x,
             const T* b, const T* inv, T* y, const unsigned short* col16, int rel, cudaStream_t s,
             cudaEvent_t e0, cudaEvent_t e1) {
  if (n <= 0 || avg > 96) return 0;
  const int nb = (int)std::lround(2.0 * std::log2((double)n));
  const auto key = std::make_tuple(slot, kind, nb, avg);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) return it->second;
  }
  // the fewest lanes within 3 % of the fastest: timing noise between near-equal
  // candidates does not flip the choice
  int cand[6], nc = 0;
  float ms[6];
  for (int lpr : {1, 2, 4, 8, 16, 32}) {
    if (lpr > 1 && lpr > 4 * avg) break;
    cand[nc] = lpr;
    ms[nc++] = time_lpr<T, MODE>(lpr, n, avg, rowptr, col, val, x, b, inv, y, col16, rel, s, e0, e1);
  }
  float best_ms = 1e30f;
  for (int q = 0; q < nc; ++q) best_ms = std::min(best_ms, ms[q]);
  int best = default_lpr(avg);
  for (int q = 0; q < nc; ++q)
    if (ms[q] <= 1.03f * best_ms) { best = cand[q]; break; }
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto ins = g_tune_cache.emplace(key, best);   // another thread may have decided first
  return ins.first->second;
}

// IMPES_SELL=1 (read at setup) puts every level that has a SELL copy on it,
// whatever the timings say (and no level on its DIA copy).
bool sell_forced() {
  const char* ev = getenv("IMPES_SELL");
  return ev && ev[0] == '1';
}

// SELL-32 against the level's tuned CSR sweep: kept when it is more than 3 %
// faster (cached by shape like the lanes per row).
template <typename T>
bool tune_sell(Level& L, int slot, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
  if (L.sell_slices <= 0 || !sell_values<T>(L)) return false;
  const int nb = (int)std::lround(2.0 * std::log2((double)L.n));
  const auto key = std::make_tuple(slot, 3, nb, L.avg_row);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) return it->second != 0;
  }
  const double bytes = level_bytes(sizeof(T), L.n, L.avg_row, L.col16.p != nullptr);
  auto timed = [&](bool sell) {
    L.sell_on[slot] = sell;
    return time_trials([&] { launch_a<T, Y_SMOOTH>(L, slot, LV<T>::x(L), LV<T>::b(L), LV<T>::inv(L), LV<T>::t(L), s); },
                       bytes, s, e0, e1);
  };
  const float t_csr = timed(false), t_sell = timed(true);
  const int pick = t_sell < 0.97f * t_csr ? 1 : 0;
  L.sell_on[slot] = false;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto ins = g_tune_cache.emplace(key, pick);
  return ins.first->second != 0;
}

// The DIA copy against the level's tuned CSR/SELL sweep: kept when it is more
// than 3 % faster (cached by shape).
template <typename T>
bool tune_dia(Level& L, int slot, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
  if (L.dia_nd <= 0 || !dia_values<T>(L)) return false;
  const int nb = (int)std::lround(2.0 * std::log2((double)L.n));
  const auto key = std::make_tuple(slot, 4, nb, L.avg_row);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      if (it->second > 0) L.dia_rpt = it->second;   // the cached choice: rows per thread, 0 = no DIA
      return it->second != 0;
    }
  }
  const double bytes = level_bytes(sizeof(T), L.n, L.avg_row, L.col16.p != nullptr);
  auto timed = [&](bool dia) {
    L.dia_on[slot] = dia;
    return time_trials([&] { launch_a<T, Y_SMOOTH>(L, slot, LV<T>::x(L), LV<T>::b(L), LV<T>::inv(L), LV<T>::t(L), s); },
                       bytes, s, e0, e1);
  };
  const float t_other = timed(false);
  L.dia_rpt = 1;
  float t_dia = timed(true);
  int rpt = 1;
  if (L.dia_nd == 7) {   // two rows per thread: kept when more than 3 % faster
    L.dia_rpt = 2;
    const float t2 = timed(true);
    if (t2 < 0.97f * t_dia) { t_dia = t2; rpt = 2; }
  }
  L.dia_rpt = rpt;
  const int pick = t_dia < 0.97f * t_other ? rpt : 0;
  L.dia_on[slot] = false;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto ins = g_tune_cache.emplace(key, pick);
  if (ins.first->second > 0) L.dia_rpt = ins.first->second;
  return ins.first->second != 0;
}

// IMPES_DIA=1 (read at setup) puts every level that has a DIA copy on it.
bool dia_forced() {
  const char* ev = getenv("IMPES_DIA");
  return ev && ev[0] == '1';
}

template <typename T>
void tune_levels(AMG& h, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1) {
  const int slot = LV<T>::slot;
  for (auto& up : h.levels) {
    Level& L = *up;
    if (L.coarsest || !LV<T>::val(L)) continue;
    L.lpr_a[slot] = tune_one<T, Y_SMOOTH>(slot, 0, L.n, L.avg_row, L.rowptr.p, L.col.p, LV<T>::val(L),
                                          LV<T>::x(L), LV<T>::b(L), LV<T>::inv(L), LV<T>::t(L), L.col16.p,
                                          L.col16_rel, s, e0, e1);
    L.sell_on[slot] = sell_forced() ? (L.sell_slices > 0 && sell_values<T>(L) != nullptr)
                                    : tune_sell<T>(L, slot, s, e0, e1);
    // a forced layout is the one used (IMPES_SELL=1 keeps DIA off)
    L.dia_on[slot] = dia_forced()    ? (L.dia_nd > 0 && dia_values<T>(L) != nullptr)
                     : sell_forced() ? false
                                     : tune_dia<T>(L, slot, s, e0, e1);
    L.lpr_r[slot] = tune_one<T, Y_AX>(slot, 1, L.nc, L.r_avg, L.rrow.p, L.rcol.p, LV<T>::rval(L), LV<T>::r(L),
                                      nullptr, nullptr, LV<T>::t(*h.levels[&up - &h.levels[0] + 1]), nullptr, 0,
                                      s, e0, e1);
    L.lpr_p[slot] = tune_one<T, Y_ADD_AX>(slot, 2, L.n, L.p_avg, L.prow.p, L.pcol.p, LV<T>::pval(L),
                                          LV<T>::x(*h.levels[&up - &h.levels[0] + 1]), nullptr, nullptr,
                                          LV<T>::t(L), nullptr, 0, s, e0, e1);
  }
}
}  // namespace

// Per-level kernel times of the V-cycle (instrumentation): for each level, the
// mean device time of one l1-Jacobi sweep, one residual, one restriction and
// one prolongation in the given precision, each launched `reps` times back to
// back between CUDA events on the level's own work vectors (warm caches), with
// the level's tuned lanes per row.  out[4 * level + {0,1,2,3}] in microseconds
// (0 on the coarsest level).
void amg_profile_levels(AMG& h, int precision, int reps, double* out, cudaStream_t s) {
  if (precision == 0) amg_ensure_fp64(h, s);
  cudaEvent_t e0, e1;
  IMPES_CUDA(cudaEventCreate(&e0));
  IMPES_CUDA(cudaEventCreate(&e1));
  auto timed = [&](auto&& launch) {
    launch();
    IMPES_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) launch();
    IMPES_CUDA(cudaEventRecord(e1, s));
    IMPES_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    IMPES_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    return 1e3 * (double)ms / reps;
  };
  auto run = [&](auto tag) {
    using T = decltype(tag);
    const int slot = LV<T>::slot;
    for (size_t l = 0; l < h.levels.size(); ++l) {
      Level& L = *h.levels[l];
      double* o = out + 4 * l;
      o[0] = o[1] = o[2] = o[3] = 0.0;
      if (L.coarsest || !LV<T>::val(L)) continue;
      Level& Nc = *h.levels[l + 1];
      o[0] = timed([&] {
        launch_a<T, Y_SMOOTH>(L, slot, LV<T>::x(L), LV<T>::b(L), LV<T>::inv(L), LV<T>::t(L), s);
      });
      o[1] = timed([&] {
        launch_a<T, Y_B_MINUS_AX>(L, slot, LV<T>::x(L), LV<T>::b(L), nullptr, LV<T>::r(L), s);
      });
      o[2] = timed([&] {
        launch_csr<T, Y_AX>(L.nc, L.r_avg, L.rrow.p, L.rcol.p, LV<T>::rval(L), LV<T>::r(L), nullptr, nullptr,
                            LV<T>::t(Nc), s, nullptr, 0, L.lpr_r[slot]);
      });
      o[3] = timed([&] {
        launch_csr<T, Y_ADD_AX>(L.n, L.p_avg, L.prow.p, L.pcol.p, LV<T>::pval(L), LV<T>::x(Nc), nullptr, nullptr,
                                LV<T>::t(L), s, nullptr, 0, L.lpr_p[slot]);
      });
    }
  };
  try {
    if (precision == 1) {
      IMPES_REQUIRE(h.prm.mixed_precision, IMPES_ERR_STATE, "fp32 levels need mixed_precision=1");
      run(float{});
    } else {
      run(double{});
    }
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

// The largest cluster (16, else 8 CTAs of kTailThreads) that can be resident.
template <typename T>
int tail_cluster_size() {
  cudaFuncSetAttribute((const void*)k_vcycle_tail<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaGetLastError();
  for (int c : {16, 8}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(kTailThreads);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = c;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_vcycle_tail<T>, &cfg) == cudaSuccess && nclusters >= 1)
      return c;
    cudaGetLastError();
  }
  return 0;
}

int amg_tail_level(AMG& h) {
  // the shared-memory fp32 tail, unless the cluster tail is asked for
  h.stail_level = h.use_tail ? -1 : amg_stail_level(h);
  for (size_t l = 1; l < h.levels.size(); ++l) {
    if (!tail_eligible(h, (int)l)) continue;
    if (h.levels[l]->coarsest) return -1;
    const int c = std::min(tail_cluster_size<double>(), h.prm.mixed_precision ? tail_cluster_size<float>() : 16);
    if (c <= 0) return -1;
    h.tail_cluster = c;
    return (int)l;
  }
  return -1;
}

void amg_autotune(AMG& h, cudaStream_t s) {
  {
    const char* ev = getenv("IMPES_NO_TUNE");
    if (ev && ev[0] == '1') return;
  }
  cudaEvent_t e0, e1;
  IMPES_CUDA(cudaEventCreate(&e0));
  IMPES_CUDA(cudaEventCreate(&e1));
  try {
    // the work vectors hold whatever they hold: clear them so the trial
    // kernels read finite numbers
    for (auto& L : h.levels) {
      const size_t n = std::max(L->n, 1);
      IMPES_CUDA(cudaMemsetAsync(L->x.p, 0, n * sizeof(double), s));
      IMPES_CUDA(cudaMemsetAsync(L->b.p, 0, n * sizeof(double), s));
      IMPES_CUDA(cudaMemsetAsync(L->r.p, 0, n * sizeof(double), s));
      IMPES_CUDA(cudaMemsetAsync(L->xf.p, 0, n * sizeof(float), s));
      IMPES_CUDA(cudaMemsetAsync(L->bf.p, 0, n * sizeof(float), s));
      IMPES_CUDA(cudaMemsetAsync(L->rf.p, 0, n * sizeof(float), s));
    }
    tune_cache_load();
    DBuf<char> flush(kFlushBytes);
    g_flush = flush.p;
    tune_levels<double>(h, s, e0, e1);
    if (h.prm.mixed_precision) tune_levels<float>(h, s, e0, e1);
    IMPES_CUDA(cudaStreamSynchronize(s));
    g_flush = nullptr;
    tune_cache_save();
  } catch (...) {
    g_flush = nullptr;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

// V-cycle on the equilibrated system: xs = V(0, bs)  (FP64 or FP32 inside)
void amg_vcycle_scaled(AMG& h, const double* bs, double* xs, int precision, cudaStream_t s) {
  if (precision == 0) amg_ensure_fp64(h, s);
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  if (precision == 1) {
    IMPES_REQUIRE(h.prm.mixed_precision, IMPES_ERR_STATE, "fp32 V-cycle needs mixed_precision=1");
    launch_pdl(k_convert<double, float>, grid_for(n, TB), TB, 0, s, n, bs, L0.bf.p);
    float* x = vcycle_top<float>(h, true, s);
    launch_pdl(k_convert<float, double>, grid_for(n, TB), TB, 0, s, n, x, xs);
  } else {
    IMPES_CUDA(cudaMemcpyAsync(L0.b.p, bs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    double* x = vcycle_top<double>(h, true, s);
    IMPES_CUDA(cudaMemcpyAsync(xs, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  }
  IMPES_CHECK_LAUNCH();
}

// ClassicalAMG.solve (classical_amg.py:1108-1155).  norm = IMPES_NORM_JACOBI
// measures the stopping test in ||D^-1 r|| / ||D^-1 b|| instead.
void amg_solve_vcycles(AMG& h, const double* b, double* x, double tol, int max_cycles, int* cycles,
                       double* rel, cudaStream_t s, int norm) {
  amg_ensure_fp64(h, s);
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  DBuf<double> bs(n), r(n), wb(n);
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, b, bs.p);
  IMPES_CHECK_LAUNCH();
  const bool jac = norm == IMPES_NORM_JACOBI;
  if (jac) { launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.jac_w.p, bs.p, wb.p); }
  const double bn = std::sqrt(jac ? dot_host(h, wb.p, wb.p, n, s) : dot_host(h, bs.p, bs.p, n, s));
  IMPES_CUDA(cudaMemcpyAsync(L0.b.p, bs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  double rr = INFINITY;
  int c = 0;
  double* xs = nullptr;
  for (c = 1; c <= max_cycles; ++c) {
    xs = vcycle_top<double>(h, c == 1, s);
    if (xs != L0.x.p)
      IMPES_CUDA(cudaMemcpyAsync(L0.x.p, xs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    xs = L0.x.p;
    launch_csr<double, Y_B_MINUS_AX>(n, L0.avg_row, L0.rowptr.p, L0.col.p, L0.val.p, xs, bs.p,
                                     nullptr, r.p, s);
    if (jac) { launch_pdl(k_mul_inplace, grid_for(n, TB), TB, 0, s, n, r.p, h.jac_w.p); }
    rr = std::sqrt(dot_host(h, r.p, r.p, n, s)) / (bn + 1e-30);
    if (!(rr == rr)) throw Error(IMPES_ERR_NAN, "NaN residual in V-cycle solve");
    if (rr < tol) break;
  }
  if (c > max_cycles) c = max_cycles;
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, L0.x.p, x);
  IMPES_CHECK_LAUNCH();
  if (cycles) *cycles = c;
  if (rel) *rel = rr;
}

// ClassicalAMG.apply (classical_amg.py:1157-1180)
void amg_apply(AMG& h, const double* b, double* x, int cycles, double apply_tol,
               int apply_max_cycles, cudaStream_t s) {
  amg_ensure_fp64(h, s);
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  DBuf<double> bs(n), r(n);
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, b, bs.p);
  IMPES_CUDA(cudaMemcpyAsync(L0.b.p, bs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  const double bn = std::sqrt(dot_host(h, bs.p, bs.p, n, s));
  int c = 0;
  while (c < apply_max_cycles) {
    double* xs = vcycle_top<double>(h, c == 0, s);
    if (xs != L0.x.p)
      IMPES_CUDA(cudaMemcpyAsync(L0.x.p, xs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    ++c;
    launch_csr<double, Y_B_MINUS_AX>(n, L0.avg_row, L0.rowptr.p, L0.col.p, L0.val.p, L0.x.p, bs.p,
                                     nullptr, r.p, s);
    double rel = std::sqrt(dot_host(h, r.p, r.p, n, s)) / (bn + 1e-30);
    if (c >= cycles && rel < apply_tol) break;
  }
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, L0.x.p, x);
  IMPES_CHECK_LAUNCH();
}

// ------------------------------------------------------------------ FGMRES
namespace {

__global__ void k_givens(int j, int ldh, double* H, double* cs, double* sn, double* g, double* est) {
  pdl_wait_release();
  double* hj = H + (long long)j * ldh;  // column j, rows 0..j+1
  for (int i = 0; i < j; ++i) {
    double t = cs[i] * hj[i] + sn[i] * hj[i + 1];
    hj[i + 1] = -sn[i] * hj[i] + cs[i] * hj[i + 1];
    hj[i] = t;
  }
  double a = hj[j], b = hj[j + 1];
  double d = hypot(a, b);
  double c = d > 0 ? a / d : 1.0, s = d > 0 ? b / d : 0.0;
  cs[j] = c; sn[j] = s;
  hj[j] = d; hj[j + 1] = 0.0;
  g[j + 1] = -s * g[j];
  g[j] = c * g[j];
  *est = fabs(g[j + 1]);
}
__global__ void k_set_hcol(int j, int ldh, double* H, const double* nrm2) {
  pdl_wait_release();
  H[(long long)j * ldh + j + 1] = sqrt(*nrm2);
}
// y = R^{-1} g (upper triangular k x k, column-major with leading dim ldh)
__global__ void k_backsolve(int k, int ldh, const double* H, const double* g, double* y) {
  pdl_wait_release();
  for (int i = k - 1; i >= 0; --i) {
    double s = g[i];
    for (int j = i + 1; j < k; ++j) s -= H[(long long)j * ldh + i] * y[j];
    y[i] = s / H[(long long)i * ldh + i];
  }
}
__global__ void k_combine(long long n, const double* __restrict__ Z, long long ldz, int k,
                          const double* __restrict__ y, double* __restrict__ x) {
  pdl_wait_release();
  __shared__ double sy[128];
  for (int q = threadIdx.x; q < k; q += blockDim.x) sy[q] = y[q];
  __syncthreads();
  GRID_LOOP(i, n) x[i] = axpy_rows<1>(x[i], sy, k, Z, ldz, i);
}
__global__ void k_hadd(int k, double* h, const double* y, const int* pred) {
  pdl_wait_release();
  if (pred && *pred == 0) return;
  for (int i = threadIdx.x; i < k; i += blockDim.x) h[i] += y[i];
}
__global__ void k_fill(long long n, double* a, double v) {
  pdl_wait_release(); GRID_LOOP(i, n) a[i] = v; }
__global__ void k_init_g(double* g, int m1, const double* nrm2) {
  pdl_wait_release();
  for (int i = 0; i < m1; ++i) g[i] = 0.0;
  g[0] = sqrt(*nrm2);
}

}  // namespace

// Right-preconditioned flexible GMRES on the equilibrated system, with a row
// weighting wt that selects the minimised norm: wt = 1 gives the reference's
// equilibrated norm, wt = D^-1/2 (or 1/|a_ii| without equilibration) the Jacobi
// norm ||D^-1 r||.  Operator K = diag(wt) A_s, preconditioner M(v) = V(v ./ wt).
// Orthogonalisation is classical Gram-Schmidt with one re-orthogonalisation
// pass; all reductions use a fixed block count (deterministic).
namespace {
struct KrylovModeGuard {
  AMG& h;
  explicit KrylovModeGuard(AMG& a) : h(a) { h.krylov_mode = true; }
  ~KrylovModeGuard() { h.krylov_mode = false; }
};
}  // namespace

void amg_fgmres(AMG& h, const double* b, double* x, const impes_krylov_params& kp,
                impes_krylov_stats& st, cudaStream_t s) {
  if (kp.precision == 0) amg_ensure_fp64(h, s);
  KrylovModeGuard guard(h);
  struct SolveTimer {
    cudaStream_t s;
    int id;
    ~SolveTimer() { try { timers().end(id, s, 0.0); } catch (...) {} }
  } solve_timer{s, timers().begin(IMPES_PH_SOLVE, s)};
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  const int m = std::max(1, std::min(kp.restart, 120));
  if (h.krylov_m != m || h.V.n < (size_t)(m + 1) * n) {
    h.V.alloc((size_t)(m + 1) * n);
    h.Z.alloc((size_t)m * n);
    h.H.alloc((size_t)(m + 2) * (m + 1));
    h.cs.alloc(m + 1); h.sn.alloc(m + 1); h.g.alloc(m + 2); h.y.alloc(m + 1);
    h.kw.alloc(n); h.kb.alloc(n); h.kx.alloc(n);
    h.krylov_m = m;
  }
  h.red.ensure((size_t)(m + 2) * kDotBlocks + kDotBlocks);
  const int ldh = m + 2;
  const bool jac = kp.norm == IMPES_NORM_JACOBI;
  double* wt = jac ? h.jac_w.p : h.kw.p;
  if (!jac) { launch_pdl(k_fill, grid_for(n, TB), TB, 0, s, n, h.kw.p, 1.0); }
  double* bs = h.kb.p;   // b_s = dhalf .* b
  double* xs = h.kx.p;   // x_s
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, b, bs);
  if (kp.use_x0)
    { launch_pdl(k_div_convert<double, double>, grid_for(n, TB), TB, 0, s, n, x, h.dhalf_inv.p, xs); }
  else
    { launch_pdl(k_zero, grid_for(n, TB), TB, 0, s, n, xs); }
  IMPES_CHECK_LAUNCH();
  double* r0 = h.V.p;
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, wt, bs, r0);
  const double bnorm = std::sqrt(dot_host(h, r0, r0, n, s));
  st = impes_krylov_stats{0, 0, 0, 0.0, 0.0};
  if (!(bnorm > 0.0)) {
    if (!(bnorm == bnorm)) throw Error(IMPES_ERR_NAN, "non-finite right-hand side");
    launch_pdl(k_zero, grid_for(n, TB), TB, 0, s, n, x);
    st.converged = 1;
    return;
  }
  double* dscal = h.scal.p;  // [0] squared norm, [1] residual estimate
  int total = 0;
  double est_rel = INFINITY;
  const int prec = kp.precision;
  if (prec == 1)
    IMPES_REQUIRE(h.prm.mixed_precision, IMPES_ERR_STATE, "fp32 V-cycle needs mixed_precision=1");
  while (true) {
    // V[0] = wt .* (b_s - A_s x_s), beta = ||V[0]||
    launch_csr<double, Y_B_MINUS_AX>(n, L0.avg_row, L0.rowptr.p, L0.col.p, L0.val.p, xs, bs,
                                     nullptr, h.V.p, s);
    launch_pdl(k_mul_inplace, grid_for(n, TB), TB, 0, s, n, h.V.p, wt);
    launch_pdl(k_multidot, kDotBlocks, TB, 0, s, n, h.V.p, 0, 1, h.V.p, h.red.p);
    launch_pdl(k_dot_finalize, 1, 32, 0, s, 1, (const double*)h.red.p, dscal, 0, (const int*)nullptr);
    IMPES_CUDA(cudaMemcpyAsync(h.hbuf.p, dscal, sizeof(double), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    const double beta = std::sqrt(h.hbuf.p[0]);
    if (!(beta == beta)) throw Error(IMPES_ERR_NAN, "NaN residual in FGMRES");
    est_rel = beta / bnorm;
    st.rel_res = est_rel;
    if (est_rel < kp.tol || total >= kp.max_iters) break;
    launch_pdl(k_init_g, 1, 1, 0, s, h.g.p, m + 1, dscal);
    launch_pdl(k_scale_by_inv_sqrt, grid_for(n, TB), TB, 0, s, n, h.V.p, h.V.p, dscal);
    int j = 0;
    for (; j < m && total < kp.max_iters; ++j) {
      double* vj = h.V.p + (size_t)j * n;
      double* zj = h.Z.p + (size_t)j * n;
      double* w = h.V.p + (size_t)(j + 1) * n;
      // z_j = V(v_j ./ wt)
      if (prec == 1) {
        launch_pdl(k_div_convert<double, float>, grid_for(n, TB), TB, 0, s, n, vj, wt, L0.bf.p);
        float* zf = vcycle_top<float>(h, true, s);
        launch_pdl(k_convert<float, double>, grid_for(n, TB), TB, 0, s, n, zf, zj);
      } else {
        launch_pdl(k_div_convert<double, double>, grid_for(n, TB), TB, 0, s, n, vj, wt, L0.b.p);
        double* zd = vcycle_top<double>(h, true, s);
        IMPES_CUDA(cudaMemcpyAsync(zj, zd, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      }
      // w = wt .* (A_s z_j)
      const int tsp = timers().begin(IMPES_PH_SPMV_L0, s);
      launch_a<double, Y_W_AX>(L0, 0, zj, nullptr, wt, w, s);
      timers().end(tsp, s, L0.dia_on[0] ? 8.0 * L0.dia_nd * (double)n + 24.0 * n
                                        : spmv_bytes(8.0, 8.0, L0.nnz, n, n, L0.col16.p ? 2.0 : 4.0) + 8.0 * n);
      // classical Gram-Schmidt; the second pass only when the first cancelled
      // more than 0.3 of the norm (flag on the device).  H[j+1, j] holds
      // ||w||^2 before the first pass until k_set_hcol overwrites it.
      const int tor = timers().begin(IMPES_PH_ORTHO, s);
      double* hcol = h.H.p + (size_t)j * ldh;
      int* reorth = h.iflag.p + 4;
      const dim3 g1(kDotBlocks, (unsigned)((j + 2 + kMD - 1) / kMD));
      launch_pdl(k_multidot_g, g1, dim3(TB), 0, s, (long long)n, (const double*)h.V.p, (long long)n, j + 1, 1,
                 (const double*)w, h.red.p, (const int*)nullptr);
      launch_pdl(k_dot_finalize, j + 2, 32, 0, s, j + 2, (const double*)h.red.p, hcol, 0, (const int*)nullptr);
      launch_pdl(k_update, kDotBlocks, TB, 0, s, n, h.V.p, n, j + 1, hcol, w, h.red.p, (const int*)nullptr);
      launch_pdl(k_dot_finalize, 1, 32, 0, s, 1, (const double*)h.red.p, dscal, 0, (const int*)nullptr);
      launch_pdl(k_reorth_flag, 1, 1, 0, s, (const double*)dscal, (const double*)(hcol + j + 1), reorth);
      const dim3 g2(kDotBlocks, (unsigned)((j + 1 + kMD - 1) / kMD));
      launch_pdl(k_multidot_g, g2, dim3(TB), 0, s, (long long)n, (const double*)h.V.p, (long long)n, j + 1, 0,
                 (const double*)w, h.red.p, (const int*)reorth);
      launch_pdl(k_dot_finalize, j + 1, 32, 0, s, j + 1, (const double*)h.red.p, h.y.p, 0, (const int*)reorth);
      launch_pdl(k_update, kDotBlocks, TB, 0, s, n, h.V.p, n, j + 1, (const double*)h.y.p, w, h.red.p,
                 (const int*)reorth);
      launch_pdl(k_dot_finalize, 1, 32, 0, s, 1, (const double*)h.red.p, dscal, 0, (const int*)reorth);
      launch_pdl(k_hadd, 1, 128, 0, s, j + 1, hcol, (const double*)h.y.p, (const int*)reorth);
      launch_pdl(k_set_hcol, 1, 1, 0, s, j, ldh, h.H.p, dscal);
      launch_pdl(k_scale_by_inv_sqrt, grid_for(n, TB), TB, 0, s, n, w, w, dscal);
      timers().end(tor, s, 8.0 * n * (2.0 * (j + 1) + 3.0));
      launch_pdl(k_givens, 1, 1, 0, s, j, ldh, h.H.p, h.cs.p, h.sn.p, h.g.p, dscal + 1);
      IMPES_CHECK_LAUNCH();
      ++total;
      IMPES_CUDA(cudaMemcpyAsync(h.hbuf.p, dscal + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
      IMPES_CUDA(cudaStreamSynchronize(s));
      timers().harvest();
      est_rel = h.hbuf.p[0] / bnorm;
      if (!(est_rel == est_rel)) throw Error(IMPES_ERR_NAN, "NaN in FGMRES");
      if (est_rel < kp.tol) { ++j; break; }
    }
    // x_s += Z y with y = R^-1 g; the loop head re-checks the true residual
    launch_pdl(k_backsolve, 1, 1, 0, s, j, ldh, h.H.p, h.g.p, h.y.p);
    launch_pdl(k_combine, grid_for(n, TB), TB, 0, s, n, h.Z.p, n, j, h.y.p, xs);
    IMPES_CHECK_LAUNCH();
    st.restarts++;
  }
  st.iterations = total;
  st.converged = est_rel < kp.tol;
  st.true_rel_res = est_rel;
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, xs, x);
  IMPES_CHECK_LAUNCH();
}

// ===================================================== device-driven FGMRES
// The FGMRES above with its control on the device, for capture into a CUDA
// graph: the iteration count, the Arnoldi index j, the convergence test and
// the restart decision live in FgState, every kernel reads j from there, and a
// conditional WHILE node repeats the iteration body until the last kernel of
// an iteration clears the node's condition.  One body pass is one iteration
// (preconditioner application, operator product, Gram-Schmidt with the
// optional second pass, Givens rotation); at the end of a cycle (converged,
// j == restart or the iteration cap) the same pass also back-solves, updates
// x_s and recomputes the true residual, which decides whether to stop or to
// restart.  Same arithmetic and order as amg_fgmres; no host synchronisation
// until the caller reads the state after the graph.
namespace {
__global__ void k_fg_init(FgState* st, const double* part_b, const double* part_r, int nb, double tol,
                          int max_iters, int m1, double* g, cudaGraphConditionalHandle cond) {
  pdl_wait_release();
  double b2 = 0.0, r2 = 0.0;
  for (int q = 0; q < nb; ++q) { b2 += part_b[q]; r2 += part_r[q]; }
  FgState t{};
  t.bnorm = sqrt(b2);
  t.beta = sqrt(r2);
  t.rel = t.bnorm > 0.0 ? t.beta / t.bnorm : 0.0;
  t.true_rel = t.rel;
  t.bzero = !(t.bnorm > 0.0);
  t.nan = !(t.beta == t.beta) || !(t.bnorm == t.bnorm);
  t.converged = t.bzero || t.rel < tol;
  t.done = t.bzero || t.nan || t.rel < tol || max_iters <= 0;
  *st = t;
  for (int i = 0; i < m1; ++i) g[i] = 0.0;
  g[0] = t.beta;
  cudaGraphSetConditional(cond, t.done ? 0u : 1u);
}
// V[0] /= beta while the solve goes on (after k_fg_init or a restart)
__global__ void k_fg_scale_v0(long long n, double* V, const FgState* st, int after_restart) {
  pdl_wait_release();
  if (st->done || (after_restart && !st->cycle_end)) return;
  const double inv = 1.0 / st->beta;
  GRID_LOOP(i, n) V[i] *= inv;
}
// preconditioner input: V[j] ./ wt in the V-cycle's precision; a new pass
// clears the cycle-end flag of the previous one
template <typename T>
__global__ void k_fg_prec_in(long long n, double* __restrict__ V, const double* __restrict__ wt,
                             T* __restrict__ out, FgState* st) {
  pdl_wait_release();
  const long long j = st->j;
  // V[j] (j > 0) still holds the orthogonalised w of the last iteration: it is
  // normalised here, times 1 / ||w|| (||w||^2 from k_fg_update), and written back
  const bool sc = j > 0;
  const double inv = sc ? 1.0 / sqrt(st->wn2) : 1.0;
  GRID_LOOP(i, n) {
    double v = V[j * n + i];
    if (sc) {
      v *= inv;
      V[j * n + i] = v;
    }
    out[i] = (T)(v / wt[i]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->cycle_end = 0;
}
// k_fg_prec_in fused with the V-cycle's first level-0 sweep from zero
// (Y_SMOOTH0, same arithmetic): b = V[j] ./ wt and x = w inv b
template <typename T>
__global__ void k_fg_prec_smooth0(long long n, double* __restrict__ V, const double* __restrict__ wt,
                                  const T* __restrict__ inv, T* __restrict__ b, T* __restrict__ x, FgState* st) {
  pdl_wait_release();
  const long long j = st->j;
  const bool sc = j > 0;   // normalise V[j] as k_fg_prec_in does
  const double iw = sc ? 1.0 / sqrt(st->wn2) : 1.0;
  GRID_LOOP(i, n) {
    double v = V[j * n + i];
    if (sc) {
      v *= iw;
      V[j * n + i] = v;
    }
    const T bi = (T)(v / wt[i]);
    b[i] = bi;
    x[i] = T(kOmega) * inv[i] * bi;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->cycle_end = 0;
}
// Z[j] = z (the preconditioner's output, widened exactly to fp64) and
// V[j+1] = wt .* (A_s z), LPR lanes per row (the level-0 Y_W_AX product)
template <typename XT, typename CT, int LPR>
__global__ void __launch_bounds__(TB) k_fg_op(int n, const int* __restrict__ rowptr, const CT* __restrict__ col,
                                              const double* __restrict__ val, const XT* __restrict__ x,
                                              double* __restrict__ Z, const double* __restrict__ wt,
                                              double* __restrict__ V, int rel, const FgState* st) {
  pdl_wait_release();
  const long long j = st->j;
  double* zj = Z + j * n;
  double* y = V + (j + 1) * (long long)n;
  const int g = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  const int rows_per_block = TB / LPR;
  for (long long row = (long long)blockIdx.x * rows_per_block + g; row < n;
       row += (long long)gridDim.x * rows_per_block) {
    double acc = 0.0;
    const int a = rowptr[row], e = rowptr[row + 1];
    const int cb = col_base<CT>(row, rel);
    acc = row_dot(a + lane, e, LPR, val, col, x, cb, acc);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
    if (lane == 0) {
      y[row] = wt[row] * acc;
      zj[row] = (double)x[row];
    }
  }
}
// Gram-Schmidt dots of pass `pass` against w = V[j+1]: pass 0 over V[0..j] and
// w.w (k_multidot_g's self); pass 1 only when the reorth flag is set.
__global__ void __launch_bounds__(TB, 4) k_fg_multidot(long long n, const double* __restrict__ V,
                                                    double* __restrict__ partial, double* __restrict__ H, int ldh,
                                                    double* __restrict__ y, FgState* st, int pass) {
  pdl_wait_release();
  if (pass == 1 && !st->reorth) return;
  const int j = st->j, k = j + 1, self = pass == 0;
  const int q0 = blockIdx.y * kMD;
  if (q0 >= k + self) return;
  const double* w = V + (long long)(j + 1) * n;
  __shared__ double sm[kMD][TB / 32];
  __shared__ int s_last;
  double acc[kMD];
#pragma unroll
  for (int u = 0; u < kMD; ++u) acc[u] = 0.0;
  multidot_acc(acc, n, V, n, q0, k, self, w);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int u = 0; u < kMD; ++u) {
    double v = warp_sum(acc[u]);
    if (lane == 0) sm[u][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kMD && q0 + (int)threadIdx.x < k + self) {
    double t = 0.0;
    for (int u = 0; u < TB / 32; ++u) t += sm[threadIdx.x][u];
    partial[(q0 + threadIdx.x) * kDotBlocks + blockIdx.x] = t;
    __threadfence();
  }
  __syncthreads();
  // the last block of the launch to finish sums every dot's partials in block
  // order (warp w takes dots w, w + 8, ...): into column j of H in pass 0
  // (entry j + 1 is ||w||^2 until k_fg_column), into y in pass 1
  if (threadIdx.x == 0) {
    const int active = kDotBlocks * ((k + self + kMD - 1) / kMD);
    s_last = atomicAdd(&st->gs_count, 1) == active - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double* out = pass == 0 ? H + (long long)j * ldh : y;
  for (int q = wid; q < k + self; q += TB / 32) {
    double t = 0.0;
    for (int b = lane; b < kDotBlocks; b += 32) t += __ldcg(partial + (long long)q * kDotBlocks + b);
    t = warp_sum(t);
    if (lane == 0) out[q] = t;
  }
  if (threadIdx.x == 0) st->gs_count = 0;
}
// w -= sum_q h_q V[q] (h = column j of H, or y in pass 1); the last block to
// finish sums the blocks' partial squares (||w||^2, FgState::wn2) and, after
// pass 0, sets the reorthogonalisation flag, which also opens the conditional
// node of pass 1
__global__ void __launch_bounds__(TB) k_fg_update(long long n, double* __restrict__ V, const double* __restrict__ H,
                                                  int ldh, const double* __restrict__ y,
                                                  double* __restrict__ partial, FgState* st, int pass,
                                                  cudaGraphConditionalHandle reorth_if) {
  pdl_wait_release();
  if (pass == 1 && !st->reorth) return;
  __shared__ double sh[128];
  __shared__ double sm[TB / 32];
  __shared__ int s_last;
  const int j = st->j, k = j + 1;
  const double* h = pass == 0 ? H + (long long)j * ldh : y;
  for (int q = threadIdx.x; q < k; q += blockDim.x) sh[q] = h[q];
  __syncthreads();
  double* w = V + (long long)(j + 1) * n;
  const double acc = update_rows(n, V, n, sh, k, w);
  double t = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int q = 0; q < TB / 32; ++q) u += sm[q];
    partial[blockIdx.x] = u;
    __threadfence();
    s_last = atomicAdd(&st->gs_count, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x >= 32) return;
  __threadfence();
  double nt = 0.0;
  for (int b = threadIdx.x; b < kDotBlocks; b += 32) nt += __ldcg(partial + b);
  nt = warp_sum(nt);
  if (threadIdx.x == 0) {
    st->gs_count = 0;
    st->wn2 = nt;
    if (pass == 0) {
      st->reorth = nt < 0.49 * H[(long long)st->j * ldh + st->j + 1];
      st->reorths += st->reorth;
      cudaGraphSetConditional(reorth_if, st->reorth ? 1u : 0u);
    }
  }
}
// Column j of the Hessenberg matrix in one block: the reorthogonalisation
// terms and h[j+1][j], then on thread 0 the Givens rotation (k_givens), the
// estimate |g[j+1]|, the counters, the continue/cycle-end decision and, at a
// cycle's end, y = R^-1 g (k_backsolve over the j columns).
__global__ void k_fg_column(double* H, int ldh, double* cs, double* sn, double* g, double* y, FgState* st,
                            double tol, int max_iters, int m, cudaGraphConditionalHandle cond,
                            cudaGraphConditionalHandle end_if) {
  pdl_wait_release();
  const int j = st->j;
  double* hj = H + (long long)j * ldh;
  if (st->reorth)
    for (int q = threadIdx.x; q <= j; q += blockDim.x) hj[q] += y[q];
  if (threadIdx.x == 0) hj[j + 1] = sqrt(st->wn2);
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int i = 0; i < j; ++i) {
    double t = cs[i] * hj[i] + sn[i] * hj[i + 1];
    hj[i + 1] = -sn[i] * hj[i] + cs[i] * hj[i + 1];
    hj[i] = t;
  }
  double a = hj[j], b = hj[j + 1];
  double d = hypot(a, b);
  double c = d > 0 ? a / d : 1.0, sv = d > 0 ? b / d : 0.0;
  cs[j] = c; sn[j] = sv;
  hj[j] = d; hj[j + 1] = 0.0;
  g[j + 1] = -sv * g[j];
  g[j] = c * g[j];
  const double est = fabs(g[j + 1]) / st->bnorm;
  st->rel = est;
  st->total += 1;
  st->j = j + 1;
  const bool nan = !(est == est);
  if (nan) st->nan = 1;
  const bool conv = est < tol;
  st->cycle_end = nan || conv || st->j >= m || st->total >= max_iters;
  cudaGraphSetConditional(end_if, st->cycle_end ? 1u : 0u);
  if (!st->cycle_end) {
    cudaGraphSetConditional(cond, 1u);
    return;
  }
  if (st->nan) return;
  const int k = st->j;
  for (int i = k - 1; i >= 0; --i) {
    double s = g[i];
    for (int jj = i + 1; jj < k; ++jj) s -= H[(long long)jj * ldh + i] * y[jj];
    y[i] = s / H[(long long)i * ldh + i];
  }
}
// at a cycle's end x_s += Z y ...
__global__ void k_fg_combine(long long n, const double* __restrict__ Z, const double* __restrict__ y,
                             double* __restrict__ x, const FgState* st) {
  pdl_wait_release();
  if (!st->cycle_end || st->nan) return;
  __shared__ double sy[128];
  const int k = st->j;
  for (int q = threadIdx.x; q < k; q += blockDim.x) sy[q] = y[q];
  __syncthreads();
  GRID_LOOP(i, n) x[i] = axpy_rows<1>(x[i], sy, k, Z, n, i);
}
// ... the true residual V[0] = wt .* (b_s - A_s x_s) and its norm partials ...
template <typename CT, int LPR>
__global__ void __launch_bounds__(TB) k_fg_resid(int n, const int* __restrict__ rowptr, const CT* __restrict__ col,
                                                 const double* __restrict__ val, const double* __restrict__ xs,
                                                 const double* __restrict__ bs, const double* __restrict__ wt,
                                                 double* __restrict__ V, int rel, double* __restrict__ partial,
                                                 const FgState* st) {
  pdl_wait_release();
  if (!st->cycle_end || st->nan) return;
  __shared__ double sm[TB / 32];
  const int g = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  const int rows_per_block = TB / LPR;
  double nrm = 0.0;
  for (long long row = (long long)blockIdx.x * rows_per_block + g; row < n;
       row += (long long)gridDim.x * rows_per_block) {
    double acc = 0.0;
    const int a = rowptr[row], e = rowptr[row + 1];
    const int cb = col_base<CT>(row, rel);
    acc = row_dot(a + lane, e, LPR, val, col, xs, cb, acc);
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
    if (lane == 0) {
      const double v = wt[row] * (bs[row] - acc);
      V[row] = v;
      nrm += v * v;
    }
  }
  double t = warp_sum(nrm);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int q = 0; q < TB / 32; ++q) u += sm[q];
    partial[blockIdx.x] = u;
  }
}
// ... and the decision: stop (converged in the true residual, or the cap) or
// restart with g = beta e_1.
__global__ void k_fg_restart(const double* partial, int nb, FgState* st, double* g, int m1, double tol,
                             int max_iters, cudaGraphConditionalHandle cond) {
  pdl_wait_release();
  if (!st->cycle_end) return;
  if (st->nan) {
    st->done = 1;
    st->converged = 0;
    cudaGraphSetConditional(cond, 0u);
    return;
  }
  double r2 = 0.0;
  for (int q = 0; q < nb; ++q) r2 += partial[q];
  const double beta = sqrt(r2);
  st->beta = beta;
  st->true_rel = beta / st->bnorm;
  st->rel = st->true_rel;
  st->restarts += 1;
  if (!(beta == beta)) st->nan = 1;
  st->converged = st->true_rel < tol;
  st->done = st->nan || st->converged || st->total >= max_iters;
  if (!st->done) {
    st->j = 0;
    for (int i = 0; i < m1; ++i) g[i] = 0.0;
    g[0] = beta;
  }
  cudaGraphSetConditional(cond, st->done ? 0u : 1u);
}
__global__ void k_fg_final(long long n, const double* dhalf, const double* xs, double* x, const FgState* st) {
  pdl_wait_release();
  const bool zero = st->bzero;
  GRID_LOOP(i, n) x[i] = zero ? 0.0 : dhalf[i] * xs[i];
}
// residual-norm partials of a plain vector (the FGMRES right-hand side)
__global__ void __launch_bounds__(TB) k_fg_norm_partials(long long n, const double* __restrict__ v,
                                                         double* __restrict__ partial) {
  pdl_wait_release();
  __shared__ double sm[TB / 32];
  double acc = 0.0;
  GRID_LOOP(i, n) acc += v[i] * v[i];
  double t = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double u = 0.0;
    for (int q = 0; q < TB / 32; ++q) u += sm[q];
    partial[blockIdx.x] = u;
  }
}

// k_fg_op on level 0's 7-diagonal DIA copy (fp64 values): the loads of a row
// issued together, x indices clamped as in k_dia_n
template <typename XT>
__global__ void __launch_bounds__(TB) k_fg_op_dia(int n, DiaOffsets o, const double* __restrict__ val,
                                                  const XT* __restrict__ x, double* __restrict__ Z,
                                                  const double* __restrict__ wt, double* __restrict__ V,
                                                  const FgState* st) {
  pdl_wait_release();
  const long long j = st->j;
  double* zj = Z + j * n;
  double* y = V + (j + 1) * (long long)n;
  for (int i = blockIdx.x * TB + threadIdx.x; i < n; i += gridDim.x * TB) {
    double v[7];
    XT xv[7];
#pragma unroll
    for (int d = 0; d < 7; ++d) {
      int c = i + o.off[d];
      c = c < 0 ? 0 : (c >= n ? n - 1 : c);
      v[d] = val[(long long)d * n + i];
      xv[d] = x[c];
    }
    double acc = 0.0;
#pragma unroll
    for (int d = 0; d < 7; ++d) acc += v[d] * xv[d];
    y[i] = wt[i] * acc;
    zj[i] = (double)x[i];
  }
}

// level-0 products of the device FGMRES: the DIA copy when the level's fp64
// sweeps use it, else CSR with the lanes per row the level was tuned to
template <typename XT, typename CT>
void fg_op(const Level& L0, const CT* col, const XT* z, double* Z, const double* wt, double* V, int rel,
           const FgState* st, cudaStream_t s) {
  const int n = L0.n;
  if (L0.dia_on[0] && L0.dia_nd == 7 && L0.dia_val.p) {
    DiaOffsets o{};
    for (int d = 0; d < Level::kDiaMax; ++d) o.off[d] = L0.dia_off[d];
    launch_pdl(k_fg_op_dia<XT>, grid_for(n, TB, 16), TB, 0, s, n, o, (const double*)L0.dia_val.p, z, Z, wt, V, st);
    return;
  }
  const int lpr = L0.lpr_a[0] > 0 ? L0.lpr_a[0] : (L0.avg_row <= 8 ? 1 : L0.avg_row <= 16 ? 4 : 8);
  auto grid = [&](int l) { return grid_for(((size_t)n * l + TB - 1) / TB * TB, TB, 16); };
  switch (lpr) {
    case 1: launch_pdl(k_fg_op<XT, CT, 1>, grid(1), TB, 0, s, n, L0.rowptr.p, col, L0.val.p, z, Z, wt, V, rel, st); break;
    case 2: launch_pdl(k_fg_op<XT, CT, 2>, grid(2), TB, 0, s, n, L0.rowptr.p, col, L0.val.p, z, Z, wt, V, rel, st); break;
    case 4: launch_pdl(k_fg_op<XT, CT, 4>, grid(4), TB, 0, s, n, L0.rowptr.p, col, L0.val.p, z, Z, wt, V, rel, st); break;
    default: launch_pdl(k_fg_op<XT, CT, 8>, grid(8), TB, 0, s, n, L0.rowptr.p, col, L0.val.p, z, Z, wt, V, rel, st); break;
  }
}
template <typename CT>
void fg_resid(const Level& L0, const CT* col, const double* xs, const double* bs, const double* wt, double* V,
              int rel, double* partial, const FgState* st, cudaStream_t s) {
  const int n = L0.n;
  // a fixed grid of kDotBlocks blocks: the partials are summed in block order
  launch_pdl(k_fg_resid<CT, 1>, kDotBlocks, TB, 0, s, n, L0.rowptr.p, col, L0.val.p, xs, bs, wt, V, rel, partial,
             st);
}

// Appends an IF conditional node on `hc` to the graph that `s` is capturing,
// captures emit(q) into the node's body on the handle's third stream, and
// continues the capture of `s` after the node.
template <typename F>
void capture_if(cudaStream_t s, AMG& h, cudaGraphConditionalHandle hc, F emit) {
  cudaStreamCaptureStatus cst;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  IMPES_CUDA(cudaStreamGetCaptureInfo(s, &cst, nullptr, &g, &deps, &ndeps));
  IMPES_REQUIRE(cst == cudaStreamCaptureStatusActive, IMPES_ERR_STATE, "conditional block needs a capturing stream");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  IMPES_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
  if (!h.if_stream) IMPES_CUDA(cudaStreamCreateWithFlags(&h.if_stream, cudaStreamNonBlocking));
  IMPES_CUDA(cudaStreamBeginCaptureToGraph(h.if_stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
  try {
    emit(h.if_stream);
  } catch (...) {
    cudaGraph_t dummy = nullptr;
    cudaStreamEndCapture(h.if_stream, &dummy);
    throw;
  }
  cudaGraph_t out = nullptr;
  IMPES_CUDA(cudaStreamEndCapture(h.if_stream, &out));
  IMPES_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
}
}  // namespace

void amg_fgmres_prepare(AMG& h, const impes_krylov_params& kp) {
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  const int m = std::max(1, std::min(kp.restart, 120));
  if (h.krylov_m != m || h.V.n < (size_t)(m + 1) * n) {
    h.V.alloc((size_t)(m + 1) * n);
    h.Z.alloc((size_t)m * n);
    h.H.alloc((size_t)(m + 2) * (m + 1));
    h.cs.alloc(m + 1); h.sn.alloc(m + 1); h.g.alloc(m + 2); h.y.alloc(m + 1);
    h.kw.alloc(n); h.kb.alloc(n); h.kx.alloc(n);
    h.krylov_m = m;
  }
  h.red.ensure((size_t)(m + 2) * kDotBlocks + 2 * kDotBlocks);
  h.fgst.ensure(1);
  if (kp.precision == 1)
    IMPES_REQUIRE(h.prm.mixed_precision, IMPES_ERR_STATE, "fp32 V-cycle needs mixed_precision=1");
}

void amg_fgmres_capture(AMG& h, const double* b, double* x, const impes_krylov_params& kp, cudaStream_t s) {
  KrylovModeGuard guard(h);
  Level& L0 = *h.levels[0];
  const long long n = L0.n;
  const int m = h.krylov_m;
  const int ldh = m + 2;
  const bool jac = kp.norm == IMPES_NORM_JACOBI;
  double* wt = jac ? h.jac_w.p : h.kw.p;
  double* bs = h.kb.p;
  double* xs = h.kx.p;
  double* part_b = h.red.p + (size_t)(m + 2) * kDotBlocks;
  double* part_r = part_b + kDotBlocks;
  FgState* st = h.fgst.p;
  const unsigned gn = grid_for(n, TB);
  // prologue: b_s, x_s, ||wt b_s||, V[0] = wt (b_s - A x_s) and its norm
  if (!jac) launch_pdl(k_fill, gn, TB, 0, s, n, h.kw.p, 1.0);
  launch_pdl(k_mul, gn, TB, 0, s, n, (const double*)h.dhalf_inv.p, b, bs);
  if (kp.use_x0)
    launch_pdl(k_div_convert<double, double>, gn, TB, 0, s, n, (const double*)x, (const double*)h.dhalf_inv.p, xs);
  else
    launch_pdl(k_zero, gn, TB, 0, s, n, xs);
  launch_pdl(k_mul, gn, TB, 0, s, n, (const double*)wt, (const double*)bs, h.V.p);
  launch_pdl(k_fg_norm_partials, kDotBlocks, TB, 0, s, n, (const double*)h.V.p, part_b);
  launch_csr<double, Y_B_MINUS_AX>((int)n, L0.avg_row, L0.rowptr.p, L0.col.p, L0.val.p, xs, bs, nullptr, h.V.p, s,
                                   L0.col16.p, L0.col16_rel, L0.lpr_a[0]);
  launch_pdl(k_mul_inplace, gn, TB, 0, s, n, h.V.p, (const double*)wt);
  launch_pdl(k_fg_norm_partials, kDotBlocks, TB, 0, s, n, (const double*)h.V.p, part_r);
  // the while node; the init kernel sets its condition (0: nothing to do)
  cudaStreamCaptureStatus cst;
  cudaGraph_t cap = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  IMPES_CUDA(cudaStreamGetCaptureInfo(s, &cst, nullptr, &cap, &deps, &ndeps));
  IMPES_REQUIRE(cst == cudaStreamCaptureStatusActive, IMPES_ERR_STATE, "device FGMRES needs a capturing stream");
  cudaGraphConditionalHandle cond;
  IMPES_CUDA(cudaGraphConditionalHandleCreate(&cond, cap, 1, cudaGraphCondAssignDefault));
  launch_pdl(k_fg_init, 1, 1, 0, s, st, (const double*)part_b, (const double*)part_r, (int)kDotBlocks, kp.tol,
             kp.max_iters, m + 1, h.g.p, cond);
  launch_pdl(k_fg_scale_v0, gn, TB, 0, s, n, h.V.p, (const FgState*)st, 0);
  IMPES_CUDA(cudaStreamGetCaptureInfo(s, &cst, nullptr, &cap, &deps, &ndeps));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t wnode;
  IMPES_CUDA(cudaGraphAddNode(&wnode, cap, deps, ndeps, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // the body, captured on a second stream into the node's graph
  if (!h.body_stream) IMPES_CUDA(cudaStreamCreateWithFlags(&h.body_stream, cudaStreamNonBlocking));
  cudaStream_t bsm = h.body_stream;
  IMPES_CUDA(cudaStreamBeginCaptureToGraph(bsm, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  const unsigned long long body_start = thread_launches();
  try {
    const unsigned gb = grid_for(n, TB);
    // z = M^-1 (V[j] / wt); Z[j] = z is written by the operator kernel
    // the l1-Jacobi V-cycle's first level-0 sweep is fused with the input
    // conversion (not for Chebyshev smoothing or a one-level hierarchy)
    const bool fuse0 = h.prm.smoother != IMPES_SMOOTHER_CHEBYSHEV && !L0.coarsest;
    if (kp.precision == 1) {
      if (fuse0)
        launch_pdl(k_fg_prec_smooth0<float>, gb, TB, 0, bsm, n, h.V.p, (const double*)wt,
                   (const float*)L0.inv_relaxf.p, L0.bf.p, L0.xf.p, st);
      else
        launch_pdl(k_fg_prec_in<float>, gb, TB, 0, bsm, n, h.V.p, (const double*)wt, L0.bf.p, st);
      const float* zf = vcycle<float>(h, 0, true, bsm, fuse0);
      if (L0.col16.p)
        fg_op(L0, (const unsigned short*)L0.col16.p, zf, h.Z.p, wt, h.V.p, L0.col16_rel, st, bsm);
      else
        fg_op(L0, (const int*)L0.col.p, zf, h.Z.p, wt, h.V.p, 0, st, bsm);
    } else {
      if (fuse0)
        launch_pdl(k_fg_prec_smooth0<double>, gb, TB, 0, bsm, n, h.V.p, (const double*)wt,
                   (const double*)L0.inv_relax.p, L0.b.p, L0.x.p, st);
      else
        launch_pdl(k_fg_prec_in<double>, gb, TB, 0, bsm, n, h.V.p, (const double*)wt, L0.b.p, st);
      const double* zd = vcycle<double>(h, 0, true, bsm, fuse0);
      if (L0.col16.p)
        fg_op(L0, (const unsigned short*)L0.col16.p, zd, h.Z.p, wt, h.V.p, L0.col16_rel, st, bsm);
      else
        fg_op(L0, (const int*)L0.col.p, zd, h.Z.p, wt, h.V.p, 0, st, bsm);
    }
    // Gram-Schmidt: pass 0, then pass 1 inside an IF node that k_fg_update opens
    // when the first pass lost too much of the vector's norm
    const dim3 gd(kDotBlocks, (unsigned)((m + 2 + kMD - 1) / kMD));
    cudaGraphConditionalHandle reorth_if, end_if;
    IMPES_CUDA(cudaGraphConditionalHandleCreate(&reorth_if, body, 0, cudaGraphCondAssignDefault));
    IMPES_CUDA(cudaGraphConditionalHandleCreate(&end_if, body, 0, cudaGraphCondAssignDefault));
    auto gs_pass = [&](int pass, cudaStream_t q) {
      launch_pdl(k_fg_multidot, gd, dim3(TB), 0, q, n, (const double*)h.V.p, h.red.p, h.H.p, ldh, h.y.p, st, pass);
      launch_pdl(k_fg_update, kDotBlocks, TB, 0, q, n, h.V.p, (const double*)h.H.p, ldh, (const double*)h.y.p,
                 h.red.p, st, pass, reorth_if);
    };
    gs_pass(0, bsm);
    unsigned long long mark = thread_launches();
    capture_if(bsm, h, reorth_if, [&](cudaStream_t q) { gs_pass(1, q); });
    h.fg_reorth_kernels = (long long)(thread_launches() - mark);
    // (V[j+1] is normalised by the next iteration's input kernel)
    launch_pdl(k_fg_column, 1, 128, 0, bsm, h.H.p, ldh, h.cs.p, h.sn.p, h.g.p, h.y.p, st, kp.tol, kp.max_iters, m,
               cond, end_if);
    // a cycle's end (IF node opened by k_fg_column): x_s += Z y, the true
    // residual, the restart/stop decision and the new V[0]
    mark = thread_launches();
    capture_if(bsm, h, end_if, [&](cudaStream_t q) {
      launch_pdl(k_fg_combine, gb, TB, 0, q, n, (const double*)h.Z.p, (const double*)h.y.p, xs, (const FgState*)st);
      if (L0.col16.p)
        fg_resid<unsigned short>(L0, L0.col16.p, xs, bs, wt, h.V.p, L0.col16_rel, part_r, st, q);
      else
        fg_resid<int>(L0, L0.col.p, xs, bs, wt, h.V.p, 0, part_r, st, q);
      launch_pdl(k_fg_restart, 1, 1, 0, q, (const double*)part_r, (int)kDotBlocks, st, h.g.p, m + 1, kp.tol,
                 kp.max_iters, cond);
      launch_pdl(k_fg_scale_v0, gb, TB, 0, q, n, h.V.p, (const FgState*)st, 1);
    });
    h.fg_end_kernels = (long long)(thread_launches() - mark);
  } catch (...) {
    cudaGraph_t dummy = nullptr;
    cudaStreamEndCapture(bsm, &dummy);
    throw;
  }
  cudaGraph_t body_out = nullptr;
  IMPES_CUDA(cudaStreamEndCapture(bsm, &body_out));
  h.fg_body_kernels = (long long)(thread_launches() - body_start) - h.fg_reorth_kernels - h.fg_end_kernels;
  IMPES_CUDA(cudaStreamUpdateCaptureDependencies(s, &wnode, 1, cudaStreamSetCaptureDependencies));
  // epilogue: x = D^-1/2 x_s (zero for a zero right-hand side)
  launch_pdl(k_fg_final, gn, TB, 0, s, n, (const double*)h.dhalf_inv.p, (const double*)xs, x, (const FgState*)st);
}

}  // namespace impes

// ============================================================ no-alloc solve
// Work space of impes_amg_solve_vcycles_noalloc: the scaled right-hand side, the
// residual and the weighted right-hand side (3 vectors of up to
// kNoAllocMaxRows doubles, 6 MiB).  It is static device storage: every GPU that
// loads this library holds it until the process exits, and every call on a
// device shares it.
namespace impes {
constexpr int kNoAllocMaxRows = 262144;
}
static __device__ __align__(256) double g_solve_scratch[3 * (size_t)impes::kNoAllocMaxRows];

namespace impes {
namespace {
std::mutex g_scratch_mu;
double* g_scratch_dev[128] = {};
void* g_scratch_ctx[128] = {};

// The driver context current on this thread (CUcontext as void*), through the
// runtime's driver entry point so the library needs no link to libcuda; null
// when the entry point is unavailable.
void* current_context() {
  using CtxGetCurrent = int (*)(void**);
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of g_solve_scratch on the current device, looked up with that
// device current (the host-side symbol is not a device address) on the first
// call per device, and again only if the device's context has changed since
// (after cudaDeviceReset the module is loaded anew and the array may move).
double* solve_scratch() {
  int dev = 0;
  IMPES_CUDA(cudaGetDevice(&dev));
  IMPES_REQUIRE(dev >= 0 && dev < 128, IMPES_ERR_ARG, "device ordinal out of range");
  void* ctx = current_context();
  if (!ctx) {                      // no context current on this thread yet
    IMPES_CUDA(cudaSetDevice(dev));
    ctx = current_context();
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_dev[dev] || g_scratch_ctx[dev] != ctx) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_solve_scratch);
    if (e != cudaSuccess || !ptr)
      throw Error(IMPES_ERR_CUDA, std::string("cudaGetSymbolAddress(g_solve_scratch): ") +
                                      cudaGetErrorString(e));
    g_scratch_dev[dev] = static_cast<double*>(ptr);
    g_scratch_ctx[dev] = ctx;
  }
  return g_scratch_dev[dev];
}

// The stand-alone V-cycle solve of amg_solve_vcycles with its three vectors in
// the static array and the V-cycles launched directly (no graph instantiation).
void solve_vcycles_noalloc(AMG& h, const double* b, double* x, double tol, int max_cycles,
                           int* cycles, double* rel, int norm, cudaStream_t s) {
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  IMPES_REQUIRE(n <= kNoAllocMaxRows, IMPES_ERR_ARG,
                "impes_amg_solve_vcycles_noalloc: n exceeds the 262144-row static work space");
  IMPES_REQUIRE(h.red.n >= (size_t)kMD * kDotBlocks, IMPES_ERR_STATE, "hierarchy not set up");
  amg_ensure_fp64(h, s);
  double* base = solve_scratch();
  double* bs = base;
  double* r = base + kNoAllocMaxRows;
  double* wb = base + 2 * (size_t)kNoAllocMaxRows;
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, b, bs);
  IMPES_CHECK_LAUNCH();
  const bool jac = norm == IMPES_NORM_JACOBI;
  if (jac) { launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.jac_w.p, bs, wb); }
  const double bn = std::sqrt(jac ? dot_host(h, wb, wb, n, s) : dot_host(h, bs, bs, n, s));
  IMPES_CUDA(cudaMemcpyAsync(L0.b.p, bs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  double rr = INFINITY;
  int c = 0;
  for (c = 1; c <= max_cycles; ++c) {
    double* xs = vcycle<double>(h, 0, c == 1, s);
    if (xs != L0.x.p)
      IMPES_CUDA(cudaMemcpyAsync(L0.x.p, xs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    launch_csr<double, Y_B_MINUS_AX>(n, L0.avg_row, L0.rowptr.p, L0.col.p, L0.val.p, L0.x.p, bs,
                                     nullptr, r, s);
    if (jac) { launch_pdl(k_mul_inplace, grid_for(n, TB), TB, 0, s, n, r, h.jac_w.p); }
    rr = std::sqrt(dot_host(h, r, r, n, s)) / (bn + 1e-30);
    if (!(rr == rr)) throw Error(IMPES_ERR_NAN, "NaN residual in V-cycle solve");
    if (rr < tol) break;
  }
  if (c > max_cycles) c = max_cycles;
  launch_pdl(k_mul, grid_for(n, TB), TB, 0, s, n, h.dhalf_inv.p, L0.x.p, x);
  IMPES_CHECK_LAUNCH();
  if (cycles) *cycles = c;
  if (rel) *rel = rr;
}
}  // namespace
}  // namespace impes

extern "C" int impes_amg_solve_vcycles_noalloc(impes_amg* h, const double* b, double* x, double tol,
                                               int max_cycles, int* cycles, double* rel_res, int norm,
                                               void* stream) {
  try {
    IMPES_REQUIRE(h && b && x, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(impes_amg_handle_built(h), IMPES_ERR_STATE, "solve before setup");
    IMPES_REQUIRE(max_cycles >= 1, IMPES_ERR_ARG, "max_cycles must be >= 1");
    impes::solve_vcycles_noalloc(*impes_amg_handle_core(h), b, x, tol, max_cycles, cycles, rel_res, norm,
                                 reinterpret_cast<cudaStream_t>(stream));
    return IMPES_OK;
  } catch (const impes::Error& e) {
    impes::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    impes::set_last_error(e.what());
    return IMPES_ERR_ARG;
  }
}
