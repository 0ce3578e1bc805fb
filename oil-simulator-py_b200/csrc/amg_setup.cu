// Ruge-Stueben AMG setup and matrix update on the device.
//
// Reference: researchim-ai/oil-simulator-py src/solver/classical_amg.py
//   find_strong_connections :34-82, classical_coarsening :85-146,
//   build_prolongation_rs_full :149-427, solve_energy_weights :1469-1501,
//   generate_nullspace / orthonormalize_columns :1395-1466, _csr_spmm/rap_torch
//   :519-657, ClassicalAMG.__init__ :699-938, update_matrix :1308-1392.
//
// Setup runs once per hierarchy (host-orchestrated, it syncs for sizes);
// amg_update() is the per-step path: equilibration + Galerkin numeric products
// for every level on a frozen pattern, all on the stream without host syncs.
//
// Galerkin products use a two-level "union" SpGEMM: the symbolic phase forms
// each output row as the union of inner rows selected by an outer row, through a
// per-warp open-addressing hash table in shared memory; the numeric phase keeps
// each output row in shared memory and accumulates inner rows one outer entry at
// a time (lanes own distinct output columns, so the sums are deterministic).
#include "amg.cuh"
#include <algorithm>
#include <cmath>

namespace impes {
namespace {

constexpr int TB = 256;

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Deterministic [0,1) tie-break replacing torch.rand (classical_amg.py:125).
__device__ __forceinline__ double tiebreak(uint32_t seed, int level, int i) {
  uint64_t key = ((uint64_t)(seed & 0xFFFFFFu) << 40) | ((uint64_t)(level & 0xFF) << 32) |
                 (uint64_t)(uint32_t)i;
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

#define GRID_LOOP(i, n) \
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// ------------------------------------------------------------ validation
__global__ void k_validate_csr(int n, int nnz, const int* rowptr, const int* col, int* flag) {
  GRID_LOOP(i, n) {
    int a = rowptr[i], b = rowptr[i + 1];
    if (a > b || a < 0 || b > nnz) atomicOr(flag, 1);
    for (int e = a; e < b && e < nnz && e >= 0; ++e) {
      int c = col[e];
      if (c < 0 || c >= n) atomicOr(flag, 2);
      if (e > a && col[e - 1] >= c) atomicOr(flag, 4);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (rowptr[0] != 0 || rowptr[n] != nnz) atomicOr(flag, 1);
  }
}

__global__ void k_nonfinite(const double* v, long long n, int* flag) {
  GRID_LOOP(i, n) if (!isfinite(v[i])) atomicOr(flag, 8);
}

// ------------------------------------------------------- diag / scaling
// _extract_diag (classical_amg.py:940-955): value of the diagonal entry, 0 if none.
__global__ void k_narrow_cols(int nnz, const int* col, unsigned short* col16) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz;
       e += (long long)gridDim.x * blockDim.x)
    col16[e] = (unsigned short)col[e];
}
// flag = 1 when some entry lies more than 32768 columns left or 32767 right of
// its row (the row-relative 16-bit form cannot hold it)
__global__ void k_rel16_check(int n, const int* rowptr, const int* col, int* flag) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
      const long long d = (long long)col[e] - r;
      if (d < -32768 || d > 32767) { atomicOr(flag, 1); break; }
    }
  }
}
__global__ void k_narrow_cols_rel(int n, const int* rowptr, const int* col, unsigned short* col16) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x)
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) col16[e] = (unsigned short)(col[e] - r + 32768);
}
__global__ void k_diag(int n, const int* rowptr, const int* col, const double* val, double* d) {
  GRID_LOOP(i, n) {
    double v = 0.0;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
      if (col[e] == i) v = val[e];
    d[i] = v;
  }
}
// count of |d| (clamped at 1e-30) below the threshold -> lower-median test
__global__ void k_count_below(int n, const double* d, double thr, int* cnt) {
  int local = 0;
  GRID_LOOP(i, n) local += (fmax(fabs(d[i]), 1e-30) < thr);
  local = warp_sum_int(local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(cnt, local);
}
// dhalf = D^-1/2 when the lower median of |diag| is below the threshold, else 1;
// Jacobi weights of the FGMRES norm in the scaled space.
__global__ void k_equil_prepare(int n, const double* d, const int* below, double* dh, double* jw,
                                int* flag_out) {
  const bool on = below[0] >= (n - 1) / 2 + 1;
  GRID_LOOP(i, n) {
    const double a = fmax(fabs(d[i]), 1e-30);
    const double hv = on ? 1.0 / sqrt(a) : 1.0;
    dh[i] = hv;
    jw[i] = on ? hv : 1.0 / a;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *flag_out = on ? 1 : 0;
}
// A_s = D^-1/2 A D^-1/2 as vals * dh[row] * dh[col] (classical_amg.py:776-780)
// with dval set, also into the level's DIA copy (dval[dmap[e]])
__global__ void k_equilibrate(int n, const int* rowptr, const int* col, const double* vin,
                              const double* dh, double* vout, const int* dmap, double* dval) {
  GRID_LOOP(i, n) {
    double di = dh[i];
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      const double v = vin[e] * di * dh[col[e]];
      vout[e] = v;
      if (dval) dval[dmap[e]] = v;
    }
  }
}

// l1-Jacobi weights (classical_amg.py:885-889, 1298-1306)
// With lmax non-null each row also contributes inv_i * sum_j |a_ij| to the
// Gershgorin bound of diag(inv) A (the Chebyshev smoother's interval), kept as
// the bits of a non-negative double so atomicMax orders them.
template <typename TO>
__device__ __forceinline__ void lmax_update(unsigned long long* lmax, TO inv, double ra) {
  if (lmax) atomicMax(lmax, (unsigned long long)__double_as_longlong((double)inv * ra));
}
template <typename TV, typename TO>
__global__ void k_inv_relax(int n, const int* rowptr, const int* col, const TV* val, TO* inv,
                            unsigned long long* lmax) {
  GRID_LOOP(i, n) {
    double d = 0.0, ra = 0.0;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      double v = val[e];
      if (col[e] == i) d = v;
      ra += fabs(v);
    }
    double denom = fmax(fabs(d), 0.3 * ra);
    denom = denom < 1e-30 ? 1e-30 : denom;
    double r = 1.0 / denom;
    const TO w = (TO)(r > 1e2 ? 1e2 : r);
    inv[i] = w;
    lmax_update(lmax, w, ra);
  }
}

// The same with LPR lanes per row (4 to 32, by the level's mean row length),
// so a row's entries load in about one round instead of one after another: the
// diagonal comes from the lane that holds it, the absolute row sum from a
// fixed-order reduction over the row's lanes.  The loop runs per warp (its
// first row decides), so every lane of a warp reaches the shuffles; rows past
// n only skip their loads.
template <typename TV, typename TO, int LPR>
__global__ void k_inv_relax_lanes(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                  const TV* __restrict__ val, TO* __restrict__ inv,
                                  unsigned long long* lmax) {
  const int lane = threadIdx.x % LPR;
  const long long rows_per_block = blockDim.x / LPR;
  const long long warp_row0 = blockIdx.x * rows_per_block + (threadIdx.x / 32) * (32 / LPR);
  for (long long w0 = warp_row0; w0 < n; w0 += gridDim.x * rows_per_block) {
    const long long i = w0 + (threadIdx.x % 32) / LPR;
    const bool live = i < n;
    double d = 0.0, ra = 0.0;
    if (live)
      for (int e = rowptr[i] + lane; e < rowptr[i + 1]; e += LPR) {
        const double v = val[e];
        if (col[e] == i) d = v;
        ra += fabs(v);
      }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) {
      ra += __shfl_down_sync(0xffffffffu, ra, o, LPR);
      d += __shfl_down_sync(0xffffffffu, d, o, LPR);   // one lane holds the diagonal
    }
    if (live && lane == 0) {
      double denom = fmax(fabs(d), 0.3 * ra);
      denom = denom < 1e-30 ? 1e-30 : denom;
      const double r = 1.0 / denom;
      const TO w = (TO)(r > 1e2 ? 1e2 : r);
      inv[i] = w;
      lmax_update(lmax, w, ra);
    }
  }
}

// --------------------------------------------------------------- strength
// find_strong_connections (classical_amg.py:34-82)
__global__ void k_strength(int n, const int* rowptr, const int* col, const double* val,
                           double theta, unsigned char* strong) {
  GRID_LOOP(i, n) {
    const int a = rowptr[i], b = rowptr[i + 1];
    double diag = 0.0;
    for (int e = a; e < b; ++e)
      if (col[e] == i) diag = fabs(val[e]);
    const double den = fabs(diag) + 1e-30;
    double mx = 0.0;
    for (int e = a; e < b; ++e) {
      double s = val[e] / den;
      bool cand = (col[e] != i) && (s < 0);
      double na = cand ? -s : 0.0;
      mx = fmax(mx, na);
    }
    const double thr = theta * mx;
    for (int e = a; e < b; ++e) {
      double s = val[e] / den;
      bool cand = (col[e] != i) && (s < 0);
      strong[e] = (cand && (-s >= thr)) ? 1 : 0;
    }
  }
}

// ------------------------------------------------- symmetric strong graph
__global__ void k_sym_count(int n, const int* rowptr, const int* col, const unsigned char* strong,
                            int* cnt) {
  GRID_LOOP(i, n) {
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
      if (strong[e]) { atomicAdd(&cnt[i], 1); atomicAdd(&cnt[col[e]], 1); }
  }
}
__global__ void k_sym_fill(int n, const int* rowptr, const int* col, const unsigned char* strong,
                           int* fill, int* gcol) {
  GRID_LOOP(i, n) {
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
      if (strong[e]) {
        int j = col[e];
        gcol[atomicAdd(&fill[i], 1)] = j;
        gcol[atomicAdd(&fill[j], 1)] = (int)i;
      }
  }
}
// sort + unique each row of the symmetric graph (the {min,max} coalesce at :113-116)
__global__ void k_sym_unique(int n, const int* gptr, int* gcol, int* ucnt) {
  GRID_LOOP(i, n) {
    int a = gptr[i], b = gptr[i + 1];
    for (int x = a + 1; x < b; ++x) {
      int v = gcol[x], y = x - 1;
      while (y >= a && gcol[y] > v) { gcol[y + 1] = gcol[y]; --y; }
      gcol[y + 1] = v;
    }
    int u = 0;
    for (int x = a; x < b; ++x)
      if (u == 0 || gcol[a + u - 1] != gcol[x]) gcol[a + u++] = gcol[x];
    ucnt[i] = u;
  }
}
// score = deg + 1e-3 * w (classical_amg.py:124-126)
__global__ void k_score(int n, const int* ucnt, uint32_t seed, int level, double* score) {
  GRID_LOOP(i, n) score[i] = (double)ucnt[i] + 1e-3 * tiebreak(seed, level, (int)i);
}
// C = score > neighbour max.  The reference's two scatter_reduce_(amax,
// include_self=False) passes (:129-132) leave, for every node with a
// lower-index neighbour, the max over lower-index neighbours only; else the max
// over higher-index neighbours; else 0.
__global__ void k_cselect(int n, const int* gptr, const int* gcol, const int* ucnt,
                          const double* score, unsigned char* C) {
  GRID_LOOP(i, n) {
    double lo = -INFINITY, up = -INFINITY;
    bool hlo = false, hup = false;
    for (int x = gptr[i]; x < gptr[i] + ucnt[i]; ++x) {
      int j = gcol[x];
      double s = score[j];
      if (j < i) { hlo = true; lo = fmax(lo, s); }
      else { hup = true; up = fmax(up, s); }
    }
    double nm = hlo ? lo : (hup ? up : 0.0);
    C[i] = score[i] > nm;
  }
}
// coverage lift (:136-141); has_C is int8 in the reference, so the count wraps mod 256
__global__ void k_lift(int n, const int* gptr, const int* gcol, const int* ucnt,
                       const unsigned char* C, signed char* cf, int* nc) {
  int local = 0;
  GRID_LOOP(i, n) {
    int h = 0;
    for (int x = gptr[i]; x < gptr[i] + ucnt[i]; ++x) h += C[gcol[x]];
    signed char f = C[i] ? 0 : (((h & 0xFF) == 0) ? 0 : 1);
    cf[i] = f;
    local += (f == 0);
  }
  local = warp_sum_int(local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(nc, local);
}
// orphan promotion (:178-189): F rows without a strong C neighbour become C
__global__ void k_orphans(int n, const int* rowptr, const int* col, const unsigned char* strong,
                          const signed char* cf_in, signed char* cf_out, int* cflag) {
  GRID_LOOP(i, n) {
    signed char f = cf_in[i];
    if (f == 1) {
      bool has = false;
      for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
        if (strong[e] && col[e] != i && cf_in[col[e]] == 0) { has = true; break; }
      if (!has) f = 0;
    }
    cf_out[i] = f;
    cflag[i] = (f == 0);
  }
}

// ----------------------------------------------------------- interpolation
// Per-row sums of build_prolongation_rs_full (:193-236).
__global__ void k_p_stats(int n, const int* rowptr, const int* col, const double* val,
                          const unsigned char* strong, const signed char* cf, double* pdiag,
                          double* ssum, double* wcsum, double* wfsum, int* scnt) {
  GRID_LOOP(i, n) {
    double d = 0.0, s = 0.0, wc = 0.0, wf = 0.0;
    int c = 0;
    const bool F = cf[i] == 1;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      int j = col[e];
      double v = val[e];
      if (j == i) { d += v; continue; }
      if (!F) continue;
      bool jC = cf[j] == 0;
      if (strong[e] && jC) { s += -v; ++c; }
      else if (!strong[e] && jC) wc += -v;
      else if (!strong[e] && !jC) wf += -v;
    }
    pdiag[i] = fabs(d) > 1e-14 ? d : 1.0;
    ssum[i] = s; wcsum[i] = wc; wfsum[i] = wf; scnt[i] = c;
  }
}
__device__ __forceinline__ bool ff_valid(int j, const int* scnt, const double* ssum) {
  return scnt[j] > 0 && ssum[j] > 1e-14;
}
__global__ void k_p_count(int n, const int* rowptr, const int* col, const unsigned char* strong,
                          const signed char* cf, const int* scnt, const double* ssum, int* cnt) {
  GRID_LOOP(i, n) {
    if (cf[i] == 0) { cnt[i] = 1; continue; }
    int c = scnt[i];
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) {
      int j = col[e];
      if (j != i && strong[e] && cf[j] == 1 && ff_valid(j, scnt, ssum)) c += scnt[j];
    }
    cnt[i] = c;
  }
}
__device__ __forceinline__ double nan_to_zero(double v) { return isfinite(v) ? v : 0.0; }

__global__ void k_p_fill(int n, const int* rowptr, const int* col, const double* val,
                         const unsigned char* strong, const signed char* cf, const int* f2c,
                         const double* pdiag, const double* ssum, const double* wcsum,
                         const double* wfsum, const int* scnt, const int* cptr, int* ccol,
                         double* cval) {
  GRID_LOOP(i, n) {
    int o = cptr[i];
    if (cf[i] == 0) { ccol[o] = f2c[i]; cval[o] = 1.0; continue; }
    const int a = rowptr[i], b = rowptr[i + 1];
    const double di = pdiag[i];
    double fws = wfsum[i];
    for (int e = a; e < b; ++e) {  // invalid F-F entries join the weak sum (:280-284)
      int j = col[e];
      if (j != i && strong[e] && cf[j] == 1 && !ff_valid(j, scnt, ssum)) fws += -val[e];
    }
    const double tw = wcsum[i] + fws;
    const double corr = ssum[i] > 1e-14 ? tw / ssum[i] : 0.0;
    for (int e = a; e < b; ++e) {  // direct RS weights (:240-246, 292-296)
      int j = col[e];
      if (j != i && strong[e] && cf[j] == 0) {
        double v = nan_to_zero(-val[e] / di) * (1.0 + corr);
        ccol[o] = f2c[j];
        cval[o] = v < 0.0 ? 0.0 : v;
        ++o;
      }
    }
    for (int e = a; e < b; ++e) {  // F-F distribution (:248-278)
      int j = col[e];
      if (j == i || !strong[e] || cf[j] != 1 || !ff_valid(j, scnt, ssum)) continue;
      const double fac = nan_to_zero(-val[e] / di);
      const double sj = ssum[j];
      for (int f = rowptr[j]; f < rowptr[j + 1]; ++f) {
        int c = col[f];
        if (c != j && strong[f] && cf[c] == 0) {
          double w = sj > 1e-14 ? -val[f] / sj : 0.0;
          double v = fac * w;
          ccol[o] = f2c[c];
          cval[o] = v < 0.0 ? 0.0 : v;
          ++o;
        }
      }
    }
  }
}
// stable sort by column and sum duplicates (the COO coalesce at :323-331)
__global__ void k_p_merge(int n, const int* cptr, int* ccol, double* cval, int* mcnt) {
  GRID_LOOP(i, n) {
    int a = cptr[i], b = cptr[i + 1];
    for (int x = a + 1; x < b; ++x) {
      int c = ccol[x]; double v = cval[x]; int y = x - 1;
      while (y >= a && ccol[y] > c) { ccol[y + 1] = ccol[y]; cval[y + 1] = cval[y]; --y; }
      ccol[y + 1] = c; cval[y + 1] = v;
    }
    int u = 0;
    for (int x = a; x < b; ++x) {
      if (u > 0 && ccol[a + u - 1] == ccol[x]) cval[a + u - 1] += cval[x];
      else { ccol[a + u] = ccol[x]; cval[a + u] = cval[x]; ++u; }
    }
    mcnt[i] = u;
  }
}
__global__ void k_p_compact(int n, const int* cptr, const int* ccol, const double* cval,
                            const int* prow, int* pcol, double* pval) {
  GRID_LOOP(i, n) {
    int a = cptr[i], o = prow[i], m = prow[i + 1] - prow[i];
    for (int x = 0; x < m; ++x) { pcol[o + x] = ccol[a + x]; pval[o + x] = cval[a + x]; }
  }
}
// row sums of F rows; zero rows need the injection fallback (:347-385)
__global__ void k_p_rowsum(int n, const int* prow, const double* pval, const signed char* cf,
                           double* rsum, int* nzero) {
  int local = 0;
  GRID_LOOP(i, n) {
    double s = 0.0;
    for (int e = prow[i]; e < prow[i + 1]; ++e) s += pval[e];
    rsum[i] = s;
    local += (cf[i] == 1 && !(s > 1e-14));
  }
  local = warp_sum_int(local);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(nzero, local);
}
// injection target of a zero F row: first coarse neighbour in A's row
__global__ void k_p_zero_extra(int n, const int* rowptr, const int* col, const signed char* cf,
                               const int* f2c, const double* rsum, int* extra, const int* prow,
                               int* newcnt) {
  GRID_LOOP(i, n) {
    int x = -1;
    if (cf[i] == 1 && !(rsum[i] > 1e-14)) {
      for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
        if (cf[col[e]] == 0) { x = f2c[col[e]]; break; }
    }
    extra[i] = x;
    newcnt[i] = prow[i + 1] - prow[i] + (x >= 0);
  }
}
__global__ void k_p_insert(int n, const int* prow, const int* pcol, const double* pval,
                           const int* extra, const int* nrow, int* ncol, double* nval) {
  GRID_LOOP(i, n) {
    int o = nrow[i];
    if (extra[i] >= 0) { ncol[o] = extra[i]; nval[o] = 1.0; ++o; }
    for (int e = prow[i]; e < prow[i + 1]; ++e) { ncol[o] = pcol[e]; nval[o] = pval[e]; ++o; }
  }
}
// scale F rows by 1/row_sum and clamp at 0 (:386-388)
__global__ void k_p_scale(int n, const int* prow, double* pval, const signed char* cf,
                          const double* rsum) {
  GRID_LOOP(i, n) {
    double sc = (cf[i] == 1 && rsum[i] > 1e-14) ? 1.0 / rsum[i] : 1.0;
    for (int e = prow[i]; e < prow[i + 1]; ++e) {
      double v = pval[e] * sc;
      pval[e] = v < 0.0 ? 0.0 : v;
    }
  }
}
// Energy-minimising blend (:390-419, solve_energy_weights :1469-1501).
// (A^T A + reg I)^-1 A^T y = A^T (A A^T + reg I)^-1 y with A = [B_c; 1^T] of
// size (m+1) x k, so each F row solves an (m+1) x (m+1) SPD system (m <= 3).
// B_c takes the FINE basis rows at the row's COARSE column indices, as the
// reference indexes basis_dev[cols_row].
__global__ void k_p_blend(int n, const int* prow, const int* pcol, double* pval,
                          const signed char* cf, const double* basis, int m, double blend,
                          double reg) {
  GRID_LOOP(i, n) {
    if (cf[i] != 1) continue;
    const int a = prow[i], b = prow[i + 1];
    if (b <= a) continue;
    const int M = m + 1;
    double G[4][4];
    for (int p = 0; p < M; ++p)
      for (int q = 0; q < M; ++q) G[p][q] = 0.0;
    for (int e = a; e < b; ++e) {
      double col_[4];
      const double* br = basis + (long long)pcol[e] * m;
      for (int p = 0; p < m; ++p) col_[p] = br[p];
      col_[m] = 1.0;
      for (int p = 0; p < M; ++p)
        for (int q = 0; q < M; ++q) G[p][q] += col_[p] * col_[q];
    }
    for (int p = 0; p < M; ++p) G[p][p] += reg;
    double y[4];
    for (int p = 0; p < m; ++p) y[p] = basis[(long long)i * m + p];
    y[m] = 1.0;
    // Cholesky G = L L^T, then two triangular solves
    double L[4][4];
    bool ok = true;
    for (int p = 0; p < M; ++p) {
      for (int q = 0; q <= p; ++q) {
        double s = G[p][q];
        for (int r = 0; r < q; ++r) s -= L[p][r] * L[q][r];
        if (p == q) {
          if (!(s > 0.0)) { ok = false; s = 1.0; }
          L[p][p] = sqrt(s);
        } else {
          L[p][q] = s / L[q][q];
        }
      }
    }
    if (!ok) continue;
    double z[4];
    for (int p = 0; p < M; ++p) {
      double s = y[p];
      for (int r = 0; r < p; ++r) s -= L[p][r] * z[r];
      z[p] = s / L[p][p];
    }
    for (int p = M - 1; p >= 0; --p) {
      double s = z[p];
      for (int r = p + 1; r < M; ++r) s -= L[r][p] * z[r];
      z[p] = s / L[p][p];
    }
    double wsum = 0.0;
    for (int e = a; e < b; ++e) {
      const double* br = basis + (long long)pcol[e] * m;
      double w = z[m];
      for (int p = 0; p < m; ++p) w += br[p] * z[p];
      w = w < 0.0 ? 0.0 : w;
      wsum += w;
    }
    if (wsum <= 1e-12) continue;
    for (int e = a; e < b; ++e) {
      const double* br = basis + (long long)pcol[e] * m;
      double w = z[m];
      for (int p = 0; p < m; ++p) w += br[p] * z[p];
      w = w < 0.0 ? 0.0 : w;
      pval[e] = (1.0 - blend) * pval[e] + blend * (w / wsum);
    }
  }
}

// Interpolation truncation (an option of this library; the reference keeps
// every entry).  An F row keeps entry e when fewer than kmax entries outrank it
// (larger weight, or equal weight and lower position) and its weight is at least
// tf times the row's largest; the kept entries are rescaled to the row's old
// sum.  kmax = 0 means no cap.  Weights are >= 0 here (clamped above).
__device__ __forceinline__ bool p_keep(const double* w, int a, int b, int e, int kmax, double tf,
                                       double wmax) {
  if (w[e] < tf * wmax) return false;
  if (kmax <= 0) return true;
  int rank = 0;
  for (int f = a; f < b && rank < kmax; ++f)
    if (w[f] > w[e] || (w[f] == w[e] && f < e)) ++rank;
  return rank < kmax;
}
__global__ void k_p_trunc_count(int n, const int* prow, const double* pval, const signed char* cf,
                                int kmax, double tf, int* cnt) {
  GRID_LOOP(i, n) {
    const int a = prow[i], b = prow[i + 1];
    if (cf[i] != 1) { cnt[i] = b - a; continue; }
    double wmax = 0.0;
    for (int e = a; e < b; ++e) wmax = fmax(wmax, pval[e]);
    int c = 0;
    for (int e = a; e < b; ++e) c += p_keep(pval, a, b, e, kmax, tf, wmax);
    cnt[i] = c;
  }
}
__global__ void k_p_trunc_fill(int n, const int* prow, const int* pcol, const double* pval,
                               const signed char* cf, int kmax, double tf, const int* nrow,
                               int* ncol, double* nval) {
  GRID_LOOP(i, n) {
    const int a = prow[i], b = prow[i + 1];
    int o = nrow[i];
    if (cf[i] != 1) {
      for (int e = a; e < b; ++e, ++o) { ncol[o] = pcol[e]; nval[o] = pval[e]; }
      continue;
    }
    double wmax = 0.0, all = 0.0, kept = 0.0;
    for (int e = a; e < b; ++e) { wmax = fmax(wmax, pval[e]); all += pval[e]; }
    for (int e = a; e < b; ++e)
      if (p_keep(pval, a, b, e, kmax, tf, wmax)) kept += pval[e];
    const double sc = kept > 0.0 ? all / kept : 1.0;
    for (int e = a; e < b; ++e)
      if (p_keep(pval, a, b, e, kmax, tf, wmax)) { ncol[o] = pcol[e]; nval[o] = pval[e] * sc; ++o; }
  }
}

// ---------------------------------------------------------- R = P^T
__global__ void k_col_count(int n, const int* prow, const int* pcol, int* cnt) {
  GRID_LOOP(i, n) for (int e = prow[i]; e < prow[i + 1]; ++e) atomicAdd(&cnt[pcol[e]], 1);
}
__global__ void k_r_fill(int n, const int* prow, const int* pcol, int* fill, int* rcol, int* rsrc) {
  GRID_LOOP(i, n) {
    for (int e = prow[i]; e < prow[i + 1]; ++e) {
      int s = atomicAdd(&fill[pcol[e]], 1);
      rcol[s] = (int)i;
      rsrc[s] = e;
    }
  }
}
__global__ void k_r_sort(int nc, const int* rrow, int* rcol, int* rsrc) {
  GRID_LOOP(I, nc) {
    int a = rrow[I], b = rrow[I + 1];
    for (int x = a + 1; x < b; ++x) {
      int c = rcol[x], s = rsrc[x], y = x - 1;
      while (y >= a && rcol[y] > c) { rcol[y + 1] = rcol[y]; rsrc[y + 1] = rsrc[y]; --y; }
      rcol[y + 1] = c; rsrc[y + 1] = s;
    }
  }
}
__global__ void k_gather(long long n, const int* src, const double* in, double* out) {
  GRID_LOOP(e, n) out[e] = in[src[e]];
}

// ------------------------------------------------ union SpGEMM (symbolic)
// candidate upper bound of each output row: sum of inner row lengths
__global__ void k_union_bound(int rows, const int* optr, const int* ocol, const int* iptr, int* bound) {
  GRID_LOOP(r, rows) {
    int s = 0;
    for (int e = optr[r]; e < optr[r + 1]; ++e) s += iptr[ocol[e] + 1] - iptr[ocol[e]];
    bound[r] = s;
  }
}
__global__ void k_max_i32(long long n, const int* v, int* out) {
  int m = 0;
  GRID_LOOP(i, n) m = max(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// max of the bounds that stay in shared memory
__global__ void k_max_narrow(long long n, const int* v, int limit, int* out) {
  int m = 0;
  GRID_LOOP(i, n) if (v[i] <= limit) m = max(m, v[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}
__device__ __forceinline__ unsigned hash_slot(int key, unsigned mask) {
  return ((unsigned)key * 2654435761u) & mask;
}
// Hash capacity of a row with `bound` candidates: power of two >= 2*bound.
__host__ __device__ __forceinline__ int hash_cap(int bound) {
  int h = 32;
  while (h < 2 * bound) h <<= 1;
  return h;
}
// Rows with more than kWideBound candidates keep their hash table in global
// scratch (offset goff[r], table + list of cap ints each); others use shared memory.
constexpr int kWideBound = 2048;
__global__ void k_wide_size(int rows, const int* bound, long long* gsize) {
  GRID_LOOP(r, rows) gsize[r] = bound[r] > kWideBound ? 2LL * hash_cap(bound[r]) : 0LL;
}

// One warp per output row.  Pass 1 (outcol == nullptr): count distinct columns.
// Pass 2: write the sorted distinct columns at outptr[row].
__global__ void k_union_rows(int rows, const int* optr, const int* ocol, const int* iptr,
                             const int* icol, int hsize, const int* bound, const long long* goff,
                             int* gscratch, int* ucnt, const int* outptr, int* outcol) {
  extern __shared__ int sh[];
  const int wpb = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* lcount = sh + warp * (2 * hsize + 1);
  for (long long r = (long long)blockIdx.x * wpb + warp; r < rows; r += (long long)gridDim.x * wpb) {
    const bool wide = bound[r] > kWideBound;
    const int cap = wide ? hash_cap(bound[r]) : hsize;
    int* table = wide ? gscratch + goff[r] : lcount + 1;
    int* list = table + cap;
    const unsigned mask = (unsigned)cap - 1;
    for (int q = lane; q < cap; q += 32) table[q] = -1;
    if (lane == 0) *lcount = 0;
    __syncwarp();
    for (int e = optr[r]; e < optr[r + 1]; ++e) {
      const int j = ocol[e];
      for (int f = iptr[j] + lane; f < iptr[j + 1]; f += 32) {
        const int key = icol[f];
        unsigned h = hash_slot(key, mask);
        while (true) {
          int prev = atomicCAS(&table[h], -1, key);
          if (prev == -1) { list[atomicAdd(lcount, 1)] = key; break; }
          if (prev == key) break;
          h = (h + 1) & mask;
        }
      }
      __syncwarp();
    }
    __threadfence_block();
    __syncwarp();
    const int u = *lcount;
    if (outcol == nullptr) {
      if (lane == 0) ucnt[r] = u;
    } else {
      const int base = outptr[r];
      for (int x = lane; x < u; x += 32) {
        int v = list[x], rank = 0;
        for (int y = 0; y < u; ++y) rank += (list[y] < v);
        outcol[base + rank] = v;
      }
    }
    __syncwarp();
  }
}

// --------------------------------------------------- Galerkin product plans
// Output position of every (outer entry, inner entry) product, enumerated row
// by row in (outer, inner) order; kbase = exclusive scan of the row bounds.
__global__ void k_plan_pos(int rows, const int* optr, const int* ocol, const int* iptr,
                           const int* icol, const int* outptr, const int* outcol,
                           const long long* kbase, int* ppos) {
  GRID_LOOP(r, rows) {
    long long k = kbase[r];
    const int ob = outptr[r], L = outptr[r + 1] - ob;
    for (int e = optr[r]; e < optr[r + 1]; ++e) {
      const int j = ocol[e];
      for (int f = iptr[j]; f < iptr[j + 1]; ++f, ++k) {
        const int key = icol[f];
        int lo = 0, hi = L - 1;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (outcol[ob + mid] < key) lo = mid + 1; else hi = mid;
        }
        ppos[k] = ob + lo;
      }
    }
  }
}
__global__ void k_plan_count(long long nprod, const int* ppos, int* cnt) {
  GRID_LOOP(k, nprod) atomicAdd(&cnt[ppos[k]], 1);
}
// Scatter products into their output segments; outer index is remapped by
// `omap` (R entry -> P entry) when given.
__global__ void k_plan_fill(int rows, const int* optr, const int* ocol, const int* iptr,
                            const long long* kbase, const int* ppos, const int* omap, int* fill,
                            long long* key, int* pe, int* pf) {
  GRID_LOOP(r, rows) {
    long long k = kbase[r];
    for (int e = optr[r]; e < optr[r + 1]; ++e) {
      const int j = ocol[e];
      const int eo = omap ? omap[e] : e;
      for (int f = iptr[j]; f < iptr[j + 1]; ++f, ++k) {
        const int slot = atomicAdd(&fill[ppos[k]], 1);
        key[slot] = k;
        pe[slot] = eo;
        pf[slot] = f;
      }
    }
  }
}
// Order every segment by product index: the sums then run in enumeration order.
__global__ void k_plan_sort(int nout, const int* seg, long long* key, int* pe, int* pf) {
  GRID_LOOP(o, nout) {
    const int a = seg[o], b = seg[o + 1];
    for (int x = a + 1; x < b; ++x) {
      long long kk = key[x];
      int e = pe[x], f = pf[x], y = x - 1;
      while (y >= a && key[y] > kk) { key[y + 1] = key[y]; pe[y + 1] = pe[y]; pf[y + 1] = pf[y]; --y; }
      key[y + 1] = kk; pe[y + 1] = e; pf[y + 1] = f;
    }
  }
}
// out[o] = sum over the segment of a[pe] * b[pf]; one thread per output walks
// its own run of the plan (consecutive terms share cache lines).  Interleaving
// the runs of 32 outputs so that a warp's index loads coalesce was slower on the
// 1e6-cell hierarchy (update 10.9 -> 13.0 ms per step): the padding to each
// group's longest run grows the index stream, while the runs' L1 reuse (~80 %
// hits) already absorbs the uncoalesced pattern.
template <typename T>
__global__ void __launch_bounds__(256) k_plan_apply(int nout, const int* __restrict__ seg,
                                                    const int* __restrict__ pe,
                                                    const int* __restrict__ pf,
                                                    const T* __restrict__ a,
                                                    const T* __restrict__ b,
                                                    T* __restrict__ out) {
  GRID_LOOP(o, nout) {
    T acc = T(0);
    for (int t = seg[o]; t < seg[o + 1]; ++t) acc += a[pe[t]] * b[pf[t]];
    out[o] = acc;
  }
}

// out[o] = sum over the segment of v[idx] * cf, cf the term's frozen P factor
// (same products and order as k_plan_apply, one gather fewer per term).
template <typename T>
__global__ void __launch_bounds__(256) k_plan_apply_cf(int nout, const int* __restrict__ seg,
                                                       const int* __restrict__ idx,
                                                       const T* __restrict__ cf,
                                                       const T* __restrict__ v,
                                                       T* __restrict__ out) {
  GRID_LOOP(o, nout) {
    T acc = T(0);
    for (int t = seg[o]; t < seg[o + 1]; ++t) acc += v[idx[t]] * cf[t];
    out[o] = acc;
  }
}
__global__ void k_gather_f(long long n, const int* src, const float* in, float* out) {
  GRID_LOOP(i, n) out[i] = in[src[i]];
}
// out[o] = sum over the segment of v[base[o] + idx16] * cf (k_plan_apply_cf with
// the A*P term indices stored as offsets into the output's A row)
template <typename T>
__global__ void __launch_bounds__(256) k_plan_apply_cf16(int nout, const int* __restrict__ seg,
                                                         const int* __restrict__ base,
                                                         const unsigned short* __restrict__ idx16,
                                                         const T* __restrict__ cf,
                                                         const T* __restrict__ v,
                                                         T* __restrict__ out) {
  GRID_LOOP(o, nout) {
    T acc = T(0);
    const T* __restrict__ vr = v + base[o];
    for (int t = seg[o]; t < seg[o + 1]; ++t) acc += vr[idx16[t]] * cf[t];
    out[o] = acc;
  }
}
// k_plan_apply_cf / k_plan_apply_cf16 with LPR lanes per output (the small
// levels' outputs have long term segments and few outputs, so one thread per
// output leaves most of the GPU idle while it walks its segment): each lane
// sums the terms t = seg[o] + lane, + LPR, ... in order, then a fixed-order
// reduction over the output's lanes.  The loop runs per warp so that every
// lane reaches the shuffles.  BASE16: v indexed by base[o] + idx16[t].
template <typename T, int LPR, bool BASE16>
__global__ void __launch_bounds__(256) k_plan_apply_lanes(int nout, const int* __restrict__ seg,
                                                          const int* __restrict__ base,
                                                          const int* __restrict__ idx,
                                                          const unsigned short* __restrict__ idx16,
                                                          const T* __restrict__ cf, const T* __restrict__ v,
                                                          T* __restrict__ out) {
  const int lane = threadIdx.x % LPR;
  const long long outs_per_block = blockDim.x / LPR;
  const long long warp_o0 = blockIdx.x * outs_per_block + (threadIdx.x / 32) * (32 / LPR);
  for (long long w0 = warp_o0; w0 < nout; w0 += gridDim.x * outs_per_block) {
    const long long o = w0 + (threadIdx.x % 32) / LPR;
    T acc = T(0);
    if (o < nout) {
      if constexpr (BASE16) {
        const T* __restrict__ vr = v + base[o];
        for (int t = seg[o] + lane; t < seg[o + 1]; t += LPR) acc += vr[idx16[t]] * cf[t];
      } else {
        for (int t = seg[o] + lane; t < seg[o + 1]; t += LPR) acc += v[idx[t]] * cf[t];
      }
    }
#pragma unroll
    for (int q = LPR / 2; q > 0; q >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, q, LPR);
    if (o < nout && lane == 0) out[o] = acc;
  }
}
// Lanes per output of the fp32 chain's plan kernels: 1 (one thread per output)
// unless the level has few outputs with long segments.
inline int plan_lanes(long long nout, long long terms) {
  if (nout <= 0 || nout > (1 << 18)) return 1;
  const long long avg = terms / nout;
  return avg >= 24 ? 8 : (avg >= 6 ? 4 : 1);
}
template <typename T, bool BASE16>
void launch_plan_lanes(int lpr, int nout, const int* seg, const int* base, const int* idx,
                       const unsigned short* idx16, const T* cf, const T* v, T* out, cudaStream_t s) {
  const unsigned grid = grid_for((size_t)nout * lpr, 256, 16);
  if (lpr == 8)
    k_plan_apply_lanes<T, 8, BASE16><<<grid, 256, 0, s>>>(nout, seg, base, idx, idx16, cf, v, out);
  else
    k_plan_apply_lanes<T, 4, BASE16><<<grid, 256, 0, s>>>(nout, seg, base, idx, idx16, cf, v, out);
  ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
}
// base[o] = rowptr[i] for every output o of A*P row i
__global__ void k_ap_ebase(int n, const int* aprow, const int* rowptr, int* base) {
  GRID_LOOP(i, n) for (int o = aprow[i]; o < aprow[i + 1]; ++o) base[o] = rowptr[i];
}
// e16[t] = pe[t] - base[o]; flag = 1 when an offset does not fit 16 bits
__global__ void k_ap_e16(int nout, const int* seg, const int* pe, const int* base,
                         unsigned short* e16, int* flag) {
  GRID_LOOP(o, nout) {
    for (int t = seg[o]; t < seg[o + 1]; ++t) {
      const int d = pe[t] - base[o];
      if (d < 0 || d > 65535) { atomicOr(flag, 1); return; }
      e16[t] = (unsigned short)d;
    }
  }
}

template <typename T>
void plan_apply_cf(int nout, const int* seg, const int* idx, const T* cf, const T* v, T* out,
                   cudaStream_t s) {
  if (nout <= 0) return;
  k_plan_apply_cf<T><<<grid_for(nout, 256, 16), 256, 0, s>>>(nout, seg, idx, cf, v, out); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
}

template <typename T>
void plan_apply(int nout, const int* seg, const int* pe, const int* pf, const T* a, const T* b,
                T* out, cudaStream_t s) {
  if (nout <= 0) return;
  k_plan_apply<T><<<grid_for(nout, 256, 16), 256, 0, s>>>(nout, seg, pe, pf, a, b, out); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
}

// ------------------------------------------------ union SpGEMM (numeric)
// out[r, J] = sum_e oval[e] * inner[ocol[e], J]; each output row lives in shared
// memory; for one outer entry the lanes own distinct columns (deterministic).
template <int WPB>
__global__ void k_union_numeric(int rows, const int* __restrict__ optr, const int* __restrict__ ocol,
                                const double* __restrict__ oval, const int* __restrict__ iptr,
                                const int* __restrict__ icol, const double* __restrict__ ival,
                                const int* __restrict__ outptr, const int* __restrict__ outcol,
                                double* __restrict__ outval, int maxrow) {
  extern __shared__ unsigned char shraw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int* scol = (int*)shraw + warp * maxrow;
  double* sacc = (double*)((int*)shraw + WPB * maxrow + ((WPB * maxrow) & 1)) + warp * maxrow;
  for (long long r = (long long)blockIdx.x * WPB + warp; r < rows; r += (long long)gridDim.x * WPB) {
    const int ob = outptr[r], L = outptr[r + 1] - ob;
    for (int x = lane; x < L; x += 32) { scol[x] = outcol[ob + x]; sacc[x] = 0.0; }
    __syncwarp();
    for (int e = optr[r]; e < optr[r + 1]; ++e) {
      const int j = ocol[e];
      const double a = oval[e];
      for (int f = iptr[j] + lane; f < iptr[j + 1]; f += 32) {
        const int key = icol[f];
        int lo = 0, hi = L - 1;
        while (lo < hi) {
          int mid = (lo + hi) >> 1;
          if (scol[mid] < key) lo = mid + 1; else hi = mid;
        }
        sacc[lo] += a * ival[f];
      }
      __syncwarp();
    }
    for (int x = lane; x < L; x += 32) outval[ob + x] = sacc[x];
    __syncwarp();
  }
}

// ---------------------------------------------------------- basis (nullspace)
// torch.linspace(0, 1, n) evaluated from both ends about the midpoint.
__global__ void k_linspace(int n, double* c) {
  GRID_LOOP(i, n) {
    double step = n > 1 ? 1.0 / (double)(n - 1) : 0.0;
    long long half = n / 2;
    c[i] = (i < half) ? 0.0 + step * (double)i : 1.0 - step * (double)(n - i - 1);
  }
}
__global__ void k_fill_col(int n, int m, int c, double* B, const double* v, double a, double sub) {
  GRID_LOOP(i, n) B[(long long)i * m + c] = (v ? v[i] : 1.0) * a - sub;
}
__global__ void k_col_extract(int n, int m, int c, const double* B, double* v) {
  GRID_LOOP(i, n) v[i] = B[(long long)i * m + c];
}
__global__ void k_axpy(int n, double a, const double* x, double* y) {
  GRID_LOOP(i, n) y[i] += a * x[i];
}
__global__ void k_scale_into(int n, double a, const double* x, double* y) {
  GRID_LOOP(i, n) y[i] = x[i] * a;
}
__global__ void k_square(int n, const double* x, double* y) {
  GRID_LOOP(i, n) y[i] = x[i] * x[i];
}
__global__ void k_add_scalar(int n, double* x, double a) {
  GRID_LOOP(i, n) x[i] -= a;
}
// Bc = R * B (n_c x m)
__global__ void k_restrict_basis(int nc, int m, const int* rrow, const int* rcol, const double* rval,
                                 const double* B, double* Bc) {
  GRID_LOOP(I, nc) {
    double acc[3] = {0, 0, 0};
    for (int e = rrow[I]; e < rrow[I + 1]; ++e) {
      const double* br = B + (long long)rcol[e] * m;
      for (int p = 0; p < m; ++p) acc[p] += rval[e] * br[p];
    }
    for (int p = 0; p < m; ++p) Bc[(long long)I * m + p] = acc[p];
  }
}

__global__ void k_to_float(long long n, const double* in, float* out) {
  GRID_LOOP(i, n) out[i] = (float)in[i];
}
// k_to_float of a level's values that also fills its fp32 DIA copy
__global__ void k_to_float_dia(long long n, const double* in, float* out, const int* dmap, float* dval) {
  GRID_LOOP(i, n) {
    const float f = (float)in[i];
    out[i] = f;
    dval[dmap[i]] = f;
  }
}

}  // namespace

// =================================================================== host
namespace {

void union_numeric(int rows, const int* optr, const int* ocol, const double* oval, const int* iptr,
                   const int* icol, const double* ival, const int* outptr, const int* outcol,
                   double* outval, int maxrow, cudaStream_t s);

struct Ctx {
  AMG& h;
  cudaStream_t s;
};

int to_host_int(AMG& h, const int* d, cudaStream_t s) {
  IMPES_CUDA(cudaMemcpyAsync(h.hint.p, d, sizeof(int), cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  return h.hint.p[0];
}

// orthonormalize_columns (classical_amg.py:1395-1407) on an n x m row-major basis.
// Returns the number of kept columns (compacted to the front).
int orthonormalize(AMG& h, double* B, int n, int m, cudaStream_t s) {
  DBuf<double> v(n), q(n), out((size_t)n * m);
  std::vector<DBuf<double>> kept;
  for (int c = 0; c < m; ++c) {
    k_col_extract<<<grid_for(n, TB), TB, 0, s>>>(n, m, c, B, v.p); ::impes::count_launch();
    for (auto& qq : kept) {
      double d = dot_host(h, v.p, qq.p, n, s);
      k_axpy<<<grid_for(n, TB), TB, 0, s>>>(n, -d, qq.p, v.p); ::impes::count_launch();
    }
    double nv = std::sqrt(dot_host(h, v.p, v.p, n, s));
    if (nv > 1e-10) {
      DBuf<double> qn(n);
      k_scale_into<<<grid_for(n, TB), TB, 0, s>>>(n, 1.0 / nv, v.p, qn.p); ::impes::count_launch();
      kept.push_back(std::move(qn));
    }
  }
  int mk = (int)kept.size();
  if (mk == 0) {
    DBuf<double> one(n);
    k_fill_col<<<grid_for(n, TB), TB, 0, s>>>(n, 1, 0, one.p, nullptr, 1.0 / (std::sqrt((double)n) + 1e-30), 0.0); ::impes::count_launch();
    kept.push_back(std::move(one));
    mk = 1;
  }
  for (int c = 0; c < mk; ++c)
    { k_fill_col<<<grid_for(n, TB), TB, 0, s>>>(n, mk, c, B, kept[c].p, 1.0, 0.0); ::impes::count_launch(); }
  IMPES_CUDA(cudaStreamSynchronize(s));
  return mk;
}

// generate_nullspace (classical_amg.py:1426-1466) for dim <= 3.
int level0_basis(AMG& h, DBuf<double>& B, int n, int dim, cudaStream_t s) {
  if (dim <= 0) return 0;
  dim = std::min(dim, 3);
  B.alloc((size_t)n * 3);
  DBuf<double> coords(n), tmp(n), c0(n), cur(n);
  std::vector<DBuf<double>> basis;
  {
    DBuf<double> one(n);
    double inv = 1.0 / (std::sqrt((double)n) + 1e-30);
    k_fill_col<<<grid_for(n, TB), TB, 0, s>>>(n, 1, 0, one.p, nullptr, inv, 0.0); ::impes::count_launch();
    basis.push_back(std::move(one));
  }
  k_linspace<<<grid_for(n, TB), TB, 0, s>>>(n, coords.p); ::impes::count_launch();
  k_fill_col<<<grid_for(n, TB), TB, 0, s>>>(n, 1, 0, c0.p, nullptr, 1.0, 0.0); ::impes::count_launch();  // ones
  double mean = dot_host(h, coords.p, c0.p, n, s) / n;
  if ((int)basis.size() < dim) {
    k_scale_into<<<grid_for(n, TB), TB, 0, s>>>(n, 1.0, coords.p, cur.p); ::impes::count_launch();
    k_add_scalar<<<grid_for(n, TB), TB, 0, s>>>(n, cur.p, mean); ::impes::count_launch();
    double nr = std::sqrt(dot_host(h, cur.p, cur.p, n, s));
    if (nr > 1e-8) {
      DBuf<double> q(n);
      k_scale_into<<<grid_for(n, TB), TB, 0, s>>>(n, 1.0 / nr, cur.p, q.p); ::impes::count_launch();
      basis.push_back(std::move(q));
    }
  }
  if ((int)basis.size() < dim) {
    k_square<<<grid_for(n, TB), TB, 0, s>>>(n, coords.p, cur.p); ::impes::count_launch();
    double m2 = dot_host(h, cur.p, c0.p, n, s) / n;
    k_add_scalar<<<grid_for(n, TB), TB, 0, s>>>(n, cur.p, m2); ::impes::count_launch();
    double nr = std::sqrt(dot_host(h, cur.p, cur.p, n, s));
    if (nr > 1e-8) {
      for (auto& b : basis) {
        double d = dot_host(h, cur.p, b.p, n, s);
        k_axpy<<<grid_for(n, TB), TB, 0, s>>>(n, -d, b.p, cur.p); ::impes::count_launch();
      }
      double nr2 = std::sqrt(dot_host(h, cur.p, cur.p, n, s));
      if (nr2 > 1e-8) {
        DBuf<double> q(n);
        k_scale_into<<<grid_for(n, TB), TB, 0, s>>>(n, 1.0 / nr2, cur.p, q.p); ::impes::count_launch();
        basis.push_back(std::move(q));
      }
    }
  }
  int m = (int)basis.size();
  for (int c = 0; c < m; ++c)
    { k_fill_col<<<grid_for(n, TB), TB, 0, s>>>(n, m, c, B.p, basis[c].p, 1.0, 0.0); ::impes::count_launch(); }
  return orthonormalize(h, B.p, n, m, s);
}

// symbolic union product: output pattern (ptr, col), returns nnz and max row length
void union_symbolic(AMG& h, int rows, const int* optr, const int* ocol, const int* iptr,
                    const int* icol, DBuf<int>& outptr, DBuf<int>& outcol, int& maxrow,
                    cudaStream_t s) {
  DBuf<int> bound(rows), ucnt(rows + 1);
  k_union_bound<<<grid_for(rows, TB), TB, 0, s>>>(rows, optr, ocol, iptr, bound.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  // global scratch for the wide rows
  DBuf<long long> gsize(rows + 1), goff(rows + 1);
  k_wide_size<<<grid_for(rows, TB), TB, 0, s>>>(rows, bound.p, gsize.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  std::vector<long long> hs(rows);
  IMPES_CUDA(cudaMemcpyAsync(hs.data(), gsize.p, sizeof(long long) * rows, cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  std::vector<long long> ho(rows + 1, 0);
  for (int r = 0; r < rows; ++r) ho[r + 1] = ho[r] + hs[r];
  IMPES_CUDA(cudaMemcpyAsync(goff.p, ho.data(), sizeof(long long) * (rows + 1), cudaMemcpyHostToDevice, s));
  DBuf<int> gscratch(std::max<long long>(ho[rows], 1));
  // shared-memory table size for the narrow rows
  IMPES_CUDA(cudaMemsetAsync(h.iflag.p, 0, sizeof(int), s));
  k_max_narrow<<<grid_for(rows, TB), TB, 0, s>>>(rows, bound.p, kWideBound, h.iflag.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  const int maxc = to_host_int(h, h.iflag.p, s);
  const int hsize = hash_cap(maxc);
  const size_t per_warp = sizeof(int) * (2 * (size_t)hsize + 1);
  const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (64u << 10) / per_warp));
  const size_t smem = per_warp * wpb;
  raise_smem_limit((const void*)k_union_rows, smem);
  unsigned grid = (unsigned)std::min<long long>((rows + wpb - 1) / wpb, (long long)num_sms() * 32);
  k_union_rows<<<std::max(1u, grid), 32 * wpb, smem, s>>>(rows, optr, ocol, iptr, icol, hsize, bound.p,
                                                          goff.p, gscratch.p, ucnt.p, nullptr, nullptr); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  outptr.alloc(rows + 1);
  int nnz = exclusive_scan_i32(ucnt.p, outptr.p, rows, s);
  outcol.alloc(std::max(nnz, 1));
  k_union_rows<<<std::max(1u, grid), 32 * wpb, smem, s>>>(rows, optr, ocol, iptr, icol, hsize, bound.p,
                                                          goff.p, gscratch.p, nullptr, outptr.p, outcol.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  IMPES_CUDA(cudaMemsetAsync(h.iflag.p, 0, sizeof(int), s));
  k_max_i32<<<grid_for(rows, TB), TB, 0, s>>>(rows, ucnt.p, h.iflag.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  maxrow = to_host_int(h, h.iflag.p, s);
}

// Product plan of out = outer * inner on a known output pattern (see Level).
// Returns false (no plan) when the product count does not fit the memory budget.
bool build_plan(int rows, const int* optr, const int* ocol, const int* iptr, const int* icol,
                const int* outptr, const int* outcol, int nout, const int* omap, DBuf<int>& seg,
                DBuf<int>& pe, DBuf<int>& pf, long long& nterms, cudaStream_t s) {
  nterms = 0;
  DBuf<int> bound(std::max(rows, 1));
  k_union_bound<<<grid_for(rows, TB), TB, 0, s>>>(rows, optr, ocol, iptr, bound.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  std::vector<int> hb(rows);
  IMPES_CUDA(cudaMemcpyAsync(hb.data(), bound.p, sizeof(int) * rows, cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  std::vector<long long> hk(rows + 1, 0);
  for (int r = 0; r < rows; ++r) hk[r + 1] = hk[r] + hb[r];
  const long long nprod = hk[rows];
  if (nprod >= (1LL << 31) - 1) return false;
  size_t free_b = 0, total_b = 0;
  IMPES_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const double keep = 8.0 * nprod + 4.0 * nout, temp = 16.0 * nprod;
  if (keep + temp > 0.5 * (double)free_b) return false;
  DBuf<long long> kbase(rows + 1);
  IMPES_CUDA(cudaMemcpyAsync(kbase.p, hk.data(), sizeof(long long) * (rows + 1), cudaMemcpyHostToDevice, s));
  DBuf<int> ppos(std::max<long long>(nprod, 1));
  k_plan_pos<<<grid_for(rows, TB), TB, 0, s>>>(rows, optr, ocol, iptr, icol, outptr, outcol, kbase.p, ppos.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  DBuf<int> cnt(nout + 1), fill(nout + 1);
  IMPES_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (nout + 1), s));
  k_plan_count<<<grid_for(nprod, TB), TB, 0, s>>>(nprod, ppos.p, cnt.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  seg.alloc(nout + 1);
  exclusive_scan_i32(cnt.p, seg.p, nout, s);
  IMPES_CUDA(cudaMemcpyAsync(fill.p, seg.p, sizeof(int) * nout, cudaMemcpyDeviceToDevice, s));
  DBuf<long long> key(std::max<long long>(nprod, 1));
  pe.alloc(std::max<long long>(nprod, 1));
  pf.alloc(std::max<long long>(nprod, 1));
  k_plan_fill<<<grid_for(rows, TB), TB, 0, s>>>(rows, optr, ocol, iptr, kbase.p, ppos.p, omap, fill.p,
                                                key.p, pe.p, pf.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  k_plan_sort<<<grid_for(nout, TB), TB, 0, s>>>(nout, seg.p, key.p, pe.p, pf.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  IMPES_CUDA(cudaStreamSynchronize(s));
  nterms = nprod;
  return true;
}

// Galerkin numeric update of level l -> l+1 (plan when available).
void galerkin_numeric(Level& L, Level& Nc, cudaStream_t s) {
  if (L.planned) {
    const int apn = (int)L.apval.n;
    plan_apply<double>(apn, L.ap_seg.p, L.ap_e.p, L.ap_f.p, L.val.p, L.pval.p, L.apval.p, s);
    plan_apply<double>(Nc.nnz, L.ac_seg.p, L.ac_r.p, L.ac_f.p, L.pval.p, L.apval.p, Nc.val.p, s);
    return;
  }
  union_numeric(L.n, L.rowptr.p, L.col.p, L.val.p, L.prow.p, L.pcol.p, L.pval.p, L.aprow.p,
                L.apcol.p, L.apval.p, L.ap_maxrow, s);
  union_numeric(L.nc, L.rrow.p, L.rcol.p, L.rval.p, L.aprow.p, L.apcol.p, L.apval.p, Nc.rowptr.p,
                Nc.col.p, Nc.val.p, L.ac_maxrow, s);
}

void union_numeric(int rows, const int* optr, const int* ocol, const double* oval, const int* iptr,
                   const int* icol, const double* ival, const int* outptr, const int* outcol,
                   double* outval, int maxrow, cudaStream_t s) {
  if (rows == 0) return;
  maxrow = std::max(maxrow, 1);
  size_t per_warp = (size_t)maxrow * (sizeof(int) + sizeof(double));
  if (per_warp * 8 + 16 <= (96u << 10)) {
    constexpr int W = 8;
    size_t smem = per_warp * W + 16;
    raise_smem_limit((const void*)k_union_numeric<W>, smem);
    unsigned grid = (unsigned)std::min<long long>((rows + W - 1) / W, (long long)num_sms() * 16);
    k_union_numeric<W><<<grid, 32 * W, smem, s>>>(rows, optr, ocol, oval, iptr, icol, ival, outptr,
                                                   outcol, outval, maxrow); ::impes::count_launch();
  } else {
    constexpr int W = 1;
    size_t smem = per_warp * W + 16;
    IMPES_REQUIRE(smem <= (220u << 10), IMPES_ERR_ARG, "Galerkin row too wide for shared memory");
    raise_smem_limit((const void*)k_union_numeric<W>, smem);
    unsigned grid = (unsigned)std::min<long long>(rows, (long long)num_sms() * 32);
    k_union_numeric<W><<<grid, 32 * W, smem, s>>>(rows, optr, ocol, oval, iptr, icol, ival, outptr,
                                                   outcol, outval, maxrow); ::impes::count_launch();
  }
  IMPES_CHECK_LAUNCH();
}

template <typename TV, typename TO>
void launch_inv_relax(const Level& L, const TV* val, TO* out, unsigned long long* lmax, cudaStream_t s) {
  if (lmax) IMPES_CUDA(cudaMemsetAsync(lmax, 0, sizeof(unsigned long long), s));
  // lanes per row: about half the mean row length, so each lane loads one or
  // two entries (one thread per row for rows of at most 4 entries)
  const int avg = L.n > 0 ? (int)((L.nnz + L.n - 1) / L.n) : 1;
  auto go = [&](auto kernel, int lpr) {
    kernel<<<grid_for((size_t)L.n * lpr, TB, 16), TB, 0, s>>>(L.n, L.rowptr.p, L.col.p, val, out, lmax);
    ::impes::count_launch();
  };
  if (avg > 32) go(k_inv_relax_lanes<TV, TO, 32>, 32);
  else if (avg > 16) go(k_inv_relax_lanes<TV, TO, 16>, 16);
  else if (avg > 8) go(k_inv_relax_lanes<TV, TO, 8>, 8);
  else if (avg > 4) go(k_inv_relax_lanes<TV, TO, 4>, 4);
  else go(k_inv_relax<TV, TO>, 1);
  IMPES_CHECK_LAUNCH();
}

// The Chebyshev bound of level L (slot 0: fp64 values, 1: fp32 chain), or null
// when the hierarchy smooths with l1-Jacobi.
unsigned long long* cheb_slot(AMG& h, Level& L, int slot) {
  if (h.prm.smoother != IMPES_SMOOTHER_CHEBYSHEV) return nullptr;
  L.cheb_lmax.ensure(2);
  return L.cheb_lmax.p + slot;
}

void compute_inv_relax(AMG& h, Level& L, cudaStream_t s) {
  L.inv_relax.ensure(std::max(L.n, 1));
  launch_inv_relax<double, double>(L, L.val.p, L.inv_relax.p, cheb_slot(h, L, 0), s);
}

// l1 weights of the fp32 chain, from the fp32 values
void compute_inv_relax_f(AMG& h, Level& L, cudaStream_t s) {
  L.inv_relaxf.ensure(std::max(L.n, 1));
  launch_inv_relax<float, float>(L, L.valf.p, L.inv_relaxf.p, cheb_slot(h, L, 1), s);
}

// fp32 weights rounded from the fp64 ones: the fp32 path's Chebyshev bound is
// the fp64 one
void cheb_copy_to_fp32(AMG& h, Level& L, cudaStream_t s) {
  if (h.prm.smoother != IMPES_SMOOTHER_CHEBYSHEV) return;
  L.cheb_lmax.ensure(2);
  IMPES_CUDA(cudaMemcpyAsync(L.cheb_lmax.p + 1, L.cheb_lmax.p, sizeof(unsigned long long),
                             cudaMemcpyDeviceToDevice, s));
}

void alloc_level_vectors(Level& L) {
  size_t n = std::max(L.n, 1);
  L.x.ensure(n); L.b.ensure(n); L.r.ensure(n); L.t.ensure(n); L.u.ensure(n);
  L.xf.ensure(n); L.bf.ensure(n); L.rf.ensure(n); L.tf.ensure(n); L.uf.ensure(n);
}

// Equilibration of level-0 values (classical_amg.py:763-788 / 1334-1355).  The
// ON/OFF decision (lower median of |diag| below the threshold) stays on the
// device: with it OFF, dhalf = 1 and the scaling kernel copies values exactly.
void equilibrate_level0(AMG& h, const double* val_in, cudaStream_t s) {
  Level& L0 = *h.levels[0];
  const int n = L0.n;
  h.dhalf_inv.ensure(n);
  h.jac_w.ensure(n);
  h.diag_tmp.ensure(n);
  k_diag<<<grid_for(n, TB), TB, 0, s>>>(n, L0.rowptr.p, L0.col.p, val_in, h.diag_tmp.p); ::impes::count_launch();
  IMPES_CUDA(cudaMemsetAsync(h.iflag.p, 0, sizeof(int), s));
  k_count_below<<<grid_for(n, TB), TB, 0, s>>>(n, h.diag_tmp.p, h.prm.equilibration_threshold, h.iflag.p); ::impes::count_launch();
  k_equil_prepare<<<grid_for(n, TB), TB, 0, s>>>(n, h.diag_tmp.p, h.iflag.p, h.dhalf_inv.p,
                                                 h.jac_w.p, h.iflag.p + 1); ::impes::count_launch();
  const bool dia = L0.dia_nd > 0 && L0.dia_on[0] && L0.dia_val.p;
  k_equilibrate<<<grid_for(n, TB), TB, 0, s>>>(n, L0.rowptr.p, L0.col.p, val_in, h.dhalf_inv.p, L0.val.p,
                                               dia ? L0.dia_map.p : nullptr, dia ? L0.dia_val.p : nullptr);
  ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
}

}  // namespace

void level_precision_copies(AMG& h, Level& L, cudaStream_t s) {
  if (!h.prm.mixed_precision) return;
  L.valf.ensure(std::max(L.nnz, 1));
  L.inv_relaxf.ensure(std::max(L.n, 1));
  k_to_float<<<grid_for(L.nnz, TB), TB, 0, s>>>(L.nnz, L.val.p, L.valf.p); ::impes::count_launch();
  k_to_float<<<grid_for(L.n, TB), TB, 0, s>>>(L.n, L.inv_relax.p, L.inv_relaxf.p); ::impes::count_launch();
  cheb_copy_to_fp32(h, L, s);
  if (!L.coarsest && L.pnnz) {
    L.pvalf.ensure(L.pnnz);
    L.rvalf.ensure(L.pnnz);
    k_to_float<<<grid_for(L.pnnz, TB), TB, 0, s>>>(L.pnnz, L.pval.p, L.pvalf.p); ::impes::count_launch();
    k_to_float<<<grid_for(L.pnnz, TB), TB, 0, s>>>(L.pnnz, L.rval.p, L.rvalf.p); ::impes::count_launch();
  }
  IMPES_CHECK_LAUNCH();
}

namespace {
// ------------------------------------------------ SELL-32 copies of A
// Levels of at least kSellMinRows rows with at most 96 entries per row get a
// SELL-32 copy of A (Level::sell_*), which the autotuner may pick for the
// sweeps and residuals.  Built on the host from the fixed pattern: lanes per
// row by the mean row length (1 up to 12 entries, 4 up to 30, else 8), rows
// sorted by length (longest first, stable) inside windows of 256 rows (one
// lane per row) or 32 rows, so a slice's rows have similar lengths; padding
// points at the row's own column (row-relative 32768, or the row itself) with
// value 0.  The rule and windows are the fastest of 1, 2, 4, 8 lanes and
// 32/256-row windows on the 1e6-cell hierarchy's levels 0-6.
constexpr int kSellMinRows = 8192;
inline int sell_lanes(int avg) { return avg <= 12 ? 1 : avg <= 30 ? 4 : 8; }

// IMPES_NO_SELL=1 (read at setup) builds no SELL or DIA copies.
bool sell_enabled() {
  const char* ev = getenv("IMPES_NO_SELL");
  return !(ev && ev[0] == '1');
}

__global__ void k_sell_gather(long long len, const int* __restrict__ map, const double* __restrict__ v,
                              double* __restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < len; k += (long long)gridDim.x * blockDim.x) {
    const int m = map[k];
    out[k] = m >= 0 ? v[m] : 0.0;
  }
}
__global__ void k_sell_gather_f(long long len, const int* __restrict__ map, const float* __restrict__ v,
                                float* __restrict__ out) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < len; k += (long long)gridDim.x * blockDim.x) {
    const int m = map[k];
    out[k] = m >= 0 ? v[m] : 0.0f;
  }
}

void build_sell(Level& L, cudaStream_t s) {
  L.sell_slices = 0;
  L.sell_len = 0;
  if (L.coarsest || L.n < kSellMinRows || L.avg_row > 96 || L.nnz <= 0) return;
  const int n = L.n;
  std::vector<int> rp(n + 1), col(L.nnz);
  std::vector<unsigned short> c16;
  IMPES_CUDA(cudaMemcpyAsync(rp.data(), L.rowptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
  if (L.col16.p) {
    c16.resize(L.nnz);
    IMPES_CUDA(cudaMemcpyAsync(c16.data(), L.col16.p, sizeof(unsigned short) * L.nnz, cudaMemcpyDeviceToHost, s));
  } else {
    IMPES_CUDA(cudaMemcpyAsync(col.data(), L.col.p, sizeof(int) * L.nnz, cudaMemcpyDeviceToHost, s));
  }
  IMPES_CUDA(cudaStreamSynchronize(s));
  const int lpr = sell_lanes(L.avg_row), R = 32 / lpr;
  const int window = lpr == 1 ? 256 : 32;
  std::vector<int> perm(n);
  for (int r = 0; r < n; ++r) perm[r] = r;
  for (int w0 = 0; w0 < n; w0 += window) {
    const int w1 = std::min(n, w0 + window);
    std::stable_sort(perm.begin() + w0, perm.begin() + w1,
                     [&](int a, int b) { return rp[a + 1] - rp[a] > rp[b + 1] - rp[b]; });
  }
  const int nsl = (n + R - 1) / R;
  std::vector<int> sptr(nsl + 1, 0);
  long long tot = 0;
  for (int q = 0; q < nsl; ++q) {
    int w = 0;   // steps of 32 entries: the slice's longest row over its lanes
    for (int r = q * R; r < std::min(n, q * R + R); ++r)
      w = std::max(w, (rp[perm[r] + 1] - rp[perm[r]] + lpr - 1) / lpr);
    tot += 32LL * w;
    IMPES_REQUIRE(tot < (1LL << 31), IMPES_ERR_OOM, "SELL copy of a level exceeds 2^31 entries");
    sptr[q + 1] = (int)tot;
  }
  std::vector<int> map((size_t)tot, -1);
  std::vector<int> scol(L.col16.p ? 0 : (size_t)tot);
  std::vector<unsigned short> scol16(L.col16.p ? (size_t)tot : 0);
  for (int r = 0; r < nsl * R; ++r) {
    const int q = r / R, rq = r % R;
    const int row = perm[r < n ? r : n - 1];
    const int len = r < n ? rp[row + 1] - rp[row] : 0;
    const int w = (sptr[q + 1] - sptr[q]) / 32;
    for (int j = 0; j < w * lpr; ++j) {
      const size_t k = (size_t)sptr[q] + 32 * (size_t)(j / lpr) + (size_t)rq * lpr + j % lpr;
      if (j < len) {
        map[k] = rp[row] + j;
        if (L.col16.p) scol16[k] = c16[rp[row] + j];
        else scol[k] = col[rp[row] + j];
      } else if (L.col16.p) {
        scol16[k] = L.col16_rel ? (unsigned short)32768 : (unsigned short)row;
      } else {
        scol[k] = row;
      }
    }
  }
  L.sell_ptr.alloc(nsl + 1);
  L.sell_perm.alloc(n);
  L.sell_map.alloc(std::max<long long>(tot, 1));
  IMPES_CUDA(cudaMemcpyAsync(L.sell_ptr.p, sptr.data(), sizeof(int) * (nsl + 1), cudaMemcpyHostToDevice, s));
  IMPES_CUDA(cudaMemcpyAsync(L.sell_perm.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  IMPES_CUDA(cudaMemcpyAsync(L.sell_map.p, map.data(), sizeof(int) * tot, cudaMemcpyHostToDevice, s));
  if (L.col16.p) {
    L.sell_col16.alloc(std::max<long long>(tot, 1));
    IMPES_CUDA(cudaMemcpyAsync(L.sell_col16.p, scol16.data(), sizeof(unsigned short) * tot, cudaMemcpyHostToDevice, s));
  } else {
    L.sell_col.alloc(std::max<long long>(tot, 1));
    IMPES_CUDA(cudaMemcpyAsync(L.sell_col.p, scol.data(), sizeof(int) * tot, cudaMemcpyHostToDevice, s));
  }
  IMPES_CUDA(cudaStreamSynchronize(s));   // the host vectors go out of scope
  L.sell_slices = nsl;
  L.sell_len = tot;
  L.sell_lpr = lpr;
}

// DIA copy (Level::dia_*) of a level of at least kSellMinRows rows whose
// entries lie on at most Level::kDiaMax diagonals, from the fixed pattern.
template <typename T>
__global__ void k_dia_scatter(int nnz, const int* __restrict__ map, const T* __restrict__ v, T* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) out[map[k]] = v[k];
}

void build_dia(Level& L, cudaStream_t s) {
  L.dia_nd = 0;
  if (L.coarsest || L.n < kSellMinRows || L.nnz <= 0) return;
  const int n = L.n;
  std::vector<int> rp(n + 1), col(L.nnz);
  IMPES_CUDA(cudaMemcpyAsync(rp.data(), L.rowptr.p, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaMemcpyAsync(col.data(), L.col.p, sizeof(int) * L.nnz, cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  std::vector<int> offs;
  for (int r = 0; r < n; ++r)
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      const int d = col[k] - r;
      if (std::find(offs.begin(), offs.end(), d) == offs.end()) {
        offs.push_back(d);
        if ((int)offs.size() > Level::kDiaMax) return;
      }
    }
  std::sort(offs.begin(), offs.end());
  std::vector<int> map(L.nnz);
  for (int r = 0; r < n; ++r)
    for (int k = rp[r]; k < rp[r + 1]; ++k) {
      const int d = (int)(std::lower_bound(offs.begin(), offs.end(), col[k] - r) - offs.begin());
      map[k] = d * n + r;
    }
  IMPES_REQUIRE((long long)offs.size() * n < (1LL << 31), IMPES_ERR_OOM, "DIA copy exceeds 2^31 entries");
  L.dia_map.alloc(L.nnz);
  IMPES_CUDA(cudaMemcpyAsync(L.dia_map.p, map.data(), sizeof(int) * L.nnz, cudaMemcpyHostToDevice, s));
  IMPES_CUDA(cudaStreamSynchronize(s));   // the host vectors go out of scope
  L.dia_nd = (int)offs.size();
  for (int d = 0; d < Level::kDiaMax; ++d) L.dia_off[d] = d < L.dia_nd ? offs[d] : 0;
  // a grid's 7-point stencil: offsets -a, -b, -1, 0, 1, b, a with b | a | n,
  // and no entry of offset +-1 crossing a z line's end nor of offset +-b a
  // y line's end (grid_nz = b, grid_ny = a / b, grid_nx = n / a)
  L.grid_nx = L.grid_ny = L.grid_nz = 0;
  if (L.dia_nd == 7) {
    const int a = offs[6], b = offs[5];
    bool grid = offs[0] == -a && offs[1] == -b && offs[2] == -1 && offs[3] == 0 && offs[4] == 1 && b > 1 &&
                a > b && a % b == 0 && n % a == 0;
    for (int r = 0; grid && r < n; ++r)
      for (int k = rp[r]; k < rp[r + 1]; ++k) {
        const int c = col[k], d = c - r;
        if ((d == 1 || d == -1) && r / b != c / b) grid = false;
        if ((d == b || d == -b) && r / a != c / a) grid = false;
      }
    if (grid) {
      L.grid_nz = b;
      L.grid_ny = a / b;
      L.grid_nx = n / a;
    }
  }
}

// Gather the SELL values and scatter the DIA values of the levels whose sweeps
// read them (all levels with a copy when `all`, before the autotuner has
// chosen) from their CSR values: slot 0 the fp64 values, 1 the fp32 ones.  A
// DIA array is zeroed when first allocated; the pattern's entries overwrite
// the same places every time.
void sell_refresh(AMG& h, int slot, cudaStream_t s, bool all = false, bool l0_fp32_done = false) {
  for (auto& up : h.levels) {
    Level& L = *up;
    // level 0's fp64 DIA copy is written by the equilibration, and its fp32
    // one, when l0_fp32_done, by the fp32 conversion
    const bool l0_written = !all && &L == h.levels[0].get() && (slot == 0 || l0_fp32_done);
    if (L.dia_nd > 0 && (all || L.dia_on[slot]) && !l0_written) {
      const size_t len = (size_t)L.dia_nd * L.n;
      if (slot == 0 && L.val.p) {
        if (L.dia_val.n < len) {
          L.dia_val.alloc(len);
          IMPES_CUDA(cudaMemsetAsync(L.dia_val.p, 0, len * sizeof(double), s));
        }
        k_dia_scatter<double><<<grid_for(L.nnz, TB), TB, 0, s>>>(L.nnz, L.dia_map.p, L.val.p, L.dia_val.p);
        ::impes::count_launch();
      } else if (slot == 1 && L.valf.p) {
        if (L.dia_valf.n < len) {
          L.dia_valf.alloc(len);
          IMPES_CUDA(cudaMemsetAsync(L.dia_valf.p, 0, len * sizeof(float), s));
        }
        k_dia_scatter<float><<<grid_for(L.nnz, TB), TB, 0, s>>>(L.nnz, L.dia_map.p, L.valf.p, L.dia_valf.p);
        ::impes::count_launch();
      }
      IMPES_CHECK_LAUNCH();
    }
    if (L.sell_slices <= 0 || !(all || L.sell_on[slot])) continue;
    if (slot == 0) {
      if (!L.val.p) continue;
      L.sell_val.ensure(L.sell_len);
      k_sell_gather<<<grid_for(L.sell_len, TB), TB, 0, s>>>(L.sell_len, L.sell_map.p, L.val.p, L.sell_val.p);
    } else {
      if (!L.valf.p) continue;
      L.sell_valf.ensure(L.sell_len);
      k_sell_gather_f<<<grid_for(L.sell_len, TB), TB, 0, s>>>(L.sell_len, L.sell_map.p, L.valf.p, L.sell_valf.p);
    }
    ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
  }
}

}  // namespace

void amg_setup(AMG& h, int n, int nnz, const int* rowptr, const int* col, const double* val,
               cudaStream_t s) {
  IMPES_REQUIRE(n > 0 && nnz > 0, IMPES_ERR_ARG, "empty matrix");
  h.drop_graphs();
  {
    const char* ev = getenv("IMPES_NO_GRAPHS");
    h.use_graphs = !(ev && ev[0] == '1');
    const char* es = getenv("IMPES_NO_STEP_GRAPH");
    h.use_step_graph = !(es && es[0] == '1');
    const char* et = getenv("IMPES_TAIL");
    h.use_tail = et && et[0] == '1';
    h.tail_level = -1;
    const char* eg = getenv("IMPES_DIA_TILE");
    h.use_dia_tile = eg && eg[0] == '1';
  }
  h.levels.clear();
  h.built = false;
  h.fp64_stale = false;
  h.iflag.ensure(8);
  h.red.ensure(4096);
  h.scal.ensure(256);
  // validate the caller's CSR before reading it
  IMPES_CUDA(cudaMemsetAsync(h.iflag.p, 0, sizeof(int), s));
  k_validate_csr<<<grid_for(n, TB), TB, 0, s>>>(n, nnz, rowptr, col, h.iflag.p); ::impes::count_launch();
  k_nonfinite<<<grid_for(nnz, TB), TB, 0, s>>>(val, nnz, h.iflag.p); ::impes::count_launch();
  int bad = to_host_int(h, h.iflag.p, s);
  IMPES_REQUIRE(!(bad & 7), IMPES_ERR_BAD_CSR, "malformed CSR (row pointers, column range or order)");
  IMPES_REQUIRE(!(bad & 8), IMPES_ERR_NAN, "non-finite matrix value");

  auto L0p = std::make_unique<Level>();
  Level& L0 = *L0p;
  L0.n = n; L0.nnz = nnz;
  L0.rowptr.alloc(n + 1); L0.col.alloc(nnz); L0.val.alloc(nnz);
  IMPES_CUDA(cudaMemcpyAsync(L0.rowptr.p, rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
  IMPES_CUDA(cudaMemcpyAsync(L0.col.p, col, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
  h.levels.push_back(std::move(L0p));
  equilibrate_level0(h, val, s);

  DBuf<double> basis;
  int m = level0_basis(h, basis, n, h.prm.nullspace_dim, s);
  const double theta = h.prm.theta;
  for (int lvl = 0; lvl < h.prm.max_levels; ++lvl) {
    Level& L = *h.levels.back();
    L.avg_row = std::max(1, L.nnz / std::max(L.n, 1));
    const int nl = L.n;
    compute_inv_relax(h, L, s);
    alloc_level_vectors(L);
    if (nl <= h.prm.coarsest_size) { L.coarsest = true; break; }
    // strength + C/F split
    DBuf<unsigned char> strong(L.nnz);
    k_strength<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, L.val.p, theta, strong.p); ::impes::count_launch();
    DBuf<int> gcnt(nl + 1), gptr(nl + 1), fill(nl + 1);
    IMPES_CUDA(cudaMemsetAsync(gcnt.p, 0, sizeof(int) * (nl + 1), s));
    k_sym_count<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, strong.p, gcnt.p); ::impes::count_launch();
    int gn = exclusive_scan_i32(gcnt.p, gptr.p, nl, s);
    DBuf<int> gcol(std::max(gn, 1)), ucnt(nl);
    IMPES_CUDA(cudaMemcpyAsync(fill.p, gptr.p, sizeof(int) * nl, cudaMemcpyDeviceToDevice, s));
    k_sym_fill<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, strong.p, fill.p, gcol.p); ::impes::count_launch();
    k_sym_unique<<<grid_for(nl, TB), TB, 0, s>>>(nl, gptr.p, gcol.p, ucnt.p); ::impes::count_launch();
    DBuf<double> score(nl);
    k_score<<<grid_for(nl, TB), TB, 0, s>>>(nl, ucnt.p, h.prm.tiebreak_seed, lvl, score.p); ::impes::count_launch();
    DBuf<unsigned char> C(nl);
    k_cselect<<<grid_for(nl, TB), TB, 0, s>>>(nl, gptr.p, gcol.p, ucnt.p, score.p, C.p); ::impes::count_launch();
    DBuf<signed char> cf(nl), cf2(nl);
    IMPES_CUDA(cudaMemsetAsync(h.iflag.p, 0, sizeof(int), s));
    k_lift<<<grid_for(nl, TB), TB, 0, s>>>(nl, gptr.p, gcol.p, ucnt.p, C.p, cf.p, h.iflag.p); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
    int n_coarse = to_host_int(h, h.iflag.p, s);
    if ((double)n_coarse >= nl * 0.9) { L.coarsest = true; break; }  // :832
    // orphans + fine->coarse map
    DBuf<int> cflag(nl + 1), f2c(nl + 1);
    k_orphans<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, strong.p, cf.p, cf2.p, cflag.p); ::impes::count_launch();
    const int nc = exclusive_scan_i32(cflag.p, f2c.p, nl, s);
    // interpolation
    DBuf<double> pdiag(nl), ssum(nl), wcsum(nl), wfsum(nl);
    DBuf<int> scnt(nl), ccnt(nl + 1), cptr(nl + 1);
    k_p_stats<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, L.val.p, strong.p, cf2.p,
                                              pdiag.p, ssum.p, wcsum.p, wfsum.p, scnt.p); ::impes::count_launch();
    k_p_count<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, strong.p, cf2.p, scnt.p,
                                              ssum.p, ccnt.p); ::impes::count_launch();
    int ctot = exclusive_scan_i32(ccnt.p, cptr.p, nl, s);
    DBuf<int> ccol(std::max(ctot, 1));
    DBuf<double> cval(std::max(ctot, 1));
    k_p_fill<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, L.val.p, strong.p, cf2.p,
                                             f2c.p, pdiag.p, ssum.p, wcsum.p, wfsum.p, scnt.p,
                                             cptr.p, ccol.p, cval.p); ::impes::count_launch();
    DBuf<int> mcnt(nl + 1);
    k_p_merge<<<grid_for(nl, TB), TB, 0, s>>>(nl, cptr.p, ccol.p, cval.p, mcnt.p); ::impes::count_launch();
    L.nc = nc;
    L.prow.alloc(nl + 1);
    L.pnnz = exclusive_scan_i32(mcnt.p, L.prow.p, nl, s);
    L.pcol.alloc(std::max(L.pnnz, 1));
    L.pval.alloc(std::max(L.pnnz, 1));
    k_p_compact<<<grid_for(nl, TB), TB, 0, s>>>(nl, cptr.p, ccol.p, cval.p, L.prow.p, L.pcol.p, L.pval.p); ::impes::count_launch();
    DBuf<double> rsum(nl);
    IMPES_CUDA(cudaMemsetAsync(h.iflag.p, 0, sizeof(int), s));
    k_p_rowsum<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pval.p, cf2.p, rsum.p, h.iflag.p); ::impes::count_launch();
    int nzero = to_host_int(h, h.iflag.p, s);
    if (nzero > 0) {
      DBuf<int> extra(nl), ncnt(nl + 1), nrow(nl + 1);
      k_p_zero_extra<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.rowptr.p, L.col.p, cf2.p, f2c.p, rsum.p,
                                                     extra.p, L.prow.p, ncnt.p); ::impes::count_launch();
      int nn = exclusive_scan_i32(ncnt.p, nrow.p, nl, s);
      DBuf<int> ncol(nn);
      DBuf<double> nval(nn);
      k_p_insert<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pcol.p, L.pval.p, extra.p, nrow.p,
                                                 ncol.p, nval.p); ::impes::count_launch();
      IMPES_CUDA(cudaStreamSynchronize(s));
      L.prow = std::move(nrow); L.pcol = std::move(ncol); L.pval = std::move(nval);
      L.pnnz = nn;
      k_p_rowsum<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pval.p, cf2.p, rsum.p, h.iflag.p); ::impes::count_launch();
    }
    k_p_scale<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pval.p, cf2.p, rsum.p); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
    if (m > 0 && h.prm.nullspace_blend > 0.0) {
      m = orthonormalize(h, basis.p, nl, m, s);   // build_prolongation_rs_full :393-396
      k_p_blend<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pcol.p, L.pval.p, cf2.p, basis.p, m,
                                                h.prm.nullspace_blend, h.prm.nullspace_reg); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
    }
    if (h.prm.p_max_elements > 0 || h.prm.p_trunc_factor > 0.0) {
      DBuf<int> tcnt(nl + 1), trow(nl + 1);
      k_p_trunc_count<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pval.p, cf2.p, h.prm.p_max_elements,
                                                      h.prm.p_trunc_factor, tcnt.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      const int tn = exclusive_scan_i32(tcnt.p, trow.p, nl, s);
      DBuf<int> tcol(std::max(tn, 1));
      DBuf<double> tval(std::max(tn, 1));
      k_p_trunc_fill<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pcol.p, L.pval.p, cf2.p,
                                                     h.prm.p_max_elements, h.prm.p_trunc_factor, trow.p,
                                                     tcol.p, tval.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      IMPES_CUDA(cudaStreamSynchronize(s));
      L.prow = std::move(trow); L.pcol = std::move(tcol); L.pval = std::move(tval);
      L.pnnz = tn;
    }
    // R = P^T (sorted rows) and its values
    DBuf<int> rcnt(nc + 1), rfill(nc + 1);
    IMPES_CUDA(cudaMemsetAsync(rcnt.p, 0, sizeof(int) * (nc + 1), s));
    k_col_count<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pcol.p, rcnt.p); ::impes::count_launch();
    L.rrow.alloc(nc + 1);
    exclusive_scan_i32(rcnt.p, L.rrow.p, nc, s);
    L.rcol.alloc(std::max(L.pnnz, 1)); L.rsrc.alloc(std::max(L.pnnz, 1)); L.rval.alloc(std::max(L.pnnz, 1));
    IMPES_CUDA(cudaMemcpyAsync(rfill.p, L.rrow.p, sizeof(int) * nc, cudaMemcpyDeviceToDevice, s));
    k_r_fill<<<grid_for(nl, TB), TB, 0, s>>>(nl, L.prow.p, L.pcol.p, rfill.p, L.rcol.p, L.rsrc.p); ::impes::count_launch();
    k_r_sort<<<grid_for(nc, TB), TB, 0, s>>>(nc, L.rrow.p, L.rcol.p, L.rsrc.p); ::impes::count_launch();
    k_gather<<<grid_for(L.pnnz, TB), TB, 0, s>>>(L.pnnz, L.rsrc.p, L.pval.p, L.rval.p); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
    L.p_avg = std::max(1, L.pnnz / std::max(nl, 1));
    L.r_avg = std::max(1, L.pnnz / std::max(nc, 1));
    // Galerkin: AP = A P, A_c = R (AP)
    auto Ncp = std::make_unique<Level>();
    Level& Nc = *Ncp;
    Nc.n = nc;
    union_symbolic(h, nl, L.rowptr.p, L.col.p, L.prow.p, L.pcol.p, L.aprow, L.apcol, L.ap_maxrow, s);
    int apnnz;
    IMPES_CUDA(cudaMemcpyAsync(h.hint.p, L.aprow.p + nl, sizeof(int), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    apnnz = h.hint.p[0];
    L.apval.alloc(std::max(apnnz, 1));
    union_symbolic(h, nc, L.rrow.p, L.rcol.p, L.aprow.p, L.apcol.p, Nc.rowptr, Nc.col, L.ac_maxrow, s);
    IMPES_CUDA(cudaMemcpyAsync(h.hint.p, Nc.rowptr.p + nc, sizeof(int), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    Nc.nnz = h.hint.p[0];
    Nc.val.alloc(std::max(Nc.nnz, 1));
    L.planned = build_plan(nl, L.rowptr.p, L.col.p, L.prow.p, L.pcol.p, L.aprow.p, L.apcol.p, apnnz,
                           nullptr, L.ap_seg, L.ap_e, L.ap_f, L.ap_terms, s) &&
                build_plan(nc, L.rrow.p, L.rcol.p, L.aprow.p, L.apcol.p, Nc.rowptr.p, Nc.col.p, Nc.nnz,
                           L.rsrc.p, L.ac_seg, L.ac_r, L.ac_f, L.ac_terms, s);
    if (!L.planned) {
      L.ap_seg.release(); L.ap_e.release(); L.ap_f.release();
      L.ac_seg.release(); L.ac_r.release(); L.ac_f.release();
    }
    galerkin_numeric(L, Nc, s);
    // coarse basis (classical_amg.py:906-914)
    if (m > 0) {
      DBuf<double> Bc((size_t)std::max(nc, 1) * m);
      k_restrict_basis<<<grid_for(nc, TB), TB, 0, s>>>(nc, m, L.rrow.p, L.rcol.p, L.rval.p, basis.p, Bc.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      m = orthonormalize(h, Bc.p, nc, m, s);
      basis = std::move(Bc);
    }
    IMPES_CUDA(cudaStreamSynchronize(s));
    h.levels.push_back(std::move(Ncp));
  }
  Level& Lc = *h.levels.back();
  if (!Lc.coarsest) {  // max_levels reached (:917-934)
    Lc.avg_row = std::max(1, Lc.nnz / std::max(Lc.n, 1));
    compute_inv_relax(h, Lc, s);
    alloc_level_vectors(Lc);
    Lc.coarsest = true;
  }
  coarse_factor(h, Lc, s);
  for (auto& L : h.levels) level_precision_copies(h, *L, s);
  // frozen fp32 P factors of the plan terms (mixed precision, while memory allows)
  for (auto& L : h.levels) {
    L->ap_cf.release();
    L->ac_cf.release();
    L->ap_e16.release();
    L->ap_ebase.release();
    if (!h.prm.mixed_precision || L->coarsest || !L->planned || !L->pvalf.p) continue;
    size_t free_b = 0, total_b = 0;
    IMPES_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (4.0 * (double)(L->ap_terms + L->ac_terms) > 0.5 * (double)free_b) continue;
    if (L->ap_terms > 0) {
      L->ap_cf.alloc(L->ap_terms);
      k_gather_f<<<grid_for(L->ap_terms, TB), TB, 0, s>>>(L->ap_terms, L->ap_f.p, L->pvalf.p, L->ap_cf.p); ::impes::count_launch();
      const int apn = (int)L->apval.n;
      L->ap_ebase.alloc(apn);
      L->ap_e16.alloc(L->ap_terms);
      DBuf<int> flag(1);
      IMPES_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), s));
      k_ap_ebase<<<grid_for(L->n, TB), TB, 0, s>>>(L->n, L->aprow.p, L->rowptr.p, L->ap_ebase.p); ::impes::count_launch();
      k_ap_e16<<<grid_for(apn, TB), TB, 0, s>>>(apn, L->ap_seg.p, L->ap_e.p, L->ap_ebase.p, L->ap_e16.p, flag.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      int wide = 1;
      IMPES_CUDA(cudaMemcpyAsync(&wide, flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      IMPES_CUDA(cudaStreamSynchronize(s));
      if (wide) { L->ap_e16.release(); L->ap_ebase.release(); }
    }
    if (L->ac_terms > 0) {
      L->ac_cf.alloc(L->ac_terms);
      k_gather_f<<<grid_for(L->ac_terms, TB), TB, 0, s>>>(L->ac_terms, L->ac_r.p, L->pvalf.p, L->ac_cf.p); ::impes::count_launch();
    }
    IMPES_CHECK_LAUNCH();
  }
  // 16-bit column indices for the smoothing and residual passes (the pattern is
  // fixed from here on: update_matrix only changes values): absolute on levels
  // of <= 65536 rows, row-relative on larger levels whose entries all lie within
  // [row - 32768, row + 32767] (banded by the grid ordering, which coarsening
  // keeps: C-points are numbered in fine order); int columns otherwise.
  DBuf<int> rel_flag(1);
  for (auto& L : h.levels) {
    L->col16 = DBuf<unsigned short>();
    L->col16_rel = 0;
    if (L->nnz <= 0) continue;
    if (L->n <= 65536) {
      L->col16.alloc(L->nnz);
      k_narrow_cols<<<grid_for(L->nnz, 256), 256, 0, s>>>(L->nnz, L->col.p, L->col16.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      continue;
    }
    IMPES_CUDA(cudaMemsetAsync(rel_flag.p, 0, sizeof(int), s));
    k_rel16_check<<<grid_for(L->n, 256), 256, 0, s>>>(L->n, L->rowptr.p, L->col.p, rel_flag.p); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
    int out_of_band = 1;
    IMPES_CUDA(cudaMemcpyAsync(&out_of_band, rel_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    if (out_of_band) continue;
    L->col16.alloc(L->nnz);
    L->col16_rel = 1;
    k_narrow_cols_rel<<<grid_for(L->n, 256), 256, 0, s>>>(L->n, L->rowptr.p, L->col.p, L->col16.p); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
  }
  IMPES_CUDA(cudaStreamSynchronize(s));
  // the fp32 Galerkin chain's A*P values are allocated here, not at the first
  // update: that update may run inside a stream capture (whole-step graphs),
  // where cudaMalloc is refused
  if (h.prm.mixed_precision)
    for (auto& L : h.levels)
      if (!L->coarsest) L->apvalf.ensure(std::max<size_t>(L->apval.n, 1));
  if (sell_enabled()) {
    for (auto& L : h.levels) {
      build_sell(*L, s);
      build_dia(*L, s);
    }
    sell_refresh(h, 0, s, true);
    if (h.prm.mixed_precision) sell_refresh(h, 1, s, true);
  }
  amg_autotune(h, s);
  // the SELL copies the tuner did not pick are dropped
  for (auto& L : h.levels) {
    if (L->dia_nd > 0) {
      if (!L->dia_on[0]) L->dia_val.release();
      if (!L->dia_on[1]) L->dia_valf.release();
      if (!L->dia_on[0] && !L->dia_on[1]) {
        L->dia_map.release();
        L->dia_nd = 0;
      }
    }
    if (L->sell_slices <= 0) continue;
    if (!L->sell_on[0]) L->sell_val.release();
    if (!L->sell_on[1]) L->sell_valf.release();
    if (!L->sell_on[0] && !L->sell_on[1]) {
      L->sell_ptr.release(); L->sell_perm.release(); L->sell_map.release();
      L->sell_col16.release(); L->sell_col.release();
      L->sell_slices = 0;
      L->sell_len = 0;
    }
  }
  h.tail_level = amg_tail_level(h);
  h.built = true;
}

// The fp32 Galerkin chain of a mixed AMG (every level planned): the V-cycle of
// the mixed path reads only fp32 coarse values, so A*P and P^T(AP) gather 4-byte
// values.  The coarsest inverses come from the fp32 coarsest matrix.
void update_fp32_chain(AMG& h, cudaStream_t s) {
  Level& L0 = *h.levels[0];
  compute_inv_relax(h, L0, s);
  const bool dia0 = L0.dia_nd > 0 && L0.dia_on[1] && L0.dia_valf.p;
  if (dia0)
    k_to_float_dia<<<grid_for(L0.nnz, TB), TB, 0, s>>>(L0.nnz, L0.val.p, L0.valf.p, L0.dia_map.p, L0.dia_valf.p);
  else
    k_to_float<<<grid_for(L0.nnz, TB), TB, 0, s>>>(L0.nnz, L0.val.p, L0.valf.p);
  ::impes::count_launch();
  k_to_float<<<grid_for(L0.n, TB), TB, 0, s>>>(L0.n, L0.inv_relax.p, L0.inv_relaxf.p); ::impes::count_launch();
  cheb_copy_to_fp32(h, L0, s);
  IMPES_CHECK_LAUNCH();
  for (size_t l = 0; l < h.levels.size(); ++l) {
    Level& L = *h.levels[l];
    if (L.coarsest) break;
    Level& Nc = *h.levels[l + 1];
    const int apn = (int)L.apval.n;
    L.apvalf.ensure(std::max(apn, 1));
    Nc.valf.ensure(std::max(Nc.nnz, 1));
    const int lap = plan_lanes(apn, L.ap_terms), lac = plan_lanes(Nc.nnz, L.ac_terms);
    if (L.ap_e16.p && lap > 1) {
      launch_plan_lanes<float, true>(lap, apn, L.ap_seg.p, L.ap_ebase.p, nullptr, L.ap_e16.p, L.ap_cf.p, L.valf.p,
                                     L.apvalf.p, s);
    } else if (L.ap_e16.p) {
      k_plan_apply_cf16<float><<<grid_for(apn, 256, 16), 256, 0, s>>>(apn, L.ap_seg.p, L.ap_ebase.p, L.ap_e16.p,
                                                                      L.ap_cf.p, L.valf.p, L.apvalf.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
    } else if (L.ap_terms > 0 && L.ap_cf.p && lap > 1)
      launch_plan_lanes<float, false>(lap, apn, L.ap_seg.p, nullptr, L.ap_e.p, nullptr, L.ap_cf.p, L.valf.p,
                                      L.apvalf.p, s);
    else if (L.ap_terms == 0 || L.ap_cf.p)
      plan_apply_cf<float>(apn, L.ap_seg.p, L.ap_e.p, L.ap_cf.p, L.valf.p, L.apvalf.p, s);
    else
      plan_apply<float>(apn, L.ap_seg.p, L.ap_e.p, L.ap_f.p, L.valf.p, L.pvalf.p, L.apvalf.p, s);
    if (L.ac_terms > 0 && L.ac_cf.p && lac > 1)
      launch_plan_lanes<float, false>(lac, Nc.nnz, L.ac_seg.p, nullptr, L.ac_f.p, nullptr, L.ac_cf.p, L.apvalf.p,
                                      Nc.valf.p, s);
    else if (L.ac_terms == 0 || L.ac_cf.p)
      plan_apply_cf<float>(Nc.nnz, L.ac_seg.p, L.ac_f.p, L.ac_cf.p, L.apvalf.p, Nc.valf.p, s);
    else
      plan_apply<float>(Nc.nnz, L.ac_seg.p, L.ac_r.p, L.ac_f.p, L.pvalf.p, L.apvalf.p, Nc.valf.p, s);
    compute_inv_relax_f(h, Nc, s);
  }
  coarse_factor(h, *h.levels.back(), s, true);
  sell_refresh(h, 1, s, false, true);
  h.fp64_stale = true;
}

void amg_ensure_fp64(AMG& h, cudaStream_t s) {
  if (!h.fp64_stale) return;
  for (size_t l = 0; l < h.levels.size(); ++l) {
    Level& L = *h.levels[l];
    compute_inv_relax(h, L, s);
    if (L.coarsest) break;
    galerkin_numeric(L, *h.levels[l + 1], s);
  }
  coarse_factor(h, *h.levels.back(), s);
  sell_refresh(h, 0, s);
  h.fp64_stale = false;
}

void amg_update(AMG& h, const double* val, cudaStream_t s) {
  IMPES_REQUIRE(h.built, IMPES_ERR_STATE, "update before setup");
  const int tid = timers().begin(IMPES_PH_GALERKIN, s);
  double bytes = 0.0;
  bool all_planned = true;
  for (size_t l = 0; l + 1 < h.levels.size(); ++l) {
    const Level& L = *h.levels[l];
    bytes += 12.0 * L.nnz + 24.0 * L.pnnz + 8.0 * h.levels[l + 1]->nnz;
    if (!L.coarsest && !L.planned) all_planned = false;
  }
  equilibrate_level0(h, val, s);
  if (h.prm.mixed_precision && all_planned && h.levels.size() > 1) {
    update_fp32_chain(h, s);
    timers().end(tid, s, bytes * 0.6);   // 4-byte values instead of 8
    return;
  }
  h.fp64_stale = false;
  for (size_t l = 0; l < h.levels.size(); ++l) {
    Level& L = *h.levels[l];
    compute_inv_relax(h, L, s);
    if (L.coarsest) break;
    galerkin_numeric(L, *h.levels[l + 1], s);
  }
  coarse_factor(h, *h.levels.back(), s);
  for (auto& L : h.levels) {
    if (!h.prm.mixed_precision) break;
    L->valf.ensure(std::max(L->nnz, 1));
    L->inv_relaxf.ensure(std::max(L->n, 1));
    k_to_float<<<grid_for(L->nnz, TB), TB, 0, s>>>(L->nnz, L->val.p, L->valf.p); ::impes::count_launch();
    k_to_float<<<grid_for(L->n, TB), TB, 0, s>>>(L->n, L->inv_relax.p, L->inv_relaxf.p); ::impes::count_launch();
    cheb_copy_to_fp32(h, *L, s);
  }
  IMPES_CHECK_LAUNCH();
  sell_refresh(h, 0, s);
  if (h.prm.mixed_precision) sell_refresh(h, 1, s);
  timers().end(tid, s, bytes);
}

}  // namespace impes
