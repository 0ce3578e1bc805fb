// Pressure assembly (K1) and explicit saturation update (K4) of the IMPES step.
//
// Reference: researchim-ai/oil-simulator-py src/simulator/simulation.py
//   transmissibilities :52-74, pressure step :867-904, matrix :1546-1580,
//   right-hand side :1582-1620, well terms :1622-1660, saturation :968-1544;
//   src/simulator/fluid.py relperm :224-248/:377-435, densities :129-158/:330-375,
//   total compressibility :190-222, capillary pressure :273-296; pvt.py :48-64.
//
// This translation unit is compiled with -fmad=false: every expression keeps the
// reference's operation order and rounding (no fused multiply-add), so the
// assembled system matches the reference's float64 evaluation to the last bit
// wherever the reference's arithmetic is elementwise.
//
// K1 and K4a stage a 3-D brick of cells plus a one-cell face halo in shared
// memory: per-cell phase properties (mobilities, densities, capillary pressure,
// pressure) are evaluated once per brick cell, then every interior cell reads its
// six neighbours from shared memory.
#include "model.cuh"
#include <algorithm>
#include <math.h>
#include <mutex>

namespace impes {

namespace {

constexpr int kPvtCols = 9;  // P, Bo, Bw, Bg, mu_o, mu_w, mu_g, Rs, Rv
enum { C_P = 0, C_BO = 1, C_BW = 2, C_BG = 3, C_MUO = 4, C_MUW = 5, C_MUG = 6, C_RS = 7, C_RV = 8 };

// torch's scalar-exponent pow special cases (x*x, x*x*x, 1/sqrt, 1/x, 1/(x*x)).
__device__ __forceinline__ double tpow(double x, double e) {
  if (e == 0.0) return 1.0;
  if (e == 1.0) return x;
  if (e == 2.0) return x * x;
  if (e == 3.0) return x * x * x;
  if (e == -0.5) return 1.0 / sqrt(x);
  if (e == -1.0) return 1.0 / x;
  if (e == -2.0) return 1.0 / (x * x);
  return pow(x, e);
}
// torch.clamp semantics (NaN passes through; lo > hi yields hi).
__device__ __forceinline__ double tclamp(double x, double lo, double hi) {
  double y = (x < lo) ? lo : x;
  return (y > hi) ? hi : y;
}
__device__ __forceinline__ double tclamp_min(double x, double lo) { return (x < lo) ? lo : x; }
__device__ __forceinline__ double tclamp_max(double x, double hi) { return (x > hi) ? hi : x; }
// torch.maximum: NaN-propagating.
__device__ __forceinline__ double tmaximum(double a, double b) {
  if (isnan(a) || isnan(b)) return __longlong_as_double(0x7ff8000000000000LL);
  return a > b ? a : b;
}

// PVT table staged in shared memory: columns [9][rows] and slopes [8][rows-1].
struct PvtSmem {
  int rows;
  const double* col;    // 9 * rows
  const double* slope;  // 8 * (rows - 1)
};

__device__ void pvt_stage(const double* __restrict__ g, int rows, double* s_col, double* s_slope) {
  for (int t = threadIdx.x; t < rows * kPvtCols; t += blockDim.x) {
    int r = t / kPvtCols, c = t % kPvtCols;
    s_col[c * rows + r] = g[t];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < (kPvtCols - 1) * (rows - 1); t += blockDim.x) {
    int c = 1 + t / (rows - 1), r = t % (rows - 1);
    const double* xp = s_col;
    const double* fp = s_col + c * rows;
    s_slope[(c - 1) * (rows - 1) + r] = (fp[r + 1] - fp[r]) / (xp[r + 1] - xp[r]);
  }
  __syncthreads();
}

// numpy.interp(x, xp, fp) with flat extrapolation (pvt.py:48-50).
__device__ double pvt_interp(const PvtSmem& t, int c, double x) {
  const int n = t.rows;
  const double* xp = t.col;
  const double* fp = t.col + c * n;
  if (isnan(x)) return x;
  if (x < xp[0]) return fp[0];
  if (x >= xp[n - 1]) return fp[n - 1];
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid; else hi = mid;
  }
  if (xp[lo] == x) return fp[lo];
  double sl = t.slope[(c - 1) * (n - 1) + lo];
  double r = sl * (x - xp[lo]) + fp[lo];
  if (isnan(r)) {
    r = sl * (x - xp[lo + 1]) + fp[lo + 1];
    if (isnan(r) && fp[lo] == fp[lo + 1]) r = fp[lo];
  }
  return r;
}
// Fluid._eval_pvt(p, key): interpolation at p / 1e6 MPa (fluid.py:186-187).
__device__ __forceinline__ double pvt_at(const PvtSmem& t, int c, double p_pa) {
  return pvt_interp(t, c, p_pa / 1e6);
}

struct KR { double kro, krw, krg; };

// Fluid.get_rel_perms(sw, sg) (fluid.py:231-248, 377-435).
__device__ KR relperms(const ModelParams& P, double sw, double sg) {
  KR r;
  const double den = (1 - P.sw_cr) - P.so_r;
  double s_norm = tclamp((sw - P.sw_cr) / den, 0.0, 1.0);
  r.krw = tpow(s_norm, P.nw);
  if (P.relperm_model == 1) {
    const double dw = (1.0 - P.sw_cr) - P.so_r;
    double swn = tclamp((sw - P.sw_cr) / (dw + 1e-12), 0.0, 1.0);
    const double dg = (1.0 - P.sg_cr) - P.so_r;
    double sgn = tclamp((sg - P.sg_cr) / (dg + 1e-12), 0.0, 1.0);
    double krow = P.ko_end_w * tpow(1.0 - swn, P.now);
    double krog = P.ko_end_g * tpow(1.0 - sgn, P.nog);
    double kmin = P.ko_end_w < P.ko_end_g ? P.ko_end_w : P.ko_end_g;
    r.kro = tclamp_min(krow + krog - kmin, 0.0);
  } else {
    r.kro = tpow(1 - s_norm, P.no);
  }
  double sgn2 = tclamp(sg / ((1.0 - P.sw_cr) - P.so_r + 1e-10), 0.0, 1.0);
  r.krg = tpow(sgn2, P.ng);
  return r;
}

struct Visc { double o, w, g; };
__device__ __forceinline__ Visc viscosities(const ModelParams& P, const PvtSmem& t, double p) {
  Visc v;
  if (P.pvt_rows > 0) {
    v.o = pvt_at(t, C_MUO, p) * 1e-3;
    v.w = pvt_at(t, C_MUW, p) * 1e-3;
    v.g = pvt_at(t, C_MUG, p) * 1e-3;
  } else {
    v.o = P.mu_o; v.w = P.mu_w; v.g = P.mu_g;
  }
  return v;
}

struct Rho { double w, o, g; };
// Fluid.rho_w / rho_o / rho_g at pressure p (fluid.py:129-158, 330-375).
__device__ Rho densities(const ModelParams& P, const PvtSmem& t, double p) {
  Rho r;
  if (P.pvt_rows > 0) {
    double bw = pvt_at(t, C_BW, p), bo = pvt_at(t, C_BO, p), rs = pvt_at(t, C_RS, p);
    double bg = pvt_at(t, C_BG, p), rv = pvt_at(t, C_RV, p);
    r.w = P.rho_w_ref / (bw + 1e-12);
    r.o = (P.rho_o_ref + rs * P.rho_g_ref) / (bo + 1e-12);
    r.g = (P.rho_g_ref + rv * P.rho_o_ref) / (bg + 1e-12);
  } else {
    r.w = P.rho_w_ref * (1.0 + P.c_w * (p - 1e5));
    r.o = P.rho_o_ref * (1.0 + P.c_o * (p - 1e5));
    r.g = P.rho_g_ref * (1.0 + P.c_g * (p - 1e5));
  }
  return r;
}

// calc_total_compressibility (fluid.py:190-222).
__device__ double total_compressibility(const ModelParams& P, const PvtSmem& t, double p, double sw,
                                        double sg) {
  if (P.pvt_rows == 0) return P.cf;
  const double P_mpa = p / 1e6;
  const double Pp = P_mpa + 0.1, Pm = P_mpa - 0.1;
  const double x0 = P_mpa * 1e6, xp = Pp * 1e6, xm = Pm * 1e6;
  double c[3];
  const int cols[3] = {C_BW, C_BO, C_BG};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double B = pvt_at(t, cols[q], x0), Bp = pvt_at(t, cols[q], xp), Bm = pvt_at(t, cols[q], xm);
    double dB = (Bp - Bm) / (2 * 0.1);
    c[q] = -(dB / (B + 1e-12)) / 1e6;
  }
  const double so = 1.0 - sw - sg;
  return P.c_r + sw * c[0] + so * c[1] + sg * c[2];
}

__device__ __forceinline__ double capillary(const ModelParams& P, double sw) {
  if (P.pc_scale == 0.0) return 0.0;
  double s_norm = tclamp((sw - P.sw_cr) / ((1 - P.sw_cr) - P.so_r), 0.0, 1.0);
  return P.pc_scale * tpow(1.0 - s_norm + 1e-6, -P.pc_exponent);
}
__device__ __forceinline__ double capillary_og(const ModelParams& P, double sg) {
  if (P.pc_og_scale == 0.0) return 0.0;
  const double denom = (1 - P.sw_cr) - P.so_r;
  double sgn = tclamp(sg / (denom + 1e-12), 0.0, 1.0);
  return P.pc_og_scale * tpow(1.0 - sgn + 1e-6, -P.pc_og_exponent);
}

// Brick geometry shared by K1 and K4a.
struct Brick {
  int TI, TJ, TK;      // interior extents
  int hi, hj, hk;      // halo widths (0 or 1)
  int HI, HJ, HK;      // halo box extents
  int nbi, nbj, nbk;   // bricks per dimension
};

// Interior extents <= 8 (z), <= 8 or 16 (y), and at most 256 cells per brick;
// each dimension is split evenly so no brick is mostly empty.
Brick make_brick(const ModelParams& P) {
  Brick b;
  b.nbk = (P.nz + 7) / 8;
  b.TK = (P.nz + b.nbk - 1) / b.nbk;
  int tj = std::min(P.ny, P.nz == 1 ? 16 : 8);
  b.nbj = (P.ny + tj - 1) / tj;
  b.TJ = (P.ny + b.nbj - 1) / b.nbj;
  int ti = std::max(1, std::min(P.nx, 256 / (b.TK * b.TJ)));
  b.nbi = (P.nx + ti - 1) / ti;
  b.TI = (P.nx + b.nbi - 1) / b.nbi;
  b.hi = P.nx > 1; b.hj = P.ny > 1; b.hk = P.nz > 1;
  b.HI = b.TI + 2 * b.hi; b.HJ = b.TJ + 2 * b.hj; b.HK = b.TK + 2 * b.hk;
  return b;
}

// Raise a kernel's dynamic shared-memory limit when a launch needs more.
template <typename K>
void ensure_smem(K kernel, size_t bytes, size_t& current) {
  static std::mutex mu;   // several host threads may step different models
  std::lock_guard<std::mutex> lock(mu);
  if (bytes > current) {
    raise_smem_limit((const void*)kernel, bytes);
    current = bytes;
  }
}
size_t g_smem_k1 = 48 << 10, g_smem_k4 = 48 << 10;

__device__ __forceinline__ void brick_origin(const Brick& b, int& i0, int& j0, int& k0) {
  int bid = blockIdx.x;
  int bk = bid % b.nbk; bid /= b.nbk;
  int bj = bid % b.nbj; bid /= b.nbj;
  int bi = bid;
  i0 = bi * b.TI; j0 = bj * b.TJ; k0 = bk * b.TK;
}

// Binary search of `cell` in the sorted distinct well-cell list.
__device__ __forceinline__ int well_slot(const int* wc, int nwc, int cell) {
  int lo = 0, hi = nwc - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int v = wc[mid];
    if (v == cell) return mid;
    if (v < cell) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// ------------------------------------------------------------ static data
__global__ void k_transmissibility(ModelParams P, const double* __restrict__ kx,
                                   const double* __restrict__ ky, const double* __restrict__ kz,
                                   const double* __restrict__ poro, double* tx, double* ty,
                                   double* tz, double* pv) {
  const long long N = P.N;
  const double cell_volume = (P.dx * P.dy) * P.dz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N;
       c += (long long)gridDim.x * blockDim.x) {
    int k = c % P.nz;
    long long r = c / P.nz;
    int j = r % P.ny;
    int i = r / P.ny;
    pv[c] = cell_volume * poro[c];
    if (i < P.nx - 1) {
      double a = kx[c], b = kx[c + (long long)P.ny * P.nz];
      tx[c] = 2 * a * b / (a + b + 1e-15) * P.dy * P.dz / P.dx;          // simulation.py:66-67
    }
    if (j < P.ny - 1) {
      double a = ky[c], b = ky[c + P.nz];
      ty[((long long)i * (P.ny - 1) + j) * P.nz + k] = 2 * a * b / (a + b + 1e-15) * P.dx * P.dz / P.dy;
    }
    if (k < P.nz - 1) {
      double a = kz[c], b = kz[c + 1];
      tz[((long long)i * P.ny + j) * (P.nz - 1) + k] = 2 * a * b / (a + b + 1e-15) * P.dx * P.dy / P.dz;
    }
  }
}

__global__ void k_pattern(ModelParams P, int* rowptr, int* col) {
  const long long N = P.N;
  const long long plane = (long long)P.ny * P.nz;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c <= N;
       c += (long long)gridDim.x * blockDim.x) {
    long long rp = pattern_rowptr(c, P.nx, P.ny, P.nz);
    rowptr[c] = (int)rp;
    if (c == N) continue;
    int k = c % P.nz;
    long long r = c / P.nz;
    int j = r % P.ny;
    int i = r / P.ny;
    int e = (int)rp;
    if (i > 0) col[e++] = (int)(c - plane);
    if (j > 0) col[e++] = (int)(c - P.nz);
    if (k > 0) col[e++] = (int)(c - 1);
    col[e++] = (int)c;
    if (k < P.nz - 1) col[e++] = (int)(c + 1);
    if (j < P.ny - 1) col[e++] = (int)(c + P.nz);
    if (i < P.nx - 1) col[e++] = (int)(c + plane);
  }
}

// ------------------------------------------------------------ K1 assembly
// Shared layout per halo cell: p, mw, mo, mg, rw, ro, rg, pc (8 doubles).
constexpr int kK1Fields = 8;

__global__ void __launch_bounds__(256, 4) k_assemble(
    ModelParams P, Brick B, const double* __restrict__ pvt_g, const double* __restrict__ p,
    const double* __restrict__ sw, const double* __restrict__ sg, const double* __restrict__ tx,
    const double* __restrict__ ty, const double* __restrict__ tz, const double* __restrict__ pv,
    const WellDev* __restrict__ wells, const int* __restrict__ wc_cells,
    const int* __restrict__ wc_ptr, const int* __restrict__ wc_wells, int* __restrict__ well_mode,
    double dt, double* __restrict__ val, double* __restrict__ rhs) {
  extern __shared__ double smem[];
  double* s_pvt_col = smem;
  const int pvt_r = P.pvt_rows > 0 ? P.pvt_rows : 1;     // tables sized by the actual rows
  double* s_pvt_slope = s_pvt_col + kPvtCols * pvt_r;
  double* s_cells = s_pvt_slope + (kPvtCols - 1) * pvt_r;
  const int H = B.HI * B.HJ * B.HK;
  double* s_p = s_cells;
  double* s_mw = s_p + H;
  double* s_mo = s_mw + H;
  double* s_mg = s_mo + H;
  double* s_rw = s_mg + H;
  double* s_ro = s_rw + H;
  double* s_rg = s_ro + H;
  double* s_pc = s_rg + H;

  PvtSmem T{P.pvt_rows, s_pvt_col, s_pvt_slope};
  if (P.pvt_rows > 0) pvt_stage(pvt_g, P.pvt_rows, s_pvt_col, s_pvt_slope);

  int i0, j0, k0;
  brick_origin(B, i0, j0, k0);
  const bool grav = (P.dz > 0) && (P.nz > 1);
  const long long plane = (long long)P.ny * P.nz;

  // phase 1: per-cell properties on the brick + face halo (simulation.py:870-882)
  for (int t = threadIdx.x; t < H; t += blockDim.x) {
    int lk = t % B.HK, lj = (t / B.HK) % B.HJ, li = t / (B.HK * B.HJ);
    int i = i0 + li - B.hi, j = j0 + lj - B.hj, k = k0 + lk - B.hk;
    int out = (li < B.hi || li >= B.hi + B.TI) + (lj < B.hj || lj >= B.hj + B.TJ) +
              (lk < B.hk || lk >= B.hk + B.TK);
    if (out > 1 || i < 0 || j < 0 || k < 0 || i >= P.nx || j >= P.ny || k >= P.nz) continue;
    long long c = ((long long)i * P.ny + j) * P.nz + k;
    double pc_ = p[c], swc = sw[c], sgc = sg[c];
    KR kr = relperms(P, swc, sgc);
    Visc mu = viscosities(P, T, pc_);
    s_p[t] = pc_;
    s_mw[t] = kr.krw / mu.w;
    s_mo[t] = kr.kro / mu.o;
    s_mg[t] = kr.krg / mu.g;
    if (grav) {
      Rho r = densities(P, T, pc_);
      s_rw[t] = r.w; s_ro[t] = r.o; s_rg[t] = r.g;
    }
    s_pc[t] = capillary(P, swc);
  }
  __syncthreads();

  // phase 2: one matrix row and RHS entry per interior cell
  const int TI = B.TI, TJ = B.TJ, TK = B.TK;
  for (int t = threadIdx.x; t < TI * TJ * TK; t += blockDim.x) {
    int tk = t % TK, tj = (t / TK) % TJ, ti = t / (TK * TJ);
    int i = i0 + ti, j = j0 + tj, k = k0 + tk;
    if (i >= P.nx || j >= P.ny || k >= P.nz) continue;
    long long c = ((long long)i * P.ny + j) * P.nz + k;
    int li = ti + B.hi, lj = tj + B.hj, lk = tk + B.hk;
    auto sidx = [&](int a, int b_, int d) { return (a * B.HJ + b_) * B.HK + d; };
    int s0 = sidx(li, lj, lk);
    auto mt_at = [&](int s) { return s_mw[s] + s_mo[s] + s_mg[s]; };
    // total-mobility transmissibility of the face (a lower, b upper), upwind by
    // dp_prev = p_a - p_b > 0 (simulation.py:885-895)
    auto face_t = [&](double T_, int sa, int sb) {
      double dp = s_p[sa] - s_p[sb];
      return T_ * (dp > 0 ? mt_at(sa) : mt_at(sb));
    };
    double txm = 0, typ_ = 0, tym = 0, tzp = 0, tzm = 0, txp = 0;
    const bool hxm = i > 0, hxp = i < P.nx - 1, hym = j > 0, hyp = j < P.ny - 1;
    const bool hzm = k > 0, hzp = k < P.nz - 1;
    int sxm = hxm ? sidx(li - 1, lj, lk) : 0, sxp = hxp ? sidx(li + 1, lj, lk) : 0;
    int sym_ = hym ? sidx(li, lj - 1, lk) : 0, syp = hyp ? sidx(li, lj + 1, lk) : 0;
    int szm = hzm ? sidx(li, lj, lk - 1) : 0, szp = hzp ? sidx(li, lj, lk + 1) : 0;
    const long long iy = ((long long)i * (P.ny - 1) + j) * P.nz + k;
    const long long iz = ((long long)i * P.ny + j) * (P.nz - 1) + k;
    if (hxm) txm = face_t(tx[c - plane], sxm, s0);
    if (hxp) txp = face_t(tx[c], s0, sxp);
    if (hym) tym = face_t(ty[iy - P.nz], sym_, s0);
    if (hyp) typ_ = face_t(ty[iy], s0, syp);
    if (hzm) tzm = face_t(tz[iz - 1], szm, s0);
    if (hzp) tzp = face_t(tz[iz], s0, szp);

    // wells at this cell (simulation.py:1622-1660), in configuration order
    double well_diag = 0.0, q_well = 0.0;
    if (P.nwc > 0) {
      int slot = well_slot(wc_cells, P.nwc, (int)c);
      if (slot >= 0) {
        double mt = mt_at(s0);
        for (int q = wc_ptr[slot]; q < wc_ptr[slot + 1]; ++q) {
          int w = wc_wells[q];
          const WellDev W = wells[w];
          if (W.control_bhp == 0) {
            double rate_si = (W.value * P.rate_scale) / 86400.0 * (W.is_injector ? 1 : -1);
            if (!W.is_injector && W.has_bhp_min) {
              double denom = W.well_index * mt + 1e-12;
              double p_req = s_p[s0] - rate_si / denom;
              double p_min = W.bhp_min * 1e6;
              if (p_req < p_min) {
                well_mode[w] = 1;
                well_diag += W.well_index * mt;
                q_well += W.well_index * mt * p_min;
                continue;
              }
            }
            well_mode[w] = 0;
            q_well += rate_si;
          } else {
            well_diag += W.well_index * mt;
            q_well += W.well_index * mt * (W.value * 1e6);
          }
        }
      }
    }

    // accumulation (simulation.py:1569-1576, 1586-1591)
    const double ct = total_compressibility(P, T, s_p[s0], sw[c], sg[c]);
    const double acc = pv[c] * ct / dt;
    // diagonal in the reference's scatter_add order: x+, x-, y+, y-, z+, z-
    double diag = 0.0;
    if (hxp) diag += txp;
    if (hxm) diag += txm;
    if (hyp) diag += typ_;
    if (hym) diag += tym;
    if (hzp) diag += tzp;
    if (hzm) diag += tzm;
    diag += acc;
    diag += well_diag;

    // row in CSR order: x-, y-, z-, diag, z+, y+, x+
    long long e = pattern_rowptr(c, P.nx, P.ny, P.nz);
    if (hxm) val[e++] = -txm;
    if (hym) val[e++] = -tym;
    if (hzm) val[e++] = -tzm;
    val[e++] = diag;
    if (hzp) val[e++] = -tzp;
    if (hyp) val[e++] = -typ_;
    if (hxp) val[e++] = -txp;

    // right-hand side (simulation.py:1582-1620)
    const double comp = acc * s_p[s0];
    double qg = 0.0;
    if (grav) {
      auto gflow = [&](double T_, int sa, int sb) {
        int su = (s_p[sa] - s_p[sb] > 0) ? sa : sb;
        return T_ * P.gravity * P.dz *
               (s_mw[su] * s_rw[su] + s_mo[su] * s_ro[su] + s_mg[su] * s_rg[su]);
      };
      if (hzp) qg -= gflow(tz[iz], s0, szp);
      if (hzm) qg += gflow(tz[iz - 1], szm, s0);
    }
    double qpc = 0.0;
    if (P.pc_scale > 0) {
      auto pflow = [&](double T_, int sa, int sb) {
        double mo = (s_p[sa] - s_p[sb] > 0) ? s_mo[sa] : s_mo[sb];
        return T_ * mo * (s_pc[sb] - s_pc[sa]);
      };
      if (hxm) qpc += pflow(tx[c - plane], sxm, s0);
      if (hxp) qpc -= pflow(tx[c], s0, sxp);
      if (hym) qpc += pflow(ty[iy - P.nz], sym_, s0);
      if (hyp) qpc -= pflow(ty[iy], s0, syp);
      if (hzm) qpc += pflow(tz[iz - 1], szm, s0);
      if (hzp) qpc -= pflow(tz[iz], s0, szp);
    }
    rhs[c] = comp + q_well + qg + qpc;
  }
}

// ------------------------------------------------ K4: saturation update
// Well sources of the saturation step (simulation.py:1044-1347), one thread,
// wells in configuration order; component balance of the step (non-substep part).
__device__ void well_cell_phase(const ModelParams& P, const PvtSmem& T, double p, double sw,
                                double sg, double& mt, double& fw, double& fg, double& fo) {
  KR kr = relperms(P, sw, sg);
  Visc mu = viscosities(P, T, p);
  double mw = kr.krw / mu.w, mo = kr.kro / mu.o, mg = kr.krg / mu.g;
  mt = mw + mo + mg;
  fw = mw / (mt + 1e-10);
  fg = mg / (mt + 1e-10);
  fo = mo / (mt + 1e-10);
}

__global__ void k_well_sources(ModelParams P, const double* __restrict__ pvt_g,
                               const WellDev* __restrict__ wells, const int* __restrict__ wc_cells,
                               const double* __restrict__ p_new, const double* __restrict__ sw,
                               const double* __restrict__ sg, const double* __restrict__ pv,
                               double dt, double* wq /*3*nwc*/, double* bal /*12*/,
                               double* well_q, double* well_rates, const int* pred) {
  if (pred && *pred == 0) return;
  __shared__ double s_col[kPvtCols * kMaxPvtRows];
  __shared__ double s_slope[(kPvtCols - 1) * kMaxPvtRows];
  // per well: its additions to the (water, gas, oil) sources of its cell and to
  // the component balance (oil in, oil out, gas in, gas out), which phase 2 adds
  // up in well order; bit k of s_mask marks addition k as made
  __shared__ double s_q[kMaxWells][3];
  __shared__ double s_b[kMaxWells][4];
  __shared__ int s_mask[kMaxWells];
  __shared__ int s_slot[kMaxWells];
  PvtSmem T{P.pvt_rows, s_col, s_slope};
  if (P.pvt_rows > 0) pvt_stage(pvt_g, P.pvt_rows, s_col, s_slope);
  const bool pvt = P.pvt_rows > 0;
  const double so_r = P.so_r, sw_min = P.sw_cr, sg_min = P.sg_cr;
  // phase 1: every well on its own thread (a well's numbers depend only on its
  // cell's state)
  for (int w = threadIdx.x; w < P.nwells; w += blockDim.x) {
    const WellDev W = wells[w];
    const int c = W.cell;
    int mask = 0;
    double dq[3] = {0.0, 0.0, 0.0}, db[4] = {0.0, 0.0, 0.0, 0.0};
    s_slot[w] = -1;
    if (c >= 0) {  // a well outside the grid contributes nothing (simulation.py:1053-1054)
      s_slot[w] = well_slot(wc_cells, P.nwc, c);
      const double p = p_new[c], sw_c = sw[c], sg_c = sg[c], pv_c = pv[c];
      double mt, fw_, fg_, fo_;
      well_cell_phase(P, T, p, sw_c, sg_c, mt, fw_, fg_, fo_);
      double Bo = 0, Bw = 0, Bg = 0, Rs = 0, Rv = 0;
      if (pvt) {
        Bo = pvt_at(T, C_BO, p); Bw = pvt_at(T, C_BW, p); Bg = pvt_at(T, C_BG, p);
        Rs = pvt_at(T, C_RS, p); Rv = pvt_at(T, C_RV, p);
      }
      if (W.control_bhp == 0) {
        const double q_base = (W.value * P.rate_scale) / 86400.0;
        double q_total;
        if (W.is_injector && W.surface_rate && pvt)
          q_total = q_base * (W.injected_phase == 1 ? Bg : Bw);
        else
          q_total = q_base;
        q_total *= (W.is_injector ? 1 : -1);
        if (W.is_injector) {
          if (W.injected_phase == 1) {
            double sg_up = fmax(0.0, (1.0 - so_r - sw_c) - sg_c);
            double dS = (dt / fmax(pv_c, 1e-12)) * q_total;
            double alpha = 1.0;
            if (dS > 0.0) alpha = fmin(alpha, sg_up / fmax(dS, 1e-12));
            else alpha = fmin(alpha, (sg_c - sg_min) / fmax(fabs(dS), 1e-12));
            q_total *= fmax(0.0, fmin(1.0, alpha));
            dq[1] = q_total; mask |= 2;
            if (pvt) {
              double qg_surf = fmax(q_total, 0.0) / fmax(Bg, 1e-12) * 86400.0;
              double scale = dt / 86400.0;
              db[2] = qg_surf * scale;        // gas in
              db[0] = Rv * qg_surf * scale;   // oil in
              mask |= 8 | 32;
            }
          } else {
            double sw_up = fmax(0.0, (1.0 - so_r - sg_c) - sw_c);
            double dS = (dt / fmax(pv_c, 1e-12)) * q_total;
            double alpha = 1.0;
            if (dS > 0.0) alpha = fmin(alpha, sw_up / fmax(dS, 1e-12));
            else alpha = fmin(alpha, (sw_c - sw_min) / fmax(fabs(dS), 1e-12));
            q_total *= fmax(0.0, fmin(1.0, alpha));
            dq[0] = q_total; mask |= 1;
          }
        } else {
          // producer at rate
          if (pvt) {
            if (W.surface_rate) {
              switch (W.surface_phase) {
                case 0: q_total = -(q_base / fmax(fo_ / fmax(Bo, 1e-12) + fg_ * Rv / fmax(Bg, 1e-12), 1e-12)); break;
                case 1: q_total = -(q_base * Bw) / fmax(fw_, 1e-8); break;
                case 2: q_total = -(q_base / fmax(fg_ / fmax(Bg, 1e-12) + fo_ * Rs / fmax(Bo, 1e-12), 1e-12)); break;
                default:
                  q_total = -(q_base / fmax(fo_ / fmax(Bo, 1e-12) + fg_ * Rv / fmax(Bg, 1e-12) +
                                                fw_ / fmax(Bw, 1e-12), 1e-12));
              }
            }
            double sw_up = fmax(0.0, (1.0 - so_r - sg_c) - sw_c);
            double sw_dn = fmax(0.0, sw_c - sw_min);
            double sg_up = fmax(0.0, (1.0 - so_r - sw_c) - sg_c);
            double sg_dn = fmax(0.0, sg_c - sg_min);
            double dSw = (dt / fmax(pv_c, 1e-12)) * (q_total * fw_);
            double dSg = (dt / fmax(pv_c, 1e-12)) * (q_total * fg_);
            double alpha = 1.0;
            alpha = dSw > 0.0 ? fmin(alpha, sw_up / fmax(dSw, 1e-12)) : fmin(alpha, sw_dn / fmax(fabs(dSw), 1e-12));
            alpha = dSg > 0.0 ? fmin(alpha, sg_up / fmax(dSg, 1e-12)) : fmin(alpha, sg_dn / fmax(fabs(dSg), 1e-12));
            alpha = fmax(0.0, fmin(1.0, alpha));
            q_total *= alpha;
            if (W.limit_mask) {
              double d_o = fo_ / fmax(Bo, 1e-12) + fg_ * Rv / fmax(Bg, 1e-12);
              double d_w = fw_ / fmax(Bw, 1e-12);
              double d_g = fg_ / fmax(Bg, 1e-12) + fo_ * Rs / fmax(Bo, 1e-12);
              double d_l = d_o + d_w;
              double mx = INFINITY;
              bool any = false;
              if ((W.limit_mask & 1) && d_o > 0) { mx = fmin(mx, (W.limits[0] / 86400.0) / d_o); any = true; }
              if ((W.limit_mask & 2) && d_w > 0) { mx = fmin(mx, (W.limits[1] / 86400.0) / d_w); any = true; }
              if ((W.limit_mask & 4) && d_g > 0) { mx = fmin(mx, (W.limits[2] / 86400.0) / d_g); any = true; }
              if ((W.limit_mask & 8) && d_l > 0) { mx = fmin(mx, (W.limits[3] / 86400.0) / d_l); any = true; }
              if (any && fabs(q_total) > mx) q_total = -mx;
            }
            double aq = fabs(q_total);
            double oil_s = aq * (fo_ / fmax(Bo, 1e-12) + fg_ * Rv / fmax(Bg, 1e-12)) * 86400.0;
            double wat_s = aq * (fw_ / fmax(Bw, 1e-12)) * 86400.0;
            double gas_s = aq * (fg_ / fmax(Bg, 1e-12) + fo_ * Rs / fmax(Bo, 1e-12)) * 86400.0;
            well_rates[4 * w + 0] = oil_s;
            well_rates[4 * w + 1] = wat_s;
            well_rates[4 * w + 2] = gas_s;
            well_rates[4 * w + 3] = oil_s + wat_s;
            well_q[w] = q_total;
            double qo_res = -q_total * fo_, qg_res = -q_total * fg_;
            db[1] = dt * (fmax(qo_res, 0.0) / fmax(Bo, 1e-12) + Rv * fmax(qg_res, 0.0) / fmax(Bg, 1e-12));
            db[3] = dt * (fmax(qg_res, 0.0) / fmax(Bg, 1e-12) + Rs * fmax(qo_res, 0.0) / fmax(Bo, 1e-12));
            mask |= 16 | 64;
          }
          dq[0] = q_total * fw_;
          dq[1] = q_total * fg_;
          dq[2] = q_total * fo_;
          mask |= 1 | 2 | 4;
        }
      } else {
        const double p_bhp = W.value * 1e6;
        const double q_total = W.well_index * mt * (p - p_bhp);
        if (W.is_injector) {
          if (W.injected_phase == 1) {
            dq[1] = -q_total; mask |= 2;
            if (pvt) {
              double qg_surf = fmax(-q_total, 0.0) / fmax(Bg, 1e-12) * 86400.0;
              double scale = dt / 86400.0;
              db[2] = qg_surf * scale;
              db[0] = Rv * qg_surf * scale;
              mask |= 8 | 32;
            }
          } else {
            dq[0] = -q_total; mask |= 1;
          }
        } else {
          dq[0] = (-q_total) * fw_;
          dq[1] = (-q_total) * fg_;
          dq[2] = (-q_total) * fo_;
          mask |= 1 | 2 | 4;
          if (pvt) {
            double qabs = fabs(q_total);
            double qo_res = qabs * fo_, qg_res = qabs * fg_;
            db[1] = dt * (qo_res / fmax(Bo, 1e-12) + Rv * qg_res / fmax(Bg, 1e-12));
            db[3] = dt * (qg_res / fmax(Bg, 1e-12) + Rs * qo_res / fmax(Bo, 1e-12));
            mask |= 16 | 64;
          }
        }
      }
    }
    s_mask[w] = mask;
    for (int k = 0; k < 3; ++k) s_q[w][k] = dq[k];
    for (int k = 0; k < 4; ++k) s_b[w][k] = db[k];
  }
  __syncthreads();
  // phase 2: the sums in the reference's well order (one thread)
  if (threadIdx.x != 0) return;
  for (int t = 0; t < 3 * P.nwc; ++t) wq[t] = 0.0;
  for (int w = 0; w < P.nwells; ++w) {
    const int slot = s_slot[w], mask = s_mask[w];
    if (slot < 0) continue;
    if (mask & 1) wq[slot] += s_q[w][0];
    if (mask & 2) wq[P.nwc + slot] += s_q[w][1];
    if (mask & 4) wq[2 * P.nwc + slot] += s_q[w][2];
    // balance additions in the order the serial loop made them: gas in then
    // oil in (gas injectors), oil out then gas out (producers)
    if (mask & 32) bal[6 + 3] += s_b[w][2];
    if (mask & 8) bal[6 + 0] += s_b[w][0];
    if (mask & 16) bal[6 + 1] += s_b[w][1];
    if (mask & 64) bal[6 + 4] += s_b[w][3];
  }
}

// K4a: fluxes, divergence, dS and the substep ratio (simulation.py:968-1042, 1351-1379).
constexpr int kK4Fields = 6;  // p, mw, mg, rw, rg, pcog

__global__ void __launch_bounds__(256, 4) k_saturation_flux(
    ModelParams P, Brick B, const double* __restrict__ pvt_g, const double* __restrict__ p,
    const double* __restrict__ sw, const double* __restrict__ sg, const double* __restrict__ tx,
    const double* __restrict__ ty, const double* __restrict__ tz, const double* __restrict__ pv,
    const int* __restrict__ wc_cells, const double* __restrict__ wq, double dt,
    double* __restrict__ dsw_out, double* __restrict__ dsg_out, double* __restrict__ red,
    unsigned* __restrict__ counter, int* __restrict__ nsub_out, const int* pred) {
  if (pred && *pred == 0) return;
  extern __shared__ double smem[];
  double* s_pvt_col = smem;
  const int pvt_r = P.pvt_rows > 0 ? P.pvt_rows : 1;     // tables sized by the actual rows
  double* s_pvt_slope = s_pvt_col + kPvtCols * pvt_r;
  double* s_cells = s_pvt_slope + (kPvtCols - 1) * pvt_r;
  const int H = B.HI * B.HJ * B.HK;
  double* s_p = s_cells;
  double* s_mw = s_p + H;
  double* s_mg = s_mw + H;
  double* s_rw = s_mg + H;
  double* s_rg = s_rw + H;
  double* s_pcg = s_rg + H;
  __shared__ double s_red[3 * 8];
  __shared__ bool s_last;

  PvtSmem T{P.pvt_rows, s_pvt_col, s_pvt_slope};
  if (P.pvt_rows > 0) pvt_stage(pvt_g, P.pvt_rows, s_pvt_col, s_pvt_slope);
  int i0, j0, k0;
  brick_origin(B, i0, j0, k0);
  const bool grav = (P.dz > 0) && (P.nz > 1);
  const long long plane = (long long)P.ny * P.nz;
  for (int t = threadIdx.x; t < H; t += blockDim.x) {
    int lk = t % B.HK, lj = (t / B.HK) % B.HJ, li = t / (B.HK * B.HJ);
    int i = i0 + li - B.hi, j = j0 + lj - B.hj, k = k0 + lk - B.hk;
    int out = (li < B.hi || li >= B.hi + B.TI) + (lj < B.hj || lj >= B.hj + B.TJ) +
              (lk < B.hk || lk >= B.hk + B.TK);
    if (out > 1 || i < 0 || j < 0 || k < 0 || i >= P.nx || j >= P.ny || k >= P.nz) continue;
    long long c = ((long long)i * P.ny + j) * P.nz + k;
    double pc_ = p[c], swc = sw[c], sgc = sg[c];
    KR kr = relperms(P, swc, sgc);
    Visc mu = viscosities(P, T, pc_);
    s_p[t] = pc_;
    s_mw[t] = kr.krw / mu.w;
    s_mg[t] = kr.krg / mu.g;
    if (grav) {
      Rho r = densities(P, T, pc_);
      s_rw[t] = r.w; s_rg[t] = r.g;
    }
    s_pcg[t] = capillary_og(P, sgc);
  }
  __syncthreads();

  double rmax = 0.0, rnan = 0.0, rinf = 0.0;
  const int TI = B.TI, TJ = B.TJ, TK = B.TK;
  for (int t = threadIdx.x; t < TI * TJ * TK; t += blockDim.x) {
    int tk = t % TK, tj = (t / TK) % TJ, ti = t / (TK * TJ);
    int i = i0 + ti, j = j0 + tj, k = k0 + tk;
    if (i >= P.nx || j >= P.ny || k >= P.nz) continue;
    long long c = ((long long)i * P.ny + j) * P.nz + k;
    int li = ti + B.hi, lj = tj + B.hj, lk = tk + B.hk;
    auto sidx = [&](int a, int b_, int d) { return (a * B.HJ + b_) * B.HK + d; };
    int s0 = sidx(li, lj, lk);
    const long long iy = ((long long)i * (P.ny - 1) + j) * P.nz + k;
    const long long iz = ((long long)i * P.ny + j) * (P.nz - 1) + k;
    const bool pcog = P.pc_og_scale > 0;
    // water / gas flux through face (sa lower, sb upper) in direction d (0 x, 1 y, 2 z)
    auto flux = [&](double T_, int sa, int sb, bool zdir, double& fw, double& fg) {
      double dp = s_p[sa] - s_p[sb];
      bool up = dp > 0;
      double mw = up ? s_mw[sa] : s_mw[sb];
      double mg = up ? s_mg[sa] : s_mg[sb];
      double pw = dp, pg = dp;
      if (zdir && grav) {
        double rwa = 0.5 * (s_rw[sa] + s_rw[sb]);
        double rga = 0.5 * (s_rg[sa] + s_rg[sb]);
        pw = dp + P.gravity * rwa * P.dz;
        pg = dp + P.gravity * rga * P.dz;
      }
      fw = T_ * mw * pw;
      if (pcog) fg = T_ * mg * (pg - (s_pcg[sb] - s_pcg[sa]));
      else fg = T_ * mg * pg;
    };
    double dw = 0.0, dg = 0.0, fw, fg;
    if (i < P.nx - 1) { flux(tx[c], s0, sidx(li + 1, lj, lk), false, fw, fg); dw += fw; dg += fg; }
    if (i > 0) { flux(tx[c - plane], sidx(li - 1, lj, lk), s0, false, fw, fg); dw -= fw; dg -= fg; }
    if (j < P.ny - 1) { flux(ty[iy], s0, sidx(li, lj + 1, lk), false, fw, fg); dw += fw; dg += fg; }
    if (j > 0) { flux(ty[iy - P.nz], sidx(li, lj - 1, lk), s0, false, fw, fg); dw -= fw; dg -= fg; }
    if (k < P.nz - 1) { flux(tz[iz], s0, sidx(li, lj, lk + 1), true, fw, fg); dw += fw; dg += fg; }
    if (k > 0) { flux(tz[iz - 1], sidx(li, lj, lk - 1), s0, true, fw, fg); dw -= fw; dg -= fg; }
    double qwc = 0.0, qgc = 0.0;
    if (P.nwc > 0) {
      int slot = well_slot(wc_cells, P.nwc, (int)c);
      if (slot >= 0) { qwc = wq[slot]; qgc = wq[P.nwc + slot]; }
    }
    const double f = dt / pv[c];
    const double dSw = f * (qwc - dw);
    const double dSg = f * (qgc - dg);
    dsw_out[c] = dSw;
    dsg_out[c] = dSg;
    const double swc = sw[c], sgc = sg[c], eps = 1e-12;
    const double sw_up = tclamp_min(1.0 - P.so_r - sgc - swc, 0.0);
    const double sw_dn = tclamp_min(swc - P.sw_cr, 0.0);
    const double sg_up = tclamp_min(1.0 - P.so_r - swc - sgc, 0.0);
    const double sg_dn = tclamp_min(sgc - P.sg_cr, 0.0);
    double rw = dSw > 0 ? dSw / tclamp_min(sw_up, eps) : (-dSw) / tclamp_min(sw_dn, eps);
    double rg = dSg > 0 ? dSg / tclamp_min(sg_up, eps) : (-dSg) / tclamp_min(sg_dn, eps);
    double rl = tmaximum(fabs(dSw) / P.max_dS, fabs(dSg) / P.max_dS);
    double rat = tmaximum(tmaximum(rw, rg), rl);
    if (isnan(rat)) rnan = 1.0;
    else if (isinf(rat)) rinf = 1.0;
    else rmax = fmax(rmax, rat);
  }
  // block max -> partials; the last block derives N (simulation.py:1371-1379)
  rmax = warp_max(rmax); rnan = warp_max(rnan); rinf = warp_max(rinf);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { s_red[wid] = rmax; s_red[8 + wid] = rnan; s_red[16 + wid] = rinf; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a = fmax(a, s_red[w]); b = fmax(b, s_red[8 + w]); c = fmax(c, s_red[16 + w]);
    }
    red[3 * blockIdx.x + 0] = a; red[3 * blockIdx.x + 1] = b; red[3 * blockIdx.x + 2] = c;
    __threadfence();
    unsigned done = atomicAdd(counter, 1u);
    s_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {   // the whole last block reduces the block maxima
    __threadfence();
    double a = 0, b = 0, c = 0;
    for (unsigned q = threadIdx.x; q < gridDim.x; q += blockDim.x) {
      a = fmax(a, ((volatile double*)red)[3 * q]);
      b = fmax(b, ((volatile double*)red)[3 * q + 1]);
      c = fmax(c, ((volatile double*)red)[3 * q + 2]);
    }
    a = warp_max(a); b = warp_max(b); c = warp_max(c);
    __syncthreads();
    if (lane == 0) { s_red[wid] = a; s_red[8 + wid] = b; s_red[16 + wid] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
      a = 0; b = 0; c = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        a = fmax(a, s_red[w]); b = fmax(b, s_red[8 + w]); c = fmax(c, s_red[16 + w]);
      }
      double rat_max = (b > 0 || c > 0) ? 0.0 : a;  // nan_to_num(nan=0, posinf=0)
      double n = ceil(rat_max);
      int N = n > 2.0e9 ? 2000000000 : (int)n;
      if (N < 1) N = 1;
      if (N > P.max_substeps) N = P.max_substeps;
      *nsub_out = N;
      *counter = 0u;
    }
  }
}

// Per-substep component balance of PVT runs (simulation.py:1396-1505): one
// thread replays the substeps at the well cells.
__global__ void k_well_substeps(ModelParams P, const double* __restrict__ pvt_g,
                                const WellDev* __restrict__ wells, const double* __restrict__ p_new,
                                const double* __restrict__ sw, const double* __restrict__ sg,
                                const double* __restrict__ dsw, const double* __restrict__ dsg,
                                const int* __restrict__ nsub, double dt, double* __restrict__ contrib,
                                double* bal, const int* pred) {
  if (pred && *pred == 0) return;
  // contrib[(s * nwells + w) * 4 + q]: the addend of bal[6 + {0, 1, 3, 4}[q]] for
  // substep s and well w (never negative), -1 where the reference adds nothing
  __shared__ double s_col[kPvtCols * kMaxPvtRows];
  __shared__ double s_slope[(kPvtCols - 1) * kMaxPvtRows];
  PvtSmem T{P.pvt_rows, s_col, s_slope};
  pvt_stage(pvt_g, P.pvt_rows, s_col, s_slope);
  const int N = *nsub;
  const double dt_sub = dt / N;
  const double so_r = P.so_r;
  const int items = N * P.nwells;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int s = it / P.nwells, w = it % P.nwells;
    double add[4] = {-1.0, -1.0, -1.0, -1.0};   // bal[6+0], bal[6+1], bal[6+3], bal[6+4]
    const WellDev W = wells[w];
    const int c = W.cell;
    if (c >= 0) {
      double swc = sw[c], sgc = sg[c];
      const double dws = dsw[c] / N, dgs = dsg[c] / N;
      for (int q = 0; q <= s; ++q) {   // the cell's state after substep s (as K4b)
        swc = swc + dws;
        sgc = sgc + dgs;
        swc = tclamp(swc, P.sw_cr, 1.0 - so_r - sgc);
        sgc = tclamp(sgc, P.sg_cr, 1.0 - so_r - swc);
      }
      const double p = p_new[c];
      const double Bo = pvt_at(T, C_BO, p), Bw = pvt_at(T, C_BW, p), Bg = pvt_at(T, C_BG, p);
      const double Rs = pvt_at(T, C_RS, p), Rv = pvt_at(T, C_RV, p);
      const double mu_w = pvt_at(T, C_MUW, p), mu_o = pvt_at(T, C_MUO, p), mu_g = pvt_at(T, C_MUG, p);
      KR kr = relperms(P, swc, sgc);
      double mw = kr.krw / (mu_w + 1e-12), mo = kr.kro / (mu_o + 1e-12), mg = kr.krg / (mu_g + 1e-12);
      double mt = mw + mo + mg;
      double fw_ = mw / (mt + 1e-12), fg_ = mg / (mt + 1e-12), fo_ = mo / (mt + 1e-12);
      if (W.control_bhp == 0) {
        const double q_base = (W.value * P.rate_scale) / 86400.0;
        if (W.is_injector) {
          double q_sub = W.surface_rate ? q_base * (W.injected_phase == 1 ? Bg : Bw) : q_base;
          if (W.injected_phase == 1) {
            double qg_surf = fmax(q_sub, 0.0) / fmax(Bg, 1e-12) * 86400.0;
            add[2] = qg_surf * (dt_sub / 86400.0);
            add[0] = Rv * qg_surf * (dt_sub / 86400.0);
          }
        } else {
          double q_sub;
          if (W.surface_rate) {
            switch (W.surface_phase) {
              case 0: q_sub = -(q_base / fmax(fo_ / fmax(Bo, 1e-12) + fg_ * Rv / fmax(Bg, 1e-12), 1e-12)); break;
              case 1: q_sub = -(q_base * Bw) / fmax(fw_, 1e-12); break;
              case 2: q_sub = -(q_base / fmax(fg_ / fmax(Bg, 1e-12) + fo_ * Rs / fmax(Bo, 1e-12), 1e-12)); break;
              default:
                q_sub = -(q_base / fmax(fo_ / fmax(Bo, 1e-12) + fg_ * Rv / fmax(Bg, 1e-12) +
                                          fw_ / fmax(Bw, 1e-12), 1e-12));
            }
          } else {
            q_sub = -q_base;
          }
          double qo_res = fmax(-q_sub * fo_, 0.0), qg_res = fmax(-q_sub * fg_, 0.0);
          add[1] = dt_sub * (qo_res / fmax(Bo, 1e-12) + Rv * qg_res / fmax(Bg, 1e-12));
          add[3] = dt_sub * (qg_res / fmax(Bg, 1e-12) + Rs * qo_res / fmax(Bo, 1e-12));
        }
      } else {
        double q_sub = W.well_index * mt * (p - W.value * 1e6);
        if (W.is_injector) {
          if (W.injected_phase == 1) {
            double qg_surf = fmax(-q_sub, 0.0) / fmax(Bg, 1e-12) * 86400.0;
            add[2] = qg_surf * (dt_sub / 86400.0);
            add[0] = Rv * qg_surf * (dt_sub / 86400.0);
          }
        } else {
          double qabs = fabs(q_sub);
          double qo_res = qabs * fo_, qg_res = qabs * fg_;
          add[1] = dt_sub * (qo_res / fmax(Bo, 1e-12) + Rv * qg_res / fmax(Bg, 1e-12));
          add[3] = dt_sub * (qg_res / fmax(Bg, 1e-12) + Rs * qo_res / fmax(Bo, 1e-12));
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) contrib[(size_t)it * 4 + q] = add[q];
  }
  __syncthreads();
  // the reference's accumulation order: substeps outer, wells inner (simulation.py:1396-1505)
  if (threadIdx.x < 4) {
    const int q = threadIdx.x;
    const int slot = q == 0 ? 0 : q == 1 ? 1 : q == 2 ? 3 : 4;
    double acc = bal[6 + slot];
    for (int it = 0; it < items; ++it) {
      const double v = contrib[(size_t)it * 4 + q];
      if (!(v < 0.0)) acc += v;   // NaN propagates as before
    }
    bal[6 + slot] = acc;
  }
}

// K4b: N clamped substeps per cell, So, and the mass balance (simulation.py:1381-1527).
constexpr int kSatBlock = 256;
__global__ void __launch_bounds__(kSatBlock) k_saturation_substeps(
    ModelParams P, const double* __restrict__ pvt_g, const double* __restrict__ p_new,
    double* __restrict__ sw, double* __restrict__ sg, double* __restrict__ so,
    const double* __restrict__ dsw, const double* __restrict__ dsg, const double* __restrict__ pv,
    const int* __restrict__ nsub, double* __restrict__ red, unsigned* __restrict__ counter,
    double* __restrict__ bal, const int* pred) {
  if (pred && *pred == 0) return;
  __shared__ double s_col[kPvtCols * kMaxPvtRows];
  __shared__ double s_slope[(kPvtCols - 1) * kMaxPvtRows];
  __shared__ double s_w[kSatBlock / 32];
  __shared__ bool s_last;
  PvtSmem T{P.pvt_rows, s_col, s_slope};
  if (P.pvt_rows > 0) pvt_stage(pvt_g, P.pvt_rows, s_col, s_slope);
  const int N = *nsub;
  const double so_r = P.so_r;
  double acc[6] = {0, 0, 0, 0, 0, 0};  // water in/out, oil in/out, gas in/out
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N;
       c += (long long)gridDim.x * blockDim.x) {
    const double sw0 = sw[c], sg0 = sg[c];
    const double dws = dsw[c] / N, dgs = dsg[c] / N;
    double swc = sw0, sgc = sg0;
    for (int s = 0; s < N; ++s) {
      swc = swc + dws;
      sgc = sgc + dgs;
      swc = tclamp(swc, P.sw_cr, 1.0 - so_r - sgc);
      sgc = tclamp(sgc, P.sg_cr, 1.0 - so_r - swc);
    }
    sw[c] = swc;
    sg[c] = sgc;
    so[c] = 1.0 - swc - sgc;
    const double dwe = swc - sw0, dge = sgc - sg0;
    Rho r = densities(P, T, p_new[c]);
    const double mw = dwe * pv[c] * r.w;
    const double mg = dge * pv[c] * r.g;
    const double mo = (-(dwe + dge)) * pv[c] * r.o;
    acc[0] += tclamp_min(mw, 0.0); acc[1] += -tclamp_max(mw, 0.0);
    acc[2] += tclamp_min(mo, 0.0); acc[3] += -tclamp_max(mo, 0.0);
    acc[4] += tclamp_min(mg, 0.0); acc[5] += -tclamp_max(mg, 0.0);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double v = block_sum<kSatBlock>(acc[q], s_w);
    if (threadIdx.x == 0) red[6 * blockIdx.x + q] = v;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned done = atomicAdd(counter, 1u);
    s_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {   // the whole last block sums the block partials (fixed order)
    __threadfence();
    double tot[6] = {0, 0, 0, 0, 0, 0};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
      for (int q = 0; q < 6; ++q) tot[q] += ((volatile double*)red)[6 * b + q];
#pragma unroll
    for (int q = 0; q < 6; ++q) tot[q] = block_sum<kSatBlock>(tot[q], s_w);
    if (threadIdx.x == 0) {
      // mass_balance[water/oil/gas][in/out] (simulation.py:1521-1526)
      for (int q = 0; q < 6; ++q) bal[q] += tot[q];
      // component accum = in - out (simulation.py:1529-1530)
      bal[6 + 2] = bal[6 + 0] - bal[6 + 1];
      bal[6 + 5] = bal[6 + 3] - bal[6 + 4];
      *counter = 0u;
    }
  }
}

size_t brick_smem(const Brick& b, int fields, int pvt_rows) {
  const size_t r = pvt_rows > 0 ? (size_t)pvt_rows : 1;
  return sizeof(double) * ((size_t)kPvtCols * r + (size_t)(kPvtCols - 1) * r +
                           (size_t)fields * b.HI * b.HJ * b.HK);
}

}  // namespace

// ---------------------------------------------------------------- host API
void model_build_static(Model& m, const double* kx, const double* ky, const double* kz,
                        const double* poro, cudaStream_t s) {
  const ModelParams& P = m.P;
  m.tx.alloc(std::max<long long>(1, (long long)(P.nx - 1) * P.ny * P.nz));
  m.ty.alloc(std::max<long long>(1, (long long)P.nx * (P.ny - 1) * P.nz));
  m.tz.alloc(std::max<long long>(1, (long long)P.nx * P.ny * (P.nz - 1)));
  m.pv.alloc(P.N);
  k_transmissibility<<<grid_for(P.N, 256), 256, 0, s>>>(P, kx, ky, kz, poro, m.tx.p, m.ty.p,
                                                        m.tz.p, m.pv.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  m.nnz = (int)pattern_rowptr(P.N, P.nx, P.ny, P.nz);
  m.rowptr.alloc(P.N + 1);
  m.col.alloc(m.nnz);
  k_pattern<<<grid_for(P.N + 1, 256), 256, 0, s>>>(P, m.rowptr.p, m.col.p); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  Brick b = make_brick(P);
  int blocks = b.nbi * b.nbj * b.nbk;
  m.red_blocks = std::max(blocks, (int)grid_for(P.N, kSatBlock));
  m.red.alloc((size_t)6 * m.red_blocks + 16);
  m.counter.alloc(2);
  IMPES_CUDA(cudaMemsetAsync(m.counter.p, 0, 2 * sizeof(unsigned), s));
  m.nsub.alloc(1);
  m.dsw.alloc(P.N);
  m.dsg.alloc(P.N);
  m.wq.alloc(std::max(1, 3 * P.nwc));
  m.wsub.alloc(std::max<size_t>(1, (size_t)4 * std::max(P.max_substeps, 1) * std::max(P.nwells, 1)));
}

void model_pattern(Model& m, int* rowptr, int* col, cudaStream_t s) {
  IMPES_CUDA(cudaMemcpyAsync(rowptr, m.rowptr.p, sizeof(int) * (m.P.N + 1), cudaMemcpyDeviceToDevice, s));
  IMPES_CUDA(cudaMemcpyAsync(col, m.col.p, sizeof(int) * m.nnz, cudaMemcpyDeviceToDevice, s));
}

void model_assemble(Model& m, const double* p, const double* sw, const double* sg, double dt,
                    double* csr_val, double* rhs, cudaStream_t s) {
  Brick b = make_brick(m.P);
  int blocks = b.nbi * b.nbj * b.nbk;
  ensure_smem(k_assemble, brick_smem(b, kK1Fields, m.P.pvt_rows), g_smem_k1);
  const double F = 0.5 * (double)(m.nnz - m.P.N);
  const int tid = timers().begin(IMPES_PH_ASSEMBLE, s);
  k_assemble<<<blocks, 256, brick_smem(b, kK1Fields, m.P.pvt_rows), s>>>(
      m.P, b, m.pvt.p, p, sw, sg, m.tx.p, m.ty.p, m.tz.p, m.pv.p, m.wells.p, m.wc_cells.p,
      m.wc_ptr.p, m.wc_wells.p, m.well_mode.p, dt, csr_val, rhs); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  timers().end(tid, s, 8.0 * (6.0 * m.P.N + 3.0 * F));   // reads p, Sw, Sg, PV, T; writes A, b
}

void model_saturation(Model& m, const double* p_new, double* sw, double* sg, double* so, double dt,
                      cudaStream_t s, const int* pred) {
  const ModelParams& P = m.P;
  const int tid = timers().begin(IMPES_PH_SATURATION, s);
  if (P.nwells > 0) {
    k_well_sources<<<1, kMaxWells, 0, s>>>(P, m.pvt.p, m.wells.p, m.wc_cells.p, p_new, sw, sg, m.pv.p,
                                     dt, m.wq.p, m.balances.p, m.well_q.p, m.well_rates.p, pred); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
  }
  Brick b = make_brick(P);
  int blocks = b.nbi * b.nbj * b.nbk;
  ensure_smem(k_saturation_flux, brick_smem(b, kK4Fields, P.pvt_rows), g_smem_k4);
  k_saturation_flux<<<blocks, 256, brick_smem(b, kK4Fields, P.pvt_rows), s>>>(
      P, b, m.pvt.p, p_new, sw, sg, m.tx.p, m.ty.p, m.tz.p, m.pv.p, m.wc_cells.p, m.wq.p, dt,
      m.dsw.p, m.dsg.p, m.red.p, m.counter.p, m.nsub.p, pred); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  if (P.pvt_rows > 0 && P.nwells > 0) {
    k_well_substeps<<<1, 256, 0, s>>>(P, m.pvt.p, m.wells.p, p_new, sw, sg, m.dsw.p, m.dsg.p,
                                      m.nsub.p, dt, m.wsub.p, m.balances.p, pred); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
  }
  unsigned g = grid_for(P.N, kSatBlock);
  k_saturation_substeps<<<g, kSatBlock, 0, s>>>(P, m.pvt.p, p_new, sw, sg, so, m.dsw.p, m.dsg.p,
                                                m.pv.p, m.nsub.p, m.red.p, m.counter.p + 1,
                                                m.balances.p, pred); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  timers().end(tid, s, 8.0 * (6.0 * P.N + 0.5 * (double)(m.nnz - P.N)));
}

}  // namespace impes
