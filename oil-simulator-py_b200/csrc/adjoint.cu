// Discrete adjoint of the oil-water IMPES step (no reference counterpart).
//
// Objective: J = sum_steps sum_producers (q_o - q_target)^2, q_o the producer's
// oil rate in m3/day from the flux balance of its pressure row,
//   q_fb = sum_f c_f (p1_nb - p1_c) - PV_c ct/dt (p1_c - p0_c) + Qg_c,
// times the oil fractional flow at the previous saturation.  (The well's own
// WI*lambda_t*(p1_c - p_bhp), simulation.py:1297, is the same number
// algebraically but p1_c sits within an ulp of p_bhp, so it is round-off.)
// Gradients are taken with respect to ln k (kx, ky, kz of a cell scaled together)
// and porosity.
//
// Forward step (the library's own): assembly (simulation.py:867-904, 1546-1620)
// on (p0, sw0), FGMRES with the AMG V-cycle, saturation (simulation.py:968-1544)
// on (p1, sw0).  Reverse step n, with adjoints gp = dJ/dp1 and gs = dJ/dsw1:
//   1. saturation: replay the clamped substeps from the stored increment and
//      substep count -> dJ/d(dSw), dJ/dsw0; chain through dSw = dt/PV (q_w - div)
//      to the face fluxes, well sources, sw0 (upwind mobility), p1 and PV;
//   2. objective term of step n: adds to gp and gs, and d/dq_fb to the producer
//      rows of the pressure adjoint;
//   3. A mu = gp.  A is symmetric (one upwinded value at (i,j) and (j,i),
//      simulation.py:1563-1565), so the forward hierarchy and FGMRES solve it;
//   4. pressure parameters: d/dc_f = -(mu'_a - mu'_b)(p1_a - p1_b),
//      d/dacc_i = mu'_i (p0_i - p1_i), d/dQg_i = mu'_i, d/dp0_i = mu'_i acc_i, with
//      mu' = mu plus the objective's d/dq_fb at producer cells; well diagonal
//      and BHP source terms use mu.
// Upwind directions, substep counts and the availability choke's branch follow
// the forward values; a clamp passes the gradient on its bounds.
//
// Scope: two phases (s_g = 0, no gas wells), no PVT table, no capillarity,
// Corey relative permeability, no bhp_min switching.  Other models are refused.
#include "amg.cuh"
#include "model.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace impes {

namespace {

constexpr int TBA = 256;

__device__ __forceinline__ double apow(double x, double e) {
  if (e == 0.0) return 1.0;
  if (e == 1.0) return x;
  if (e == 2.0) return x * x;
  if (e == 3.0) return x * x * x;
  return pow(x, e);
}
// d/dx x^e
__device__ __forceinline__ double dapow(double x, double e) {
  if (e == 0.0) return 0.0;
  if (e == 1.0) return 1.0;
  if (e == 2.0) return 2.0 * x;
  if (e == 3.0) return 3.0 * x * x;
  return e * pow(x, e - 1.0);
}

struct MobD {
  double mw, mo, dmw, dmo;
};
// Corey mobilities and their derivatives in sw (fluid.py:224-248, 377-435).
__device__ __forceinline__ MobD mob_d(const ModelParams& P, double sw) {
  const double den = (1 - P.sw_cr) - P.so_r;
  const double x = (sw - P.sw_cr) / den;
  const double s = (x < 0.0) ? 0.0 : ((x > 1.0) ? 1.0 : x);
  const double ds = (x >= 0.0 && x <= 1.0) ? 1.0 / den : 0.0;
  MobD r;
  r.mw = apow(s, P.nw) / P.mu_w;
  r.mo = apow(1 - s, P.no) / P.mu_o;
  r.dmw = dapow(s, P.nw) * ds / P.mu_w;
  r.dmo = -dapow(1 - s, P.no) * ds / P.mu_o;
  return r;
}
__device__ __forceinline__ double rho_w(const ModelParams& P, double p) {
  return P.rho_w_ref * (1.0 + P.c_w * (p - 1e5));
}
__device__ __forceinline__ double rho_o(const ModelParams& P, double p) {
  return P.rho_o_ref * (1.0 + P.c_o * (p - 1e5));
}

struct Nb {
  long long j;    // neighbour cell
  long long fid;  // face index in its direction's array
  double T;       // transmissibility
  int dir;        // 0 x, 1 y, 2 z
  int lower;      // this cell is the face's lower-index cell
};
// Faces of cell c in the layout of k_transmissibility.
__device__ __forceinline__ int cell_faces(const ModelParams& P, const double* __restrict__ tx,
                                          const double* __restrict__ ty,
                                          const double* __restrict__ tz, long long c, Nb* f) {
  const int k = (int)(c % P.nz);
  const long long r = c / P.nz;
  const int j = (int)(r % P.ny);
  const int i = (int)(r / P.ny);
  const long long plane = (long long)P.ny * P.nz;
  int n = 0;
  if (i > 0) f[n++] = Nb{c - plane, c - plane, tx[c - plane], 0, 0};
  if (i < P.nx - 1) f[n++] = Nb{c + plane, c, tx[c], 0, 1};
  const long long iy = ((long long)i * (P.ny - 1) + j) * P.nz + k;
  if (j > 0) f[n++] = Nb{c - P.nz, iy - P.nz, ty[iy - P.nz], 1, 0};
  if (j < P.ny - 1) f[n++] = Nb{c + P.nz, iy, ty[iy], 1, 1};
  const long long iz = ((long long)i * P.ny + j) * (P.nz - 1) + k;
  if (k > 0) f[n++] = Nb{c - 1, iz - 1, tz[iz - 1], 2, 0};
  if (k < P.nz - 1) f[n++] = Nb{c + 1, iz, tz[iz], 2, 1};
  return n;
}

struct ProdTerms {
  int nf;
  Nb f[6];
  double cf[6];
  double csum, acc, qfb, fo, dfo;
};
// Flux-balance rate of the producer at cell c and the coefficients of its row.
__device__ void producer_terms(const ModelParams& P, const double* tx, const double* ty,
                               const double* tz, const double* pv, const double* P0,
                               const double* S0, const double* P1, long long c, double dt,
                               ProdTerms& t) {
  t.nf = cell_faces(P, tx, ty, tz, c, t.f);
  const bool grav = (P.dz > 0) && (P.nz > 1);
  double inflow = 0.0, csum = 0.0, qg = 0.0;
  for (int q = 0; q < t.nf; ++q) {
    const long long nb = t.f[q].j;
    const long long a = t.f[q].lower ? c : nb, b = t.f[q].lower ? nb : c;
    const long long up = (P0[a] - P0[b] > 0) ? a : b;
    const MobD m = mob_d(P, S0[up]);
    const double cf = t.f[q].T * (m.mw + m.mo);
    t.cf[q] = cf;
    inflow += cf * (P1[nb] - P1[c]);
    csum += cf;
    if (grav && t.f[q].dir == 2) {
      const double gf = t.f[q].T * P.gravity * P.dz * (m.mw * rho_w(P, P0[up]) + m.mo * rho_o(P, P0[up]));
      qg += t.f[q].lower ? -gf : gf;
    }
  }
  t.csum = csum;
  t.acc = pv[c] * P.cf / dt;
  t.qfb = inflow - t.acc * (P1[c] - P0[c]) + qg;
  const MobD mc = mob_d(P, S0[c]);
  const double mt = mc.mw + mc.mo + 1e-10;
  t.fo = mc.mo / mt;
  t.dfo = (mc.dmo * mt - mc.mo * (mc.dmw + mc.dmo)) / (mt * mt);
}

__global__ void k_producer_rates(ModelParams P, const double* tx, const double* ty,
                                 const double* tz, const double* pv, const int* prod_cells,
                                 int nprod, const double* P0, const double* S0, const double* P1,
                                 double dt, double* out) {
  for (int w = threadIdx.x; w < nprod; w += blockDim.x) {
    ProdTerms t;
    producer_terms(P, tx, ty, tz, pv, P0, S0, P1, prod_cells[w], dt, t);
    out[w] = t.qfb * t.fo * 86400.0;
  }
}

// 1. replay of the clamped substeps (k_saturation_substeps) per cell.
__global__ void k_adj_sat_cell(ModelParams P, const double* __restrict__ S0,
                               const double* __restrict__ DS, const int* __restrict__ NS,
                               const double* __restrict__ pv, const double* __restrict__ gs,
                               double dt, double* __restrict__ gs_prev,
                               double* __restrict__ gam, double* __restrict__ gpv) {
  const int N = *NS;
  const double lo = P.sw_cr, hi = 1.0 - P.so_r - 0.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N;
       c += (long long)gridDim.x * blockDim.x) {
    const double inc = DS[c] / N;
    double s = S0[c], du = 0.0, dv = 1.0;
    for (int q = 0; q < N; ++q) {
      const double x = s + inc;
      if (x < lo) { s = lo; du = 0.0; dv = 0.0; }
      else if (x > hi) { s = hi; du = 0.0; dv = 0.0; }
      else { s = x; du += 1.0 / N; }
    }
    const double g = gs[c];
    const double gds = g * du;
    gs_prev[c] = g * dv;
    gam[c] = gds * dt / pv[c];
    gpv[c] += -gds * DS[c] / pv[c];
  }
}

// Saturation-step well sources (simulation.py:1051-1347, oil-water): one thread.
__global__ void k_adj_sat_wells(ModelParams P, const WellDev* __restrict__ wells,
                                const double* __restrict__ S0, const double* __restrict__ P1,
                                const double* __restrict__ pv, const double* __restrict__ gam,
                                double dt, double* gs_prev, double* gp, double* gpv) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int w = 0; w < P.nwells; ++w) {
    const WellDev W = wells[w];
    const int c = W.cell;
    if (c < 0) continue;
    const double g = gam[c];
    const double sw = S0[c], pvc = pv[c];
    const MobD m = mob_d(P, sw);
    const double mt = m.mw + m.mo, dmt = m.dmw + m.dmo;
    if (W.control_bhp == 0) {
      const double q_base = (W.value * P.rate_scale) / 86400.0;
      if (W.is_injector) {
        // q_w = q * clip(alpha), alpha = sw_up / dS (dS > 0) or (sw - sw_min) / |dS|
        const double q = q_base;
        const double sw_up = fmax(0.0, (1.0 - P.so_r - 0.0) - sw);
        const double dS = (dt / fmax(pvc, 1e-12)) * q;
        if (dS > 0.0) {
          const double ratio = sw_up / fmax(dS, 1e-12);
          if (ratio < 1.0 && ratio >= 0.0 && dS > 1e-12) {
            // q * sw_up * pv / (dt q) = sw_up * pv / dt
            if (sw_up > 0.0) gs_prev[c] += g * (-pvc / dt);
            gpv[c] += g * sw_up / dt;
          }
        } else if (dS < 0.0) {
          const double ratio = (sw - P.sw_cr) / fmax(fabs(dS), 1e-12);
          if (ratio < 1.0 && ratio >= 0.0 && fabs(dS) > 1e-12) {
            // q * (sw - sw_min) * pv / (dt |q|)
            gs_prev[c] += g * q * pvc / (dt * fabs(q));
            gpv[c] += g * q * (sw - P.sw_cr) / (dt * fabs(q));
          }
        }
      } else {
        // q_w = -q_base * fw
        const double mtt = mt + 1e-10;
        const double dfw = (m.dmw * mtt - m.mw * dmt) / (mtt * mtt);
        gs_prev[c] += g * (-q_base) * dfw;
      }
    } else {
      const double dpw = P1[c] - W.value * 1e6;
      if (W.is_injector) {
        // q_w = -WI mt (p - p_bhp)
        gp[c] += -g * W.well_index * mt;
        gs_prev[c] += -g * W.well_index * dmt * dpw;
      } else {
        // q_w = -WI mt (p - p_bhp) fw
        const double mtt = mt + 1e-10;
        const double fw = m.mw / mtt;
        const double dfw = (m.dmw * mtt - m.mw * dmt) / (mtt * mtt);
        gp[c] += -g * W.well_index * mt * fw;
        gs_prev[c] += -g * W.well_index * dpw * (dmt * fw + mt * dfw);
      }
    }
  }
}

// Saturation-step face fluxes f = T mw_up pot: gather over each cell's faces.
__global__ void k_adj_sat_faces(ModelParams P, const double* __restrict__ tx,
                                const double* __restrict__ ty, const double* __restrict__ tz,
                                const double* __restrict__ S0, const double* __restrict__ P1,
                                const double* __restrict__ gam, double* __restrict__ gs_prev,
                                double* __restrict__ gp, double* __restrict__ gtx,
                                double* __restrict__ gty, double* __restrict__ gtz) {
  const bool grav = (P.dz > 0) && (P.nz > 1);
  const double drw = P.rho_w_ref * P.c_w;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N;
       c += (long long)gridDim.x * blockDim.x) {
    Nb f[6];
    const int nf = cell_faces(P, tx, ty, tz, c, f);
    double dgs = 0.0, dgp = 0.0;
    for (int q = 0; q < nf; ++q) {
      const long long nb = f[q].j;
      const long long a = f[q].lower ? c : nb, b = f[q].lower ? nb : c;
      const double dp = P1[a] - P1[b];
      const long long up = (dp > 0) ? a : b;
      const MobD m = mob_d(P, S0[up]);
      double pot = dp, dpot_a = 1.0, dpot_b = -1.0;
      if (grav && f[q].dir == 2) {
        const double rwa = 0.5 * (rho_w(P, P1[a]) + rho_w(P, P1[b]));
        pot = dp + P.gravity * rwa * P.dz;
        dpot_a += P.gravity * 0.5 * drw * P.dz;
        dpot_b += P.gravity * 0.5 * drw * P.dz;
      }
      // div_a += f, div_b -= f, d/ddiv = -gam
      const double gf = -gam[a] + gam[b];
      if (up == c) dgs += gf * f[q].T * pot * m.dmw;
      dgp += gf * f[q].T * m.mw * (f[q].lower ? dpot_a : dpot_b);
      if (f[q].lower) {
        double* gt = f[q].dir == 0 ? gtx : (f[q].dir == 1 ? gty : gtz);
        gt[f[q].fid] += gf * m.mw * pot;
      }
    }
    gs_prev[c] += dgs;
    gp[c] += dgp;
  }
}

// Objective of step n: one thread over the producers.
__global__ void k_adj_objective(ModelParams P, const double* tx, const double* ty,
                                const double* tz, const double* pv, const int* prod_cells,
                                int nprod, const double* P0, const double* S0, const double* P1,
                                double dt, const double* target, double* gs_prev, double* gp,
                                double* dmu) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int w = 0; w < nprod; ++w) {
    const long long c = prod_cells[w];
    ProdTerms t;
    producer_terms(P, tx, ty, tz, pv, P0, S0, P1, c, dt, t);
    const double rate = t.qfb * t.fo * 86400.0;
    const double gq = 2.0 * (rate - target[w]);
    const double gqfb = gq * t.fo * 86400.0;
    gs_prev[c] += gq * t.qfb * 86400.0 * t.dfo;
    for (int q = 0; q < t.nf; ++q) gp[t.f[q].j] += gqfb * t.cf[q];
    gp[c] += -gqfb * (t.csum + t.acc);
    dmu[w] = gqfb;
  }
}

// Pressure-step well terms (wd = WI mt, q = wd p_bhp) with mu, then mu' = mu + d/dq_fb.
__global__ void k_adj_press_wells(ModelParams P, const WellDev* __restrict__ wells,
                                  const double* __restrict__ S0, const double* __restrict__ P1,
                                  const int* prod_cells, int nprod, const double* dmu,
                                  double* mu, double* gs_prev) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int w = 0; w < P.nwells; ++w) {
    const WellDev W = wells[w];
    const int c = W.cell;
    if (c < 0 || W.control_bhp == 0) continue;
    const MobD m = mob_d(P, S0[c]);
    const double gwd = mu[c] * (W.value * 1e6 - P1[c]);
    gs_prev[c] += gwd * W.well_index * (m.dmw + m.dmo);
  }
  for (int w = 0; w < nprod; ++w) mu[prod_cells[w]] += dmu[w];
}

// Pressure-step parameters with mu': faces, gravity, accumulation.
__global__ void k_adj_press_cell(ModelParams P, const double* __restrict__ tx,
                                 const double* __restrict__ ty, const double* __restrict__ tz,
                                 const double* __restrict__ pv, const double* __restrict__ P0,
                                 const double* __restrict__ S0, const double* __restrict__ P1,
                                 const double* __restrict__ mu, double dt,
                                 double* __restrict__ gs_prev, double* __restrict__ gp_prev,
                                 double* __restrict__ gpv, double* __restrict__ gtx,
                                 double* __restrict__ gty, double* __restrict__ gtz) {
  const bool grav = (P.dz > 0) && (P.nz > 1);
  const double drw = P.rho_w_ref * P.c_w, dro = P.rho_o_ref * P.c_o;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N;
       c += (long long)gridDim.x * blockDim.x) {
    Nb f[6];
    const int nf = cell_faces(P, tx, ty, tz, c, f);
    double dgs = 0.0, dgp = 0.0;
    for (int q = 0; q < nf; ++q) {
      const long long nb = f[q].j;
      const long long a = f[q].lower ? c : nb, b = f[q].lower ? nb : c;
      const long long up = (P0[a] - P0[b] > 0) ? a : b;
      const MobD m = mob_d(P, S0[up]);
      const double mt = m.mw + m.mo;
      const double gc = -(mu[a] - mu[b]) * (P1[a] - P1[b]);
      if (up == c) dgs += gc * f[q].T * (m.dmw + m.dmo);
      double gtf = gc * mt;
      if (grav && f[q].dir == 2) {
        // Qg[a] -= gf, Qg[b] += gf; gf = Tz g dz (mw rw + mo ro) at the upwind cell
        const double gg = mu[b] - mu[a];
        const double rw = rho_w(P, P0[up]), ro = rho_o(P, P0[up]);
        const double k = P.gravity * P.dz;
        gtf += gg * k * (m.mw * rw + m.mo * ro);
        if (up == c) {
          dgs += gg * f[q].T * k * (m.dmw * rw + m.dmo * ro);
          dgp += gg * f[q].T * k * (m.mw * drw + m.mo * dro);
        }
      }
      if (f[q].lower) {
        double* gt = f[q].dir == 0 ? gtx : (f[q].dir == 1 ? gty : gtz);
        gt[f[q].fid] += gtf;
      }
    }
    const double acc = pv[c] * P.cf / dt;
    gs_prev[c] += dgs;
    gp_prev[c] = dgp + mu[c] * acc;
    gpv[c] += mu[c] * (P0[c] - P1[c]) * P.cf / dt;
  }
}

// dJ/dln k and dJ/dphi from the accumulated dJ/dT and dJ/dPV.
__global__ void k_adj_params(ModelParams P, const double* __restrict__ kx,
                             const double* __restrict__ ky, const double* __restrict__ kz,
                             const double* __restrict__ gtx, const double* __restrict__ gty,
                             const double* __restrict__ gtz, const double* __restrict__ gpv,
                             double* __restrict__ g_lnk, double* __restrict__ g_poro) {
  const double vol = (P.dx * P.dy) * P.dz;
  const double geo[3] = {P.dy * P.dz / P.dx, P.dx * P.dz / P.dy, P.dx * P.dy / P.dz};
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < P.N;
       c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c % P.nz);
    const long long r = c / P.nz;
    const int j = (int)(r % P.ny);
    const int i = (int)(r / P.ny);
    const long long plane = (long long)P.ny * P.nz;
    const long long iy = ((long long)i * (P.ny - 1) + j) * P.nz + k;
    const long long iz = ((long long)i * P.ny + j) * (P.nz - 1) + k;
    // k_c dT/dk_c for T = geo 2 a b / (a + b + eps): 2 geo k_c k_o (k_o + eps) / (k_c + k_o + eps)^2
    auto term = [&](double gT, double kc, double ko, double g) {
      const double s = kc + ko + 1e-15;
      return gT * g * 2.0 * kc * ko * (ko + 1e-15) / (s * s);
    };
    double acc = 0.0;
    if (i > 0) acc += term(gtx[c - plane], kx[c], kx[c - plane], geo[0]);
    if (i < P.nx - 1) acc += term(gtx[c], kx[c], kx[c + plane], geo[0]);
    if (j > 0) acc += term(gty[iy - P.nz], ky[c], ky[c - P.nz], geo[1]);
    if (j < P.ny - 1) acc += term(gty[iy], ky[c], ky[c + P.nz], geo[1]);
    if (k > 0) acc += term(gtz[iz - 1], kz[c], kz[c - 1], geo[2]);
    if (k < P.nz - 1) acc += term(gtz[iz], kz[c], kz[c + 1], geo[2]);
    g_lnk[c] = acc;
    g_poro[c] = vol * gpv[c];
  }
}

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  Events() {
    IMPES_CUDA(cudaEventCreate(&a));
    IMPES_CUDA(cudaEventCreate(&b));
  }
  ~Events() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  double ms() {
    float t = 0.f;
    IMPES_CUDA(cudaEventSynchronize(b));
    IMPES_CUDA(cudaEventElapsedTime(&t, a, b));
    return t;
  }
};

std::vector<int> producer_cells(const Model& m) {
  std::vector<int> v;
  for (const WellDev& w : m.wells_host)
    if (!w.is_injector && w.cell >= 0) v.push_back(w.cell);
  return v;
}

// One forward IMPES step of the adjoint runs: p (p0 in, p1 out), sw updated.
void forward_step(Model& m, AMG& a, double* p, double* pold, double* sw, double* sg, double* so,
                  double dt, const impes_krylov_params& kp, const int* prod, int nprod,
                  double* rates, long long& iters, cudaStream_t s) {
  const ModelParams& P = m.P;
  model_assemble(m, p, sw, sg, dt, m.csr_val.p, m.rhs.p, s);
  if (!a.built || a.levels[0]->n != P.N)
    amg_setup(a, P.N, m.nnz, m.rowptr.p, m.col.p, m.csr_val.p, s);
  else
    amg_update(a, m.csr_val.p, s);
  IMPES_CUDA(cudaMemcpyAsync(pold, p, sizeof(double) * P.N, cudaMemcpyDeviceToDevice, s));
  impes_krylov_stats st{};
  amg_fgmres(a, m.rhs.p, p, kp, st, s);
  iters += st.iterations;
  if (!st.converged) throw Error(IMPES_ERR_NOT_CONVERGED, "adjoint forward: FGMRES did not converge");
  if (nprod > 0) {
    k_producer_rates<<<1, 32, 0, s>>>(P, m.tx.p, m.ty.p, m.tz.p, m.pv.p, prod, nprod, pold, sw, p,
                                      dt, rates); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
  }
  model_saturation(m, p, sw, sg, so, dt, s);
}

}  // namespace

void adjoint_check_model(const Model& m) {
  const ModelParams& P = m.P;
  IMPES_REQUIRE(P.pvt_rows == 0, IMPES_ERR_ARG, "adjoint: PVT tables are outside its scope");
  IMPES_REQUIRE(P.pc_scale == 0.0 && P.pc_og_scale == 0.0, IMPES_ERR_ARG,
                "adjoint: capillary pressure is outside its scope");
  IMPES_REQUIRE(P.relperm_model == 0, IMPES_ERR_ARG, "adjoint: Corey relative permeability only");
  IMPES_REQUIRE(P.sg_cr == 0.0, IMPES_ERR_ARG, "adjoint: oil-water only (sg_cr must be 0)");
  for (const WellDev& w : m.wells_host) {
    IMPES_REQUIRE(!(w.is_injector && w.injected_phase == 1), IMPES_ERR_ARG,
                  "adjoint: gas injection is outside its scope");
    IMPES_REQUIRE(!(w.control_bhp == 0 && !w.is_injector && w.has_bhp_min), IMPES_ERR_ARG,
                  "adjoint: bhp_min switching is outside its scope");
  }
}

int adjoint_num_producers(const Model& m) { return (int)producer_cells(m).size(); }

void adjoint_rates(Model& m, AMG& a, double* p, double* sw, int steps, double dt,
                   const impes_krylov_params& kp, double* rates_host, long long& iters,
                   cudaStream_t s) {
  adjoint_check_model(m);
  IMPES_REQUIRE(steps >= 1 && dt > 0, IMPES_ERR_ARG, "steps >= 1 and dt > 0 required");
  const int N = m.P.N;
  const std::vector<int> pc = producer_cells(m);
  const int np = (int)pc.size();
  DBuf<int> prod(std::max(np, 1));
  if (np) IMPES_CUDA(cudaMemcpyAsync(prod.p, pc.data(), sizeof(int) * np, cudaMemcpyHostToDevice, s));
  DBuf<double> sg(N), so(N), pold(N), rates((size_t)std::max(1, steps * np));
  IMPES_CUDA(cudaMemsetAsync(sg.p, 0, sizeof(double) * N, s));
  DBuf<double> bal(12);
  IMPES_CUDA(cudaMemcpyAsync(bal.p, m.balances.p, sizeof(double) * 12, cudaMemcpyDeviceToDevice, s));
  for (int n = 0; n < steps; ++n)
    forward_step(m, a, p, pold.p, sw, sg.p, so.p, dt, kp, prod.p, np, rates.p + (size_t)n * np,
                 iters, s);
  IMPES_CUDA(cudaMemcpyAsync(m.balances.p, bal.p, sizeof(double) * 12, cudaMemcpyDeviceToDevice, s));
  if (np && rates_host)
    IMPES_CUDA(cudaMemcpyAsync(rates_host, rates.p, sizeof(double) * steps * np,
                               cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
}

void adjoint_gradient(Model& m, AMG& a, const double* p0, const double* sw0, const double* kx,
                      const double* ky, const double* kz, int steps, int ckpt, double dt,
                      const impes_krylov_params& kf, const impes_krylov_params& ka,
                      const double* target_host, double* rates_host, double* g_lnk,
                      double* g_poro, impes_adjoint_stats& out, cudaStream_t s) {
  adjoint_check_model(m);
  IMPES_REQUIRE(steps >= 1 && dt > 0, IMPES_ERR_ARG, "steps >= 1 and dt > 0 required");
  const ModelParams& P = m.P;
  const int N = P.N;
  const int K = (ckpt <= 0 || ckpt > steps) ? steps : ckpt;
  const int nseg = (steps + K - 1) / K;
  const std::vector<int> pc = producer_cells(m);
  const int np = (int)pc.size();
  IMPES_REQUIRE(np >= 1, IMPES_ERR_ARG, "adjoint: the model has no producer");
  out = impes_adjoint_stats{};
  out.checkpoints = nseg;
  DBuf<int> prod(np);
  IMPES_CUDA(cudaMemcpyAsync(prod.p, pc.data(), sizeof(int) * np, cudaMemcpyHostToDevice, s));
  DBuf<double> rates((size_t)steps * np), tgt((size_t)steps * np), scratch_rates(np);
  IMPES_CUDA(cudaMemcpyAsync(tgt.p, target_host, sizeof(double) * steps * np, cudaMemcpyHostToDevice, s));
  DBuf<double> p(N), sw(N), sg(N), so(N), pold(N);
  IMPES_CUDA(cudaMemsetAsync(sg.p, 0, sizeof(double) * N, s));
  DBuf<double> ck_p((size_t)nseg * N), ck_s((size_t)nseg * N);
  DBuf<double> tp((size_t)(K + 1) * N), ts((size_t)K * N), tds((size_t)K * N);
  DBuf<int> tns(K);
  const size_t Fx = std::max<size_t>(1, (size_t)(P.nx - 1) * P.ny * P.nz);
  const size_t Fy = std::max<size_t>(1, (size_t)P.nx * (P.ny - 1) * P.nz);
  const size_t Fz = std::max<size_t>(1, (size_t)P.nx * P.ny * (P.nz - 1));
  DBuf<double> gp(N), gs(N), gp2(N), gs2(N), gam(N), mu(N), gpv(N), gtx(Fx), gty(Fy), gtz(Fz),
      dmu(np);
  DBuf<double> bal(12);
  IMPES_CUDA(cudaMemcpyAsync(bal.p, m.balances.p, sizeof(double) * 12, cudaMemcpyDeviceToDevice, s));
  const size_t bN = sizeof(double) * N;
  auto d2d = [&](double* dst, const double* src) {
    IMPES_CUDA(cudaMemcpyAsync(dst, src, bN, cudaMemcpyDeviceToDevice, s));
  };
  // states of segment `seg` are recorded into tp/ts/tds/tns while stepping
  auto record_step = [&](int t) {
    d2d(tp.p + (size_t)t * N, p.p);
    d2d(ts.p + (size_t)t * N, sw.p);
  };
  auto record_after = [&](int t) {
    d2d(tds.p + (size_t)t * N, m.dsw.p);
    IMPES_CUDA(cudaMemcpyAsync(tns.p + t, m.nsub.p, sizeof(int), cudaMemcpyDeviceToDevice, s));
  };

  // ---- forward run with checkpoints (the last segment is kept whole)
  Events ef;
  IMPES_CUDA(cudaEventRecord(ef.a, s));
  d2d(p.p, p0);
  d2d(sw.p, sw0);
  const int last0 = (nseg - 1) * K;
  for (int n = 0; n < steps; ++n) {
    if (n % K == 0) {
      d2d(ck_p.p + (size_t)(n / K) * N, p.p);
      d2d(ck_s.p + (size_t)(n / K) * N, sw.p);
    }
    if (n >= last0) record_step(n - last0);
    forward_step(m, a, p.p, pold.p, sw.p, sg.p, so.p, dt, kf, prod.p, np,
                 rates.p + (size_t)n * np, out.forward_iterations, s);
    if (n >= last0) record_after(n - last0);
  }
  d2d(tp.p + (size_t)(steps - last0) * N, p.p);
  IMPES_CUDA(cudaEventRecord(ef.b, s));
  std::vector<double> rh((size_t)steps * np), th((size_t)steps * np);
  IMPES_CUDA(cudaMemcpyAsync(rh.data(), rates.p, sizeof(double) * steps * np, cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  std::copy(target_host, target_host + (size_t)steps * np, th.begin());
  double J = 0.0;
  for (size_t q = 0; q < rh.size(); ++q) J += (rh[q] - th[q]) * (rh[q] - th[q]);
  out.J = J;
  out.forward_ms = ef.ms();
  if (rates_host) std::copy(rh.begin(), rh.end(), rates_host);

  // ---- reverse sweep
  Events er;
  IMPES_CUDA(cudaEventRecord(er.a, s));
  for (DBuf<double>* b : {&gp, &gs, &gpv})
    IMPES_CUDA(cudaMemsetAsync(b->p, 0, bN, s));
  IMPES_CUDA(cudaMemsetAsync(gtx.p, 0, sizeof(double) * Fx, s));
  IMPES_CUDA(cudaMemsetAsync(gty.p, 0, sizeof(double) * Fy, s));
  IMPES_CUDA(cudaMemsetAsync(gtz.p, 0, sizeof(double) * Fz, s));
  double *g_p = gp.p, *g_s = gs.p, *g_p2 = gp2.p, *g_s2 = gs2.p;
  const unsigned grid = grid_for(N, TBA);
  for (int seg = nseg - 1; seg >= 0; --seg) {
    const int n0 = seg * K, n1 = std::min(steps, n0 + K);
    if (seg != nseg - 1) {
      d2d(p.p, ck_p.p + (size_t)seg * N);
      d2d(sw.p, ck_s.p + (size_t)seg * N);
      for (int n = n0; n < n1; ++n) {
        record_step(n - n0);
        forward_step(m, a, p.p, pold.p, sw.p, sg.p, so.p, dt, kf, prod.p, np, scratch_rates.p,
                     out.forward_iterations, s);
        record_after(n - n0);
        ++out.recomputed_steps;
      }
      d2d(tp.p + (size_t)(n1 - n0) * N, p.p);
    }
    for (int n = n1 - 1; n >= n0; --n) {
      const int t = n - n0;
      const double* P0 = tp.p + (size_t)t * N;
      const double* P1 = tp.p + (size_t)(t + 1) * N;
      const double* S0 = ts.p + (size_t)t * N;
      const double* DS = tds.p + (size_t)t * N;
      // A^n into the hierarchy
      model_assemble(m, P0, S0, sg.p, dt, m.csr_val.p, m.rhs.p, s);
      amg_update(a, m.csr_val.p, s);
      k_adj_sat_cell<<<grid, TBA, 0, s>>>(P, S0, DS, tns.p + t, m.pv.p, g_s, dt, g_s2, gam.p, gpv.p); ::impes::count_launch();
      k_adj_sat_wells<<<1, 32, 0, s>>>(P, m.wells.p, S0, P1, m.pv.p, gam.p, dt, g_s2, g_p, gpv.p); ::impes::count_launch();
      k_adj_sat_faces<<<grid, TBA, 0, s>>>(P, m.tx.p, m.ty.p, m.tz.p, S0, P1, gam.p, g_s2, g_p,
                                           gtx.p, gty.p, gtz.p); ::impes::count_launch();
      k_adj_objective<<<1, 32, 0, s>>>(P, m.tx.p, m.ty.p, m.tz.p, m.pv.p, prod.p, np, P0, S0, P1, dt,
                                       tgt.p + (size_t)n * np, g_s2, g_p, dmu.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      impes_krylov_stats st{};
      impes_krylov_params k = ka;
      k.use_x0 = 0;
      amg_fgmres(a, g_p, mu.p, k, st, s);
      out.adjoint_iterations += st.iterations;
      if (!st.converged)
        throw Error(IMPES_ERR_NOT_CONVERGED, "adjoint: FGMRES did not converge on A mu = dJ/dp");
      k_adj_press_wells<<<1, 32, 0, s>>>(P, m.wells.p, S0, P1, prod.p, np, dmu.p, mu.p, g_s2); ::impes::count_launch();
      k_adj_press_cell<<<grid, TBA, 0, s>>>(P, m.tx.p, m.ty.p, m.tz.p, m.pv.p, P0, S0, P1, mu.p, dt,
                                            g_s2, g_p2, gpv.p, gtx.p, gty.p, gtz.p); ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      std::swap(g_p, g_p2);
      std::swap(g_s, g_s2);
    }
  }
  k_adj_params<<<grid, TBA, 0, s>>>(P, kx, ky, kz, gtx.p, gty.p, gtz.p, gpv.p, g_lnk, g_poro); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  IMPES_CUDA(cudaEventRecord(er.b, s));
  IMPES_CUDA(cudaMemcpyAsync(m.balances.p, bal.p, sizeof(double) * 12, cudaMemcpyDeviceToDevice, s));
  out.reverse_ms = er.ms();
  IMPES_CUDA(cudaStreamSynchronize(s));
}

}  // namespace impes
