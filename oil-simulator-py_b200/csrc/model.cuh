// IMPES model: static data of Reservoir + Fluid + WellManager on the device.
#pragma once
#include "common.cuh"

namespace impes {

constexpr int kMaxPvtRows = 128;
constexpr int kMaxWells = 256;

// Plain parameters copied by value into kernels.
struct ModelParams {
  int nx, ny, nz, N;
  double dx, dy, dz;
  double mu_o, mu_w, mu_g;
  double rho_o_ref, rho_w_ref, rho_g_ref;
  double c_o, c_w, c_g, c_r, cf;
  int relperm_model;
  double nw, no, ng, now, nog, ko_end_w, ko_end_g;
  double sw_cr, so_r, sg_cr;
  double pc_scale, pc_exponent, pc_og_scale, pc_og_exponent;
  double gravity, rate_scale, max_dS;
  int max_substeps;
  int pvt_rows;
  int nwells;       // wells
  int nwc;          // distinct well cells
};

// Device-side well record (same fields as impes_well_desc + derived).
struct WellDev {
  int cell;
  int is_injector, control_bhp;
  double value, well_index;
  int injected_phase, surface_rate, surface_phase, limit_mask;
  double limits[4];
  int has_bhp_min;
  double bhp_min;
};

struct Model {
  ModelParams P;
  int nnz = 0;
  std::vector<WellDev> wells_host;
  std::vector<int> wc_cells_host;      // sorted distinct well cells
  DBuf<double> tx, ty, tz, pv;         // transmissibilities, pore volume
  DBuf<double> pvt;                    // rows x 9, row-major
  DBuf<WellDev> wells;
  DBuf<int> wc_cells, wc_ptr, wc_wells;// well-cell -> wells (original order)
  // per-step scratch
  DBuf<double> dsw, dsg;               // saturation increments
  DBuf<double> wq;                     // 3 x nwc well sources (q_w, q_g, q_o)
  DBuf<double> wsub;                   // per (substep, well) component-balance addends
  DBuf<double> red;                    // block partials for reductions
  DBuf<unsigned> counter;              // last-block counters
  DBuf<int> nsub;                      // substep count (device)
  DBuf<double> balances;               // 12: mass[6], component[6]
  DBuf<int> well_mode;                 // per well last_mode (-1 unset)
  DBuf<double> well_q;                 // per well last_q_total (NaN unset)
  DBuf<double> well_rates;             // per well 4 surface rates (NaN unset)
  DBuf<double> csr_val, rhs;           // assembled system (owned for impes_step)
  DBuf<double> p_save;                 // pressure before the solve (restored on failure)
  DBuf<double> p_prev;                 // pressure before the last accepted step
  double dt_prev = 0.0;                // and that step's dt (extrapolated first iterate)
  bool have_prev = false;
  DBuf<double> p_prev2;                // the one before (quadratic extrapolation)
  double dt_prev2 = 0.0;
  bool have_prev2 = false;
  DBuf<int> rowptr, col;               // static pattern
  int red_blocks = 0;
};

// Kernels implemented in physics.cu (compiled with -fmad=false).
void model_build_static(Model& m, const double* kx, const double* ky, const double* kz,
                        const double* poro, cudaStream_t s);
void model_pattern(Model& m, int* rowptr, int* col, cudaStream_t s);
void model_assemble(Model& m, const double* p, const double* sw, const double* sg, double dt,
                    double* csr_val, double* rhs, cudaStream_t s);
// pred (device int, may be null): the kernels do nothing unless *pred != 0
void model_saturation(Model& m, const double* p_new, double* sw, double* sg, double* so,
                      double dt, cudaStream_t s, const int* pred = nullptr);

// Closed-form CSR row pointer of the 7-point pattern (no scan needed).
__host__ __device__ inline long long pattern_rowptr(long long c, int nx, int ny, int nz) {
  long long plane = (long long)ny * nz;
  long long i = c / plane, rem = c % plane, j = rem / nz, k = rem % nz;
  long long cnt = c;                                           // diagonals
  long long xm = c - plane; cnt += xm > 0 ? xm : 0;            // rows with i >= 1
  long long xp_lim = (long long)(nx - 1) * plane; cnt += c < xp_lim ? c : xp_lim;  // i <= nx-2
  long long jk = j * nz + k;
  long long ym = jk - nz; cnt += i * (long long)(ny - 1) * nz + (ym > 0 ? ym : 0);
  long long yp_lim = (long long)(ny - 1) * nz; cnt += i * (long long)(ny - 1) * nz + (jk < yp_lim ? jk : yp_lim);
  long long col_ = i * ny + j;                                 // columns before
  cnt += col_ * (nz - 1) + (k - 1 > 0 ? k - 1 : 0);            // k >= 1
  cnt += col_ * (nz - 1) + (k < nz - 1 ? k : nz - 1);          // k <= nz-2
  return cnt;
}

}  // namespace impes
