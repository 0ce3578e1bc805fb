// Classical Ruge-Stueben AMG hierarchy on the device.
#pragma once
#include "common.cuh"
#include <memory>

namespace impes {

struct Level {
  int n = 0, nnz = 0;
  DBuf<int> rowptr, col;
  DBuf<double> val;
  DBuf<float> valf;
  DBuf<double> inv_relax;
  DBuf<float> inv_relaxf;
  int avg_row = 7;                 // nnz / n, selects the SpMV row mapping
  bool coarsest = false;
  // interpolation P (n x nc) and restriction R = P^T (nc x n)
  int nc = 0, pnnz = 0;
  DBuf<int> prow, pcol;
  DBuf<double> pval;
  DBuf<float> pvalf;
  DBuf<int> rrow, rcol, rsrc;      // rsrc: P entry feeding each R entry
  DBuf<double> rval;
  DBuf<float> rvalf;
  int p_avg = 1, r_avg = 1;
  // Galerkin helper: pattern of A*P (n x nc)
  DBuf<int> aprow, apcol;
  DBuf<double> apval;
  int ap_maxrow = 0;               // longest A*P row
  int ac_maxrow = 0;               // longest row of the next level's A (computed here)
  // cycle vectors (fp64 and fp32)
  DBuf<double> x, b, r, t;
  DBuf<float> xf, bf, rf, tf;
  // coarsest level (n <= 500): inverse of the dense matrix with DOF 0 pinned
  // (the reference's coarse solve), row-major; when the coarsest level is also
  // level 0, lu_free holds the unpinned inverse used as FGMRES preconditioner
  DBuf<double> lu, lu_free;
  DBuf<int> piv;
};

struct AMG {
  impes_amg_params prm;
  std::vector<std::unique_ptr<Level>> levels;
  bool built = false;
  bool equilibrated = false;
  DBuf<double> dhalf_inv;          // D^-1/2 when equilibrated
  DBuf<double> jac_w;              // Jacobi weights in the scaled space
  DBuf<double> diag_tmp;
  DBuf<double> red;                // reduction partials
  DBuf<double> scal;               // device scalars
  DBuf<int> iflag;                 // device int flags / counters
  HostPinned<double> hbuf{64};
  HostPinned<int> hint{16};
  // FGMRES workspace
  int krylov_m = 0;
  DBuf<double> V, Z, H, cs, sn, g, y, kw, kb, kx;
  bool krylov_mode = false;        // V-cycles issued by FGMRES
};

// amg_setup.cu
void amg_setup(AMG& h, int n, int nnz, const int* rowptr, const int* col, const double* val,
               cudaStream_t s);
void amg_update(AMG& h, const double* val, cudaStream_t s);
// amg_cycle.cu
void amg_vcycle(AMG& h, int lvl, bool zero_x, int precision, cudaStream_t s);
void amg_solve_vcycles(AMG& h, const double* b, double* x, double tol, int max_cycles,
                       int* cycles, double* rel, cudaStream_t s);
void amg_apply(AMG& h, const double* b, double* x, int cycles, double apply_tol,
               int apply_max_cycles, cudaStream_t s);
void amg_vcycle_scaled(AMG& h, const double* bs, double* xs, int precision, cudaStream_t s);
void amg_fgmres(AMG& h, const double* b, double* x, const impes_krylov_params& kp,
                impes_krylov_stats& st, cudaStream_t s);

// shared kernels (amg_cycle.cu)
void spmv(const Level& L, const double* x, double* y, cudaStream_t s);
double dot_host(AMG& h, const double* a, const double* b, int n, cudaStream_t s);
void coarse_factor(AMG& h, Level& L, cudaStream_t s);
void level_precision_copies(AMG& h, Level& L, cudaStream_t s);

}  // namespace impes
