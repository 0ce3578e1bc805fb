// Classical Ruge-Stueben AMG hierarchy on the device.
#pragma once
#include "common.cuh"
#include <memory>

namespace impes {

struct Level {
  int n = 0, nnz = 0;
  DBuf<int> rowptr, col;
  DBuf<unsigned short> col16;      // col as 16-bit indices, or empty (int columns only)
  int col16_rel = 0;               // 1: column = row - 32768 + col16 (levels of > 65536 rows)
  DBuf<double> val;
  DBuf<float> valf;
  DBuf<double> inv_relax;
  DBuf<float> inv_relaxf;
  // Chebyshev smoother: Gershgorin bound of diag(inv) A as double bits, [0] from
  // the fp64 values, [1] from the fp32 chain (atomicMax of non-negative doubles)
  DBuf<unsigned long long> cheb_lmax;
  // SELL-32 copy of A (sliced ELLPACK) for the sweeps and residuals, sell_lpr
  // lanes per row: rows in sell_perm order (sorted by length, longest first,
  // inside windows of 256 rows with one lane per row, 32 otherwise),
  // 32 / sell_lpr rows per slice; entry j of the slice's row q at
  // sell_ptr[s] + 32 (j / sell_lpr) + q sell_lpr + j % sell_lpr.  Padding
  // entries hold value 0 and the row's own column.  sell_map is the CSR index
  // of each entry (-1: padding); the values are gathered from the CSR values
  // after every value change.
  int sell_slices = 0, sell_lpr = 1;
  long long sell_len = 0;
  DBuf<int> sell_ptr, sell_perm, sell_map;
  DBuf<unsigned short> sell_col16;  // when col16 exists (same encoding), else sell_col
  DBuf<int> sell_col;
  DBuf<double> sell_val;
  DBuf<float> sell_valf;
  bool sell_on[2] = {false, false};  // autotuned: the sweeps/residuals of this precision use SELL
  // Diagonal (DIA) copy of A when the level has at most kDiaMax distinct
  // offsets col - row (a structured-grid stencil, like a TPFA level 0):
  // dia_off[d] ascending, dia_val[d n + i] = A(i, i + dia_off[d]), 0 where the
  // pattern has no entry; dia_map[k] = d n + i of CSR entry k.
  static constexpr int kDiaMax = 8;
  int dia_nd = 0;
  int dia_rpt = 1;                   // rows per thread of the 7-diagonal kernel (1 or 2, tuned)
  int dia_off[kDiaMax] = {0, 0, 0, 0, 0, 0, 0, 0};
  DBuf<int> dia_map;
  DBuf<double> dia_val;
  DBuf<float> dia_valf;
  bool dia_on[2] = {false, false};   // autotuned: the sweeps/residuals of this precision use DIA
  // > 0 when the 7 diagonals are the stencil of a grid_nx x grid_ny x grid_nz
  // grid (row = (ix grid_ny + iy) grid_nz + iz) and no entry joins the end of a
  // z line or of a y line to the next one: the sweeps may then run fused on
  // grid tiles (k_dia_tile)
  int grid_nx = 0, grid_ny = 0, grid_nz = 0;
  int avg_row = 7;                 // nnz / n, selects the SpMV row mapping
  // autotuned lanes per row ([0] fp64, [1] fp32; 0 = the mean-row-length rule)
  // of the kernels on A (sweeps, residuals), R (restriction) and P (prolongation)
  int lpr_a[2] = {0, 0}, lpr_r[2] = {0, 0}, lpr_p[2] = {0, 0};
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
  DBuf<float> apvalf;              // A*P values of the fp32 Galerkin chain
  int ap_maxrow = 0;               // longest A*P row
  int ac_maxrow = 0;               // longest row of the next level's A (computed here)
  // Galerkin numeric plans (P is frozen, so both products are fixed maps of
  // values): AP[o] = sum_t A[ap_e[t]] * P[ap_f[t]] over t in [ap_seg[o], ap_seg[o+1]),
  // Ac[o] = sum_t P[ac_r[t]] * AP[ac_f[t]] (ac_r indexes P, since R = P^T)
  bool planned = false;
  DBuf<int> ap_seg, ap_e, ap_f, ac_seg, ac_r, ac_f;
  long long ap_terms = 0, ac_terms = 0;
  // the fp32 P factor of every term (P[ap_f[t]], P[ac_r[t]]), copied once since
  // P is frozen: the fp32 chain then gathers only A (or AP) values
  DBuf<float> ap_cf, ac_cf;
  // A*P terms of the fp32 chain as 16-bit offsets into their output's A row:
  // ap_e[t] = ap_ebase[o] + ap_e16[t] (empty when a row is longer than 65536)
  DBuf<unsigned short> ap_e16;
  DBuf<int> ap_ebase;
  // cycle vectors (fp64 and fp32)
  DBuf<double> x, b, r, t, u;       // u: second direction buffer of the Chebyshev smoother
  DBuf<float> xf, bf, rf, tf, uf;
  // coarsest level (n <= 500): inverse of the dense matrix with DOF 0 pinned
  // (the reference's coarse solve), row-major, and lu_free, the inverse of the
  // unpinned matrix used inside FGMRES unless it was singular (device flag)
  DBuf<double> lu, lu_free;
  DBuf<int> piv;                   // two permutations of n
};

// Solver state of the device-driven FGMRES (amg_cycle.cu), read by the host
// after the captured solve has run.
struct FgState {
  int j, total, restarts, converged, done, cycle_end, reorth, bzero, nan;
  int reorths;                          // second Gram-Schmidt passes taken
  int gs_count;                         // blocks of a Gram-Schmidt launch done (last block reduces)
  double bnorm, beta, wn2, rel, true_rel;
};

struct AMG {
  impes_amg_params prm;
  std::vector<std::unique_ptr<Level>> levels;
  bool built = false;
  bool equilibrated = false;
  // mixed AMG: update_matrix runs the Galerkin chain in fp32 (all the V-cycle
  // of the mixed path reads); the fp64 coarse levels are rebuilt on demand
  bool fp64_stale = false;
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
  // CUDA graphs of a whole V-cycle from level 0, per [fp32][zero start][krylov][timed]
  struct VGraph {
    cudaGraphExec_t exec = nullptr;
    void* out = nullptr;
    long long kernels = 0;
    std::vector<PhaseTimers::Rec> timers;
  };
  VGraph vgraph[2][2][2][2];
  cudaStream_t cap_stream = nullptr;
  cudaStream_t body_stream = nullptr;   // captures the device FGMRES's loop body
  cudaStream_t if_stream = nullptr;     // captures the IF blocks inside that body
  DBuf<FgState> fgst;                   // device FGMRES state
  long long fg_body_kernels = 0;        // kernels of one device-FGMRES iteration
  long long fg_reorth_kernels = 0;      // ... of its second Gram-Schmidt pass (IF node)
  long long fg_end_kernels = 0;         // ... of its cycle-end block (IF node)
  // whole IMPES steps captured as graphs (abi.cu), keyed by the step's inputs
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    const void* model = nullptr;
    const double *p = nullptr, *sw = nullptr, *sg = nullptr, *so = nullptr;
    double dt = 0.0, dt_prev = 0.0, dt_prev2 = 0.0;
    bool have_prev = false, have_prev2 = false;
    impes_krylov_params kp{};
    bool fp64_stale_after = false;
    long long kernels_fixed = 0, kernels_body = 0, kernels_reorth = 0, kernels_end = 0;
  };
  std::vector<StepGraph> step_graphs;
  bool step_graph_failed = false;       // capture refused once: keep the host-driven path
  bool use_graphs = true;
  bool use_step_graph = true;           // whole IMPES steps as graphs (IMPES_NO_STEP_GRAPH=1: off)
  bool use_tail = false;                // fused V-cycle tail (IMPES_TAIL=1: on)
  bool use_dia_tile = false;            // level-0 grid-tile sweeps (IMPES_DIA_TILE=1: on)
  int tail_level = -1;                  // first level of the fused tail, -1: none
  int tail_cluster = 0;                 // CTAs in the tail's cluster (16 or 8)
  int stail_level = -1;                 // first level of the shared-memory fp32 tail, -1: none
  size_t stail_smem = 0;                // its shared-memory bytes
  void drop_graphs() {
    for (auto& a : vgraph) for (auto& b : a) for (auto& c : b) for (auto& g : c) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
      for (auto& r : g.timers) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
      g.timers.clear();
    }
    for (auto& g : step_graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    step_graphs.clear();
  }
  ~AMG() {
    drop_graphs();
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (body_stream) cudaStreamDestroy(body_stream);
    if (if_stream) cudaStreamDestroy(if_stream);
  }
};

// amg_setup.cu
void amg_setup(AMG& h, int n, int nnz, const int* rowptr, const int* col, const double* val,
               cudaStream_t s);
void amg_update(AMG& h, const double* val, cudaStream_t s);
// amg_cycle.cu
void amg_vcycle(AMG& h, int lvl, bool zero_x, int precision, cudaStream_t s);
void amg_solve_vcycles(AMG& h, const double* b, double* x, double tol, int max_cycles,
                       int* cycles, double* rel, cudaStream_t s, int norm = IMPES_NORM_EQUILIBRATED);
void amg_apply(AMG& h, const double* b, double* x, int cycles, double apply_tol,
               int apply_max_cycles, cudaStream_t s);
void amg_vcycle_scaled(AMG& h, const double* bs, double* xs, int precision, cudaStream_t s);
void amg_fgmres(AMG& h, const double* b, double* x, const impes_krylov_params& kp,
                impes_krylov_stats& st, cudaStream_t s);
// Device-driven FGMRES for a graph: amg_fgmres_prepare allocates its work space
// (call it before capture); amg_fgmres_capture enqueues the whole solve on a
// stream that is being captured (a conditional WHILE node runs the
// iterations); the outcome is in h.fgst after the graph has run.
void amg_fgmres_prepare(AMG& h, const impes_krylov_params& kp);
void amg_fgmres_capture(AMG& h, const double* b, double* x, const impes_krylov_params& kp, cudaStream_t s);

// shared kernels (amg_cycle.cu)
void spmv(const Level& L, const double* x, double* y, cudaStream_t s);
double dot_host(AMG& h, const double* a, const double* b, int n, cudaStream_t s);
void coarse_factor(AMG& h, Level& L, cudaStream_t s, bool from_fp32 = false);
// Times the CSR kernels of every level with each lanes-per-row choice and keeps
// the fastest (amg_cycle.cu); choices are cached per level shape for the process.
void amg_autotune(AMG& h, cudaStream_t s);
void amg_profile_levels(AMG& h, int precision, int reps, double* out, cudaStream_t s);
// The level's sweeps in this precision (slot 0 fp64, 1 fp32) run on grid tiles.
bool amg_level_tiled(const AMG& h, int l, int slot);
// First level of the fused V-cycle tail (amg_cycle.cu), -1 when none qualifies.
int amg_tail_level(AMG& h);
// Brings the fp64 coarse levels up to date after an fp32 update (no-op otherwise).
void amg_ensure_fp64(AMG& h, cudaStream_t s);
void level_precision_copies(AMG& h, Level& L, cudaStream_t s);

}  // namespace impes
