// extern "C" entry points declared in include/impes_b200.h.
#include "amg.cuh"
#include "model.cuh"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <map>

namespace impes {
const char* last_error_cstr();
}

struct impes_amg {
  impes::AMG a;
};
struct impes_model {
  impes::Model m;
};

using namespace impes;

bool impes_amg_handle_built(impes_amg* h) { return h && h->a.built; }
impes::AMG* impes_amg_handle_core(impes_amg* h) { return &h->a; }

namespace impes {
void pcg_solve(int n, const int* rowptr, const int* col, const double* val, const double* b,
               double* x, double tol, int max_iter, int& iters, bool& converged, double& rs_out,
               cudaStream_t s);
void adjoint_check_model(const Model& m);
int adjoint_num_producers(const Model& m);
void adjoint_rates(Model& m, AMG& a, double* p, double* sw, int steps, double dt,
                   const impes_krylov_params& kp, double* rates_host, long long& iters,
                   cudaStream_t s);
void adjoint_gradient(Model& m, AMG& a, const double* p0, const double* sw0, const double* kx,
                      const double* ky, const double* kz, int steps, int ckpt, double dt,
                      const impes_krylov_params& kf, const impes_krylov_params& ka,
                      const double* target_host, double* rates_host, double* g_lnk,
                      double* g_poro, impes_adjoint_stats& out, cudaStream_t s);
}  // namespace impes

namespace {

// x0 = p + r (p - p_prev): the pressure extrapolated linearly in time
__global__ void k_extrapolate(int n, const double* __restrict__ p, const double* __restrict__ p_prev,
                              double r, double* __restrict__ x0) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x0[i] = p[i] + r * (p[i] - p_prev[i]);
}

// x0 = w0 p + w1 p_prev + w2 p_prev2: the Lagrange parabola through the last
// three accepted pressures, evaluated at the end of the step
__global__ void k_extrapolate2(int n, const double* __restrict__ p, const double* __restrict__ p_prev,
                               const double* __restrict__ p_prev2, double w0, double w1, double w2,
                               double* __restrict__ x0) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x0[i] = w0 * p[i] + w1 * p_prev[i] + w2 * p_prev2[i];
}

// After a captured step: the new pressure is accepted (p_prev takes the
// step's starting pressure for the next extrapolated iterate, and p_prev2,
// when given, the old p_prev) or, when the solve missed its tolerance, p is
// restored from p_save.
__global__ void k_accept(int n, const FgState* st, double* __restrict__ p, const double* __restrict__ p_save,
                         double* __restrict__ p_prev, double* __restrict__ p_prev2) {
  const bool ok = st->converged && !st->nan;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (ok) {
      if (p_prev2) p_prev2[i] = p_prev[i];
      p_prev[i] = p_save[i];
    } else {
      p[i] = p_save[i];
    }
  }
}

// Extrapolation weights of the first iterate: Lagrange weights at t = dt of
// the pressures at 0, -dt_prev and -(dt_prev + dt_prev2).
void quad_weights(double dt, double dt_prev, double dt_prev2, double& w0, double& w1, double& w2) {
  const double t1 = -dt_prev, t2 = -(dt_prev + dt_prev2), t = dt;
  w0 = (t - t1) * (t - t2) / (t1 * t2);
  w1 = t * (t - t2) / (t1 * (t1 - t2));
  w2 = t * (t - t1) / (t2 * (t2 - t1));
}

// The whole IMPES step of the FGMRES solver as one CUDA graph: assembly, the
// Galerkin update, the pressure-save copy, the extrapolated first iterate, the
// device-driven FGMRES (a conditional WHILE node over its iterations), the
// accept/restore kernel and the saturation update, which runs only when the
// solve converged.  One graph per (model, state pointers, dt, solver settings,
// first-iterate mode); the hierarchy must exist (the first step builds it on
// the host path).  Returns false when this build or driver refuses the capture
// (the caller then keeps the host-driven step).
// A refused step-graph capture keeps the host-driven step; IMPES_GRAPH_DEBUG=1
// prints why on stderr.
static void step_graph_refused(const char* stage, const char* why) {
  const char* ev = getenv("IMPES_GRAPH_DEBUG");
  if (ev && ev[0] == '1') fprintf(stderr, "impes: whole-step graph refused (%s): %s\n", stage, why);
}

bool step_graph_run(Model& m, AMG& a, double* p, double* sw, double* sg, double* so, double dt,
                    const impes_krylov_params& kp, impes_krylov_stats& st, cudaStream_t s) {
  if (a.step_graph_failed || !a.use_graphs || !a.use_step_graph || timers().on || kp.precision < 0) return false;
  const bool extrap = kp.use_x0 >= 2 && m.have_prev && m.dt_prev > 0;
  const bool quad = extrap && kp.use_x0 == 3 && m.have_prev2 && m.dt_prev2 > 0;
  AMG::StepGraph* g = nullptr;
  for (auto& e : a.step_graphs)
    if (e.model == &m && e.p == p && e.sw == sw && e.sg == sg && e.so == so && e.dt == dt &&
        e.have_prev == extrap && (!extrap || e.dt_prev == m.dt_prev) && e.have_prev2 == quad &&
        (!quad || e.dt_prev2 == m.dt_prev2) && e.kp.tol == kp.tol &&
        e.kp.restart == kp.restart && e.kp.max_iters == kp.max_iters && e.kp.norm == kp.norm &&
        e.kp.precision == kp.precision && e.kp.use_x0 == kp.use_x0) {
      g = &e;
      break;
    }
  if (!g) {
    if (a.step_graphs.size() >= 8) {           // dt changes (retries): keep a few
      if (a.step_graphs.front().exec) cudaGraphExecDestroy(a.step_graphs.front().exec);
      a.step_graphs.erase(a.step_graphs.begin());
    }
    impes_krylov_params k = kp;
    k.use_x0 = kp.use_x0 ? 1 : 0;
    amg_fgmres_prepare(a, k);
    m.p_prev.ensure(m.P.N);
    if (kp.use_x0 == 3) m.p_prev2.ensure(m.P.N);
    if (!a.cap_stream) IMPES_CUDA(cudaStreamCreateWithFlags(&a.cap_stream, cudaStreamNonBlocking));
    cudaStream_t cs = a.cap_stream;
    // the capture stream starts after the work already queued on s
    cudaEvent_t ev;
    IMPES_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    IMPES_CUDA(cudaEventRecord(ev, s));
    IMPES_CUDA(cudaStreamWaitEvent(cs, ev, 0));
    IMPES_CUDA(cudaEventDestroy(ev));
    const unsigned long long before = thread_launches();
    const bool stale_before = a.fp64_stale;
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) {
      step_graph_refused("begin capture", cudaGetErrorString(ce));
      a.step_graph_failed = true;
      cudaGetLastError();
      return false;
    }
    const char* stage = "assembly";
    try {
      model_assemble(m, p, sw, sg, dt, m.csr_val.p, m.rhs.p, cs);
      stage = "AMG update";
      amg_update(a, m.csr_val.p, cs);
      stage = "FGMRES";
      IMPES_CUDA(cudaMemcpyAsync(m.p_save.p, p, sizeof(double) * m.P.N, cudaMemcpyDeviceToDevice, cs));
      if (quad) {
        double w0, w1, w2;
        quad_weights(dt, m.dt_prev, m.dt_prev2, w0, w1, w2);
        k_extrapolate2<<<grid_for(m.P.N, 256), 256, 0, cs>>>(m.P.N, m.p_save.p, m.p_prev.p, m.p_prev2.p, w0, w1,
                                                             w2, p);
        ::impes::count_launch();
        IMPES_CHECK_LAUNCH();
      } else if (extrap) {
        k_extrapolate<<<grid_for(m.P.N, 256), 256, 0, cs>>>(m.P.N, m.p_save.p, m.p_prev.p, dt / m.dt_prev, p);
        ::impes::count_launch();
        IMPES_CHECK_LAUNCH();
      }
      amg_fgmres_capture(a, m.rhs.p, p, k, cs);
      stage = "saturation";
      k_accept<<<grid_for(m.P.N, 256), 256, 0, cs>>>(m.P.N, a.fgst.p, p, m.p_save.p, m.p_prev.p,
                                                     kp.use_x0 == 3 ? m.p_prev2.p : nullptr);
      ::impes::count_launch();
      IMPES_CHECK_LAUNCH();
      model_saturation(m, p, sw, sg, so, dt, cs, &a.fgst.p->converged);
    } catch (const Error& err) {
      step_graph_refused(stage, err.what());
      cudaStreamEndCapture(cs, &graph);
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      count_launches(-(long long)(thread_launches() - before));
      a.fp64_stale = stale_before;
      a.step_graph_failed = true;
      return false;
    }
    IMPES_CUDA(cudaStreamEndCapture(cs, &graph));
    AMG::StepGraph e;
    e.model = &m; e.p = p; e.sw = sw; e.sg = sg; e.so = so; e.dt = dt;
    e.have_prev = extrap; e.dt_prev = extrap ? m.dt_prev : 0.0; e.kp = kp;
    e.have_prev2 = quad; e.dt_prev2 = quad ? m.dt_prev2 : 0.0;
    e.fp64_stale_after = a.fp64_stale;
    e.kernels_body = a.fg_body_kernels;
    e.kernels_reorth = a.fg_reorth_kernels;
    e.kernels_end = a.fg_end_kernels;
    e.kernels_fixed = (long long)(thread_launches() - before) - e.kernels_body - e.kernels_reorth - e.kernels_end;
    count_launches(-(long long)(thread_launches() - before));
    a.fp64_stale = stale_before;
    cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      step_graph_refused("instantiate", cudaGetErrorString(ie));
      cudaGetLastError();
      a.step_graph_failed = true;
      return false;
    }
    a.step_graphs.push_back(e);
    g = &a.step_graphs.back();
  }
  IMPES_CUDA(cudaGraphLaunch(g->exec, s));
  a.fp64_stale = g->fp64_stale_after;
  FgState* hs = reinterpret_cast<FgState*>(a.hbuf.p);
  static_assert(sizeof(FgState) <= 64 * sizeof(double), "state must fit the pinned scratch");
  IMPES_CUDA(cudaMemcpyAsync(hs, a.fgst.p, sizeof(FgState), cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  count_launches(g->kernels_fixed + (long long)hs->total * g->kernels_body + (long long)hs->reorths * g->kernels_reorth +
                 (long long)hs->restarts * g->kernels_end);
  st = impes_krylov_stats{hs->total, hs->restarts, hs->converged && !hs->nan ? 1 : 0, hs->rel, hs->true_rel};
  if (hs->nan) throw Error(IMPES_ERR_NAN, "NaN in FGMRES");
  if (!st.converged) return true;            // p was restored by the graph
  if (kp.use_x0 == 3) {
    m.dt_prev2 = m.dt_prev;
    m.have_prev2 = m.have_prev;
  }
  m.dt_prev = dt;
  m.have_prev = true;
  return true;
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return IMPES_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return IMPES_ERR_ARG;
  } catch (...) {
    set_last_error("unknown error");
    return IMPES_ERR_ARG;
  }
}

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

const char* impes_last_error(void) { return last_error_cstr(); }
int impes_abi_version(void) { return 1; }

// ------------------------------------------------------------------ AMG
int impes_amg_create(impes_amg** out, const impes_amg_params* p) {
  return guarded([&] {
    IMPES_REQUIRE(out && p, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(p->max_levels >= 1 && p->coarsest_size >= 1, IMPES_ERR_ARG, "bad level limits");
    IMPES_REQUIRE(p->nullspace_dim >= 0 && p->nullspace_dim <= 3, IMPES_ERR_ARG,
                  "nullspace_dim must be 0..3");
    IMPES_REQUIRE(p->p_max_elements >= 0 && p->p_trunc_factor >= 0.0 && p->p_trunc_factor < 1.0,
                  IMPES_ERR_ARG, "p_max_elements must be >= 0 and p_trunc_factor in [0, 1)");
    IMPES_REQUIRE(p->smoother == IMPES_SMOOTHER_L1_JACOBI || p->smoother == IMPES_SMOOTHER_CHEBYSHEV,
                  IMPES_ERR_ARG, "unknown smoother");
    IMPES_REQUIRE(p->cheb_lower < 1.0, IMPES_ERR_ARG, "cheb_lower must be below 1");
    IMPES_REQUIRE(p->light_sweep_rows >= 0, IMPES_ERR_ARG, "light_sweep_rows must be >= 0");
    auto* h = new impes_amg();
    h->a.prm = *p;
    if (!(h->a.prm.cheb_lower > 0.0)) h->a.prm.cheb_lower = 0.3;
    h->a.prm.nullspace_blend = std::max(0.0, std::min(1.0, p->nullspace_blend));
    h->a.prm.nullspace_reg = std::max(1e-10, p->nullspace_reg);
    *out = h;
  });
}

int impes_amg_destroy(impes_amg* h) {
  return guarded([&] { delete h; });
}

int impes_amg_setup(impes_amg* h, int n, int nnz, const int* rowptr, const int* col,
                    const double* val, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && rowptr && col && val, IMPES_ERR_ARG, "null argument");
    amg_setup(h->a, n, nnz, rowptr, col, val, S(stream));
  });
}

int impes_amg_update(impes_amg* h, const double* val, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && val, IMPES_ERR_ARG, "null argument");
    amg_update(h->a, val, S(stream));
  });
}

int impes_amg_solve_vcycles(impes_amg* h, const double* b, double* x, double tol, int max_cycles,
                            int* cycles, double* rel_res, int norm, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && b && x, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(h->a.built, IMPES_ERR_STATE, "solve before setup");
    IMPES_REQUIRE(max_cycles >= 1, IMPES_ERR_ARG, "max_cycles must be >= 1");
    amg_solve_vcycles(h->a, b, x, tol, max_cycles, cycles, rel_res, S(stream), norm);
  });
}

int impes_amg_apply(impes_amg* h, const double* b, double* x, int cycles, double apply_tol,
                    int apply_max_cycles, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && b && x, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(h->a.built, IMPES_ERR_STATE, "apply before setup");
    amg_apply(h->a, b, x, cycles, apply_tol, apply_max_cycles, S(stream));
  });
}

int impes_amg_vcycle_scaled(impes_amg* h, const double* b_scaled, double* x_scaled, int precision,
                            void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && b_scaled && x_scaled, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(h->a.built, IMPES_ERR_STATE, "V-cycle before setup");
    amg_vcycle_scaled(h->a, b_scaled, x_scaled, precision, S(stream));
  });
}

int impes_amg_fgmres(impes_amg* h, const double* b, double* x, const impes_krylov_params* kp,
                     impes_krylov_stats* stats, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && b && x && kp, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(h->a.built, IMPES_ERR_STATE, "solve before setup");
    IMPES_REQUIRE(kp->restart >= 1 && kp->max_iters >= 0, IMPES_ERR_ARG, "bad Krylov limits");
    impes_krylov_stats st{};
    amg_fgmres(h->a, b, x, *kp, st, S(stream));
    if (stats) *stats = st;
  });
}

int impes_amg_num_levels(impes_amg* h, int* nlev) {
  return guarded([&] {
    IMPES_REQUIRE(h && nlev, IMPES_ERR_ARG, "null argument");
    *nlev = (int)h->a.levels.size();
  });
}

int impes_amg_level_info(impes_amg* h, int lvl, impes_amg_level_desc* info) {
  return guarded([&] {
    IMPES_REQUIRE(h && info, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(lvl >= 0 && lvl < (int)h->a.levels.size(), IMPES_ERR_ARG, "level out of range");
    const Level& L = *h->a.levels[lvl];
    info->n = L.n;
    info->nnz = L.nnz;
    info->p_cols = L.coarsest ? 0 : L.nc;
    info->p_nnz = L.coarsest ? 0 : L.pnnz;
    info->is_coarsest = L.coarsest ? 1 : 0;
    info->col_index_bytes = L.col16.p ? 2 : 4;
    info->col_row_relative = L.col16.p ? L.col16_rel : 0;
    for (int q = 0; q < 2; ++q) {
      info->lanes[3 * q + 0] = L.lpr_a[q];
      info->lanes[3 * q + 1] = L.lpr_r[q];
      info->lanes[3 * q + 2] = L.lpr_p[q];
      info->layout[q] = amg_level_tiled(h->a, lvl, q) ? 3 : L.dia_on[q] ? 2 : (L.sell_on[q] ? 1 : 0);
    }
    const AMG& A = h->a;
    info->fused_tail = (A.stail_level >= 1 && lvl >= A.stail_level) ? 1
                       : (A.tail_level >= 1 && lvl >= A.tail_level) ? 2 : 0;
  });
}

int impes_amg_profile_levels(impes_amg* h, int precision, int reps, double* out_host, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && out_host && reps >= 1, IMPES_ERR_ARG, "null argument or reps < 1");
    IMPES_REQUIRE(h->a.built, IMPES_ERR_STATE, "profile before setup");
    amg_profile_levels(h->a, precision, reps, out_host, S(stream));
  });
}

int impes_amg_step_graphs(impes_amg* h, int* graphs, int* capture_refused) {
  return guarded([&] {
    IMPES_REQUIRE(h && graphs && capture_refused, IMPES_ERR_ARG, "null argument");
    *graphs = (int)h->a.step_graphs.size();
    *capture_refused = h->a.step_graph_failed ? 1 : 0;
  });
}

int impes_amg_level_export(impes_amg* h, int lvl, int* A_rowptr, int* A_col, double* A_val,
                           double* inv_relax, int* P_rowptr, int* P_col, double* P_val,
                           void* stream) {
  return guarded([&] {
    if (h) amg_ensure_fp64(h->a, S(stream));
    IMPES_REQUIRE(h, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(lvl >= 0 && lvl < (int)h->a.levels.size(), IMPES_ERR_ARG, "level out of range");
    const Level& L = *h->a.levels[lvl];
    cudaStream_t s = S(stream);
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (dst && bytes) IMPES_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    };
    cp(A_rowptr, L.rowptr.p, sizeof(int) * (L.n + 1));
    cp(A_col, L.col.p, sizeof(int) * L.nnz);
    cp(A_val, L.val.p, sizeof(double) * L.nnz);
    cp(inv_relax, L.inv_relax.p, sizeof(double) * L.n);
    if (!L.coarsest) {
      cp(P_rowptr, L.prow.p, sizeof(int) * (L.n + 1));
      cp(P_col, L.pcol.p, sizeof(int) * L.pnnz);
      cp(P_val, L.pval.p, sizeof(double) * L.pnnz);
    }
  });
}

int impes_amg_equilibration(impes_amg* h, double* dhalf_inv, int* enabled, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && enabled, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(h->a.built, IMPES_ERR_STATE, "query before setup");
    IMPES_CUDA(cudaMemcpyAsync(h->a.hint.p, h->a.iflag.p + 1, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
    IMPES_CUDA(cudaStreamSynchronize(S(stream)));
    h->a.equilibrated = h->a.hint.p[0] != 0;
    *enabled = h->a.equilibrated ? 1 : 0;
    if (dhalf_inv && h->a.equilibrated)
      IMPES_CUDA(cudaMemcpyAsync(dhalf_inv, h->a.dhalf_inv.p, sizeof(double) * h->a.levels[0]->n,
                                 cudaMemcpyDeviceToDevice, S(stream)));
  });
}

// ---------------------------------------------------------------- model
int impes_model_create(impes_model** out, const impes_model_desc* d, const impes_well_desc* wells,
                       int nwells, const double* pvt, const double* kx, const double* ky,
                       const double* kz, const double* poro, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(out && d && kx && ky && kz && poro, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(d->nx >= 1 && d->ny >= 1 && d->nz >= 1, IMPES_ERR_ARG, "grid dims must be >= 1");
    long long N = (long long)d->nx * d->ny * d->nz;
    IMPES_REQUIRE(N * 7 < (1LL << 31), IMPES_ERR_ARG, "grid too large for int32 CSR");
    IMPES_REQUIRE(nwells >= 0 && nwells <= kMaxWells, IMPES_ERR_ARG, "too many wells");
    IMPES_REQUIRE(nwells == 0 || wells, IMPES_ERR_ARG, "null wells");
    IMPES_REQUIRE(d->pvt_rows == 0 || (pvt && d->pvt_rows >= 2 && d->pvt_rows <= kMaxPvtRows),
                  IMPES_ERR_ARG, "PVT table must have 2..128 rows");
    IMPES_REQUIRE(d->max_substeps >= 1, IMPES_ERR_ARG, "max_substeps must be >= 1");
    cudaStream_t s = S(stream);
    auto* h = new impes_model();
    Model& m = h->m;
    try {
      ModelParams& P = m.P;
      P.nx = d->nx; P.ny = d->ny; P.nz = d->nz; P.N = (int)N;
      P.dx = d->dx; P.dy = d->dy; P.dz = d->dz;
      P.mu_o = d->mu_o; P.mu_w = d->mu_w; P.mu_g = d->mu_g;
      P.rho_o_ref = d->rho_o_ref; P.rho_w_ref = d->rho_w_ref; P.rho_g_ref = d->rho_g_ref;
      P.c_o = d->c_o; P.c_w = d->c_w; P.c_g = d->c_g; P.c_r = d->c_r; P.cf = d->cf;
      P.relperm_model = d->relperm_model;
      P.nw = d->nw; P.no = d->no; P.ng = d->ng; P.now = d->now; P.nog = d->nog;
      P.ko_end_w = d->ko_end_w; P.ko_end_g = d->ko_end_g;
      P.sw_cr = d->sw_cr; P.so_r = d->so_r; P.sg_cr = d->sg_cr;
      P.pc_scale = d->pc_scale; P.pc_exponent = d->pc_exponent;
      P.pc_og_scale = d->pc_og_scale; P.pc_og_exponent = d->pc_og_exponent;
      P.gravity = d->gravity; P.rate_scale = d->global_rate_scale; P.max_dS = d->max_saturation_change;
      P.max_substeps = d->max_substeps; P.pvt_rows = d->pvt_rows;
      P.nwells = nwells;
      // wells: flat cell (simulation.py:1629), -1 when outside the grid
      std::map<int, std::vector<int>> by_cell;
      m.wells_host.resize(nwells);
      for (int w = 0; w < nwells; ++w) {
        const impes_well_desc& W = wells[w];
        WellDev& D = m.wells_host[w];
        bool inside = W.i >= 0 && W.j >= 0 && W.k >= 0 && W.i < d->nx && W.j < d->ny && W.k < d->nz;
        IMPES_REQUIRE(inside, IMPES_ERR_ARG, "well outside the grid");
        D.cell = (W.i * d->ny + W.j) * d->nz + W.k;
        D.is_injector = W.is_injector; D.control_bhp = W.control_bhp;
        D.value = W.value; D.well_index = W.well_index;
        D.injected_phase = W.injected_phase; D.surface_rate = W.surface_rate;
        D.surface_phase = W.surface_phase; D.limit_mask = W.limit_mask;
        for (int q = 0; q < 4; ++q) D.limits[q] = W.limits[q];
        D.has_bhp_min = W.has_bhp_min; D.bhp_min = W.bhp_min;
        by_cell[D.cell].push_back(w);
      }
      std::vector<int> wc_ptr(1, 0), wc_wells;
      for (auto& kv : by_cell) {
        m.wc_cells_host.push_back(kv.first);
        for (int w : kv.second) wc_wells.push_back(w);
        wc_ptr.push_back((int)wc_wells.size());
      }
      P.nwc = (int)m.wc_cells_host.size();
      m.wells.alloc(std::max(nwells, 1));
      m.wc_cells.alloc(std::max(P.nwc, 1));
      m.wc_ptr.alloc(P.nwc + 1);
      m.wc_wells.alloc(std::max(nwells, 1));
      if (nwells) {
        IMPES_CUDA(cudaMemcpyAsync(m.wells.p, m.wells_host.data(), sizeof(WellDev) * nwells, cudaMemcpyHostToDevice, s));
        IMPES_CUDA(cudaMemcpyAsync(m.wc_cells.p, m.wc_cells_host.data(), sizeof(int) * P.nwc, cudaMemcpyHostToDevice, s));
        IMPES_CUDA(cudaMemcpyAsync(m.wc_wells.p, wc_wells.data(), sizeof(int) * nwells, cudaMemcpyHostToDevice, s));
      }
      IMPES_CUDA(cudaMemcpyAsync(m.wc_ptr.p, wc_ptr.data(), sizeof(int) * (P.nwc + 1), cudaMemcpyHostToDevice, s));
      m.pvt.alloc(std::max(1, d->pvt_rows * 9));
      if (d->pvt_rows)
        IMPES_CUDA(cudaMemcpyAsync(m.pvt.p, pvt, sizeof(double) * d->pvt_rows * 9, cudaMemcpyHostToDevice, s));
      m.balances.alloc(12);
      IMPES_CUDA(cudaMemsetAsync(m.balances.p, 0, sizeof(double) * 12, s));
      m.well_mode.alloc(std::max(nwells, 1));
      m.well_q.alloc(std::max(nwells, 1));
      m.well_rates.alloc(std::max(4 * nwells, 1));
      std::vector<int> modes(std::max(nwells, 1), -1);
      std::vector<double> nan(std::max(4 * nwells, 1), std::nan(""));
      IMPES_CUDA(cudaMemcpyAsync(m.well_mode.p, modes.data(), sizeof(int) * modes.size(), cudaMemcpyHostToDevice, s));
      IMPES_CUDA(cudaMemcpyAsync(m.well_q.p, nan.data(), sizeof(double) * std::max(nwells, 1), cudaMemcpyHostToDevice, s));
      IMPES_CUDA(cudaMemcpyAsync(m.well_rates.p, nan.data(), sizeof(double) * nan.size(), cudaMemcpyHostToDevice, s));
      model_build_static(m, kx, ky, kz, poro, s);
      m.csr_val.alloc(m.nnz);
      m.rhs.alloc(P.N);
      m.p_save.alloc(P.N);
      IMPES_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int impes_model_destroy(impes_model* m) {
  return guarded([&] { delete m; });
}

int impes_model_nnz(impes_model* h, int* n, int* nnz) {
  return guarded([&] {
    IMPES_REQUIRE(h && n && nnz, IMPES_ERR_ARG, "null argument");
    *n = h->m.P.N;
    *nnz = h->m.nnz;
  });
}

int impes_csr_pattern(impes_model* h, int* rowptr, int* col, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && rowptr && col, IMPES_ERR_ARG, "null argument");
    model_pattern(h->m, rowptr, col, S(stream));
  });
}

int impes_well_cells(impes_model* h, int* cells_host) {
  return guarded([&] {
    IMPES_REQUIRE(h && (cells_host || h->m.P.nwells == 0), IMPES_ERR_ARG, "null argument");
    for (int w = 0; w < h->m.P.nwells; ++w) cells_host[w] = h->m.wells_host[w].cell;
  });
}

int impes_model_set_well_values(impes_model* h, const double* values, int nwells, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && (values || nwells == 0), IMPES_ERR_ARG, "null argument");
    Model& m = h->m;
    IMPES_REQUIRE(nwells == m.P.nwells, IMPES_ERR_ARG, "well count differs from the model's");
    if (nwells == 0) return;
    for (int w = 0; w < nwells; ++w) {
      IMPES_REQUIRE(std::isfinite(values[w]), IMPES_ERR_NAN, "non-finite well control value");
      m.wells_host[w].value = values[w];
    }
    cudaStream_t s = S(stream);
    IMPES_CUDA(cudaMemcpyAsync(m.wells.p, m.wells_host.data(), sizeof(WellDev) * nwells,
                               cudaMemcpyHostToDevice, s));
    IMPES_CUDA(cudaStreamSynchronize(s));   // wells_host is pageable and may change again
  });
}

int impes_model_export_static(impes_model* h, double* tx, double* ty, double* tz, double* pv,
                              void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h, IMPES_ERR_ARG, "null argument");
    const Model& m = h->m;
    cudaStream_t s = S(stream);
    const ModelParams& P = m.P;
    auto cp = [&](void* dst, const void* src, size_t bytes) {
      if (dst && bytes) IMPES_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    };
    cp(tx, m.tx.p, sizeof(double) * (size_t)(P.nx - 1) * P.ny * P.nz);
    cp(ty, m.ty.p, sizeof(double) * (size_t)P.nx * (P.ny - 1) * P.nz);
    cp(tz, m.tz.p, sizeof(double) * (size_t)P.nx * P.ny * (P.nz - 1));
    cp(pv, m.pv.p, sizeof(double) * P.N);
  });
}

int impes_assemble(impes_model* h, const double* p, const double* sw, const double* sg, double dt,
                   double* csr_val, double* rhs, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && p && sw && sg && csr_val && rhs, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(dt > 0, IMPES_ERR_ARG, "dt must be positive");
    model_assemble(h->m, p, sw, sg, dt, csr_val, rhs, S(stream));
  });
}

int impes_saturation(impes_model* h, const double* p_new, double* sw, double* sg, double* so,
                     double dt, impes_sat_stats* stats, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && p_new && sw && sg && so, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(dt > 0, IMPES_ERR_ARG, "dt must be positive");
    model_saturation(h->m, p_new, sw, sg, so, dt, S(stream));
    if (stats) {
      impes_sat_stats st{};
      double hb[12];
      cudaStream_t s = S(stream);
      IMPES_CUDA(cudaMemcpyAsync(hb, h->m.balances.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
      IMPES_CUDA(cudaMemcpyAsync(&st.substeps, h->m.nsub.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      IMPES_CUDA(cudaStreamSynchronize(s));
      for (int q = 0; q < 6; ++q) { st.mass_balance[q] = hb[q]; st.component[q] = hb[6 + q]; }
      *stats = st;
    }
  });
}

int impes_step(impes_model* h, impes_amg* amg, double* p, double* sw, double* sg, double* so,
               double dt, int solver, const impes_krylov_params* kp, int max_cycles,
               impes_krylov_stats* kstats, impes_sat_stats* sstats, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && p && sw && sg && so && kp, IMPES_ERR_ARG, "null argument");
    IMPES_REQUIRE(dt > 0, IMPES_ERR_ARG, "dt must be positive");
    IMPES_REQUIRE(solver >= 0 && solver <= 2, IMPES_ERR_ARG, "solver must be 0, 1 or 2");
    Model& m = h->m;
    cudaStream_t s = S(stream);
    IMPES_REQUIRE(solver == 2 || amg, IMPES_ERR_ARG, "null AMG handle");
    if (solver == 1 && amg->a.built && amg->a.levels[0]->n == m.P.N) {
      impes_krylov_stats gst{};
      if (step_graph_run(m, amg->a, p, sw, sg, so, dt, *kp, gst, s)) {
        if (kstats) *kstats = gst;
        if (!gst.converged) throw Error(IMPES_ERR_NOT_CONVERGED, "FGMRES did not reach the pressure tolerance");
        if (sstats) {
          double hb[12];
          impes_sat_stats ss{};
          IMPES_CUDA(cudaMemcpyAsync(hb, m.balances.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
          IMPES_CUDA(cudaMemcpyAsync(&ss.substeps, m.nsub.p, sizeof(int), cudaMemcpyDeviceToHost, s));
          IMPES_CUDA(cudaStreamSynchronize(s));
          for (int q = 0; q < 6; ++q) { ss.mass_balance[q] = hb[q]; ss.component[q] = hb[6 + q]; }
          *sstats = ss;
        }
        return;
      }
    }
    model_assemble(m, p, sw, sg, dt, m.csr_val.p, m.rhs.p, s);
    if (solver != 2) {
      AMG& a = amg->a;
      if (!a.built || a.levels[0]->n != m.P.N)
        amg_setup(a, m.P.N, m.nnz, m.rowptr.p, m.col.p, m.csr_val.p, s);
      else
        amg_update(a, m.csr_val.p, s);
    }
    impes_krylov_stats st{};
    // a failed pressure solve leaves the state as it was (the caller may retry
    // with a smaller dt, as _impes_step does at simulation.py:833-862)
    IMPES_CUDA(cudaMemcpyAsync(m.p_save.p, p, sizeof(double) * m.P.N, cudaMemcpyDeviceToDevice, s));
    auto restore = [&] {
      cudaMemcpyAsync(p, m.p_save.p, sizeof(double) * m.P.N, cudaMemcpyDeviceToDevice, s);
      cudaStreamSynchronize(s);
    };
    try {
      if (solver == 2) {
        // _impes_pressure_step's CG and its one relaxed retry (simulation.py:931-966)
        int it = 0;
        bool conv = false;
        double rz = 0.0;
        pcg_solve(m.P.N, m.rowptr.p, m.col.p, m.csr_val.p, m.rhs.p, p, kp->tol, kp->max_iters, it,
                  conv, rz, s);
        st.iterations = it;
        if (!conv) {
          pcg_solve(m.P.N, m.rowptr.p, m.col.p, m.csr_val.p, m.rhs.p, p, kp->tol * 10.0,
                    kp->max_iters * 4, it, conv, rz, s);
          st.iterations += it;
          st.restarts = 1;
        }
        st.rel_res = std::sqrt(std::max(rz, 0.0));
        st.true_rel_res = st.rel_res;
        st.converged = conv;
      } else if (solver == 0) {
        AMG& a = amg->a;
        int cyc = 0;
        double rel = 0.0;
        amg_solve_vcycles(a, m.rhs.p, p, kp->tol, std::max(1, max_cycles), &cyc, &rel, s, kp->norm);
        st.iterations = cyc;
        st.rel_res = rel;
        st.true_rel_res = rel;
        st.converged = rel < kp->tol;
      } else {
        impes_krylov_params k = *kp;
        if (k.use_x0 >= 2) {
          // first iterate extrapolated from the last two (or three) accepted
          // pressures (p_save holds p^n; the assembly has already used it)
          if (k.use_x0 == 3 && m.have_prev && m.dt_prev > 0 && m.have_prev2 && m.dt_prev2 > 0) {
            double w0, w1, w2;
            quad_weights(dt, m.dt_prev, m.dt_prev2, w0, w1, w2);
            k_extrapolate2<<<grid_for(m.P.N, 256), 256, 0, s>>>(m.P.N, m.p_save.p, m.p_prev.p, m.p_prev2.p, w0,
                                                                w1, w2, p); ::impes::count_launch();
            IMPES_CHECK_LAUNCH();
          } else if (m.have_prev && m.dt_prev > 0) {
            k_extrapolate<<<grid_for(m.P.N, 256), 256, 0, s>>>(m.P.N, m.p_save.p, m.p_prev.p,
                                                               dt / m.dt_prev, p); ::impes::count_launch();
            IMPES_CHECK_LAUNCH();
          }
          k.use_x0 = 1;
        }
        amg_fgmres(amg->a, m.rhs.p, p, k, st, s);
      }
    } catch (...) {
      restore();
      throw;
    }
    if (kstats) *kstats = st;
    if (solver != 0 && !st.converged) {
      restore();
      throw Error(IMPES_ERR_NOT_CONVERGED, solver == 2 ? "CG did not reach the pressure tolerance"
                                                       : "FGMRES did not reach the pressure tolerance");
    }
    // the accepted step's starting pressure, for the next extrapolated iterate
    // (and, for the quadratic one, the one before it)
    m.p_prev.ensure(m.P.N);
    if (kp->use_x0 == 3 && solver == 1) {
      m.p_prev2.ensure(m.P.N);
      if (m.have_prev)
        IMPES_CUDA(cudaMemcpyAsync(m.p_prev2.p, m.p_prev.p, sizeof(double) * m.P.N, cudaMemcpyDeviceToDevice, s));
      m.dt_prev2 = m.dt_prev;
      m.have_prev2 = m.have_prev;
    }
    IMPES_CUDA(cudaMemcpyAsync(m.p_prev.p, m.p_save.p, sizeof(double) * m.P.N, cudaMemcpyDeviceToDevice, s));
    m.dt_prev = dt;
    m.have_prev = true;
    model_saturation(m, p, sw, sg, so, dt, s);
    if (sstats) {
      double hb[12];
      impes_sat_stats ss{};
      IMPES_CUDA(cudaMemcpyAsync(hb, m.balances.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
      IMPES_CUDA(cudaMemcpyAsync(&ss.substeps, m.nsub.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      IMPES_CUDA(cudaStreamSynchronize(s));
      for (int q = 0; q < 6; ++q) { ss.mass_balance[q] = hb[q]; ss.component[q] = hb[6 + q]; }
      *sstats = ss;
    }
  });
}

int impes_model_balances(impes_model* h, impes_sat_stats* stats, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && stats, IMPES_ERR_ARG, "null argument");
    double hb[12];
    impes_sat_stats st{};
    cudaStream_t s = S(stream);
    IMPES_CUDA(cudaMemcpyAsync(hb, h->m.balances.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaMemcpyAsync(&st.substeps, h->m.nsub.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    for (int q = 0; q < 6; ++q) { st.mass_balance[q] = hb[q]; st.component[q] = hb[6 + q]; }
    *stats = st;
  });
}

int impes_model_reset_balances(impes_model* h, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h, IMPES_ERR_ARG, "null argument");
    IMPES_CUDA(cudaMemsetAsync(h->m.balances.p, 0, sizeof(double) * 12, S(stream)));
  });
}

int impes_well_states(impes_model* h, impes_well_state* out, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && (out || h->m.P.nwells == 0), IMPES_ERR_ARG, "null argument");
    const int nw = h->m.P.nwells;
    if (!nw) return;
    std::vector<int> modes(nw);
    std::vector<double> q(nw), rates(4 * nw);
    cudaStream_t s = S(stream);
    IMPES_CUDA(cudaMemcpyAsync(modes.data(), h->m.well_mode.p, sizeof(int) * nw, cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaMemcpyAsync(q.data(), h->m.well_q.p, sizeof(double) * nw, cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaMemcpyAsync(rates.data(), h->m.well_rates.p, sizeof(double) * 4 * nw, cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    for (int w = 0; w < nw; ++w) {
      out[w].last_mode = modes[w];
      out[w].has_q_total = !std::isnan(q[w]);
      out[w].last_q_total = q[w];
      out[w].has_surface_rates = !std::isnan(rates[4 * w]);
      for (int k = 0; k < 4; ++k) out[w].surface_rates[k] = rates[4 * w + k];
    }
  });
}

int impes_timing_enable(int on) {
  return guarded([&] { timers().on = on != 0; });
}

int impes_timing_collect(impes_timing* out) {
  return guarded([&] {
    IMPES_REQUIRE(out, IMPES_ERR_ARG, "null argument");
    impes_timing t{};
    PhaseTimers& T = timers();
    IMPES_CUDA(cudaDeviceSynchronize());
    T.harvest();
    for (int q = 0; q < IMPES_NUM_PHASES; ++q) {
      t.count[q] += T.acc_n[q];
      t.ms[q] += T.acc_ms[q];
      t.bytes[q] += T.acc_bytes[q];
      T.acc_n[q] = 0; T.acc_ms[q] = 0.0; T.acc_bytes[q] = 0.0;
    }
    for (auto& r : T.recs) {
      IMPES_CUDA(cudaEventSynchronize(r.b));
      float ms = 0.f;
      IMPES_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
      if (r.phase >= 0 && r.phase < IMPES_NUM_PHASES) {
        t.count[r.phase] += 1;
        t.ms[r.phase] += ms;
        t.bytes[r.phase] += r.bytes;
      }
      T.pool.push_back(r.a);
      T.pool.push_back(r.b);
    }
    T.recs.clear();
    *out = t;
  });
}

unsigned long long impes_kernel_launches(void) { return launches(); }

}  // extern "C"

int impes_adjoint_num_producers(impes_model* h, int* n) {
  return guarded([&] {
    IMPES_REQUIRE(h && n, IMPES_ERR_ARG, "null argument");
    *n = adjoint_num_producers(h->m);
  });
}

int impes_adjoint_rates(impes_model* h, impes_amg* amg, double* p, double* sw, int steps, double dt,
                        const impes_krylov_params* kp, double* rates_host, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && amg && p && sw && kp, IMPES_ERR_ARG, "null argument");
    long long iters = 0;
    adjoint_rates(h->m, amg->a, p, sw, steps, dt, *kp, rates_host, iters, S(stream));
  });
}

int impes_adjoint_gradient(impes_model* h, impes_amg* amg, const double* p0, const double* sw0,
                           const double* kx, const double* ky, const double* kz, int steps,
                           int checkpoint_every, double dt, const impes_krylov_params* forward,
                           const impes_krylov_params* adjoint, const double* target_host,
                           double* rates_host, double* g_lnk, double* g_poro,
                           impes_adjoint_stats* stats, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(h && amg && p0 && sw0 && kx && ky && kz && forward && adjoint && target_host &&
                      g_lnk && g_poro,
                  IMPES_ERR_ARG, "null argument");
    impes_adjoint_stats st{};
    adjoint_gradient(h->m, amg->a, p0, sw0, kx, ky, kz, steps, checkpoint_every, dt, *forward,
                     *adjoint, target_host, rates_host, g_lnk, g_poro, st, S(stream));
    if (stats) *stats = st;
  });
}

int impes_pcg_solve(int n, const int* rowptr, const int* col, const double* val, const double* b,
                    double* x, double tol, int max_iter, int* iterations, int* converged,
                    double* rz, void* stream) {
  return guarded([&] {
    IMPES_REQUIRE(rowptr && col && val && b && x, IMPES_ERR_ARG, "null argument");
    int it = 0;
    bool conv = false;
    double r = 0.0;
    pcg_solve(n, rowptr, col, val, b, x, tol, max_iter, it, conv, r, S(stream));
    if (iterations) *iterations = it;
    if (converged) *converged = conv ? 1 : 0;
    if (rz) *rz = r;
  });
}
