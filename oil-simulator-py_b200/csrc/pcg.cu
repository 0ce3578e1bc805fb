// Jacobi-preconditioned conjugate gradients, the reference's default pressure
// solver: Simulator._solve_pressure_cg_pytorch (simulation.py:1662-1697) as
// called by _impes_pressure_step (:931-966).
//
// Same iteration as the reference: x0 = 0, z = r / diag(A), p = z; stop when
// sqrt(r . z) < tol (absolute) after the x/r update, or after max_iter steps.
// Scalars live on the device: the fused update kernel and the reductions hand
// alpha, beta and r.z to each other through a small device array, and the host
// reads r.z once per iteration for the stopping test.  Dot products use a
// fixed grid and a fixed reduction order, so runs are bitwise repeatable.
#include "common.cuh"
#include <cmath>

namespace impes {
namespace {

constexpr int TBP = 256;
constexpr int kBlocks = 296;   // 2 x 148 SMs: fixed partial count

// scal: [0] rs_old, [1] rs_new, [2] p.Ap, [3] alpha, [4] beta
__device__ __forceinline__ double block_reduce(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < TBP / 32; ++w) t += sh[w];
  __syncthreads();
  return t;
}

// r = b, z = r / d, p = z, x = 0; partial r.z
__global__ void __launch_bounds__(TBP) k_pcg_init(int n, const double* __restrict__ b,
                                                  const double* __restrict__ d, double* __restrict__ x,
                                                  double* __restrict__ r, double* __restrict__ z,
                                                  double* __restrict__ p, double* __restrict__ part) {
  __shared__ double sh[TBP / 32];
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)TBP + threadIdx.x; i < n; i += (long long)gridDim.x * TBP) {
    const double ri = b[i];
    const double zi = ri / d[i];
    x[i] = 0.0;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    acc += ri * zi;
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// Ap = A p (7-point rows: one thread per row); partial p.Ap
__global__ void __launch_bounds__(TBP) k_pcg_spmv(int n, const int* __restrict__ rowptr,
                                                  const int* __restrict__ col,
                                                  const double* __restrict__ val,
                                                  const double* __restrict__ p, double* __restrict__ Ap,
                                                  double* __restrict__ part) {
  __shared__ double sh[TBP / 32];
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)TBP + threadIdx.x; i < n; i += (long long)gridDim.x * TBP) {
    double s = 0.0;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) s += val[e] * p[col[e]];
    Ap[i] = s;
    acc += p[i] * s;
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// out = sum of kBlocks partials in a fixed order; mode 0: p.Ap -> alpha,
// mode 1: r.z -> rs_new and beta (rs_old then takes rs_new)
__global__ void k_pcg_scalar(const double* __restrict__ part, double* scal, int mode) {
  double t = 0.0;
  for (int q = threadIdx.x; q < kBlocks; q += 32) t += part[q];
  t = warp_sum(t);
  if (threadIdx.x == 0) {
    if (mode == 0) {
      scal[2] = t;
      scal[3] = scal[0] / t;
    } else if (mode == 1) {
      scal[1] = t;
      scal[4] = t / scal[0];
      scal[0] = t;
    } else {
      scal[0] = t;
      scal[1] = t;
    }
  }
}

// x += alpha p; r -= alpha Ap; z = r / d; partial r.z
__global__ void __launch_bounds__(TBP) k_pcg_update(int n, const double* __restrict__ scal,
                                                    const double* __restrict__ d,
                                                    const double* __restrict__ p,
                                                    const double* __restrict__ Ap, double* __restrict__ x,
                                                    double* __restrict__ r, double* __restrict__ z,
                                                    double* __restrict__ part) {
  __shared__ double sh[TBP / 32];
  const double alpha = scal[3];
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)TBP + threadIdx.x; i < n; i += (long long)gridDim.x * TBP) {
    x[i] += alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    const double zi = ri / d[i];
    r[i] = ri;
    z[i] = zi;
    acc += ri * zi;
  }
  const double t = block_reduce(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// p = z + beta p
__global__ void __launch_bounds__(TBP) k_pcg_direction(int n, const double* __restrict__ scal,
                                                       const double* __restrict__ z, double* __restrict__ p) {
  const double beta = scal[4];
  for (long long i = blockIdx.x * (long long)TBP + threadIdx.x; i < n; i += (long long)gridDim.x * TBP)
    p[i] = z[i] + beta * p[i];
}

__global__ void k_diag_of(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                          const double* __restrict__ val, double* __restrict__ d) {
  for (long long i = blockIdx.x * (long long)TBP + threadIdx.x; i < n; i += (long long)gridDim.x * TBP) {
    double v = 0.0;
    for (int e = rowptr[i]; e < rowptr[i + 1]; ++e)
      if (col[e] == i) v += val[e];
    d[i] = v;
  }
}

}  // namespace

// Solves A x = b (x written); returns the iterations taken and whether the
// stopping test fired.  rs_out: the last r.z.
void pcg_solve(int n, const int* rowptr, const int* col, const double* val, const double* b,
               double* x, double tol, int max_iter, int& iters, bool& converged, double& rs_out,
               cudaStream_t s) {
  IMPES_REQUIRE(n > 0 && max_iter >= 0, IMPES_ERR_ARG, "pcg: bad size or iteration limit");
  DBuf<double> d(n), r(n), z(n), p(n), Ap(n), part(kBlocks), scal(8);
  HostPinned<double> h(1);
  k_diag_of<<<grid_for(n, TBP), TBP, 0, s>>>(n, rowptr, col, val, d.p); ::impes::count_launch();
  k_pcg_init<<<kBlocks, TBP, 0, s>>>(n, b, d.p, x, r.p, z.p, p.p, part.p); ::impes::count_launch();
  k_pcg_scalar<<<1, 32, 0, s>>>(part.p, scal.p, 2); ::impes::count_launch();
  IMPES_CHECK_LAUNCH();
  IMPES_CUDA(cudaMemcpyAsync(h.p, scal.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  IMPES_CUDA(cudaStreamSynchronize(s));
  double rs = h.p[0];
  iters = 0;
  converged = false;
  rs_out = rs;
  if (!(rs == rs)) throw Error(IMPES_ERR_NAN, "pcg: non-finite right-hand side or diagonal");
  if (rs < 1e-10) {   // simulation.py:1680-1681
    converged = true;
    return;
  }
  for (int it = 0; it < max_iter; ++it) {
    k_pcg_spmv<<<kBlocks, TBP, 0, s>>>(n, rowptr, col, val, p.p, Ap.p, part.p); ::impes::count_launch();
    k_pcg_scalar<<<1, 32, 0, s>>>(part.p, scal.p, 0); ::impes::count_launch();
    k_pcg_update<<<kBlocks, TBP, 0, s>>>(n, scal.p, d.p, p.p, Ap.p, x, r.p, z.p, part.p); ::impes::count_launch();
    k_pcg_scalar<<<1, 32, 0, s>>>(part.p, scal.p, 1); ::impes::count_launch();
    IMPES_CHECK_LAUNCH();
    IMPES_CUDA(cudaMemcpyAsync(h.p, scal.p + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    IMPES_CUDA(cudaStreamSynchronize(s));
    rs = h.p[0];
    iters = it + 1;
    rs_out = rs;
    if (!(rs == rs)) throw Error(IMPES_ERR_NAN, "pcg: NaN residual");
    if (std::sqrt(rs) < tol) {
      converged = true;
      return;
    }
    k_pcg_direction<<<kBlocks, TBP, 0, s>>>(n, scal.p, z.p, p.p); ::impes::count_launch();
  }
}

}  // namespace impes
