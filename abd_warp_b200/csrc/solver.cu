// Newton linear solve H dq = g on the block-sparse (12x12 per body pair) system.
//
// Replaces warp.optim.linear.bicgstab(hess, g, dq, 1e-4) and warp.sparse's BSR product
// (abd/abd.py:243-244).  Block-Jacobi preconditioned BiCGSTAB (the reference's solver
// choice) or PCG, FP64.  The SpMV is warp per block row: 24 lanes cover the 12 rows x 2
// half-rows of each 12x12 block, the row's blocks are the body's diagonal block and the
// off-diagonal blocks of its active body pairs in adjacency order.  Dot products are fused
// into the vector kernels as per-CTA partials on a fixed grid of kRedBlocks CTAs and summed
// in a fixed order, so the solve is bitwise reproducible.  Convergence is decided on the
// device (iteration-tagged flags); the host checks every kCheckEvery iterations.
#include <cuda_runtime.h>

#include "abd_common.cuh"

namespace abd {

namespace {

constexpr int WPB = 8;          // warps (body rows) per CTA
constexpr int kCheckEvery = 8;  // iterations launched between host checks

// slots of Sim::partials
enum { SL_R2 = 0, SL_RHR = 1, SL_RHV = 2, SL_S2 = 3, SL_TS = 4, SL_TT = 5, SL_B2 = 6, SL_X = 7 };
// Sim::scal layout
enum { SC_RHO0 = 0, SC_RHO1 = 1, SC_ALPHA = 2, SC_OMEGA = 3, SC_THR2 = 4 };
// dstat slots used by the solver
enum { DS_R_DONE = 10, DS_S_DONE = 11 };

struct SolverArgs {
  int n;
  const double *diag, *offdiag, *Minv;
  const int *row_ptr, *adj_col, *adj_pair, *pair_active, *fixed;
  const int2* ij;
  double* part;
  double* scal;
  int* dstat;
};

// all lanes of the calling warp return the fixed-order sum of the kRedBlocks partials
__device__ inline double sum_partials(const double* part) {
  const int lane = threadIdx.x & 31;
  double a = 0.0;
  for (int i = lane; i < kRedBlocks; i += 32) a += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  return a;
}

// CTA-wide broadcast of sum_partials for up to 3 slots
__device__ inline void cta_scalars(const double* part, const int* slots, int ns, double* out) {
  __shared__ double sv[3];
  if (threadIdx.x < 32)
    for (int k = 0; k < ns; ++k) {
      const double v = sum_partials(part + slots[k] * kRedBlocks);
      if (threadIdx.x == 0) sv[k] = v;
    }
  __syncthreads();
  for (int k = 0; k < ns; ++k) out[k] = sv[k];
  __syncthreads();
}

// per-CTA partial of two dot products: each warp passes its lane values (lanes 0..11)
__device__ inline void cta_partials(double d0, double d1, double* part, int slot0, int slot1) {
  __shared__ double w[WPB][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d0 += __shfl_xor_sync(0xffffffffu, d0, o);
    d1 += __shfl_xor_sync(0xffffffffu, d1, o);
  }
  if (lane == 0) {
    w[warp][0] = d0;
    w[warp][1] = d1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < WPB; ++k) {
      a += w[k][0];
      b += w[k][1];
    }
    if (slot0 >= 0) part[slot0 * kRedBlocks + blockIdx.x] = a;
    if (slot1 >= 0) part[slot1 * kRedBlocks + blockIdx.x] = b;
  }
}

// y_b (lanes 0..11 hold row lane) = (A x)_b for block row b
__device__ inline double row_product(const SolverArgs& a, int b, const double* x) {
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  if (lane < 24) {
    const int r = lane % 12, h = lane / 12;
    const double* B = a.diag + (size_t)b * 144 + r * 12 + 6 * h;
    const double* xb = x + (size_t)b * 12 + 6 * h;
#pragma unroll
    for (int c = 0; c < 6; ++c) acc += B[c] * xb[c];
    if (!a.fixed[b]) {
      for (int k = a.row_ptr[b]; k < a.row_ptr[b + 1]; ++k) {
        const int pr = a.adj_pair[k];
        if (a.pair_active[pr] <= 0) continue;
        const int J = a.adj_col[k];
        if (a.fixed[J]) continue;
        const int side = a.ij[pr].x == b ? 0 : 1;
        const double* O = a.offdiag + (size_t)pr * 288 + side * 144 + r * 12 + 6 * h;
        const double* xj = x + (size_t)J * 12 + 6 * h;
#pragma unroll
        for (int c = 0; c < 6; ++c) acc += O[c] * xj[c];
      }
    }
  }
  acc += __shfl_down_sync(0xffffffffu, acc, 12);
  return acc;  // valid on lanes 0..11
}

// lanes 0..11: (Minv_b v_b)[lane]
__device__ inline double block_apply(const double* M, int b, const double* v) {
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  if (lane < 24) {
    const int r = lane % 12, h = lane / 12;
    const double* B = M + (size_t)b * 144 + r * 12 + 6 * h;
    const double* vb = v + (size_t)b * 12 + 6 * h;
#pragma unroll
    for (int c = 0; c < 6; ++c) acc += B[c] * vb[c];
  }
  acc += __shfl_down_sync(0xffffffffu, acc, 12);
  return acc;
}

#define FOR_BODIES(b)                                                                      \
  for (int b = blockIdx.x * WPB + (int)(threadIdx.x >> 5); b < a.n; b += kRedBlocks * WPB)

__device__ inline bool solver_done(const int* dstat) {
  return ((volatile const int*)dstat)[DS_R_DONE] != 0 || ((volatile const int*)dstat)[DS_S_DONE] != 0;
}

// ---- shared setup: r = b - A x, rh = r, p = v = 0; partials r.r, rh.r ----
__global__ void __launch_bounds__(256) k_residual(SolverArgs a, const double* bvec, const double* x, double* r,
                                                  double* rh, double* pv, double* v) {
  const int lane = threadIdx.x & 31;
  double d0 = 0.0;
  FOR_BODIES(b) {
    const double ax = row_product(a, b, x);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      const double ri = bvec[i] - ax;
      r[i] = ri;
      if (rh) rh[i] = ri;
      if (pv) pv[i] = 0.0;
      if (v) v[i] = 0.0;
      d0 += ri * ri;
    }
  }
  cta_partials(d0, d0, a.part, SL_R2, SL_RHR);
}

__global__ void __launch_bounds__(256) k_norm2(SolverArgs a, const double* u, int slot) {
  const int lane = threadIdx.x & 31;
  double d0 = 0.0;
  FOR_BODIES(b) {
    if (lane < 12) {
      const double ui = u[(size_t)b * 12 + lane];
      d0 += ui * ui;
    }
  }
  cta_partials(d0, 0.0, a.part, slot, -1);
}

// ---- BiCGSTAB ----
// K1: rho = rh.r; p = r + beta (p - omega v); y = M p
__global__ void __launch_bounds__(256) k_bicg_1(SolverArgs a, int it, const double* r, double* pv, const double* v,
                                                double* y) {
  if (solver_done(a.dstat)) return;
  const int slots[2] = {SL_R2, SL_RHR};
  double sc[2];
  cta_scalars(a.part, slots, 2, sc);
  const double thr2 = a.scal[SC_THR2];
  if (sc[0] <= thr2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.dstat[DS_R_DONE] = it;
      a.dstat[DS_SOLVER_ITERS] = it - 1;
    }
    return;
  }
  const double rho = sc[1];
  const double rho_old = a.scal[(it + 1) & 1];
  const double alpha = a.scal[SC_ALPHA], omega = a.scal[SC_OMEGA];
  const double beta = (rho / rho_old) * (alpha / omega);
  const int lane = threadIdx.x & 31;
  FOR_BODIES(b) {
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      pv[i] = it == 1 ? r[i] : r[i] + beta * (pv[i] - omega * v[i]);
    }
    __syncwarp();
    const double yi = block_apply(a.Minv, b, pv);
    if (lane < 12) y[(size_t)b * 12 + lane] = yi;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.scal[it & 1] = rho;
}

// K2 / K5: out = A in; partials in2.out (slot0), out.out (slot1)
__global__ void __launch_bounds__(256) k_spmv(SolverArgs a, const double* in, double* out, const double* w0, int slot0,
                                              const double* w1, int slot1) {
  if (solver_done(a.dstat)) return;
  const int lane = threadIdx.x & 31;
  double d0 = 0.0, d1 = 0.0;
  FOR_BODIES(b) {
    const double yi = row_product(a, b, in);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      out[i] = yi;
      if (w0) d0 += w0[i] * yi;
      if (w1) d1 += w1[i] * yi;
    }
  }
  cta_partials(d0, d1, a.part, slot0, slot1);
}

// K3: alpha = rho / rh.v; s = r - alpha v; partial s.s
__global__ void __launch_bounds__(256) k_bicg_3(SolverArgs a, int it, const double* r, const double* v, double* s) {
  if (solver_done(a.dstat)) return;
  const int slots[1] = {SL_RHV};
  double sc[1];
  cta_scalars(a.part, slots, 1, sc);
  const double alpha = a.scal[it & 1] / sc[0];
  const int lane = threadIdx.x & 31;
  double d0 = 0.0;
  FOR_BODIES(b) {
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      const double si = r[i] - alpha * v[i];
      s[i] = si;
      d0 += si * si;
    }
  }
  cta_partials(d0, 0.0, a.part, SL_S2, -1);
  if (blockIdx.x == 0 && threadIdx.x == 0) a.scal[SC_ALPHA] = alpha;
}

// K4: if |s| small: x += alpha y and stop; else z = M s
__global__ void __launch_bounds__(256) k_bicg_4(SolverArgs a, int it, const double* y, const double* s, double* z,
                                                double* x) {
  const volatile int* ds = a.dstat;
  if (ds[DS_R_DONE] != 0 || (ds[DS_S_DONE] != 0 && ds[DS_S_DONE] != it)) return;
  const int slots[1] = {SL_S2};
  double sc[1];
  cta_scalars(a.part, slots, 1, sc);
  const double alpha = a.scal[SC_ALPHA];
  const int lane = threadIdx.x & 31;
  if (sc[0] <= a.scal[SC_THR2]) {
    FOR_BODIES(b) {
      if (lane < 12) {
        const size_t i = (size_t)b * 12 + lane;
        x[i] += alpha * y[i];
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.dstat[DS_S_DONE] = it;
      a.dstat[DS_SOLVER_ITERS] = it;
    }
    return;
  }
  FOR_BODIES(b) {
    const double zi = block_apply(a.Minv, b, s);
    if (lane < 12) z[(size_t)b * 12 + lane] = zi;
  }
}

// K6: omega = t.s / t.t; x += alpha y + omega z; r = s - omega t; partials r.r, rh.r
__global__ void __launch_bounds__(256) k_bicg_6(SolverArgs a, int it, const double* y, const double* z,
                                                const double* s, const double* t, const double* rh, double* x,
                                                double* r) {
  if (solver_done(a.dstat)) return;
  const int slots[2] = {SL_TS, SL_TT};
  double sc[2];
  cta_scalars(a.part, slots, 2, sc);
  const double omega = sc[0] / sc[1];
  const double alpha = a.scal[SC_ALPHA];
  const int lane = threadIdx.x & 31;
  double d0 = 0.0, d1 = 0.0;
  FOR_BODIES(b) {
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      x[i] += alpha * y[i] + omega * z[i];
      const double ri = s[i] - omega * t[i];
      r[i] = ri;
      d0 += ri * ri;
      d1 += rh[i] * ri;
    }
  }
  cta_partials(d0, d1, a.part, SL_R2, SL_RHR);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.scal[SC_OMEGA] = omega;
    a.dstat[DS_SOLVER_ITERS] = it;
  }
}

// ---- PCG ----
// init: z = M r, p = z; partials r.z (SL_RHR), r.r (SL_R2 kept from k_residual)
__global__ void __launch_bounds__(256) k_pcg_init(SolverArgs a, const double* r, double* z, double* pv) {
  const int lane = threadIdx.x & 31;
  double d0 = 0.0;
  FOR_BODIES(b) {
    const double zi = block_apply(a.Minv, b, r);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      z[i] = zi;
      pv[i] = zi;
      d0 += r[i] * zi;
    }
  }
  cta_partials(d0, 0.0, a.part, SL_RHR, -1);
}

// K1: convergence check on r.r, then Ap = A p with partial p.Ap
__global__ void __launch_bounds__(256) k_pcg_1(SolverArgs a, int it, const double* pv, double* Ap) {
  if (solver_done(a.dstat)) return;
  const int slots[1] = {SL_R2};
  double sc[1];
  cta_scalars(a.part, slots, 1, sc);
  if (sc[0] <= a.scal[SC_THR2]) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.dstat[DS_R_DONE] = it;
      a.dstat[DS_SOLVER_ITERS] = it - 1;
    }
    return;
  }
  const int lane = threadIdx.x & 31;
  double d0 = 0.0;
  FOR_BODIES(b) {
    const double yi = row_product(a, b, pv);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      Ap[i] = yi;
      d0 += pv[i] * yi;
    }
  }
  cta_partials(d0, 0.0, a.part, SL_RHV, -1);
}

// K2: alpha = rz / p.Ap; x += alpha p; r -= alpha Ap; z = M r; partials r.z (new), r.r
__global__ void __launch_bounds__(256) k_pcg_2(SolverArgs a, int it, const double* pv, const double* Ap, double* x,
                                               double* r, double* z) {
  if (solver_done(a.dstat)) return;
  const int rz_old = (it & 1) ? SL_RHR : SL_TS, rz_new = (it & 1) ? SL_TS : SL_RHR;
  const int slots[2] = {rz_old, SL_RHV};
  double sc[2];
  cta_scalars(a.part, slots, 2, sc);
  const double alpha = sc[0] / sc[1];
  const int lane = threadIdx.x & 31;
  double d0 = 0.0, d1 = 0.0;
  FOR_BODIES(b) {
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      x[i] += alpha * pv[i];
      r[i] -= alpha * Ap[i];
    }
    __syncwarp();
    const double zi = block_apply(a.Minv, b, r);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      z[i] = zi;
      d0 += r[i] * zi;
      d1 += r[i] * r[i];
    }
  }
  cta_partials(d0, d1, a.part, rz_new, SL_R2);
  if (blockIdx.x == 0 && threadIdx.x == 0) a.dstat[DS_SOLVER_ITERS] = it;
}

// K3: beta = rz_new / rz_old; p = z + beta p
__global__ void __launch_bounds__(256) k_pcg_3(SolverArgs a, int it, const double* z, double* pv) {
  if (solver_done(a.dstat)) return;
  const int rz_old = (it & 1) ? SL_RHR : SL_TS, rz_new = (it & 1) ? SL_TS : SL_RHR;
  const int slots[3] = {rz_new, rz_old, SL_R2};
  double sc[3];
  cta_scalars(a.part, slots, 3, sc);
  if (sc[2] <= a.scal[SC_THR2]) return;  // converged: K1 of the next iteration stops
  const double beta = sc[0] / sc[1];
  const int lane = threadIdx.x & 31;
  FOR_BODIES(b) {
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      pv[i] = z[i] + beta * pv[i];
    }
  }
}

// ---- block inverse by Gauss-Jordan with partial pivoting (one CTA of 144 threads per body) ----
__global__ void __launch_bounds__(144) k_block_inverse(int n, const double* diag, double* Minv) {
  const int b = blockIdx.x, t = threadIdx.x;
  __shared__ double m[12][24];
  __shared__ double f[12];
  __shared__ int piv;
  {
    const int r = t / 12, c = t % 12;
    m[r][c] = diag[(size_t)b * 144 + t];
    m[r][12 + c] = r == c ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int c = 0; c < 12; ++c) {
    if (t == 0) {
      int pr = c;
      for (int r = c + 1; r < 12; ++r)
        if (fabs(m[r][c]) > fabs(m[pr][c])) pr = r;
      piv = pr;
    }
    __syncthreads();
    if (piv != c && t < 24) {
      const double tmp = m[c][t];
      m[c][t] = m[piv][t];
      m[piv][t] = tmp;
    }
    __syncthreads();
    const double inv = 1.0 / m[c][c];
    __syncthreads();
    if (t < 24) m[c][t] *= inv;
    __syncthreads();
    if (t < 12) f[t] = m[t][c];
    __syncthreads();
    for (int e = t; e < 288; e += 144) {
      const int r = e / 24, k = e % 24;
      if (r != c && f[r] != 0.0) m[r][k] -= f[r] * m[c][k];
    }
    __syncthreads();
  }
  {
    const int r = t / 12, c = t % 12;
    Minv[(size_t)b * 144 + t] = m[r][12 + c];
  }
}

SolverArgs solver_args(Sim& s) {
  SolverArgs a;
  a.n = s.n;
  a.diag = s.diag;
  a.offdiag = s.offdiag;
  a.Minv = s.Minv;
  a.row_ptr = s.row_ptr;
  a.adj_col = s.adj_col;
  a.adj_pair = s.adj_pair;
  a.pair_active = s.pair_active;
  a.fixed = s.fixed;
  a.ij = s.ij;
  a.part = s.partials;
  a.scal = s.scal;
  a.dstat = s.dstat;
  return a;
}

}  // namespace

cudaError_t block_inverse(Sim& s) {
  k_block_inverse<<<s.n, 144, 0, s.stream>>>(s.n, s.diag, s.Minv);
  ++s.launches;
  return cudaGetLastError();
}

// Solves H x = g (x: warm start, overwritten).  Returns an ABD_* status.
int krylov_solve(Sim& s, double* x, int* iters_out) {
  SolverArgs a = solver_args(s);
  const double* bvec = s.g;
  cudaStream_t st = s.stream;
  const bool pcg = s.prm.solver == 1;
  // |b|^2 and the initial residual
  k_norm2<<<kRedBlocks, 256, 0, st>>>(a, bvec, SL_B2);
  k_residual<<<kRedBlocks, 256, 0, st>>>(a, bvec, x, s.r, pcg ? nullptr : s.rh, pcg ? nullptr : s.pv,
                                         pcg ? nullptr : s.v);
  s.launches += 2;
  if (finish_dot(s, SL_B2, s.scal + SC_THR2) != cudaSuccess) return ABD_ERR_CUDA;
  if (cudaMemcpyAsync(s.hval, s.scal + SC_THR2, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return ABD_ERR_CUDA;
  const double b2 = s.hval[0];
  if (b2 == 0.0) {
    cudaMemsetAsync(x, 0, sizeof(double) * 12 * s.n, st);
    if (iters_out) *iters_out = 0;
    return cudaGetLastError() == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
  }
  const double thr2 = (s.prm.cg_tol * s.prm.cg_tol) * b2;
  double hs[5] = {1.0, 1.0, 1.0, 1.0, thr2};  // rho (both parities), alpha, omega, thr^2
  cudaMemcpyAsync(s.scal, hs, sizeof(hs), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(s.dstat + DS_R_DONE, 0, 2 * sizeof(int), st);
  cudaMemsetAsync(s.dstat + DS_SOLVER_ITERS, 0, sizeof(int), st);
  if (pcg) {
    k_pcg_init<<<kRedBlocks, 256, 0, st>>>(a, s.r, s.z, s.pv);
    ++s.launches;
  }
  const int maxit = s.prm.cg_max_iter;
  int it = 1;
  int status = ABD_OK;
  for (;;) {
    for (int k = 0; k < kCheckEvery && it <= maxit; ++k, ++it) {
      if (pcg) {
        k_pcg_1<<<kRedBlocks, 256, 0, st>>>(a, it, s.pv, s.v);
        k_pcg_2<<<kRedBlocks, 256, 0, st>>>(a, it, s.pv, s.v, x, s.r, s.z);
        k_pcg_3<<<kRedBlocks, 256, 0, st>>>(a, it, s.z, s.pv);
        s.launches += 3;
      } else {
        k_bicg_1<<<kRedBlocks, 256, 0, st>>>(a, it, s.r, s.pv, s.v, s.y);
        k_spmv<<<kRedBlocks, 256, 0, st>>>(a, s.y, s.v, s.rh, SL_RHV, nullptr, -1);
        k_bicg_3<<<kRedBlocks, 256, 0, st>>>(a, it, s.r, s.v, s.s);
        k_bicg_4<<<kRedBlocks, 256, 0, st>>>(a, it, s.y, s.s, s.z, x);
        k_spmv<<<kRedBlocks, 256, 0, st>>>(a, s.z, s.t, s.s, SL_TS, s.t, SL_TT);
        k_bicg_6<<<kRedBlocks, 256, 0, st>>>(a, it, s.y, s.z, s.s, s.t, s.rh, x, s.r);
        s.launches += 6;
      }
    }
    if (cudaGetLastError() != cudaSuccess) return ABD_ERR_CUDA;
    cudaMemcpyAsync(s.hstat + 18, s.dstat + DS_R_DONE, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s.hstat + 20, s.dstat + DS_SOLVER_ITERS, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return ABD_ERR_CUDA;
    if (s.hstat[18] || s.hstat[19]) break;
    if (it > maxit) {
      s.host_status |= ST_SOLVER_NOCONV;  // not converged: reported through the status bits
      break;
    }
  }
  if (iters_out) *iters_out = s.hstat[20];
  return status;
}

}  // namespace abd
