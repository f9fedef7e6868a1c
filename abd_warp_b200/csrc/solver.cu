// Newton linear solve H dq = g on the block-sparse (12x12 per body pair) system.
//
// Replaces warp.optim.linear.bicgstab(hess, g, dq, 1e-4) and warp.sparse's BSR product
// (abd/abd.py:243-244).
//
// Preconditioner: contact-cluster block Jacobi.  Barrier stiffness between touching bodies is
// 1e8-1e10 times their mass, so a per-body block Jacobi leaves the Krylov method facing that
// condition number.  Bodies coupled by active contacts are grouped on the device (mutual
// strongest couplings merge in rounds, at most cluster_max bodies: k_clusters); each
// cluster's dense system is assembled and inverted (Gauss-Jordan, SPD, no pivoting) by one
// warp in registers (one body) or one CTA in shared memory (more), and applied as a dense
// product.  Clusters of one body reduce to the per-body 12x12 block.
//
// Krylov: PCG (default; the projected Hessian is SPD) or right-preconditioned BiCGSTAB (the
// reference's choice).  Convergence is measured in the preconditioned norm,
// r^T M^-1 r <= tol^2 b^T M^-1 b, which stays resolvable in FP64 although the plain residual
// of such stiff systems has a rounding floor near eps * cond.  The SpMV is warp per block row
// (24 lanes = 12 rows x 2 half-rows).  Dot products are exact (per-CTA partials summed in
// fixed point), so the solve is bitwise reproducible.  The iterations run as the body of a
// CUDA graph WHILE node: the kernel that completes an iteration's last dot product also ends
// the iteration -- it advances the device iteration counter, makes the convergence test that
// the next iteration would make, and sets the loop's condition -- so a solve runs exactly its
// iterations with no host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <utility>
#include <vector>

#include "abd_common.cuh"
#include "abd_graph.cuh"

namespace abd {

namespace {

constexpr int WPB = 8;          // warps (body rows) per CTA of the row kernels
constexpr int AT = 128;         // threads of the cluster apply kernel
constexpr int IT = 512;         // threads of the cluster inverse kernel (one CTA per cluster)

// slots of Sim::partials
enum { SL_RZ0 = 0, SL_RZ1 = 1, SL_PAP = 2, SL_BZ = 3, SL_RHR = 4, SL_RHV = 5, SL_SZ = 6, SL_TS = 7, SL_TT = 8 };
// Sim::scal layout
enum { SC_RHO0 = 0, SC_RHO1 = 1, SC_ALPHA = 2, SC_OMEGA = 3, SC_THR2 = 4 };
// dstat slots used by the solver
enum { DS_R_DONE = 10, DS_S_DONE = 11 };

struct SolverArgs {
  int n;
  const double *diag, *offdiag;
  const int *row_ptr, *adj_col, *adj_pair, *pair_active, *fixed;
  const int2* ij;
  const int* ncl_dev; // clusters (formed on the device)
  int maxit;
  const int *cl_ptr, *cl_body;
  const long long* cl_off;
  double* cl_inv;
  XSum* part;        // [kRedSlots][kRedBlocks] exact per-CTA partials
  int* red_count;    // [kRedSlots] CTAs that delivered their partial
  double* scal;
  int* dstat;
  Mailbox* tally;    // device loop: the solve's outcome goes to the step's counters (else null)
  cudaGraphConditionalHandle loop;  // the iteration loop's WHILE node
};

constexpr int SC_RED = 16;  // scal[SC_RED + slot]: the rounded total of reduction `slot`

// scalars produced by the previous kernel's reductions
__device__ inline void cta_scalars(const SolverArgs& a, const int* slots, int ns, double* out) {
  for (int k = 0; k < ns; ++k) out[k] = a.scal[SC_RED + slots[k]];
}

// The CTA's exact partial of a dot product into part[slot] (every thread passes its accumulator)
__device__ inline void cta_partial(const SolverArgs& a, XSum& x, int slot, XSum* sh) {
  xs_block_sum(x, sh);
  if (threadIdx.x == 0) a.part[slot * kRedBlocks + blockIdx.x] = x;
}

// After a CTA's partials: true in the last CTA to deliver (the launch's single counter cslot,
// reset here for the next launch), which then sees every CTA's partials
__device__ inline bool cta_last(const SolverArgs& a, int cslot) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&a.red_count[cslot], 1) == (int)gridDim.x - 1;
    if (last) a.red_count[cslot] = 0;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// In the last CTA: the sum of every CTA's partial of `slot`, rounded into scal[SC_RED + slot]
__device__ inline void total_of(const SolverArgs& a, int slot, XSum* sh) {
  XSum t;
  xs_zero(t);
  const XSum* P = a.part + slot * kRedBlocks;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
    const long long* q = reinterpret_cast<const long long*>(P + i);
#pragma unroll
    for (int j = 0; j < kXD; ++j) t.d[j] += __ldcg(q + j);
    t.flags |= __ldcg(q + kXD);
  }
  xs_block_sum(t, sh);
  if (threadIdx.x == 0) a.scal[SC_RED + slot] = xs_round(t);
}

// Exact per-CTA partials of up to two dot products (every thread passes its accumulators);
// the last CTA to deliver sums the partials of all CTAs and stores the rounded totals in
// scal[SC_RED + slot] (a single counter per launch: slot0 if >= 0, else slot1).
// Returns true in the last CTA, whose thread 0 wrote the totals.
__device__ inline bool cta_partials(const SolverArgs& a, XSum& x0, XSum& x1, int slot0, int slot1) {
  __shared__ XSum sh[8];
  if (slot0 >= 0) cta_partial(a, x0, slot0, sh);
  if (slot1 >= 0) cta_partial(a, x1, slot1, sh);
  if (!cta_last(a, slot0 >= 0 ? slot0 : slot1)) return false;
  if (slot0 >= 0) total_of(a, slot0, sh);
  if (slot1 >= 0) total_of(a, slot1, sh);
  return true;
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

#define FOR_BODIES(b) for (int b = blockIdx.x * WPB + (int)(threadIdx.x >> 5); b < a.n; b += (int)gridDim.x * WPB)

__device__ inline bool solver_done(const int* dstat) {
  return ((volatile const int*)dstat)[DS_R_DONE] != 0 || ((volatile const int*)dstat)[DS_S_DONE] != 0;
}

// the current Krylov iteration (device counter, 1 at the first iteration, advanced by
// loop_end); iterations beyond the limit do nothing
__device__ inline int iteration(const SolverArgs& a) { return a.dstat[DS_IT]; }

// The outcome of a finished solve into the device loop's step counters (a.tally): its
// iterations, and the non-convergence bit when it stopped at cg_max_iter (one thread)
__device__ inline void tally_solve(const SolverArgs& a) {
  if (!a.tally) return;
  a.tally->step.lin += a.dstat[DS_SOLVER_ITERS];
  if (!(a.dstat[DS_R_DONE] || a.dstat[DS_S_DONE])) atomicOr(&a.dstat[DS_STATUS], ST_SOLVER_NOCONV);
}

// The end of a loop iteration (one thread, in the iteration's last kernel once its last
// reduction is final): advances the iteration counter, makes the convergence test of the next
// iteration's first kernel (PCG: r.z against the threshold; BiCGSTAB: r.M^-1 r and
// rho = rh.r), records a stop as that kernel would, and sets the WHILE node's condition.  The
// loop ends at convergence or after maxit iterations (and the solve's outcome is tallied); a
// body that ran more than maxit times also ends it.
__device__ inline void loop_end(const SolverArgs& a, int pcg) {
  const int it = a.dstat[DS_IT];
  bool stop = solver_done(a.dstat) || it + 1 > a.maxit || a.dstat[DS_KRYLOV_RUNS] > a.maxit;
  if (!stop) {
    const double thr2 = a.scal[SC_THR2];
    if (pcg) {
      stop = !(a.scal[SC_RED + ((it & 1) ? SL_RZ1 : SL_RZ0)] > thr2);
    } else {
      const double rho = a.scal[SC_RED + SL_RHR];
      stop = !(a.scal[SC_RED + SL_RZ0] > thr2) || rho == 0.0 || !isfinite(rho);
    }
    if (stop) {
      a.dstat[DS_R_DONE] = it + 1;
      a.dstat[DS_SOLVER_ITERS] = it;
    }
  }
  a.dstat[DS_IT] = it + 1;
  if (stop) tally_solve(a);
  cudaGraphSetConditional(a.loop, stop ? 0u : 1u);
}

// The first kernel of an iteration counts the loop body's runs (thread 0 of CTA 0); a body
// that runs more than maxit times ends the loop (a safeguard: loop_end ends it at maxit)
__device__ inline void count_run(const SolverArgs& a) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && ++a.dstat[DS_KRYLOV_RUNS] > a.maxit)
    cudaGraphSetConditional(a.loop, 0u);
}

// ---- preconditioner setup: assemble and invert each cluster's dense block system ----
// Clusters of one body (in a resting pile nearly every cluster: most bodies touch only the
// fixed ground) are inverted by one warp each, in registers: lane j + 12 h (j < 12, h < 2)
// holds rows 6h .. 6h + 5 of column j, and the pivot values and multipliers travel by
// shuffles, so no shared memory and no barrier.  The arithmetic of every entry is the CTA
// kernel's, in the same order: at pivot k row k becomes (j == k ? 1 : K[k][j]) times the
// reciprocal of K[k][k], then every other row i with f = K[i][k] != 0 becomes
// (j == k ? 0 : K[i][j]) - f K[k][j] (f == 0: only K[i][k] = 0).
constexpr int WIT = 256;           // threads of the one-body inverse kernel
constexpr int kWarpInvGrid = 148;  // its CTAs: one wave, a warp per cluster (grid-stride past 1184)
__device__ inline void warp_inverse1(const SolverArgs& a, int c, int b, int lane) {
  const int j = lane % 12, h = lane / 12;  // lanes 24..31 (h = 2) carry values that no one reads
  double col[6];
  const double* B = a.diag + (size_t)b * 144;
#pragma unroll
  for (int t = 0; t < 6; ++t) col[t] = h < 2 ? B[(6 * h + t) * 12 + j] : 0.0;
  // The pivot loop stays rolled (the code stays small); the rows are unrolled so that they
  // live in registers, and the updates are branch-free so that the rows' shuffles overlap.
#pragma unroll 1
  for (int k = 0; k < 12; ++k) {
    const int hk = k / 6, tk = k % 6;
    double ck = 0.0;  // this lane's entry of row k (meaningful in half hk)
#pragma unroll
    for (int t = 0; t < 6; ++t)
      if (t == tk) ck = col[t];
    const double ip = 1.0 / __shfl_sync(0xffffffffu, ck, k + 12 * hk);
    const double rk = __shfl_sync(0xffffffffu, ck, j + 12 * hk);  // K[k][j]
    const double pk = (j == k ? 1.0 : rk) * ip;                     // row k scaled
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      const double f = __shfl_sync(0xffffffffu, col[t], k + 12 * h);  // K[6h + t][k]
      const double base = j == k ? 0.0 : col[t];
      const double upd = base - f * pk;
      col[t] = (h == hk && t == tk) ? pk : (f != 0.0 ? upd : base);
    }
  }
  if (h < 2) {
    double* out = a.cl_inv + a.cl_off[c];
#pragma unroll
    for (int t = 0; t < 6; ++t) out[(6 * h + t) * 12 + j] = col[t];
  }
}

// use_hc: CTA 0 also sets the condition of the IF node around k_cluster_inverse (a
// device-loop step): 1 when a cluster has more than one body
__global__ void __launch_bounds__(WIT) k_cluster_inverse_small(SolverArgs a, cudaGraphConditionalHandle hc,
                                                               int use_hc) {
  const int ncl = *a.ncl_dev;
  if (use_hc && blockIdx.x == 0) {
    int big = 0;
    for (int c = threadIdx.x; c < ncl && !big; c += WIT) big = a.cl_ptr[c + 1] - a.cl_ptr[c] > 1;
    big = __syncthreads_or(big);
    if (threadIdx.x == 0) cudaGraphSetConditional(hc, big ? 1u : 0u);
  }
  const int lane = (int)(threadIdx.x & 31);
  const int nw = gridDim.x * (WIT / 32);
  for (int c = (int)((blockIdx.x * WIT + threadIdx.x) >> 5); c < ncl; c += nw) {
    const int base = a.cl_ptr[c];
    if (a.cl_ptr[c + 1] - base == 1) warp_inverse1(a, c, a.cl_body[base], lane);
  }
}

// Clusters of two bodies or more: one CTA each, the system in shared memory.
constexpr int kInvGrid = 148;  // CTAs of the inverse kernel (one per SM at the largest clusters)
__global__ void __launch_bounds__(IT) k_cluster_inverse(SolverArgs a, const int* body_cl) {
  extern __shared__ double K[];
  const int ncl = *a.ncl_dev;
  for (int c = blockIdx.x; c < ncl; c += gridDim.x) {
    const int base = a.cl_ptr[c], s = a.cl_ptr[c + 1] - base, D = 12 * s;
    if (s == 1) continue;  // k_cluster_inverse_small's
    for (int e = threadIdx.x; e < D * D; e += IT) K[e] = 0.0;
    __syncthreads();
    // block row of every member: its diagonal block and the blocks of active pairs whose
    // other body is in the same cluster
    for (int e = threadIdx.x; e < s * 144; e += IT) {
      const int li = e / 144, rc = e % 144;
      const int b = a.cl_body[base + li];
      K[(size_t)(12 * li + rc / 12) * D + 12 * li + rc % 12] = a.diag[(size_t)b * 144 + rc];
    }
    if (s > 1) {
      for (int li = 0; li < s; ++li) {
        const int b = a.cl_body[base + li];
        for (int k = a.row_ptr[b]; k < a.row_ptr[b + 1]; ++k) {
          const int pr = a.adj_pair[k];
          if (a.pair_active[pr] <= 0) continue;
          const int J = a.adj_col[k];
          if (body_cl[J] != c || a.fixed[J] || a.fixed[b]) continue;
          int lj = 0;
          while (a.cl_body[base + lj] != J) ++lj;  // members are few (<= kMaxCluster)
          const int side = a.ij[pr].x == b ? 0 : 1;
          const double* O = a.offdiag + (size_t)pr * 288 + side * 144;
          for (int rc = threadIdx.x; rc < 144; rc += IT)
            K[(size_t)(12 * li + rc / 12) * D + 12 * lj + rc % 12] = O[rc];
        }
      }
    }
    __syncthreads();
    // In-place Gauss-Jordan inverse (SPD: no pivoting) with the oracle's arithmetic: at pivot
    // k, row k is scaled by 1 / K[k][k] (its diagonal becoming that reciprocal), then every
    // other row i with f = K[i][k] != 0 becomes (j == k ? 0 : K[i][j]) - f K[k][j] (f == 0:
    // only K[i][k] = 0).  Each row belongs to one warp for the whole inverse (rows warp,
    // warp + 16, ...), which reads its own multiplier, and the owner of row k + 1 scales that
    // row right after updating it at pivot k, so the next pivot row is ready at the one block
    // barrier per pivot.
    constexpr int NW = IT / 32;
    const int warp = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    auto scale_row = [&](int i) {  // row i / K[i][i], its diagonal the reciprocal
      double* R = K + (size_t)i * D;
      const double ip = 1.0 / R[i];
      __syncwarp();
      for (int j = lane; j < D; j += 32) R[j] = (j == i ? 1.0 : R[j]) * ip;
      __syncwarp();
    };
    if (warp == 0) scale_row(0);
    __syncthreads();
    for (int k = 0; k < D; ++k) {
      const double* P = K + (size_t)k * D;
      for (int i = warp; i < D; i += NW) {
        if (i == k) continue;
        double* R = K + (size_t)i * D;
        const double f = R[k];
        __syncwarp();
        if (f != 0.0) {
          for (int j = lane; j < D; j += 32) R[j] = (j == k ? 0.0 : R[j]) - f * P[j];
        } else if (lane == 0) {
          R[k] = 0.0;
        }
        __syncwarp();
        if (i == k + 1) scale_row(i);
      }
      __syncthreads();
    }
    double* out = a.cl_inv + a.cl_off[c];
    for (int e = threadIdx.x; e < D * D; e += IT) out[e] = K[e];
    __syncthreads();
  }
}

// One warp per cluster: the input's entries of the cluster's body rows, in = row_in(i) for the
// entry i of a member body (lanes 0..11: the row's 12 entries; row_in may also update the
// body's own entries of other vectors), then out = M^-1 in over the cluster -- lane i
// computes rows i, i + 32, ... of the cluster's dense inverse times the gathered input,
// summing over the columns in order -- with the partial in.out added to *dot (if not null);
// out null: the product only feeds the dot.
template <class RowIn>
__device__ inline void cluster_apply(const SolverArgs& a, double* out, XSum* dot, RowIn&& row_in) {
  constexpr int NWA = AT / 32;
  __shared__ double vs[NWA][12 * kMaxCluster];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncl = *a.ncl_dev;
  for (int c = blockIdx.x * NWA + warp; c < ncl; c += gridDim.x * NWA) {
    const int base = a.cl_ptr[c], sz = a.cl_ptr[c + 1] - base, D = 12 * sz;
    if (lane < 12)
      for (int m = 0; m < sz; ++m) vs[warp][12 * m + lane] = row_in((size_t)a.cl_body[base + m] * 12 + lane);
    __syncwarp();
    const double* Kc = a.cl_inv + a.cl_off[c];
    for (int i = lane; i < D; i += 32) {
      double acc = 0.0;
      const double* row = Kc + (size_t)i * D;
      for (int j = 0; j < D; ++j) acc += row[j] * vs[warp][j];
      if (out) out[(size_t)a.cl_body[base + i / 12] * 12 + i % 12] = acc;
      if (dot) xs_add(*dot, vs[warp][i] * acc);
    }
    __syncwarp();
  }
}

// ---- the solve's set-up ----
// One launch, one warp per cluster (every body is in exactly one): the residual r = b - A x of
// the cluster's bodies (BiCGSTAB: also rh = r, p = v = 0), z = M^-1 r (PCG: also p = z) and
// M^-1 b, with the exact partials of b.M^-1 b, r.r and r.z -- the arithmetic of the row
// kernels and of cluster_apply, entry for entry.  The last CTA rounds the three totals and
// starts the solve: the threshold tol^2 b.M^-1 b, the scalars, the iteration counter, the outcome
// flags and the WHILE node's condition (set at every solve: the loop's node may sit inside
// another conditional node, whose launches do not reset it).  With b.M^-1 b <= 0 the solution
// is 0 (x is cleared) and no iteration runs; a solve without iterations is tallied here.
__global__ void __launch_bounds__(AT) k_krylov_setup(SolverArgs a, const double* bvec, double* x, double* r,
                                                     double* z, double* pz, double* rh, double* p0, double* v0,
                                                     double tol2, cudaGraphConditionalHandle h) {
  constexpr int NWA = AT / 32;
  __shared__ double vr[NWA][12 * kMaxCluster], vb[NWA][12 * kMaxCluster];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  XSum bz, rr, rz;
  xs_zero(bz);
  xs_zero(rr);
  xs_zero(rz);
  const int ncl = *a.ncl_dev;
  for (int c = blockIdx.x * NWA + warp; c < ncl; c += gridDim.x * NWA) {
    const int base = a.cl_ptr[c], sz = a.cl_ptr[c + 1] - base, D = 12 * sz;
    for (int m = 0; m < sz; ++m) {
      const int b = a.cl_body[base + m];
      const double ax = row_product(a, b, x);
      if (lane < 12) {
        const size_t i = (size_t)b * 12 + lane;
        const double bi = bvec[i], ri = bi - ax;
        r[i] = ri;
        if (rh) rh[i] = ri;
        if (p0) p0[i] = 0.0;
        if (v0) v0[i] = 0.0;
        xs_add(rr, ri * ri);
        vr[warp][12 * m + lane] = ri;
        vb[warp][12 * m + lane] = bi;
      }
    }
    __syncwarp();
    const double* Kc = a.cl_inv + a.cl_off[c];
    for (int i = lane; i < D; i += 32) {
      double ar = 0.0, ab = 0.0;
      const double* row = Kc + (size_t)i * D;
      for (int j = 0; j < D; ++j) {
        const double k = row[j];
        ar += k * vr[warp][j];
        ab += k * vb[warp][j];
      }
      const size_t gi = (size_t)a.cl_body[base + i / 12] * 12 + i % 12;
      z[gi] = ar;
      if (pz) pz[gi] = ar;
      xs_add(rz, vr[warp][i] * ar);
      xs_add(bz, vb[warp][i] * ab);
    }
    __syncwarp();
  }
  __shared__ XSum sh[NWA];
  cta_partial(a, bz, SL_BZ, sh);
  cta_partial(a, rr, SL_RHR, sh);
  cta_partial(a, rz, SL_RZ0, sh);
  if (!cta_last(a, SL_BZ)) return;
  total_of(a, SL_BZ, sh);
  total_of(a, SL_RHR, sh);
  total_of(a, SL_RZ0, sh);
  __syncthreads();  // the totals, stored by thread 0
  const double b = a.scal[SC_RED + SL_BZ];
  if (!(b > 0.0))
    for (int i = threadIdx.x; i < 12 * a.n; i += AT) x[i] = 0.0;
  if (threadIdx.x == 0) {
    a.scal[SC_RHO0] = a.scal[SC_RHO1] = a.scal[SC_ALPHA] = a.scal[SC_OMEGA] = 1.0;
    a.scal[SC_THR2] = tol2 * b;
    a.dstat[DS_IT] = 1;
    a.dstat[DS_KRYLOV_RUNS] = 0;
    // the solve's outcome flags start clear (the iterations that follow set and read them)
    a.dstat[DS_R_DONE] = b > 0.0 ? 0 : 1;
    a.dstat[DS_S_DONE] = 0;
    a.dstat[DS_SOLVER_ITERS] = 0;
    const bool loop = b > 0.0 && a.maxit >= 1;
    if (!loop) tally_solve(a);
    cudaGraphSetConditional(h, loop ? 1u : 0u);
  }
}

// ---- PCG ----
// K1: converged if r.z <= thr^2; else Ap = A p with partial p.Ap
__global__ void __launch_bounds__(256) k_pcg_1(SolverArgs a, const double* pv, double* Ap) {
  count_run(a);
  const int it = iteration(a);
  if (solver_done(a.dstat) || it > a.maxit) return;
  const int rz = (it & 1) ? SL_RZ0 : SL_RZ1;
  const int slots[1] = {rz};
  double sc[1];
  cta_scalars(a, slots, 1, sc);
  if (!(sc[0] > a.scal[SC_THR2])) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.dstat[DS_R_DONE] = it;
      a.dstat[DS_SOLVER_ITERS] = it - 1;
    }
    return;
  }
  const int lane = threadIdx.x & 31;
  XSum d0, d1;
  xs_zero(d0);
  xs_zero(d1);
  FOR_BODIES(b) {
    const double yi = row_product(a, b, pv);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      Ap[i] = yi;
      xs_add(d0, pv[i] * yi);
    }
  }
  cta_partials(a, d0, d1, SL_PAP, -1);
}

// K2: alpha = rz / p.Ap; x += alpha p; r -= alpha Ap (stops on a non-positive curvature); then
// z = M^-1 r with the partial r.z into the new slot, one warp per cluster (cluster_apply: the
// update of the cluster's bodies, then the product over the updated r).  The iteration's end
// (loop_end): by the last CTA, or by CTA 0 when the solve stops here or has stopped.
__global__ void __launch_bounds__(AT) k_pcg_2(SolverArgs a, const double* pv, const double* Ap, double* x, double* r,
                                              double* z) {
  const int it = iteration(a);
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  if (solver_done(a.dstat) || it > a.maxit) {
    if (lead) loop_end(a, 1);
    return;
  }
  const int rz = (it & 1) ? SL_RZ0 : SL_RZ1;
  const int slots[2] = {rz, SL_PAP};
  double sc[2];
  cta_scalars(a, slots, 2, sc);
  if (!(sc[1] > 0.0)) {
    if (lead) {
      a.dstat[DS_R_DONE] = it;
      a.dstat[DS_SOLVER_ITERS] = it - 1;
      loop_end(a, 1);
    }
    return;
  }
  const double alpha = sc[0] / sc[1];
  XSum d0, d1;
  xs_zero(d0);
  xs_zero(d1);
  cluster_apply(a, z, &d0, [&](size_t i) {
    x[i] += alpha * pv[i];
    const double ri = r[i] - alpha * Ap[i];
    r[i] = ri;
    return ri;
  });
  if (cta_partials(a, d0, d1, (it & 1) ? SL_RZ1 : SL_RZ0, -1) && threadIdx.x == 0) {
    a.dstat[DS_SOLVER_ITERS] = it;
    loop_end(a, 1);  // (the new r.z is final)
  }
}

// K3 (after K2's z = M^-1 r and r.z in the new slot): beta = rz_new / rz_old; p = z + beta p
__global__ void __launch_bounds__(256) k_pcg_3(SolverArgs a, const double* z, double* pv) {
  const int it = iteration(a) - 1;  // (K2 ended the iteration: the counter is one ahead)
  if (solver_done(a.dstat) || it > a.maxit) return;
  const int rz_old = (it & 1) ? SL_RZ0 : SL_RZ1, rz_new = (it & 1) ? SL_RZ1 : SL_RZ0;
  const int slots[2] = {rz_new, rz_old};
  double sc[2];
  cta_scalars(a, slots, 2, sc);
  if (!(sc[0] > a.scal[SC_THR2])) return;  // converged: K1 of the next iteration stops
  const double beta = sc[0] / sc[1];
  const int lane = threadIdx.x & 31;
  FOR_BODIES(b) {
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      pv[i] = z[i] + beta * pv[i];
    }
  }
}

// ---- BiCGSTAB (right preconditioned) ----
// K1: converged if r.M^-1 r small; rho = rh.r; p = r + beta (p - omega v); then y = M^-1 p,
// one warp per cluster (cluster_apply)
__global__ void __launch_bounds__(AT) k_bicg_1(SolverArgs a, const double* r, double* pv, const double* v,
                                               double* y) {
  count_run(a);
  const int it = iteration(a);
  if (solver_done(a.dstat) || it > a.maxit) return;
  const int slots[2] = {SL_RZ0, SL_RHR};
  double sc[2];
  cta_scalars(a, slots, 2, sc);
  if (!(sc[0] > a.scal[SC_THR2]) || sc[1] == 0.0 || !isfinite(sc[1])) {
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
  cluster_apply(a, y, nullptr, [&](size_t i) {
    const double pi = it == 1 ? r[i] : r[i] + beta * (pv[i] - omega * v[i]);
    pv[i] = pi;
    return pi;
  });
  if (blockIdx.x == 0 && threadIdx.x == 0) a.scal[it & 1] = rho;
}

// out = A in; partials w0.out (slot0), w1.out (slot1)
__global__ void __launch_bounds__(256) k_spmv(SolverArgs a, const double* in, double* out, const double* w0, int slot0,
                                              const double* w1, int slot1) {
  if (solver_done(a.dstat) || iteration(a) > a.maxit) return;
  const int lane = threadIdx.x & 31;
  XSum d0, d1;
  xs_zero(d0);
  xs_zero(d1);
  FOR_BODIES(b) {
    const double yi = row_product(a, b, in);
    if (lane < 12) {
      const size_t i = (size_t)b * 12 + lane;
      out[i] = yi;
      if (w0) xs_add(d0, w0[i] * yi);
      if (w1) xs_add(d1, w1[i] * yi);
    }
  }
  cta_partials(a, d0, d1, slot0, slot1);
}

// K3: alpha = rho / rh.v; s = r - alpha v; then z = M^-1 s with the partial s.z, one warp per
// cluster (cluster_apply)
__global__ void __launch_bounds__(AT) k_bicg_3(SolverArgs a, const double* r, const double* v, double* s,
                                               double* z) {
  const int it = iteration(a);
  if (solver_done(a.dstat) || it > a.maxit) return;
  const int slots[1] = {SL_RHV};
  double sc[1];
  cta_scalars(a, slots, 1, sc);
  const double alpha = a.scal[it & 1] / sc[0];
  XSum d0, d1;
  xs_zero(d0);
  xs_zero(d1);
  cluster_apply(a, z, &d0, [&](size_t i) {
    const double si = r[i] - alpha * v[i];
    s[i] = si;
    return si;
  });
  if (blockIdx.x == 0 && threadIdx.x == 0) a.scal[SC_ALPHA] = alpha;
  cta_partials(a, d0, d1, SL_SZ, -1);
}

// K4 (after K3's z = M^-1 s and s.z): if small, x += alpha y and stop
__global__ void __launch_bounds__(256) k_bicg_4(SolverArgs a, const double* y, double* x) {
  const int it = iteration(a);
  const volatile int* ds = a.dstat;
  if (ds[DS_R_DONE] != 0 || (ds[DS_S_DONE] != 0 && ds[DS_S_DONE] != it) || it > a.maxit) return;
  const int slots[1] = {SL_SZ};
  double sc[1];
  cta_scalars(a, slots, 1, sc);
  if (sc[0] > a.scal[SC_THR2]) return;
  const double alpha = a.scal[SC_ALPHA];
  const int lane = threadIdx.x & 31;
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
}

// K6: omega = t.s / t.t; x += alpha y + omega z; r = s - omega t; partial rh.r; then the
// partial r.M^-1 r, one warp per cluster (cluster_apply; the product itself is not kept).  The
// iteration's end (loop_end): by the last CTA, or by CTA 0 when the solve has stopped.
__global__ void __launch_bounds__(AT) k_bicg_6(SolverArgs a, const double* y, const double* z, const double* s,
                                               const double* t, const double* rh, double* x, double* r) {
  const int it = iteration(a);
  if (solver_done(a.dstat) || it > a.maxit) {
    if (blockIdx.x == 0 && threadIdx.x == 0) loop_end(a, 0);
    return;
  }
  const int slots[2] = {SL_TS, SL_TT};
  double sc[2];
  cta_scalars(a, slots, 2, sc);
  const double omega = sc[0] / sc[1];
  const double alpha = a.scal[SC_ALPHA];
  XSum rz, rhr;
  xs_zero(rz);
  xs_zero(rhr);
  cluster_apply(a, nullptr, &rz, [&](size_t i) {
    x[i] += alpha * y[i] + omega * z[i];
    const double ri = s[i] - omega * t[i];
    r[i] = ri;
    xs_add(rhr, rh[i] * ri);
    return ri;
  });
  if (cta_partials(a, rz, rhr, SL_RZ0, SL_RHR) && threadIdx.x == 0) {
    a.scal[SC_OMEGA] = omega;
    a.dstat[DS_SOLVER_ITERS] = it;
    loop_end(a, 0);  // (r.M^-1 r and rh.r are final)
  }
}

SolverArgs solver_args(Sim& s) {
  SolverArgs a;
  a.tally = nullptr;
  a.loop = 0;
  a.n = s.n;
  a.diag = s.diag;
  a.offdiag = s.offdiag;
  a.row_ptr = s.row_ptr;
  a.adj_col = s.adj_col;
  a.adj_pair = s.adj_pair;
  a.pair_active = s.pair_active;
  a.fixed = s.fixed;
  a.ij = s.ij;
  a.ncl_dev = s.ncl_dev;
  a.maxit = s.prm.cg_max_iter;
  a.cl_ptr = s.cl_ptr;
  a.cl_body = s.cl_body;
  a.cl_off = s.cl_off;
  a.cl_inv = s.cl_inv;
  a.part = s.partials;
  a.red_count = s.red_count;
  a.scal = s.scal;
  a.dstat = s.dstat;
  return a;
}

}  // namespace

// Exclusive prefix sum over the 1024 threads of a CTA (one value per thread); *total gets the
// sum.  Every thread must call it.
__device__ inline long long block_scan_excl(long long v, long long* total) {
  __shared__ long long wsum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;  // inclusive prefix of the warp totals
  }
  __syncthreads();
  const long long before = (warp > 0 ? wsum[warp - 1] : 0) + x - v;
  *total = wsum[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before;
}

// The preconditioner's clusters, formed on the device by one CTA from the active-pair list
// the pair assembly appended (pair, I, J, FP32 weight bits; in any order).  Rounds: every
// cluster picks its strongest admissible pair to another cluster (weight, then the lower pair
// index, as one 64-bit key; admissible: both clusters together within cap bodies) and two
// clusters that pick the same pair merge under the lower label.  Every decision of a round
// uses the labels and sizes from its start, so the result does not depend on the order in
// which threads see the pairs.  Then the tables: clusters ordered by their first body (the
// label), members in increasing order, the offsets of the dense inverses.  Skipped when the
// list overflowed (the pass is rerun).
constexpr int KT = 1024;  // threads of the clustering CTA
__global__ void __launch_bounds__(KT) k_clusters(int n, int cap, const int4* __restrict__ act, int cap_act,
                                                 int* dstat, ClusterTables t, ClusterWork w) {
  const int tid = threadIdx.x;
  if (dstat[DS_STATUS] & (ST_ACT_OVERFLOW | ST_PAIR_OVERFLOW | ST_CONTACT_OVERFLOW)) return;
  const int m = min(dstat[DS_NACTP], cap_act);
  for (int b = tid; b < n; b += KT) {
    w.label[b] = b;
    w.size[b] = 1;
  }
  __shared__ int merged;
  __syncthreads();
  for (int round = 0; cap > 1 && round < 4 * kMaxCluster; ++round) {
    for (int b = tid; b < n; b += KT) {
      w.best[b] = 0ULL;
      w.to[b] = b;
    }
    if (tid == 0) merged = 0;
    __syncthreads();
    for (int e = tid; e < m; e += KT) {
      const int4 q = act[e];
      const int a = w.label[q.y], b = w.label[q.z];
      if (a == b || w.size[a] + w.size[b] > cap) continue;
      const unsigned long long key = ((unsigned long long)(unsigned)q.w << 32) | (0xffffffffULL - (unsigned)q.x);
      atomicMax(&w.best[a], key);
      atomicMax(&w.best[b], key);
    }
    __syncthreads();
    // a cluster has one best pair, so it takes part in at most one merge of the round
    for (int e = tid; e < m; e += KT) {
      const int4 q = act[e];
      const int a = w.label[q.y], b = w.label[q.z];
      if (a == b) continue;
      const unsigned long long key = ((unsigned long long)(unsigned)q.w << 32) | (0xffffffffULL - (unsigned)q.x);
      if (w.best[a] != key || w.best[b] != key) continue;
      const int r = min(a, b), o = max(a, b);
      w.to[o] = r;
      w.size[r] += w.size[o];
      merged = 1;
    }
    __syncthreads();
    for (int b = tid; b < n; b += KT) w.label[b] = w.to[w.label[b]];
    __syncthreads();
    if (!merged) break;
  }
  // cluster index of every label, cluster offsets and inverse offsets, in label order
  long long ccarry = 0, pcarry = 0, ocarry = 0;
  for (int b0 = 0; b0 < n; b0 += KT) {
    const int b = b0 + tid;
    const bool root = b < n && w.label[b] == b;
    const int sz = root ? w.size[b] : 0;
    long long tc, tp, to_;
    const long long c = block_scan_excl(root ? 1 : 0, &tc) + ccarry;
    const long long p = block_scan_excl(sz, &tp) + pcarry;
    const long long o = block_scan_excl(root ? 144LL * sz * sz : 0, &to_) + ocarry;
    if (root) {
      w.cidx[b] = (int)c;
      t.cl_ptr[c] = (int)p;
      t.cl_off[c] = o;
      w.fill[c] = 0;
    }
    ccarry += tc;
    pcarry += tp;
    ocarry += to_;
  }
  const int ncl = (int)ccarry;
  if (tid == 0) {
    *t.ncl = ncl;
    t.cl_ptr[ncl] = n;
    t.cl_off[ncl] = ocarry;
  }
  __syncthreads();
  for (int b = tid; b < n; b += KT) {
    const int c = w.cidx[w.label[b]];
    t.body_cl[b] = c;
    t.cl_body[t.cl_ptr[c] + atomicAdd(&w.fill[c], 1)] = b;
  }
  __syncthreads();
  for (int c = tid; c < ncl; c += KT) {  // members in increasing order (at most cap of them)
    int* mb = t.cl_body + t.cl_ptr[c];
    const int k1 = t.cl_ptr[c + 1] - t.cl_ptr[c];
    for (int i = 1; i < k1; ++i) {
      const int v = mb[i];
      int j = i - 1;
      for (; j >= 0 && mb[j] > v; --j) mb[j + 1] = mb[j];
      mb[j + 1] = v;
    }
  }
}

// Clusters of the preconditioner from the active-pair list of the last GH pass, on the device
// (k_clusters); enqueued on stream st (the pass's stream when null).
cudaError_t cluster_tables(Sim& s, cudaStream_t st) {
  const int cap = s.prm.precond == 1 ? std::max(1, std::min(kMaxCluster, s.prm.cluster_max)) : 1;
  k_clusters<<<1, KT, 0, st ? st : s.stream>>>(s.n, cap, s.act_pairs, s.cap_act, s.dstat,
                                               cluster_tables_at(s.cl_tab, s.n), s.cl_work);
  ++s.launches;
  return cudaGetLastError();
}

// Inverts every cluster's dense system (the tables k_clusters made; their count is read on the
// device): clusters of one body a warp each, larger ones (when cluster_max allows them) a CTA
// each with the shared memory of the largest.  Fixed grids; enqueued without a sync.
int cluster_inverse(Sim& s) {
  SolverArgs a = solver_args(s);
  const int cm = s.prm.precond == 1 ? std::max(1, std::min(kMaxCluster, s.prm.cluster_max)) : 1;
  // a device-loop step (in_device_loop, under capture) puts the CTA kernel in an IF node:
  // most Newton iterations of a resting pile have no cluster of more than one body
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (ABD_NOTE(cudaStreamIsCapturing(s.stream, &cs)) != cudaSuccess) return ABD_ERR_CUDA;
  const bool use_if = cm > 1 && s.in_device_loop && cs == cudaStreamCaptureStatusActive;
  cudaGraphConditionalHandle hc = 0;
  if (use_if && make_handle(s.stream, &hc) != ABD_OK) return ABD_ERR_CUDA;
  k_cluster_inverse_small<<<kWarpInvGrid, WIT, 0, s.stream>>>(a, hc, use_if ? 1 : 0);
  ++s.launches;
  if (cm > 1) {
    const size_t smem = sizeof(double) * 144 * (size_t)cm * cm;
    if (smem > 48 * 1024 && (int)smem > s.cl_smem) {
      if (cudaFuncSetAttribute(k_cluster_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
        return ABD_ERR_CUDA;
      s.cl_smem = (int)smem;
    }
    if (use_if) {  // the body's kernel is not counted among the launches (it runs now and then)
      cudaGraph_t body = nullptr;
      if (int r = add_conditional(s.stream, hc, cudaGraphCondTypeIf, &body)) return r;
      if (int r = capture_body(s, body, s.cap_stream5, [&]() -> int {
            k_cluster_inverse<<<kInvGrid, IT, smem, s.stream>>>(a, s.body_cl);
            return ABD_NOTE(cudaGetLastError()) == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
          }))
        return r;
    } else {
      k_cluster_inverse<<<kInvGrid, IT, smem, s.stream>>>(a, s.body_cl);
      ++s.launches;
    }
  }
  return cudaGetLastError() == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
}

// Opts the inverse kernel in to the shared memory of the largest cluster (once, at creation:
// the passes that launch it may be under stream capture)
int prepare_solver(Sim& s) {
  const int smem = (int)(sizeof(double) * 144 * kMaxCluster * kMaxCluster);
  if (cudaFuncSetAttribute(k_cluster_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return ABD_ERR_CUDA;
  s.cl_smem = smem;
  return ABD_OK;
}

int build_preconditioner(Sim& s) {
  if (cluster_tables(s, nullptr) != cudaSuccess) return ABD_ERR_CUDA;
  return cluster_inverse(s);
}

// kernels of one iteration of the loop's body: PCG or BiCGSTAB
constexpr int iteration_kernels(bool pcg) { return pcg ? 3 : 6; }

// Enqueues a solve on s.stream, which must be capturing: the setup kernels, then a WHILE node
// whose body is one iteration (its last kernel sets the loop condition), the body captured on
// cap_stream2.  Counts the setup's launches and, in *per_iter, one iteration's.
int krylov_capture(Sim& s, double* x, long long* per_iter_out, bool tally) {
  SolverArgs a = solver_args(s);
  a.tally = tally ? s.box : nullptr;
  const double* bvec = s.g;
  const bool pcg = s.prm.solver == 1;
  cudaStream_t st = s.stream;
  cudaStreamCaptureStatus cs;
  cudaGraph_t graph = nullptr;
  if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, nullptr, nullptr) != cudaSuccess ||
      cs != cudaStreamCaptureStatusActive)
    return ABD_ERR_CUDA;
  // the loop's handle first: k_krylov_setup sets its value
  cudaGraphConditionalHandle h;
  if (ABD_NOTE(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault)) != cudaSuccess) return ABD_ERR_CUDA;
  a.loop = h;
  k_krylov_setup<<<s.cl_grid, AT, 0, st>>>(a, bvec, x, s.r, s.z, pcg ? s.pv : nullptr, pcg ? nullptr : s.rh,
                                           pcg ? nullptr : s.pv, pcg ? nullptr : s.v, s.prm.cg_tol * s.prm.cg_tol, h);
  ++s.launches;
  // the iteration loop: a WHILE node on the capture, its body captured on a second stream
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps) != cudaSuccess ||
      cs != cudaStreamCaptureStatusActive)
    return ABD_ERR_CUDA;
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t loop;
  if (ABD_NOTE(cudaGraphAddNode(&loop, graph, deps, ndeps, &np)) != cudaSuccess) return ABD_ERR_CUDA;
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if (ABD_NOTE(cudaStreamUpdateCaptureDependencies(st, &loop, 1, cudaStreamSetCaptureDependencies)) != cudaSuccess)
    return ABD_ERR_CUDA;
  cudaStream_t bs = s.cap_stream2;
  if (ABD_NOTE(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return ABD_ERR_CUDA;
  if (pcg) {
    k_pcg_1<<<s.red_grid, 256, 0, bs>>>(a, s.pv, s.v);
    k_pcg_2<<<s.cl_grid, AT, 0, bs>>>(a, s.pv, s.v, x, s.r, s.z);
    k_pcg_3<<<s.red_grid, 256, 0, bs>>>(a, s.z, s.pv);
  } else {
    k_bicg_1<<<s.cl_grid, AT, 0, bs>>>(a, s.r, s.pv, s.v, s.y);
    k_spmv<<<s.red_grid, 256, 0, bs>>>(a, s.y, s.v, s.rh, SL_RHV, nullptr, -1);
    k_bicg_3<<<s.cl_grid, AT, 0, bs>>>(a, s.r, s.v, s.s, s.z);
    k_bicg_4<<<s.red_grid, 256, 0, bs>>>(a, s.y, x);
    k_spmv<<<s.red_grid, 256, 0, bs>>>(a, s.z, s.t, s.s, SL_TS, s.t, SL_TT);
    k_bicg_6<<<s.cl_grid, AT, 0, bs>>>(a, s.y, s.z, s.s, s.t, s.rh, x, s.r);
  }
  if (per_iter_out) *per_iter_out = iteration_kernels(pcg);
  cudaGraph_t body_out = nullptr;
  const cudaError_t eb = ABD_NOTE(cudaGetLastError());
  if (cudaStreamEndCapture(bs, &body_out) != cudaSuccess || eb != cudaSuccess) return ABD_ERR_CUDA;
  return ABD_NOTE(cudaGetLastError()) == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
}

// Solves H x = g (x: warm start, overwritten).  Returns an ABD_* status.  One replayed graph
// (krylov_capture).  With iters_out the host waits for it and reads the outcome; without, the
// solve is only enqueued and its outcome stays in the mailbox's counters (krylov_outcome
// reads it after the caller's next read of the mailbox).
int krylov_solve(Sim& s, double* x, int* iters_out, GraphSlot* slot) {
  KeyHash kh;
  kh.add(x).add(s.n).add(s.prm_version).add(s.prm.solver).add(s.prm.cg_max_iter).add(s.cl_inv).add(s.box);
  kh.add(s.cap_gen).add(s.adj_col).add(s.adj_pair).add(s.ij).add(s.offdiag).add(s.pair_active);
  int r = run_graph(s, slot ? *slot : s.g_kinit, kh.h, [&]() -> int {
    long long per_iter = 0;
    const int q = krylov_capture(s, x, &per_iter, false);
    s.launches += per_iter;  // the graph's count covers one iteration
    return q;
  });
  if (r || !iters_out) return r;
  if (cudaMemcpyAsync(s.hbox, s.box, sizeof(Mailbox), cudaMemcpyDeviceToHost, s.stream) ||
      cudaStreamSynchronize(s.stream) != cudaSuccess)
    return ABD_ERR_CUDA;
  *iters_out = krylov_outcome(s);
  return ABD_OK;
}

int krylov_issue(Sim& s, double* x) {
  long long per_iter = 0;
  const int r = krylov_capture(s, x, &per_iter, true);
  s.step_launch[2] = per_iter;  // the setup's kernels are counted with the Newton iteration's
  return r;
}

// The last solve's iterations, from the host's copy of the mailbox; non-convergence raises
// ST_SOLVER_NOCONV in the host status bits.
int krylov_outcome(Sim& s) {
  const int* ds = s.hbox->dstat;
  const int per_iter = iteration_kernels(s.prm.solver == 1);
  // the graph's launch count covers one iteration; the loop ran ds[DS_IT] - 1
  s.launches += (long long)per_iter * std::max(0, ds[DS_IT] - 2);
  if (!(ds[DS_R_DONE] || ds[DS_S_DONE])) s.host_status |= ST_SOLVER_NOCONV;
  return ds[DS_SOLVER_ITERS];
}

}  // namespace abd
