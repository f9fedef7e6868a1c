// Batched line search: the energies of several trial step lengths in one pass.
//
// The backtracking line search (abd.py:146-160) evaluates E(q - alpha dq) for
// alpha = a_cap, a_cap / 2, ... until the Armijo test passes or alpha drops below alpha_min.
// In the reference every trial is an energy pass of its own (compute_energy, abd.py:133-141:
// DOF update, transform, culling, barrier sum).  Here the CCD pass of the Newton iteration
// (the CCD_LS narrow mode) also collects every PT / EE pair that can be in the culled set at
// any DOFs between q and q - dq, and a batch of trials only re-evaluates those candidates.
// For each trial alpha_k the kernels below recompute, with the arithmetic of the energy pass:
//   - the DOFs (A, p) - alpha_k dq and the positions of the vertices involved,
//   - the exact body boxes at alpha_k (FP64 min / max of each body's vertices),
//   - the reference's culling predicate (culling2.py:32-79, 213-227): the two body boxes
//     overlap and the two primitive boxes overlap,
//   - the barrier energy of every candidate that passes (ipcsk/energy.py:9-48), the
//     vertex-ground barriers (energy.py:24-33) and the inertia + orthogonality energy of
//     every free body (orthogonal_energy.py:24-32),
// and sums each trial's terms exactly, so a trial's energy is bitwise the energy pass's at
// the same DOFs.  The host takes the first trial that the sequential search would accept.
#include <cuda_runtime.h>

#include "abd_body.cuh"
#include "abd_geometry.cuh"

namespace abd {

namespace {

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

struct LsArgs {
  abd_params prm;
  int n, V;
  const int* vbody;
  const double* x0;
  const double *A, *p, *dq;     // the iterate and the search direction
  const double* dpar;           // [kParK] trial count, [kParAlpha + k] step lengths
  abd_states st;
  const double *mass, *I0;
  const int* fixed;
  unsigned long long* bnd;      // [kLsMax][n][6] body bounds of the trials (max-keys)
  Box* box;                     // [kLsMax][n] body boxes of the trials
  const int *tris, *edges;
  const int4* ecand;            // candidates of the last CCD_LS pass
  int cap_ecand;
  const int* dstat;
  XSum* energy;                 // [kLsMax] exact energies of the trials
  int nslice;
  const int4* slice;            // vertex slices: (body, first vertex, count <= 64)
};

__device__ inline int ls_trials(const LsArgs& a) { return (int)a.dpar[kParK]; }

// the block's exact accumulators added to the trials' totals
__device__ inline void flush(XSum* dst, const XSum* acc, int K) {
  for (int e = threadIdx.x; e < K * (kXD + 1); e += blockDim.x) {
    const int k = e / (kXD + 1), i = e % (kXD + 1);
    const long long v = reinterpret_cast<const long long*>(&acc[k])[i];
    if (!v) continue;
    long long* d = reinterpret_cast<long long*>(&dst[k]);
    if (i < kXD) atomicAdd((unsigned long long*)&d[i], (unsigned long long)v);
    else atomicOr((unsigned long long*)&d[i], (unsigned long long)v);
  }
}

// Warp-wide maximum of the 64-bit keys of the lanes in seg (every lane of seg calls it): the
// maximum high word first, then the maximum low word among the lanes that hold it.
__device__ inline unsigned long long seg_max_key(unsigned seg, unsigned long long key) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned hm = __reduce_max_sync(seg, hi);
  const unsigned lm = __reduce_max_sync(seg, hi == hm ? lo : 0u);
  return ((unsigned long long)hm << 32) | lm;
}

// One warp per vertex slice (at most 64 vertices of one body: two per lane) for the exact
// bounds of each body at every trial, then one warp per 32 bodies for the inertia +
// orthogonality energy of each free body, summed exactly across the warp before one lane
// adds it to the block's accumulator.  A slice's lanes take the min / max of their vertices'
// coordinates and the warp reduces the order-preserving keys of those (the maximum key is
// the exact min / max); lane 0 updates the body's keys atomically.
__global__ void __launch_bounds__(256) k_ls_bounds(LsArgs a) {
  const int K = ls_trials(a);
  const int w = (int)((blockIdx.x * 256 + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  __shared__ XSum acc[kLsMax];
  for (int e = threadIdx.x; e < kLsMax * (kXD + 1); e += 256) reinterpret_cast<long long*>(acc)[e] = 0;
  __syncthreads();
  if (w < a.nslice) {
    const int4 sl = a.slice[w];  // body, first vertex, vertices
    const int b = sl.x;
    double r[2][3], q[12], dq[12];
    const bool has0 = lane < sl.z, has1 = lane + 32 < sl.z;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int v = sl.y + lane + 32 * h;
      const bool has = h ? has1 : has0;
#pragma unroll
      for (int j = 0; j < 3; ++j) r[h][j] = has ? a.x0[3 * v + j] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) q[i] = a.A[9 * b + i];
#pragma unroll
    for (int i = 0; i < 3; ++i) q[9 + i] = a.p[3 * b + i];
#pragma unroll
    for (int i = 0; i < 12; ++i) dq[i] = a.dq[12 * b + i];
    for (int k = 0; k < K; ++k) {
      const double al = a.dpar[kParAlpha + k];
      double M[12];  // dofs_at with the DOFs held in registers
#pragma unroll
      for (int i = 0; i < 3; ++i) M[9 + i] = q[9 + i] - dq[i] * al;
#pragma unroll
      for (int rr = 0; rr < 3; ++rr)
#pragma unroll
        for (int i = 0; i < 3; ++i) M[3 * rr + i] = q[3 * rr + i] - dq[3 * (rr + 1) + i] * al;
      unsigned long long* kb = a.bnd + 6 * ((size_t)k * a.n + b);
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double lo = INFINITY, hi = -INFINITY;
        if (has0) {
          const double c = xform(M, r[0][0], r[0][1], r[0][2], j);
          lo = c;
          hi = c;
        }
        if (has1) {
          const double c = xform(M, r[1][0], r[1][1], r[1][2], j);
          lo = fmin(lo, c);
          hi = fmax(hi, c);
        }
        const unsigned long long mlo = seg_max_key(0xffffffffu, max_key(-lo));
        const unsigned long long mhi = seg_max_key(0xffffffffu, max_key(hi));
        if (lane == 0) {
          atomicMax(&kb[j], mlo);
          atomicMax(&kb[3 + j], mhi);
        }
      }
    }
  } else if (w - a.nslice < (a.n + 31) / 32) {
    const int t = 32 * (w - a.nslice) + lane;
    const bool body = t < a.n && !a.fixed[t];
    for (int k = 0; k < K; ++k) {
      XSum r;
      xs_zero(r);
      if (body) {
        double M[12];
        dofs_at(a.A, a.p, a.dq, t, a.dpar[kParAlpha + k], M);
        xs_add(r, inertia_energy(a.prm, a.st, a.mass, a.I0, t, M, M + 9));
      }
      xs_warp_sum(r);
      if (lane == 0) {
        long long* d = reinterpret_cast<long long*>(&acc[k]);
#pragma unroll
        for (int i = 0; i < kXD; ++i)
          if (r.d[i]) atomicAdd((unsigned long long*)&d[i], (unsigned long long)r.d[i]);
        if (r.flags) atomicOr((unsigned long long*)&d[kXD], (unsigned long long)r.flags);
      }
    }
  }
  __syncthreads();
  flush(a.energy, acc, K);
}

// FP32 body boxes of every trial from its bounds (one thread per (trial, body)); the bounds
// are cleared for the next batch
__global__ void k_ls_boxes(LsArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ls_trials(a) * a.n) return;
  unsigned long long k[12];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    k[i] = a.bnd[6 * (size_t)t + i];
    a.bnd[6 * (size_t)t + i] = 0ULL;
    k[6 + i] = 0ULL;
  }
  store_box(&a.box[t], body_box_of(k, false, 0.5 * a.prm.dhat));
}

// Trial blockIdx.y: blocks [0, G) evaluate the candidates, the others the vertex-ground
// terms.  Each thread recomputes the positions of its candidate's four vertices at the
// trial's DOFs and applies the reference's culling predicate before the barrier.
__global__ void __launch_bounds__(128) k_ls_eval(LsArgs a, int G) {
  const int k = blockIdx.y;
  if (k >= ls_trials(a)) return;
  const double al = a.dpar[kParAlpha + k];
  __shared__ XSum acc;
  if (threadIdx.x <= kXD) reinterpret_cast<long long*>(&acc)[threadIdx.x] = 0;
  __syncthreads();
  const Box* bx = a.box + (size_t)k * a.n;
  const float dhf = (float)a.prm.dhat;
  const double dhh = 0.5 * a.prm.dhat;
  if ((int)blockIdx.x < G) {
    const int cnt = min(a.dstat[DS_NECAND], a.cap_ecand);
    for (int i = blockIdx.x * 128 + threadIdx.x; i < cnt; i += G * 128) {
      const int4 c = a.ecand[i];
      const int type = c.x;
      int ids[4];
      if (type == 0) {  // point c.y, triangle c.z
        ids[0] = c.y;
        ids[1] = __ldg(&a.tris[3 * c.z]);
        ids[2] = __ldg(&a.tris[3 * c.z + 1]);
        ids[3] = __ldg(&a.tris[3 * c.z + 2]);
      } else {  // edges c.y, c.z
        ids[0] = __ldg(&a.edges[2 * c.y]);
        ids[1] = __ldg(&a.edges[2 * c.y + 1]);
        ids[2] = __ldg(&a.edges[2 * c.z]);
        ids[3] = __ldg(&a.edges[2 * c.z + 1]);
      }
      const int bA = __ldg(&a.vbody[ids[0]]), bB = __ldg(&a.vbody[ids[type == 0 ? 1 : 2]]);
      if (!overlap(load_box(&bx[bA]), load_box(&bx[bB]))) continue;
      double MA[12], MB[12];
      dofs_at(a.A, a.p, a.dq, bA, al, MA);
      dofs_at(a.A, a.p, a.dq, bB, al, MB);
      d3 xs[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double* M = (q == 0 || (type == 1 && q == 1)) ? MA : MB;
        const double r0 = __ldg(&a.x0[3 * ids[q]]), r1 = __ldg(&a.x0[3 * ids[q] + 1]), r2 = __ldg(&a.x0[3 * ids[q] + 2]);
        xs[q] = mk(xform(M, r0, r1, r2, 0), xform(M, r0, r1, r2, 1), xform(M, r0, r1, r2, 2));
      }
      const bool hit = type == 0 ? overlap(point_box_at(xs[0], dhf), tri_box_at(xs[1], xs[2], xs[3]))
                                 : overlap(edge_box_at(xs[0], xs[1], dhh), edge_box_at(xs[2], xs[3], dhh));
      if (!hit) continue;
      const double e = contact_energy(type, xs, a.prm);
      if (e != 0.0) xs_add_atomic(&acc, e);
    }
  } else {
    const int nb = (int)gridDim.x - G;
    for (int v = ((int)blockIdx.x - G) * 128 + threadIdx.x; v < a.V; v += nb * 128) {
      const int b = a.vbody[v];
      const Box bb = load_box(&bx[b]);
      if (!((double)bb.lo[1] < dhh + a.prm.ground)) continue;
      double M[12];
      dofs_at(a.A, a.p, a.dq, b, al, M);
      const double r0 = a.x0[3 * v], r1 = a.x0[3 * v + 1], r2 = a.x0[3 * v + 2];
      const d3 y = mk(xform(M, r0, r1, r2, 0), xform(M, r0, r1, r2, 1), xform(M, r0, r1, r2, 2));
      if (!vg_box_test(a.prm, bb, point_box_at(y, dhf))) continue;
      const double d = y.y - a.prm.ground;
      const double e = barrier(d * d, a.prm);
      if (e != 0.0) xs_add_atomic(&acc, e);
    }
  }
  __syncthreads();
  if (threadIdx.x <= kXD) {
    const long long v = reinterpret_cast<const long long*>(&acc)[threadIdx.x];
    long long* d = reinterpret_cast<long long*>(&a.energy[k]);
    if (v) {
      if (threadIdx.x < kXD) atomicAdd((unsigned long long*)&d[threadIdx.x], (unsigned long long)v);
      else atomicOr((unsigned long long*)&d[threadIdx.x], (unsigned long long)v);
    }
  }
}

}  // namespace

cudaError_t ls_energies(Sim& s, const abd_states& st, const double* A, const double* p) {
  LsArgs a;
  a.prm = s.prm;
  a.n = s.n;
  a.V = s.V;
  a.vbody = s.vbody;
  a.x0 = s.x0;
  a.A = A;
  a.p = p;
  a.dq = s.dq;
  a.dpar = s.dpar;
  a.st = st;
  a.mass = s.mass;
  a.I0 = s.I0;
  a.fixed = s.fixed;
  a.bnd = s.ls_bnd;
  a.box = s.ls_box;
  a.tris = s.tris;
  a.edges = s.edges;
  a.ecand = s.ecand;
  a.cap_ecand = s.cap_ecand;
  a.dstat = s.dstat;
  a.energy = s.box->ls_energy;
  a.nslice = s.nslice;
  a.slice = s.slice;
  cudaError_t e = cudaMemsetAsync(a.energy, 0, sizeof(XSum) * kLsMax, s.stream);
  if (e != cudaSuccess) return e;
  const long long warps = (long long)s.nslice + (s.n + 31) / 32;
  k_ls_bounds<<<blocks(32 * warps, 256), 256, 0, s.stream>>>(a);
  k_ls_boxes<<<blocks((long long)kLsMax * s.n, 256), 256, 0, s.stream>>>(a);
  const int G = kRedBlocks;
  const int Gv = (s.prm.ground_enabled && s.prm.enable_vg) ? kRedBlocks : 0;
  k_ls_eval<<<dim3(G + Gv, kLsMax), 128, 0, s.stream>>>(a, G);
  s.launches += 3;
  return cudaGetLastError();
}

}  // namespace abd
