// Batched line search: the energies of several trial step lengths in one pass.
//
// The backtracking line search (abd.py:146-160) evaluates E(q - alpha dq) for
// alpha = a_cap, a_cap / 2, ... until the Armijo test passes or alpha drops below alpha_min.
// In the reference every trial is an energy pass of its own (compute_energy, abd.py:133-141:
// DOF update, transform, culling, barrier sum).  Here the CCD pass of the Newton iteration
// (the CCD_LS narrow mode) also collects every PT / EE pair that can be in the culled set at
// any DOFs between q and q - dq, and a batch of trials only re-evaluates those candidates.
// For each trial alpha_k, k_ls_eval recomputes with the arithmetic of the energy pass the
// DOFs (A, p) - alpha_k dq and the positions of the vertices involved, applies the
// reference's culling predicate (culling2.py:32-79, 213-227: the two body boxes overlap and
// the two primitive boxes overlap), and adds the barrier energy of every candidate that
// passes (ipcsk/energy.py:9-48), the vertex-ground barriers (energy.py:24-33) and the
// inertia + orthogonality energy of every free body (orthogonal_energy.py:24-32) to the
// trial's exact sum, so a trial's energy is bitwise the energy pass's at the same DOFs.
//
// The body-box part of the predicate needs no body bounds in all but rare cases.  Rounding
// is monotone, so a primitive's box computed from its own vertices with the body box's
// dilation (dhat / 2, FP64, then FP32) lies inside its body's box: an EE pair whose edge
// boxes overlap has overlapping body boxes, and a PT pair passes the body test when the
// point's and the triangle's dhat / 2 boxes overlap.  Only a PT pair that fails that
// sufficient test (a tie at the rounding boundary of the dhat test) computes the two body
// boxes exactly, from all their vertices; the vertex-ground terms do the same for the body
// box's lower face.  The host takes the first trial that the sequential search would accept.
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
  double* dpar;                 // [kParK] trial count, [kParAlpha + k] step lengths
  const unsigned long long* toi_key;  // the CCD pass's minimum time of impact: the trials are
                                      // derived from it (and written to dpar), or null: given
  double alpha_min;
  abd_states st;
  const double *mass, *I0;
  const int* fixed;
  const int* voff;              // [n + 1] first vertex of each body
  const int *tris, *edges;
  const int4* ecand;            // candidates of the last CCD_LS pass
  int cap_ecand;
  const int* dstat;
  XSum* energy;                 // [kLsMax] exact energies of the trials
  const FricRec* fric;          // the step's lagged friction contacts (null: friction off)
  int cap_fric;
};

// The trials of a batch from the CCD pass's minimum time of impact (its complemented bits,
// 0: none below 1): the step bound alpha = clamp(toi, 0, 1), times 0.9 below 1 (ccd,
// abd.py:278-303), then alpha, alpha / 2, ... up to the first below alpha_min, at most kLsMax
// -- the host's trial_steps.  Returns the step length of trial k (< *K) and the count *K.
__device__ inline double trial_from_toi(unsigned long long key, double alpha_min, int k, int* K) {
  double toi = 1.0;
  if (key) toi = __longlong_as_double((long long)~key);
  const double lo = toi < 1.0 ? toi : 1.0;  // std::min(1.0, toi), std::max(0.0, .)
  double t = 0.0 < lo ? lo : 0.0;
  if (t < 1.0) t *= 0.9;
  double al = t;
  int n = 1;
  for (double s = t; n < kLsMax && !(s < alpha_min); ++n) {
    s *= 0.5;
    if (n == k) al = s;
  }
  *K = n;
  return al;
}

// The exact FP32 box of body b at (A, p) - al dq (culling2.py:278-334): FP64 min / max of
// its vertices, dilated by dhat / 2 in FP64, rounded to FP32 (one thread, rare case)
__device__ Box body_box_exact(const LsArgs& a, int b, double al) {
  double M[12];
  dofs_at(a.A, a.p, a.dq, b, al, M);
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int v = a.voff[b]; v < a.voff[b + 1]; ++v) {
    const double r0 = a.x0[3 * v], r1 = a.x0[3 * v + 1], r2 = a.x0[3 * v + 2];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double c = xform(M, r0, r1, r2, j);
      lo[j] = fmin(lo[j], c);
      hi[j] = fmax(hi[j], c);
    }
  }
  Box B;
  B.pad0 = B.pad1 = 0.f;
  const double dhh = 0.5 * a.prm.dhat;
  const bool any = a.voff[b + 1] > a.voff[b];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    B.lo[j] = any ? (float)(lo[j] - dhh) : INFINITY;
    B.hi[j] = any ? (float)(hi[j] + dhh) : -INFINITY;
  }
  return B;
}

// a triangle's FP32 box dilated like a body box (FP64 min / max -+ dhat / 2, then FP32)
__device__ inline Box tri_box_dilated(const d3& a, const d3& b, const d3& c, double dhh) {
  Box B;
  const double u[3] = {a.x, a.y, a.z}, w[3] = {b.x, b.y, b.z}, q[3] = {c.x, c.y, c.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    B.lo[k] = (float)(fmin(fmin(u[k], w[k]), q[k]) - dhh);
    B.hi[k] = (float)(fmax(fmax(u[k], w[k]), q[k]) + dhh);
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}

__device__ inline d3 position_at(const LsArgs& a, const double M[12], int v) {
  const double r0 = __ldg(&a.x0[3 * v]), r1 = __ldg(&a.x0[3 * v + 1]), r2 = __ldg(&a.x0[3 * v + 2]);
  return mk(xform(M, r0, r1, r2, 0), xform(M, r0, r1, r2, 1), xform(M, r0, r1, r2, 2));
}

// Trial blockIdx.y: blocks [0, G) evaluate the candidates, blocks [G, G + Gv) the
// vertex-ground terms, blocks [G + Gv, G + Gv + Gf) the lagged friction contacts, the rest the
// bodies' inertia + orthogonality terms.
__global__ void __launch_bounds__(128) k_ls_eval(LsArgs a, int G, int Gv, int Gf) {
  const int k = blockIdx.y;
  double al;
  if (a.toi_key) {  // every CTA derives its trial; CTA (0, 0) writes the batch out for the accept
    const unsigned long long key = *a.toi_key;
    int K;
    al = trial_from_toi(key, a.alpha_min, k, &K);
    if (blockIdx.x == 0 && k == 0 && (int)threadIdx.x <= K) {
      const double aj = trial_from_toi(key, a.alpha_min, (int)threadIdx.x - 1, &K);
      if (threadIdx.x == 0) a.dpar[kParK] = K;
      else a.dpar[kParAlpha + threadIdx.x - 1] = aj;
    }
    if (k >= K) return;
  } else {
    if (k >= (int)a.dpar[kParK]) return;
    al = a.dpar[kParAlpha + k];
  }
  __shared__ XSum acc;
  if (threadIdx.x <= kXD) reinterpret_cast<long long*>(&acc)[threadIdx.x] = 0;
  __syncthreads();
  const float dhf = (float)a.prm.dhat;
  const double dhh = 0.5 * a.prm.dhat;
  const int bx = (int)blockIdx.x;
  if (bx < G) {
    const int cnt = min(a.dstat[DS_NECAND], a.cap_ecand);
    for (int i = bx * 128 + threadIdx.x; i < cnt; i += G * 128) {
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
      double MA[12], MB[12];
      dofs_at(a.A, a.p, a.dq, bA, al, MA);
      dofs_at(a.A, a.p, a.dq, bB, al, MB);
      d3 xs[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) xs[q] = position_at(a, (q == 0 || (type == 1 && q == 1)) ? MA : MB, ids[q]);
      if (type == 0) {
        if (!overlap(point_box_at(xs[0], dhf), tri_box_at(xs[1], xs[2], xs[3]))) continue;
        // body boxes: the sufficient test, else the exact boxes
        if (!overlap(edge_box_at(xs[0], xs[0], dhh), tri_box_dilated(xs[1], xs[2], xs[3], dhh)) &&
            !overlap(body_box_exact(a, bA, al), body_box_exact(a, bB, al)))
          continue;
      } else if (!overlap(edge_box_at(xs[0], xs[1], dhh), edge_box_at(xs[2], xs[3], dhh))) {
        continue;  // (the edge boxes lie inside their body boxes)
      }
      double e;
      if (a.prm.ipc_full) {  // the full model; its mollifier's scale from the rest positions
        double r[12];
#pragma unroll
        for (int k = 0; k < 12; ++k) r[k] = __ldg(&a.x0[3 * ids[k / 3] + k % 3]);
        e = full_contact_energy(type, xs, r, a.prm);
      } else {
        e = contact_energy(type, xs, a.prm);
      }
      if (e != 0.0) xs_add_atomic(&acc, e);
    }
  } else if (bx < G + Gv) {
    for (int v = (bx - G) * 128 + threadIdx.x; v < a.V; v += Gv * 128) {
      const int b = a.vbody[v];
      double M[12];
      dofs_at(a.A, a.p, a.dq, b, al, M);
      const d3 y = position_at(a, M, v);
      if (!overlap(point_box_at(y, dhf), ground_box(a.prm))) continue;
      // the body box reaches below ground + dhat / 2: the vertex's own dhat / 2 box lies
      // inside it, so its lower face suffices; else the exact body box decides
      if (!((double)edge_box_at(y, y, dhh).lo[1] < dhh + a.prm.ground) &&
          !((double)body_box_exact(a, b, al).lo[1] < dhh + a.prm.ground))
        continue;
      const double d = y.y - a.prm.ground;
      const double e = barrier(d * d, a.prm);
      if (e != 0.0) xs_add_atomic(&acc, e);
    }
  } else if (bx < G + Gv + Gf) {  // friction potentials at the trial's positions
    const int nf = min(a.dstat[DS_NFRIC], a.cap_fric);
    const double mu = a.prm.friction_mu, eps = a.prm.friction_epsv * a.prm.dt;
    for (int i = (bx - G - Gv) * 128 + threadIdx.x; i < nf; i += Gf * 128) {
      const FricRec& f = a.fric[i];
      double x12[12];
      for (int q = 0; q < 4; ++q) {
        double M[12];
        dofs_at(a.A, a.p, a.dq, __ldg(&a.vbody[f.ids[q]]), al, M);
        const d3 y = position_at(a, M, f.ids[q]);
        x12[3 * q] = y.x, x12[3 * q + 1] = y.y, x12[3 * q + 2] = y.z;
      }
      const double e = ipc::friction_d(lag_of(f), x12, f.xt, mu, eps);
      if (e != 0.0) xs_add_atomic(&acc, e);
    }
  } else {
    const int lane = threadIdx.x & 31;
    const int t = (bx - G - Gv - Gf) * 128 + threadIdx.x;
    XSum r;
    xs_zero(r);
    if (t < a.n && !a.fixed[t]) {
      double M[12];
      dofs_at(a.A, a.p, a.dq, t, al, M);
      xs_add(r, inertia_energy(a.prm, a.st, a.mass, a.I0, t, M, M + 9));
    }
    xs_warp_sum(r);
    if (lane == 0) {
      long long* d = reinterpret_cast<long long*>(&acc);
#pragma unroll
      for (int i = 0; i < kXD; ++i)
        if (r.d[i]) atomicAdd((unsigned long long*)&d[i], (unsigned long long)r.d[i]);
      if (r.flags) atomicOr((unsigned long long*)&d[kXD], (unsigned long long)r.flags);
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

cudaError_t ls_energies(Sim& s, const abd_states& st, const double* A, const double* p, bool from_ccd) {
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
  a.voff = s.voff;
  a.tris = s.tris;
  a.edges = s.edges;
  a.ecand = s.ecand;
  a.cap_ecand = s.cap_ecand;
  a.dstat = s.dstat;
  a.energy = s.box->ls_energy;
  a.toi_key = from_ccd ? s.dmin : nullptr;
  a.alpha_min = s.prm.alpha_min;
  if (!from_ccd) {  // (the CCD_LS pass clears them otherwise)
    const cudaError_t e = cudaMemsetAsync(a.energy, 0, sizeof(XSum) * kLsMax, s.stream);
    if (e != cudaSuccess) return e;
  }
  a.fric = s.prm.friction_mu > 0.0 ? s.fric : nullptr;
  a.cap_fric = s.cap_fric;
  const int G = kRedBlocks;
  const int Gv = (s.prm.ground_enabled && s.prm.enable_vg) ? kRedBlocks : 0;
  const int Gf = a.fric ? 148 : 0;
  const int Gi = (int)blocks(s.n, 128);
  k_ls_eval<<<dim3(G + Gv + Gf + Gi, kLsMax), 128, 0, s.stream>>>(a, G, Gv, Gf);
  s.launches += 1;
  return cudaGetLastError();
}

}  // namespace abd
