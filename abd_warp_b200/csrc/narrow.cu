// Narrow phase and per-body terms.
//
// One CTA per body pair {I, J} (I < J) walks the LBVH subtrees of the other body for
//   PT: every point of I against J's triangles, every point of J against I's triangles,
//   EE: every edge of I against J's edges,
// which is the reference's intended per-body-pair culling (cull_ / intersection_prims,
// abd/culling.py:32-52, 85-99) with the same float32 box predicate.  The pass mode decides
// what is done with each candidate:
//   LISTS / GH: candidates are written as contiguous, deterministically ordered per-pair
//       segments of the PT and EE lists (vec5i rows, as the reference's lists); GH then
//       evaluates the contacts of the segment (pt_ipc.py:111-190, ee_ipc.py:381-430) and
//       reduces them, in candidate order, into the pair's off-diagonal 12x12 block and its
//       contributions to the two diagonal blocks and gradients (put.py:25-66).  The
//       reduction replaces the reference's float atomics with a fixed-order sum, so the
//       assembled system is bitwise reproducible.
//   ENERGY: sum of barrier energies of the candidates (ipcsk/energy.py:9-48).
//   CCD: minimum time of impact over the candidates (ccd.py:20-40, 133-186).
// Per-body CTAs add inertia / orthogonality (orthogonal_energy.py:24-135) and the
// vertex-ground terms (vg_ipc.py:4-34, culling.py:54-82, ccd.py:9-18, energy.py:24-33).
#include <cuda_runtime.h>

#include <climits>

#include <cooperative_groups.h>

#include "abd_body.cuh"
#include "abd_graph.cuh"
#include "abd_geometry.cuh"
#include "abd_ipc_full.cuh"

namespace abd {

namespace {

constexpr int NT = 128;          // threads per pair CTA
constexpr int NW = NT / 32;
constexpr int NOUT = 456;        // 144 off-diagonal + 2 x 144 diagonal + 2 x 12 gradient

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

struct NarrowArgs {
  int mode;
  abd_params prm;
  int n, cap_adj;
  const int2* ij;
  const int *row_ptr, *adj_col, *row_cnt;
  const uint32_t* pair_mask;
  const int* pair_wpre;
  const int* nbr;
  const float* fdof;
  const Box* chunk_box;
  const int* vperm;
  int W;
  const Box* body_box;
  const int2* chunk;
  const int* adj_pair;
  int cap_ccd;
  int4* ccd_cand;
  int nch;
  int* chunk_act;               // [nch + 1] the chunks of a pass with work (k_chunk_active), then their count
  int gh_energy;                // GH: also sum the candidates' barrier energies into energy
  const int* energy_gate;       // GH in the device loop: the energy only while this counter is 0
  unsigned long long* gtime;    // CCD_LS: first start / last end of the launch (global timer)
  const int* sup_valid;         // GH: take the candidates from ecand instead of the traversal
  int cap_act;
  int4* act_pairs;              // GH: active pairs with their coupling weights (preconditioner)
  FricRec* fric;                // lagged friction contacts (null: friction off)
  int cap_fric;
  uint32_t* fric_mask;          // their body pairs, as bits of the overlap matrix
  int fric_lag;                 // GH: this pass fixes the step's friction contacts (gated by
                                // energy_gate in the device loop: its first iteration)
  const Box* body_sup;          // CCD_LS: body boxes over every DOF set between the two
  const int* vbody;
  int cap_ecand;
  int4* ecand;                  // CCD_LS: line-search candidates
  int cap_contacts;
  int4 *contacts, *contacts_by_pair;
  XSum* energy;                  // exact energy of the pass
  XSum* ls_energy;               // CCD_LS: the energies of the line-search batch that follows
  int prof;                     // kernel profiling: count the data read into prof rows
  unsigned long long* prof_rows;
  unsigned long long* toi_key;        // complemented bits of the minimum time of impact
  abd_states st;
  const double *mass, *I0;
  const int* fixed;
  const int *voff, *toff, *eoff, *tris, *edges;
  const double *y0, *y1, *x0;
  const double *A, *p, *A1, *p1;  // DOFs of y0 / y1 (affine node boxes), or null
  int affine;
  Tree tri, edge;
  int *pt_list, *ee_list;
  int cap_pt, cap_ee;
  int* pair_cand;
  int* dstat;
  double *offdiag, *pdiag, *pgrad, *pair_val;
  int* pair_active;
};

constexpr int kFricContact = 8;  // contact record y of a lagged friction contact (k_fric_pairs)

// start bringing the line at p into L2
__device__ inline void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Per-CTA view of one body's subtree boxes.  Refit mode (m0 == null): the stored boxes.
// Affine mode: internal nodes are the affine images of their rest boxes under the body's
// DOFs at y0 (m0) and, when swept, y1 (m1); leaves are computed from the positions, or, with
// sup, are the affine images of their rest boxes too (boxes that hold the leaf's box at every
// DOF set between m0 and m1).
struct NodeBoxes {
  const Tree* tr;
  const float *m0, *m1;
  float pad;
  const int* prims;   // tris or edges
  int tri;            // 1: triangle tree, 0: edge tree
  int sup;
  const double *y0, *y1;
  double dhh;
  __device__ inline Box internal(int node) const {
    if (!m0) return load_box(&tr->box[node]);
    return affine_box2(load_box(&tr->rest[node]), m0, m1, pad);
  }
  __device__ inline Box leaf(int node, int prim) const {
    if (!m0) return load_box(&tr->box[node]);
    if (sup) return affine_box2(load_box(&tr->rest[node]), m0, m1, pad);
    return tri ? tri_leaf_box(prims, y0, y1, prim) : edge_leaf_box(prims, y0, y1, prim, dhh);
  }
};

// Stack traversal of the subtree rooted at `root`; calls f(prim) for every leaf whose box
// overlaps q, in a fixed depth-first order.  A popped node's child table lists its up to four
// descendants one or two levels down, tested together: the walk is half as deep as the
// binary tree's, and in affine mode a visit costs one round of independent loads (codes and
// rest boxes, indexed by the node itself); refit mode reads the stored world boxes.
// visits: tested internal nodes and leaves (kernel profiling)
struct Visits {
  unsigned internal = 0, leaf = 0;
};

// One visit: the child table of `node` (codes and rest boxes, indexed by the node itself);
// every leaf child whose box overlaps q goes to f(prim), every internal one to push(node).
template <class F, class P>
__device__ inline void expand_node(const NodeBoxes& nb, int node, const Box& q, F&& f, P&& push, Visits& cnt) {
  const Tree& tr = *nb.tr;
  const int L0 = tr.N - 1;
  const int4 cc = __ldg(&tr.ccode[node]);
  Box R[4];
  if (nb.m0) {
#pragma unroll
    for (int h = 0; h < 4; ++h) R[h] = load_box(&tr.crest[4 * node + h]);
  }
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const int code = h == 0 ? cc.x : h == 1 ? cc.y : h == 2 ? cc.z : cc.w;
    if (code == kNoChild) continue;
    if (code < 0) {
      const int prim = ~code;
      ++cnt.leaf;
      Box B;
      if (!nb.m0) B = load_box(&tr.box[L0 + __ldg(&tr.prim_leaf[prim])]);
      else if (nb.sup) B = affine_box2(R[h], nb.m0, nb.m1, nb.pad);
      else B = nb.tri ? tri_leaf_box(nb.prims, nb.y0, nb.y1, prim) : edge_leaf_box(nb.prims, nb.y0, nb.y1, prim, nb.dhh);
      if (overlap(B, q)) f(prim);
    } else {
      ++cnt.internal;
      const Box B = nb.m0 ? affine_box2(R[h], nb.m0, nb.m1, nb.pad) : load_box(&tr.box[code]);
      if (overlap(B, q)) push(code);
    }
  }
}

// every pushed node is visited later: start bringing its child table to L2 now
__device__ inline void prefetch_node(const Tree& tr, int node) {
  prefetch_l2(&tr.ccode[node]);
  prefetch_l2(&tr.crest[4 * node]);
}

template <class F>
__device__ inline void traverse(const NodeBoxes& nb, int root, const Box& q, int* dstat, F&& f) {
  Visits v;
  traverse(nb, root, q, dstat, f, v);
}

template <class F>
__device__ inline void traverse(const NodeBoxes& nb, int root, const Box& q, int* dstat, F&& f, Visits& cnt) {
  if (root < 0) return;
  const Tree& tr = *nb.tr;
  const int L0 = tr.N - 1;
  if (root >= L0) {
    const int prim = __ldg(&tr.leaf_prim[root - L0]);
    ++cnt.leaf;
    if (overlap(nb.leaf(root, prim), q)) f(prim);
    return;
  }
  ++cnt.internal;
  if (!overlap(nb.internal(root), q)) return;
  int stack[kTraversalStack];
  int sp = 0;
  stack[sp++] = root;
  while (sp > 0) {
    const int node = stack[--sp];
    expand_node(nb, node, q, f, [&](int c) {
      if (sp < kTraversalStack) {
        stack[sp++] = c;
        if (nb.m0) prefetch_node(tr, c);
      } else {
        atomicOr(&dstat[DS_STATUS], ST_STACK_OVERFLOW);
      }
    }, cnt);
  }
}

struct PairInfo {
  int I, J, nPT1, nPT2, nEE;
  const float* dof;  // shared [2 bodies][2 times][12] FP32 DOFs (I, J), or null
};

__device__ inline PairInfo pair_info(const NarrowArgs& a, int p) {
  PairInfo P;
  const int2 ij = a.ij[p];
  P.I = ij.x;
  P.J = ij.y;
  P.nPT1 = a.prm.enable_pt ? a.voff[P.I + 1] - a.voff[P.I] : 0;
  P.nPT2 = a.prm.enable_pt ? a.voff[P.J + 1] - a.voff[P.J] : 0;
  P.nEE = a.prm.enable_ee ? a.eoff[P.I + 1] - a.eoff[P.I] : 0;
  P.dof = nullptr;
  return P;
}

// tree boxes of one body: m = its FP32 DOFs [y0: 12][y1: 12] in shared memory, or null
__device__ inline NodeBoxes node_boxes(const NarrowArgs& a, const Tree* tr, bool tri, const float* m) {
  NodeBoxes nb;
  nb.tr = tr;
  nb.m0 = m;
  nb.m1 = m && a.y1 ? m + 12 : nullptr;
  nb.pad = tri ? 0.f : __double2float_ru(0.5 * a.prm.dhat);  // triangle boxes are undilated
  nb.prims = tri ? a.tris : a.edges;
  nb.tri = tri;
  nb.sup = 0;
  nb.y0 = a.y0;
  nb.y1 = a.y1;
  nb.dhh = 0.5 * a.prm.dhat;
  return nb;
}

// Visit every candidate of item k: f(type, pointOrEdgeBody, primA_global, primB_global)
template <class F>
__device__ inline void visit_item(const NarrowArgs& a, const PairInfo& P, int k, F&& f) {
  const float dhf = (float)a.prm.dhat;
  if (k < P.nPT1 + P.nPT2) {
    const bool first = k < P.nPT1;
    const int body = first ? P.I : P.J, other = first ? P.J : P.I;
    const int v = a.voff[body] + (first ? k : k - P.nPT1);
    const Box q = point_box(a.y0, a.y1, v, dhf);
    traverse(node_boxes(a, &a.tri, true, P.dof ? P.dof + 24 * (first ? 1 : 0) : nullptr),
             __ldg(&a.tri.body_root[other]), q, a.dstat, [&](int t) { f(0, first ? 0 : 1, v, t); });
  } else {
    const int e = a.eoff[P.I] + (k - P.nPT1 - P.nPT2);
    const Box q = P.dof ? edge_leaf_box(a.edges, a.y0, a.y1, e, 0.5 * a.prm.dhat)
                        : load_box(&a.edge.box[(a.edge.N - 1) + __ldg(&a.edge.prim_leaf[e])]);
    traverse(node_boxes(a, &a.edge, false, P.dof ? P.dof + 24 : nullptr), __ldg(&a.edge.body_root[P.J]), q,
             a.dstat, [&](int eb) { f(1, 0, e, eb); });
  }
}

// A slot of an append-only list: one atomic per group of lanes that append together.
__device__ inline int append_slot(int* counter) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
  return g.shfl(base, 0) + (int)g.thread_rank();
}

// global vertex ids of a candidate: PT (point v, triangle t), EE (edge a, edge b)
__device__ inline void cand_vertices(const NarrowArgs& a, int type, int pa, int pb, int ids[4]) {
  if (type == 0) {
    ids[0] = pa;
    ids[1] = __ldg(&a.tris[3 * pb]);
    ids[2] = __ldg(&a.tris[3 * pb + 1]);
    ids[3] = __ldg(&a.tris[3 * pb + 2]);
  } else {
    ids[0] = __ldg(&a.edges[2 * pa]);
    ids[1] = __ldg(&a.edges[2 * pa + 1]);
    ids[2] = __ldg(&a.edges[2 * pb]);
    ids[3] = __ldg(&a.edges[2 * pb + 1]);
  }
}

__device__ inline void fetch(const double* y, const int ids[4], d3 xs[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) xs[k] = mk(__ldg(&y[3 * ids[k]]), __ldg(&y[3 * ids[k] + 1]), __ldg(&y[3 * ids[k] + 2]));
}

// block-wide exclusive scan of one int per thread; returns the total
__device__ inline int block_scan(int v, int* sh, int& excl) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int w = 0; w < NW; ++w) {
      const int c = sh[w];
      sh[w] = acc;
      acc += c;
    }
    sh[NW] = acc;
  }
  __syncthreads();
  excl = sh[warp] + x - v;
  const int total = sh[NW];
  __syncthreads();
  return total;
}

// Candidate lists (the reference's vec5i PT / EE lists, culling.py:85-99): one CTA per body
// pair (grid = pair capacity), each pair a contiguous segment in traversal order.
__global__ void __launch_bounds__(NT) k_pair_lists(NarrowArgs a) {
  const int p = blockIdx.x;
  // pair count of this pass (device); an overflowed pass is rerun by the host
  if (p >= a.dstat[DS_NPAIRS] || (a.dstat[DS_STATUS] & ST_PAIR_OVERFLOW)) return;
  PairInfo P = pair_info(a, p);
  const int items = P.nPT1 + P.nPT2 + P.nEE;
  const int tid = threadIdx.x;
  __shared__ int sh[NW + 1];
  __shared__ float sdof[2][2][12];  // [I, J][y0, y1][A row-major, p]
  if (a.affine) {
    if (tid < 48) {
      const int side = tid / 24, t = (tid / 12) & 1, c = tid % 12;
      const int b = side ? P.J : P.I;
      const double* A = t ? a.A1 : a.A;
      const double* q = t ? a.p1 : a.p;
      if (!t || a.y1) sdof[side][t][c] = (float)(c < 9 ? A[9 * b + c] : q[3 * b + c - 9]);
    }
    __syncthreads();
    P.dof = &sdof[0][0][0];
  }

  // ---- LISTS / GH: two passes over the candidates (count, then write in order) ----
  int cpt = 0, cee = 0;
  for (int k = tid; k < items; k += NT)
    visit_item(a, P, k, [&](int type, int, int, int) {
      if (type == 0) ++cpt;
      else ++cee;
    });
  int opt, oee;
  const int tpt = block_scan(cpt, sh, opt);
  const int tee = block_scan(cee, sh, oee);
  __shared__ int base_pt, base_ee, ok;
  if (tid == 0) {
    base_pt = atomicAdd(&a.dstat[DS_PT_COUNT], tpt);
    base_ee = atomicAdd(&a.dstat[DS_EE_COUNT], tee);
    ok = 1;
    if (base_pt + tpt > a.cap_pt) {
      atomicOr(&a.dstat[DS_STATUS], ST_PT_OVERFLOW);
      ok = 0;
    }
    if (base_ee + tee > a.cap_ee) {
      atomicOr(&a.dstat[DS_STATUS], ST_EE_OVERFLOW);
      ok = 0;
    }
    a.pair_cand[4 * p + 0] = base_pt;
    a.pair_cand[4 * p + 1] = tpt;
    a.pair_cand[4 * p + 2] = base_ee;
    a.pair_cand[4 * p + 3] = tee;
  }
  __syncthreads();
  if (!ok) {
    return;
  }
  {
    int wpt = base_pt + opt, wee = base_ee + oee;
    for (int k = tid; k < items; k += NT)
      visit_item(a, P, k, [&](int type, int swap, int pa, int pb) {
        // (I, J, pair, local prim of I, local prim of J) with I the point's / first edge's body
        int* row = type == 0 ? &a.pt_list[5 * (size_t)wpt++] : &a.ee_list[5 * (size_t)wee++];
        const int bI = swap ? P.J : P.I, bJ = swap ? P.I : P.J;
        row[0] = bI;
        row[1] = bJ;
        row[2] = p;
        row[3] = type == 0 ? pa - a.voff[bI] : pa - a.eoff[bI];
        row[4] = type == 0 ? pb - a.toff[bJ] : pb - a.eoff[bJ];
      });
  }
}

// ---------------------------------------------------------------------------------------
// GH assembly: the active contacts found by the chunk pass, grouped by body pair
// ---------------------------------------------------------------------------------------
// contacts into their pair's segment, thread k taking contacts k, k + stride, ... (the order
// inside a segment does not matter: the assembly sums exactly)
__device__ inline void scatter_contacts(int k, int stride, int cap_contacts, const int4* __restrict__ in,
                                        int* pair_cand, int4* out, const int* dstat) {
  for (const int m = min(dstat[DS_NCONTACT], cap_contacts); k < m; k += stride) {
    const int4 c = in[k];
    out[pair_cand[4 * c.x] + atomicAdd(&pair_cand[4 * c.x + 2], 1)] = c;
  }
}

// Lists of at most this many contacts are scattered by the scan's CTA itself
constexpr int kScanScatter = 16384;

// single CTA: per-pair offsets of the contact lists (pair_cand[4p] = offset, [4p+1] = count,
// [4p+2] = fill cursor); with `in` (a list of at most kScanScatter), then the contacts into
// their segments.  Skipped when the pass overflowed (the host reruns it).
__global__ void __launch_bounds__(1024) k_contact_scan(int cap_pairs, int* pair_cand, int* dstat, int cap_contacts,
                                                       const int4* __restrict__ in, int4* out) {
  if (dstat[DS_STATUS] & (ST_PAIR_OVERFLOW | ST_CONTACT_OVERFLOW)) return;
  const int np = min(dstat[DS_NPAIRS], cap_pairs);
  __shared__ int sh[33];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < np; c0 += 1024) {
    const int p = c0 + threadIdx.x;
    const int v = p < np ? pair_cand[4 * p + 1] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = carry;
      for (int w = 0; w < 32; ++w) {
        const int t = sh[w];
        sh[w] = acc;
        acc += t;
      }
      sh[32] = acc;
    }
    __syncthreads();
    if (p < np) {
      pair_cand[4 * p] = sh[warp] + x - v;
      pair_cand[4 * p + 2] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) carry = sh[32];
    __syncthreads();
  }
  // (the barrier above makes the CTA's offsets and cleared cursors visible to all its threads)
  if (in) scatter_contacts(threadIdx.x, 1024, cap_contacts, in, pair_cand, out, dstat);
}

// the contacts into their segments, one thread per contact (lists above kScanScatter)
__global__ void k_contact_scatter(int cap_contacts, const int4* __restrict__ in, int* pair_cand, int4* out,
                                  const int* dstat) {
  if (dstat[DS_STATUS] & (ST_PAIR_OVERFLOW | ST_CONTACT_OVERFLOW)) return;
  scatter_contacts(blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x, cap_contacts, in, pair_cand, out,
                   dstat);
}

// CTAs loop over the body pairs: every active contact of a pair (pt_ipc.py:111-190,
// ee_ipc.py:381-430) as 5 rank-one terms, one warp per contact; its 456 values (H_IJ, the
// contributions to H_II and H_JJ, and to g_I, g_J; put.py:25-66) are added exactly.
// EXACT (the adjoint's system): each contact's exact, unprojected Hessian instead -- the
// barrier of the point-plane (PT) or line-line (EE) squared distance, the reference's interior
// contacts, with every second-derivative term (also those of the closest-point coefficients
// that the Newton Hessian leaves out, psd/vf.py:150-176, psd/ee.py:94-116): 78 hyper-dual
// evaluations of the contact's energy per warp, one per Hessian entry, then mapped to the two
// bodies' affine DOFs.
constexpr int PT_THREADS = 256;  // threads of the pair assembly (a warp per contact)
// One contact's exact terms (EXACT pair assembly), by its warp: the local Hessian and gradient
// in the four points' coordinates into h [156], then the 456 affine values added to xred.
// Vertices 0 .. nI-1 are the first group (the point; edge a), the rest the second; the group
// of side 0 (the pair's first body) is the first unless swapped.
// full: the contact's classified feature pair and the edge-edge mollifier (the full model;
// else the reference's interior types); project: the PSD projection of the local Hessian
// (Jacobi, by the warp's first lane) before the map.
__device__ void affine_map_terms(const NarrowArgs& a, int type, int swap, const int ids[4], const double* h,
                                 XSum* xred);
__device__ void exact_contact_terms(const NarrowArgs& a, int type, int swap, const int ids[4], double* h,
                                    XSum* xred, bool full, bool project) {
  const int lane = threadIdx.x & 31;
  double x[12], rr[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    x[k] = a.y0[3 * ids[k / 3] + k % 3];
    rr[k] = __ldg(&a.x0[3 * ids[k / 3] + k % 3]);
  }
  const int ftype = full ? ipc::contact_type(type, x) : 0;
  const double ex = full && type == 1 ? ipc::ee_eps_x(rr) : 0.0;
  for (int e = lane; e < 78; e += 32) {  // the upper triangle, row by row
    int i = 0, rem = e;
    while (rem >= 12 - i) {
      rem -= 12 - i;
      ++i;
    }
    const int j = i + rem;
    ipc::V3<ipc::HD> v[4];
    for (int k = 0; k < 4; ++k) {
      ipc::HD c[3];
      for (int m = 0; m < 3; ++m) {
        const int q = 3 * k + m;
        c[m] = {x[q], q == i ? 1.0 : 0.0, q == j ? 1.0 : 0.0, 0.0};
      }
      v[k] = {c[0], c[1], c[2]};
    }
    const ipc::HD en = ipc::local_energy(type, ftype, v, ex, a.prm.d2hat, a.prm.kappa, SharedLog());
    h[12 * i + j] = en.ab;
    h[12 * j + i] = en.ab;
    if (i == j) h[144 + i] = en.a;
  }
  __syncwarp();
  if (project && lane == 0) ipc::project_psd12(h);
  __syncwarp();
  affine_map_terms(a, type, swap, ids, h, xred);
}

// A contact's local gradient and Hessian h [156] (Hessian, then gradient, in the four points'
// coordinates) as its 456 affine values, added to xred by the calling warp: vertices 0 .. nI-1
// are the first group (the point; edge a), the rest the second; the group of side 0 (the
// pair's first body) is the first unless swapped.
__device__ void affine_map_terms(const NarrowArgs& a, int type, int swap, const int ids[4], const double* h,
                                 XSum* xred) {
  const int lane = threadIdx.x & 31;
  const int nI = type == 0 ? 1 : 2;
  auto side = [&](int v) { return (v < nI ? 0 : 1) ^ swap; };
  auto wt = [&](int v, int m) { return m == 0 ? 1.0 : __ldg(&a.x0[3 * ids[v] + (m - 1)]); };
  for (int e = lane; e < NOUT; e += 32) {
    double val = 0.0;
    if (e < 432) {
      const int blk = e / 144, r = (e % 144) / 12, c = e % 12;
      const int rs = blk == 2 ? 1 : 0, cs = blk == 1 ? 0 : 1;  // H_IJ, diag I, diag J
      const int m = r / 3, ra = r % 3, n = c / 3, cb = c % 3;
      for (int u = 0; u < 4; ++u) {
        if (side(u) != rs) continue;
        for (int w = 0; w < 4; ++w)
          if (side(w) == cs) val += (wt(u, m) * h[12 * (3 * u + ra) + 3 * w + cb]) * wt(w, n);
      }
    } else {
      const int k = e - 432, sd = k / 12, m = (k % 12) / 3, comp = k % 3;
      for (int u = 0; u < 4; ++u)
        if (side(u) == sd) val += wt(u, m) * h[144 + 3 * u + comp];
    }
    xs_add_atomic(&xred[e], val);
  }
  __syncwarp();
}

constexpr int PT_WARPS = PT_THREADS / 32;
constexpr int kExactLocal = 156;  // EXACT: a warp's local Hessian (144) and gradient (12)
// the exact pair assembly's shared memory: the sums and every warp's local Hessian (49 KB: the
// kernel is opted in once, at creation, since its launches may be captured)
constexpr int kExactSmem = NOUT * (int)sizeof(XSum) + PT_WARPS * kExactLocal * (int)sizeof(double);
// MODE: kAsmRef the reference's model (5 rank-one terms); kAsmExact the adjoint's exact Hessian
// of the reference's model; kAsmFull the full IPC model, its exact local Hessian projected onto
// the PSD cone (the Newton system with ipc_full); kAsmFullExact the adjoint's exact Hessian of
// the full model
enum { kAsmRef = 0, kAsmExact = 1, kAsmFull = 2, kAsmFullExact = 3 };
template <int MODE>
__global__ void __launch_bounds__(PT_THREADS) k_pair_assemble(NarrowArgs a) {
  constexpr bool EXACT = MODE != kAsmRef;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (a.dstat[DS_STATUS] & (ST_PAIR_OVERFLOW | ST_CONTACT_OVERFLOW)) return;
  const int npairs = a.dstat[DS_NPAIRS];
  __shared__ double ush[EXACT ? 1 : PT_WARPS][5][24];
  extern __shared__ XSum xred[];  // [NOUT], then (EXACT) [PT_WARPS][kExactLocal] doubles
  double* hloc = reinterpret_cast<double*>(xred + NOUT) + warp * kExactLocal;
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {  // pairs, grid-stride
    const int cnt = a.pair_cand[4 * p + 1], off = a.pair_cand[4 * p];
    if (tid == 0) {
      a.pair_active[p] = cnt;
      if (cnt) atomicAdd(&a.dstat[DS_ACTIVE], cnt);
    }
    if (cnt == 0) continue;
    __syncthreads();  // the previous pair's results are read out of xred
    for (int e = tid; e < NOUT * (kXD + 1); e += PT_THREADS) reinterpret_cast<long long*>(xred)[e] = 0;
    __syncthreads();
    for (int ci = warp; ci < cnt; ci += PT_WARPS) {
      const int4 rec = a.contacts_by_pair[off + ci];
      if constexpr (EXACT) {
        if (rec.y == kFricContact) {  // a lagged friction contact: its potential's exact terms
          const FricRec& f = a.fric[rec.z];
          if (lane == 0) {
            double x12[12];
            for (int q = 0; q < 12; ++q) x12[q] = a.y0[3 * f.ids[q / 3] + q % 3];
            ipc::friction_gh(lag_of(f), x12, f.xt, a.prm.friction_mu, a.prm.friction_epsv * a.prm.dt, hloc + 144,
                             hloc);
          }
          __syncwarp();
          affine_map_terms(a, f.kind, f.I != a.ij[p].x ? 1 : 0, f.ids, hloc, xred);
          continue;
        }
      }
      const int type = rec.y & 1, swap = rec.y >> 1;
      int ids[4];
      cand_vertices(a, type, rec.z, rec.w, ids);
      if constexpr (EXACT) {
        exact_contact_terms(a, type, swap, ids, hloc, xred, MODE >= kAsmFull, MODE == kAsmFull);
        continue;
      }
      d3 xs[4];
      fetch(a.y0, ids, xs);
      Geo G;
      double d2;
      contact_active(type, xs, a.prm, &G, &d2);
      ContactScalars C;
      contact_scalars(type, G, d2, a.prm, C);
      if (lane < 24) {
        const int side = lane / 12, m = (lane % 12) / 3, comp = lane % 3;
        const int group = side ^ swap;  // vertex group whose body is this side
        const int v0 = type == 0 ? (group ? 1 : 0) : (group ? 2 : 0);
        const int v1 = type == 0 ? (group ? 4 : 1) : (group ? 4 : 2);
        double dw[3];
  #pragma unroll
        for (int i = 0; i < 3; ++i) {
          double sacc = 0.0;
          for (int v = v0; v < v1; ++v) {
            const double w = m == 0 ? 1.0 : __ldg(&a.x0[3 * ids[v] + (m - 1)]);
            sacc += C.D[i][v] * w;
          }
          dw[i] = sacc;
        }
  #pragma unroll
        for (int k = 0; k < 5; ++k)
          ush[warp][k][lane] = dw[0] * C.q[k][comp] + dw[1] * C.q[k][3 + comp] + dw[2] * C.q[k][6 + comp];
      }
      __syncwarp();
      for (int e = lane; e < NOUT; e += 32) {
        double v = 0.0;
        if (e < 432) {
          const int blk = e / 144, r = (e % 144) / 12, cidx = e % 12;
          const int ra = blk == 2 ? 12 + r : r;
          const int cb = blk == 1 ? cidx : 12 + cidx;
  #pragma unroll
          for (int k = 0; k < 5; ++k) v += C.coef[k] * (ush[warp][k][ra] * ush[warp][k][cb]);
        } else {
          v = C.gscale * ush[warp][4][e - 432];
        }
        xs_add_atomic(&xred[e], v);
      }
      __syncwarp();
    }
    __syncthreads();
    for (int e = tid; e < NOUT; e += PT_THREADS) {
      const double v = xs_round(xred[e]);
      if (e < 144) {
        a.offdiag[(size_t)p * 288 + e] = v;
        a.offdiag[(size_t)p * 288 + 144 + (e % 12) * 12 + e / 12] = v;
      } else if (e < 432) {
        a.pdiag[(size_t)p * 288 + (e - 144)] = v;
      } else {
        a.pgrad[(size_t)p * 24 + (e - 432)] = v;
      }
    }
    // an active pair of two free bodies joins the preconditioner's clustering with the
    // Frobenius norm of H_IJ as its weight (summed in row order, then rounded to FP32)
    __syncthreads();  // H_IJ is in global memory
    if (tid == 0) {
      const int2 ij = a.ij[p];
      if (!a.fixed[ij.x] && !a.fixed[ij.y]) {
        double f = 0.0;
        const double* O = a.offdiag + (size_t)p * 288;
        for (int k = 0; k < 144; ++k) f += O[k] * O[k];
        const float w = (float)sqrt(f);
        if (w > 0.f) {
          const int pos = atomicAdd(&a.dstat[DS_NACTP], 1);
          if (pos < a.cap_act) a.act_pairs[pos] = make_int4(p, ij.x, ij.y, __float_as_int(w));
          else atomicOr(&a.dstat[DS_STATUS], ST_ACT_OVERFLOW);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// per-body terms shared by the body kernels and the energy / CCD chunks
// ---------------------------------------------------------------------------------------
// does vertex v take part in the vertex-ground terms (culling.py:64-82)?  bb: its body box
__device__ inline bool vg_candidate_of(const abd_params& P, const Box& bb, const double* y0, const double* y1, int v) {
  return vg_box_test(P, bb, point_box(y0, y1, v, (float)P.dhat));
}

// time of impact of a vertex with the ground plane (ccd.py:9-18); 1 when none
__device__ inline double vg_toi(const abd_params& P, const double* y0, const double* y1, int v) {
  const double d1 = y1[3 * v + 1] - P.ground;
  double tt = 1.0;
  if (d1 < 0) {
    const double d0 = y0[3 * v + 1] - P.ground;
    tt = d0 / (d0 - d1);
  }
  return tt;
}

// One candidate's barrier energy at positions xs: the reference's model (ipcsk/energy.py:9-48)
// or, with ipc_full, the full model (its rest positions scale the edge-edge mollifier)
__device__ inline double candidate_energy(const NarrowArgs& a, int type, const int ids[4], const d3 xs[4]) {
  if (!a.prm.ipc_full) return contact_energy(type, xs, a.prm);
  double r[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) r[k] = __ldg(&a.x0[3 * ids[k / 3] + k % 3]);
  return full_contact_energy(type, xs, r, a.prm);
}

// minimum of non-negative doubles by atomicMax on the complemented bit patterns (0 = none)
__device__ inline void toi_min(unsigned long long* key, double t) {
  atomicMax(key, ~(unsigned long long)__double_as_longlong(t));
}

// ---------------------------------------------------------------------------------------
// energy / CCD passes: one CTA per chunk of one body's points and edges
// ---------------------------------------------------------------------------------------
constexpr int CT = 128;  // threads per chunk CTA
static_assert(kChunk <= CT && kChunk <= 256, "a chunk's queries: one thread each when loaded, 8-bit ids");
constexpr int kNoQuery = INT_MIN;  // a chunk item whose primitive kind is disabled
constexpr int NBB = 64;     // neighbours staged per batch

// The k-th neighbour (increasing order) of body I from the overlap bit matrix: the word by
// binary search over the row's prefix counts, then the bit inside it.
__device__ inline int kth_neighbour(const NarrowArgs& a, int I, int k) {
  const int* pre = a.pair_wpre + (size_t)I * a.W;
  int lo = 0, hi = a.W - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= k) lo = mid;
    else hi = mid - 1;
  }
  uint32_t m = a.pair_mask[(size_t)I * a.W + lo];
  for (int r = k - pre[lo]; r > 0; --r) m &= m - 1;
  return 32 * lo + __ffs(m) - 1;
}

// Which body of a pair {I, J} queries the other's edge tree for the EE candidates: the one
// with more edges; at equal edge counts the one with fewer neighbours (dI, dJ: the pass's row
// counts), then the higher index.  A body with many neighbours (a ground box among cubes of
// as many edges) would otherwise query every neighbour's tree from its one chunk, in series.
// The candidate set does not depend on the choice (the box predicate is symmetric).
__device__ inline bool ee_owner(int I, int nEI, int dI, int J, int nEJ, int dJ) {
  return nEI > nEJ || (nEI == nEJ && (dI < dJ || (dI == dJ && I > J)));
}

// Body I's points against the triangle trees of all its neighbours J (PT pairs (I, J); the
// pairs (J, I) come from J's chunks), and its edges against the edge trees of the neighbours
// it owns the EE candidates with -- the same candidates as the per-pair kernel, each query
// box built once.  A query is only traversed into J's tree when it overlaps J's body box,
// which contains every leaf box of J.  The overlapping (query, neighbour) combinations of a
// batch are compacted and their traversals spread over the CTA's threads.  The first chunk
// of every body also adds the body's own terms: inertia + orthogonality and the
// vertex-ground barriers (ENERGY) or the vertex-ground times of impact (CCD).
// ENERGY adds every nonzero term to one exact accumulator of the whole pass (any order gives
// the same sum); CCD takes the minimum time of impact by an atomic maximum on complemented
// bits.  (ipcsk/energy.py:9-48, orthogonal_energy.py:24-32, ccd.py:9-40, 133-186)
// CCD_LS is the CCD pass of the step: it culls with boxes that hold every box of the
// primitives at all DOF sets between the pass's two (body_sup, the affine images of the
// queries' and leaves' rest boxes) and appends every pair found to the line-search
// candidates; the pairs that also pass the CCD pass's own boxes (body pair, query and leaf)
// become CCD candidates, the same set as the CCD pass finds.
// The world box of chunk c of body I: the affine image of its rest box at the pass's DOFs
// (with y1: the union over both DOF sets), dilated by dhat.  Every query box of the chunk lies
// inside.
__device__ inline Box chunk_world_box(const NarrowArgs& a, int c, int I) {
  const Box R = load_box(&a.chunk_box[c]);
  const float pad = __double2float_ru(a.prm.dhat);
  Box b = affine_box(R, a.fdof + 24 * (size_t)I, pad);
  if (a.y1) {
    const Box B1 = affine_box(R, a.fdof + 24 * (size_t)I + 12, pad);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      b.lo[k] = fminf(b.lo[k], B1.lo[k]);
      b.hi[k] = fmaxf(b.hi[k], B1.hi[k]);
    }
  }
  return b;
}

// The chunks of a pass with work, one warp per chunk: those whose world box overlaps the body
// box of a neighbour (CCD_LS: the box over the DOF range), and a body's first chunk when the
// pass adds the body's own terms there (ENERGY; CCD with vertex-ground contacts).  They are
// appended to chunk_act, whose entry nch counts them; k_chunk_narrow's first CTAs take them.
// In a resting pile most chunks face no neighbour, and finding that out costs a chunk CTA a
// chain of dependent loads; here it costs a warp.  (The tests are k_chunk_narrow's own: a
// chunk that is left out would have found no neighbour there.)
constexpr int KA = 256;  // threads of the chunk filter
template <int MODE>
__global__ void __launch_bounds__(KA) k_chunk_active(NarrowArgs a) {
  constexpr bool ls = MODE == NARROW_CCD_LS;
  constexpr bool ccd = MODE == NARROW_CCD || ls, gh = MODE == NARROW_GH;
  if constexpr (gh) {
    if (*a.sup_valid) return;
  }
  if (ls && a.gtime && threadIdx.x == 0) atomicMin(&a.gtime[0], globaltimer_ns());
  const int lane = (int)(threadIdx.x & 31);
  const int c = (int)((blockIdx.x * KA + threadIdx.x) >> 5);
  if (c >= a.nch) return;
  const int2 ch = a.chunk[c];
  const int I = ch.x;
  const int nEI = a.eoff[I + 1] - a.eoff[I];
  const int nV = a.voff[I + 1] - a.voff[I];
  const int Q = max(0, min(kChunk, nV + nEI - ch.y));
  bool need = !gh && ch.y == 0 && (!ccd || (a.prm.ground_enabled && a.prm.enable_vg));
  int r0 = 0, deg;
  if constexpr (gh) {
    r0 = a.row_ptr[I];
    deg = (a.dstat[DS_STATUS] & ST_PAIR_OVERFLOW) ? 0 : min(a.row_ptr[I + 1], a.cap_adj) - r0;
  } else {
    deg = a.row_cnt[I];
  }
  if (Q == 0) deg = 0;
  if (ls && a.prof && lane == 0 && deg > 0)
    atomicAdd(&a.prof_rows[8 * (c & 31) + PF_NEIGHBOUR], (unsigned long long)deg);
  if (!need && deg > 0) {
    const Box cbx = chunk_world_box(a, c, I);
    for (int k0 = 0; k0 < deg && !need; k0 += 32) {
      const int k = k0 + lane;
      bool rel = false;
      if (k < deg) {
        const int J = gh ? a.adj_col[r0 + k] : (k < kNbList ? a.nbr[(size_t)I * kNbList + k] : kth_neighbour(a, I, k));
        rel = overlap(cbx, load_box(&(ls ? a.body_sup : a.body_box)[J]));
      }
      need = __any_sync(0xffffffffu, rel);
    }
  }
  if (need && lane == 0) a.chunk_act[atomicAdd(&a.chunk_act[a.nch], 1)] = c;
}

constexpr int CW = 4 * CT;  // (query, neighbour) combinations tested per round
constexpr int kFront = 512;  // entries of a breadth-first frontier
constexpr int kCandBuf = 256;  // candidates a chunk CTA gathers before it writes them out
template <int MODE>
__global__ void __launch_bounds__(CT, 5) k_chunk_narrow(NarrowArgs a) {
  constexpr bool ls = MODE == NARROW_CCD_LS;
  constexpr bool ccd = MODE == NARROW_CCD || ls, gh = MODE == NARROW_GH;
  if constexpr (gh) {
    if (*a.sup_valid) return;  // k_gh_scan takes the candidates from ecand
  }
  const int tid = threadIdx.x;
  if ((int)blockIdx.x >= a.chunk_act[a.nch]) {  // more CTAs than chunks with work
    if (ls && a.gtime && tid == 0) atomicMax(&a.gtime[1], globaltimer_ns());
    return;
  }
  const int c = a.chunk_act[blockIdx.x];
  const int2 ch = a.chunk[c];
  const int I = ch.x;
  const int nEI = a.eoff[I + 1] - a.eoff[I];
  const int nV = a.voff[I + 1] - a.voff[I];  // items: the body's points, then its edges
  const int Q = max(0, min(kChunk, nV + nEI - ch.y));
  __shared__ Box qbox[kChunk];  // query boxes (CCD_LS: over the DOF range)
  __shared__ int qprim[kChunk];  // point id, ~edge id, or kNoQuery (primitive kind disabled)
  __shared__ Box nbox[NBB];
  __shared__ __align__(16) float ndof[NBB][24];
  __shared__ int nJ[NBB], ntri[NBB], nedge[NBB], nown[NBB], npair[NBB], nrel[NBB];
  __shared__ unsigned short work[CW];
  __shared__ int nwork;
  __shared__ int2 front[2][kFront];  // breadth-first frontiers: (query | neighbour << 8, node)
  __shared__ int nfr[2];
  int fcur = 0;
  // frontier entries in use: all of them, or fewer when a test injects a small capacity
  const int fcap = a.prm.min_capacity > 0 ? min(kFront, a.prm.min_capacity) : kFront;
  __shared__ XSum xe;
  __shared__ unsigned long long tkey;
  __shared__ Box cbx;  // the chunk's world box: every query box of the chunk lies inside
  if (tid == 0 && Q > 0) cbx = chunk_world_box(a, c, I);
  // The candidates (GH, CCD, CCD_LS) gather in shared memory and go to their list in blocks,
  // one global atomic per block: a hit does not wait on the list's counter, which every CTA
  // of the launch shares.  A full buffer sends the rest straight to the list.
  constexpr bool lists = gh || ccd;
  __shared__ int4 cbuf[kCandBuf];
  __shared__ int ncb, cbase;
  int* const ccount = &a.dstat[ls ? DS_NECAND : DS_NCCD];
  int4* const cdst = ls ? a.ecand : a.ccd_cand;
  const int ccap = ls ? a.cap_ecand : a.cap_ccd;
  const int cflag = ls ? ST_ECAND_OVERFLOW : ST_CCD_OVERFLOW;
  auto emit = [&](int4 rec) {
    const int k = atomicAdd(&ncb, 1);
    if (k < kCandBuf) {
      cbuf[k] = rec;
    } else {
      const int pos = append_slot(ccount);
      if (pos < ccap) cdst[pos] = rec;
      else atomicOr(&a.dstat[DS_STATUS], cflag);
    }
  };
  // the buffer to the list: every thread, after a barrier that follows the emits
  auto flush = [&]() {
    const int n = min(ncb, kCandBuf);
    if (n == 0) return;
    if (tid == 0) cbase = atomicAdd(ccount, n);
    __syncthreads();
    for (int e = tid; e < n; e += CT) {
      if (cbase + e < ccap) cdst[cbase + e] = cbuf[e];
      else atomicOr(&a.dstat[DS_STATUS], cflag);
    }
    __syncthreads();
    if (tid == 0) ncb = 0;  // the next barrier orders it before the next emit
  };
  if (tid == 0) ncb = 0;
  if (tid == 0) nfr[0] = nfr[1] = 0;
  if (ccd) {
    if (tid == 0) tkey = 0;
  } else {
    for (int e = tid; e < kXD + 1; e += CT) reinterpret_cast<long long*>(&xe)[e] = 0;
  }
  __syncthreads();
  unsigned pf_node = 0, pf_tri = 0, pf_edge = 0, pf_cand = 0;  // profiling: entries tested, candidates
  // the body's own terms, in its first chunk (GH: the body kernel adds them)
  if (!gh && ch.y == 0) {
    const Box bb = load_box(&a.body_box[I]);
    const bool vg = a.prm.ground_enabled && a.prm.enable_vg;
    for (int v = a.voff[I] + tid; vg && v < a.voff[I + 1]; v += CT) {
      if (!vg_candidate_of(a.prm, bb, a.y0, a.y1, v)) continue;
      if constexpr (ccd) {
        const double t = vg_toi(a.prm, a.y0, a.y1, v);
        if (t < 1.0) toi_min(&tkey, t);
      } else {
        const double d = a.y0[3 * v + 1] - a.prm.ground;
        const double e = barrier(d * d, a.prm);
        if (e != 0.0) xs_add_atomic(&xe, e);
      }
    }
    if (!ccd && tid == 0 && !a.fixed[I])
      xs_add_atomic(&xe, inertia_energy(a.prm, a.st, a.mass, a.I0, I, a.A + 9 * I, a.p + 3 * I));
  }
  // neighbours of I in increasing order: GH from the adjacency (it needs the pair indices;
  // an overflowed pass is rerun), ENERGY / CCD straight from the overlap bit matrix
  int r0 = 0, deg;
  if constexpr (gh) {
    r0 = a.row_ptr[I];
    deg = (a.dstat[DS_STATUS] & ST_PAIR_OVERFLOW) ? 0 : min(a.row_ptr[I + 1], a.cap_adj) - r0;
  } else {
    deg = a.row_cnt[I];
  }
  if (Q == 0) deg = 0;
  bool loaded = false;  // queries are loaded when the first neighbour overlaps the chunk
  for (int b0 = 0; b0 < deg; b0 += NBB) {
    const int nb = min(NBB, deg - b0);
    __syncthreads();
    // ENERGY / CCD past the listed neighbours: the CTA decodes the batch from the row's overlap
    // words (their prefix counts place each word's bits), one round of loads for the batch
    const bool decode = !gh && b0 + nb > kNbList;
    if (decode) {
      for (int w = tid; w < a.W; w += CT) {
        const int pre = a.pair_wpre[(size_t)I * a.W + w];
        if (pre >= b0 + nb) continue;
        uint32_t m = a.pair_mask[(size_t)I * a.W + w];
        if (pre + __popc(m) <= b0) continue;
        for (int k = pre; m; m &= m - 1, ++k)
          if (k >= b0 && k < b0 + nb) nJ[k - b0] = 32 * w + __ffs(m) - 1;
      }
      __syncthreads();
    }
    int rel = 0;
    if (tid < nb) {
      const int k = b0 + tid;
      const int J = gh ? a.adj_col[r0 + k] : (decode ? nJ[tid] : a.nbr[(size_t)I * kNbList + k]);
      nJ[tid] = J;
      nbox[tid] = load_box(&(ls ? a.body_sup : a.body_box)[J]);
      rel = overlap(cbx, nbox[tid]) ? 1 : 0;
      nrel[tid] = rel;
      ntri[tid] = a.tri.body_root[J];
      nedge[tid] = a.edge.body_root[J];
      nown[tid] = ee_owner(I, nEI, a.row_cnt[I], J, a.eoff[J + 1] - a.eoff[J], a.row_cnt[J]);
      if (gh) npair[tid] = a.adj_pair[r0 + b0 + tid];
    }
    if (!__syncthreads_or(rel)) continue;  // the chunk touches none of these neighbours
    if (!loaded) {
      loaded = true;
      if (tid < Q) {
        const int k = ch.y + tid;
        const float* m = a.fdof + 24 * (size_t)I;
        if (k < nV) {
          const int v = __ldg(&a.vperm[a.voff[I] + k]);
          qprim[tid] = a.prm.enable_pt ? v : kNoQuery;
          if constexpr (ls) {  // the point's box over the DOF range, from its rest position
            Box R;
#pragma unroll
            for (int d = 0; d < 3; ++d) R.lo[d] = R.hi[d] = (float)__ldg(&a.x0[3 * v + d]);
            qbox[tid] = affine_box2(R, m, m + 12, __double2float_ru(a.prm.dhat));
          } else {
            qbox[tid] = point_box(a.y0, a.y1, v, (float)a.prm.dhat);
          }
        } else {
          const int e = __ldg(&a.edge.leaf_prim[a.eoff[I] + (k - nV)]);
          qprim[tid] = a.prm.enable_ee ? ~e : kNoQuery;
          if constexpr (ls)  // the edge's box over the DOF range, from its rest box
            qbox[tid] = affine_box2(load_box(&a.edge.rest[(a.edge.N - 1) + a.eoff[I] + (k - nV)]), m, m + 12,
                                    __double2float_ru(0.5 * a.prm.dhat));
          else
            qbox[tid] = edge_leaf_box(a.edges, a.y0, a.y1, e, 0.5 * a.prm.dhat);
        }
      }
      if constexpr (ls) {
        if (a.prof && tid == 0) {
          const int qp = max(0, min(Q, nV - ch.y));
          atomicAdd(&a.prof_rows[8 * (blockIdx.x & 31) + PF_POINT], (unsigned long long)qp);
          atomicAdd(&a.prof_rows[8 * (blockIdx.x & 31) + PF_EDGE], (unsigned long long)(Q - qp));
        }
      }
    }
    // FP32 DOFs of the neighbours, as the broad phase wrote them (6 x 16 B per neighbour)
    for (int e = tid; e < 6 * nb; e += CT) {
      const int j = e / 6, q = e % 6;
      if (q < 3 || a.y1)
        reinterpret_cast<float4*>(ndof[j])[q] = __ldg(reinterpret_cast<const float4*>(a.fdof + 24 * (size_t)nJ[j]) + q);
    }
    for (int w0 = 0; w0 < Q * nb; w0 += CW) {
      if (tid == 0) nwork = 0;
      __syncthreads();
      // overlapping (query, neighbour) combinations of this round
      for (int it = w0 + tid; it < min(Q * nb, w0 + CW); it += CT) {
        const int q = it % Q, j = it / Q;
        if (!nrel[j] || qprim[q] == kNoQuery || (qprim[q] < 0 && !nown[j])) continue;
        if (!overlap(qbox[q], nbox[j])) continue;
        work[atomicAdd(&nwork, 1)] = (unsigned short)(q | (j << 8));
      }
      __syncthreads();
      // the compacted (query, neighbour) combinations walk their neighbour's tree breadth
      // first: each round every thread takes frontier entries (query, neighbour, node) and
      // expands them into the next frontier, so the visits of a chunk in heavy contact spread
      // over the CTA instead of queueing on the threads that drew its longest walks.  When the
      // frontier is full a thread walks the subtree itself, depth first.
      auto visit = [&](int q, int j, int type, int pa, int pb) {
        if constexpr (gh) {
          // evaluated by k_gh_eval, one thread per candidate.  PT: the point is I's, the
          // pair's first body is min(I, J); EE: the lower body's edge comes first
          const int swap = (type == 0 && I > nJ[j]) ? 1 : 0;
          emit(make_int4(npair[j], type | (swap << 1), pa, pb));
        } else if constexpr (ls) {
          // line-search candidates; k_ccd_eval takes those that pass the CCD pass's boxes
          ++pf_cand;
          emit(make_int4(type, pa, pb, 0));
        } else if constexpr (ccd) {  // evaluated by k_ccd_eval, one thread per candidate
          emit(make_int4(type, pa, pb, 0));
        } else {
          int ids[4];
          d3 xs[4];
          cand_vertices(a, type, pa, pb, ids);
          fetch(a.y0, ids, xs);
          const double e = candidate_energy(a, type, ids, xs);
          if (e != 0.0) xs_add_atomic(&xe, e);
        }
      };
      // a leaf of J's tree reached by query q: PT (I's point, J's triangle) or EE (the lower
      // body's edge first, as the per-pair lists)
      auto hit = [&](int q, int j, int prim) {
        const int qp = qprim[q];
        if (qp >= 0) visit(q, j, 0, qp, prim);
        else if (I < nJ[j]) visit(q, j, 1, ~qp, prim);
        else visit(q, j, 1, prim, ~qp);
      };
      auto boxes_of = [&](int q, int j) {
        const bool tri = qprim[q] >= 0;
        NodeBoxes nbx = node_boxes(a, tri ? &a.tri : &a.edge, tri, ndof[j]);
        nbx.sup = ls;
        return nbx;
      };
      auto tally = [&](bool tri, const Visits& vc) {
        pf_node += vc.internal;
        if (tri) pf_tri += vc.leaf;
        else pf_edge += vc.leaf;
      };
      // frontier entry: (q | j << 8, node); a full frontier makes the pusher walk the subtree
      auto push = [&](int nxt, int q, int j, int node) {
        const NodeBoxes nbx = boxes_of(q, j);
        const int slot = atomicAdd(&nfr[nxt], 1);
        if (slot < fcap) {
          front[nxt][slot] = make_int2(q | (j << 8), node);
          prefetch_node(*nbx.tr, node);
        } else {
          Visits vc;
          traverse(nbx, node, qbox[q], a.dstat, [&](int prim) { hit(q, j, prim); }, vc);
          tally(nbx.tri, vc);
        }
      };
      // the roots
      for (int k = tid; k < nwork; k += CT) {
        const int q = work[k] & 0xff, j = work[k] >> 8;
        const NodeBoxes nbx = boxes_of(q, j);
        const int root = nbx.tri ? ntri[j] : nedge[j];
        const int L0 = nbx.tr->N - 1;
        Visits vc;
        if (root >= L0) {  // a tree of one leaf
          const int prim = __ldg(&nbx.tr->leaf_prim[root - L0]);
          ++vc.leaf;
          if (overlap(nbx.leaf(root, prim), qbox[q])) hit(q, j, prim);
        } else if (root >= 0) {
          ++vc.internal;
          if (overlap(nbx.internal(root), qbox[q])) push(fcur, q, j, root);
        }
        tally(nbx.tri, vc);
      }
      // the rounds
      for (;;) {
        __syncthreads();
        const int n = min(nfr[fcur], fcap);
        if (n == 0) break;
        const int nxt = fcur ^ 1;
        for (int e = tid; e < n; e += CT) {
          const int2 en = front[fcur][e];
          const int q = en.x & 0xff, j = en.x >> 8;
          const NodeBoxes nbx = boxes_of(q, j);
          Visits vc;
          expand_node(nbx, en.y, qbox[q], [&](int prim) { hit(q, j, prim); }, [&](int c) { push(nxt, q, j, c); }, vc);
          tally(nbx.tri, vc);
        }
        __syncthreads();
        if (lists && ncb >= kCandBuf / 2) flush();
        if (tid == 0) nfr[fcur] = 0;
        fcur = nxt;
      }
    }
  }
  if constexpr (lists) {
    __syncthreads();
    flush();
  }
  if constexpr (gh) return;
  if (ls && a.prof) {  // kernel profiling: the data this chunk read and wrote
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      pf_node += __shfl_xor_sync(0xffffffffu, pf_node, o);
      pf_tri += __shfl_xor_sync(0xffffffffu, pf_tri, o);
      pf_edge += __shfl_xor_sync(0xffffffffu, pf_edge, o);
      pf_cand += __shfl_xor_sync(0xffffffffu, pf_cand, o);
    }
    unsigned long long* row = a.prof_rows + 8 * (blockIdx.x & 31);
    if ((tid & 31) == 0) {
      atomicAdd(&row[PF_NODE], (unsigned long long)pf_node);
      atomicAdd(&row[PF_TRI], (unsigned long long)pf_tri);
      atomicAdd(&row[PF_EDGELEAF], (unsigned long long)pf_edge);
      atomicAdd(&row[PF_CAND], (unsigned long long)pf_cand);
    }
  }
  __syncthreads();
  if (tid == 0) {
    if constexpr (ls) {
      if (a.gtime) atomicMax(&a.gtime[1], globaltimer_ns());
    }
    if constexpr (ccd) {
      if (tkey) atomicMax(a.toi_key, tkey);
    } else {
      const long long* src = reinterpret_cast<const long long*>(&xe);
      long long* dst = reinterpret_cast<long long*>(a.energy);
      for (int e = 0; e < kXD; ++e)
        if (src[e]) atomicAdd((unsigned long long*)&dst[e], (unsigned long long)src[e]);
      if (src[kXD]) atomicOr((unsigned long long*)&dst[kXD], (unsigned long long)src[kXD]);
    }
  }
}

// Times of impact of the CCD candidates, one thread per candidate (ccd.py:20-40, 133-186);
// the minimum below 1 goes to the mailbox key.  LS: the candidates are the line-search
// candidates of a CCD_LS pass, and each is first put to the CCD pass's own culling
// predicate: the exact swept body boxes overlap and the two swept primitive boxes overlap;
// block 0 also clears the energies of the line-search batch that follows the pass.
template <bool LS>
__global__ void __launch_bounds__(128) k_ccd_eval(NarrowArgs a) {
  if (LS && blockIdx.x == 0) {
    static_assert(sizeof(XSum) == (kXD + 1) * sizeof(long long), "XSum layout");
    for (int i = threadIdx.x; i < kLsMax * (kXD + 1); i += blockDim.x)
      reinterpret_cast<long long*>(a.ls_energy)[i] = 0;
  }
  const int n = LS ? min(a.dstat[DS_NECAND], a.cap_ecand) : min(a.dstat[DS_NCCD], a.cap_ccd);
  if (a.dstat[DS_STATUS] & (LS ? ST_ECAND_OVERFLOW : ST_CCD_OVERFLOW)) return;
  const int4* cand = LS ? a.ecand : a.ccd_cand;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int4 c = cand[k];
    int ids[4];
    cand_vertices(a, c.x, c.y, c.z, ids);
    if (LS) {
      const int bA = __ldg(&a.vbody[ids[0]]), bB = __ldg(&a.vbody[ids[c.x == 0 ? 1 : 2]]);
      if (!overlap(load_box(&a.body_box[bA]), load_box(&a.body_box[bB]))) continue;
      const double dhh = 0.5 * a.prm.dhat;
      const bool hit = c.x == 0 ? overlap(point_box(a.y0, a.y1, c.y, (float)a.prm.dhat), tri_leaf_box(a.tris, a.y0, a.y1, c.z))
                                : overlap(edge_leaf_box(a.edges, a.y0, a.y1, c.y, dhh),
                                          edge_leaf_box(a.edges, a.y0, a.y1, c.z, dhh));
      if (!hit) continue;
    }
    d3 x0[4], x1[4];
    fetch(a.y0, ids, x0);
    fetch(a.y1, ids, x1);
    const double t = collision_time(c.x, x0, x1, a.prm.ipc_full != 0);
    if (t < 1.0) toi_min(a.toi_key, t);
  }
}

// Sets dint[kSupValid] (gh_superset_check) and, in a captured pass (use_hc), the condition of
// the IF node around the tree traversal: 1 when the traversal must run; one CTA
__global__ void k_sup_check(int n, const double* A0, const double* p0, const double* q_last, const int* have,
                            int* valid, int mode, const int* it, cudaGraphConditionalHandle hc, int use_hc) {
  if (mode == 3) mode = *it == 0 ? 1 : 2;
  __shared__ int ok;
  if (threadIdx.x == 0) ok = mode == 2 ? 1 : (mode == 1 ? (*have != 0) : 0);
  __syncthreads();
  if (mode == 1 && ok)
    for (int i = threadIdx.x; i < 12 * n; i += blockDim.x) {
      const double v = i < 9 * n ? A0[i] : p0[i - 9 * n];
      if (__double_as_longlong(v) != __double_as_longlong(q_last[i])) ok = 0;
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    *valid = ok;
    if (use_hc) cudaGraphSetConditional(hc, ok ? 0u : 1u);
  }
}

// Lagged friction (friction_mu > 0, with the full model; Li et al. 2020, section 5): at the
// step's first GH pass every contact within dhat fixes its lagged quantities (the header's
// friction_lag at the step-start positions xs) and its body pair joins the step's pair lists;
// returns the contact's friction potential there (mu lambda eps / 3: no displacement yet).
__device__ inline double friction_lag_contact(const NarrowArgs& a, int kind, const int ids[4], const d3 xs[4]) {
  double x12[12], r12[12];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x12[3 * k] = xs[k].x, x12[3 * k + 1] = xs[k].y, x12[3 * k + 2] = xs[k].z;
    for (int m = 0; m < 3; ++m) r12[3 * k + m] = __ldg(&a.x0[3 * ids[k] + m]);
  }
  ipc::FrictionLag L;
  if (!ipc::friction_lag(kind, x12, r12, a.prm.d2hat, a.prm.kappa, SharedLog(), &L)) return 0.0;
  const int I = __ldg(&a.vbody[ids[0]]), J = __ldg(&a.vbody[ids[kind == 0 ? 1 : 2]]);
  const int pos = atomicAdd(&a.dstat[DS_NFRIC], 1);
  if (pos < a.cap_fric) {
    FricRec& f = a.fric[pos];
    for (int k = 0; k < 4; ++k) f.w[k] = L.w[k];
    for (int k = 0; k < 6; ++k) f.P[k] = L.P[k];
    f.lam = L.lambda;
    for (int k = 0; k < 12; ++k) f.xt[k] = x12[k];
    for (int k = 0; k < 4; ++k) f.ids[k] = ids[k];
    f.I = I;
    f.J = J;
    f.kind = kind;
  } else {
    atomicOr(&a.dstat[DS_STATUS], ST_FRIC_OVERFLOW);
  }
  if (I != J) {
    atomicOr(&a.fric_mask[(size_t)I * a.W + (J >> 5)], 1u << (J & 31));
    atomicOr(&a.fric_mask[(size_t)J * a.W + (I >> 5)], 1u << (I & 31));
  }
  return ipc::friction_d(L, x12, x12, a.prm.friction_mu, a.prm.friction_epsv * a.prm.dt);
}

// The friction contacts of the GH pass, one thread per lagged contact: each joins its body
// pair's contact list (found in the adjacency) as a pseudo-contact (y = kFricContact, z = its
// record); the pair assembly adds its friction terms to the pair's exact sums.  They are not
// active contacts (DS_ACTIVE is compensated for the pair assembly's count).
__global__ void __launch_bounds__(128) k_fric_pairs(NarrowArgs a) {
  if (a.dstat[DS_STATUS] & (ST_PAIR_OVERFLOW | ST_CONTACT_OVERFLOW | ST_FRIC_OVERFLOW)) return;
  const int n = min(a.dstat[DS_NFRIC], a.cap_fric);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int I = a.fric[k].I, J = a.fric[k].J, lo = min(I, J), hi = max(I, J);
    int pr = -1;
    const int k1 = min(a.row_ptr[lo + 1], a.cap_adj);
    for (int q = a.row_ptr[lo]; q < k1 && pr < 0; ++q)
      if (a.adj_col[q] == hi) pr = a.adj_pair[q];
    if (pr < 0) continue;
    const int pos = atomicAdd(&a.dstat[DS_NCONTACT], 1);
    if (pos < a.cap_contacts) a.contacts[pos] = make_int4(pr, kFricContact, k, 0);
    else atomicOr(&a.dstat[DS_STATUS], ST_CONTACT_OVERFLOW);
    atomicAdd(&a.pair_cand[4 * pr + 1], 1);
    atomicSub(&a.dstat[DS_ACTIVE], 1);
  }
}

// The friction potential of every lagged contact at the pass's positions y0, into the pass's
// exact energy (the energy pass), one thread per contact
__global__ void __launch_bounds__(128) k_fric_energy(NarrowArgs a) {
  const int n = min(a.dstat[DS_NFRIC], a.cap_fric);
  XSum en;
  xs_zero(en);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const FricRec& f = a.fric[k];
    double x12[12];
    for (int q = 0; q < 12; ++q) x12[q] = a.y0[3 * f.ids[q / 3] + q % 3];
    const double e = ipc::friction_d(lag_of(f), x12, f.xt, a.prm.friction_mu, a.prm.friction_epsv * a.prm.dt);
    if (e != 0.0) xs_add(en, e);
  }
  xs_warp_sum(en);
  if ((threadIdx.x & 31) == 0) {
    long long* d = reinterpret_cast<long long*>(a.energy);
#pragma unroll
    for (int i = 0; i < kXD; ++i)
      if (en.d[i]) atomicAdd((unsigned long long*)&d[i], (unsigned long long)en.d[i]);
    if (en.flags) atomicOr((unsigned long long*)&d[kXD], (unsigned long long)en.flags);
  }
}

// One candidate of the GH pass, c = (pair, type | swap << 1, primitive a, primitive b): counted
// by kind; when active (pt_ipc.py:13-22, 114; ee_ipc.py:13-23, 382) appended for the per-pair
// assembly and counted for its pair, and at the step's first GH pass (lag) its lagged friction
// is fixed.  With gh_energy its barrier energy joins the pass's exact energy (k_body_gh adds
// the bodies' terms: the GH pass then also gives the energy at its DOFs, the same sum as an
// energy pass there).
__device__ inline void gh_candidate(const NarrowArgs& a, const int4 c, bool with_energy, bool lag, int& cpt,
                                    int& cee, XSum& en) {
  const int type = c.y & 1;
  if (type == 0) ++cpt;
  else ++cee;
  int ids[4];
  d3 xs[4];
  cand_vertices(a, type, c.z, c.w, ids);
  fetch(a.y0, ids, xs);
  if (with_energy) {
    const double e = candidate_energy(a, type, ids, xs);
    if (e != 0.0) xs_add(en, e);
  }
  Geo G;
  double d2;
  int fty;
  if (a.prm.ipc_full ? full_d2(type, xs, &fty) < a.prm.d2hat : contact_active(type, xs, a.prm, &G, &d2)) {
    const int pos = append_slot(&a.dstat[DS_NCONTACT]);
    if (pos < a.cap_contacts) a.contacts[pos] = c;
    else atomicOr(&a.dstat[DS_STATUS], ST_CONTACT_OVERFLOW);
    atomicAdd(&a.pair_cand[4 * c.x + 1], 1);
    if (lag) {
      const double e = friction_lag_contact(a, type, ids, xs);
      if (with_energy && e != 0.0) xs_add(en, e);
    }
  }
}

// the per-kind counts and the energy of a CTA's candidates into the pass's totals (every thread)
__device__ inline void gh_flush(const NarrowArgs& a, int cpt, int cee, XSum& en, bool with_energy) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cpt += __shfl_xor_sync(0xffffffffu, cpt, o);
    cee += __shfl_xor_sync(0xffffffffu, cee, o);
  }
  if (with_energy) xs_warp_sum(en);
  if ((threadIdx.x & 31) == 0) {
    if (cpt) atomicAdd(&a.dstat[DS_PT_COUNT], cpt);
    if (cee) atomicAdd(&a.dstat[DS_EE_COUNT], cee);
    long long* d = reinterpret_cast<long long*>(a.energy);
#pragma unroll
    for (int i = 0; i < kXD; ++i)
      if (en.d[i]) atomicAdd((unsigned long long*)&d[i], (unsigned long long)en.d[i]);
    if (en.flags) atomicOr((unsigned long long*)&d[kXD], (unsigned long long)en.flags);
  }
}

// the energy and the friction lag ride on the step's first GH pass
__device__ inline bool gh_with_energy(const NarrowArgs& a) {
  return a.gh_energy && (!a.energy_gate || *a.energy_gate == 0);
}
__device__ inline bool gh_lag(const NarrowArgs& a) { return a.fric_lag && (!a.energy_gate || *a.energy_gate == 0); }

// The candidates of the tree traversal (when the kept line-search candidates did not cover the
// pass; k_gh_scan evaluates them otherwise), one thread per candidate
__global__ void __launch_bounds__(128) k_gh_eval(NarrowArgs a) {
  if (*a.sup_valid || (a.dstat[DS_STATUS] & (ST_CCD_OVERFLOW | ST_PAIR_OVERFLOW))) return;
  const int n = min(a.dstat[DS_NCCD], a.cap_ccd);
  int cpt = 0, cee = 0;
  XSum en;  // the candidates' barrier energy (ipcsk/energy.py:9-48)
  xs_zero(en);
  const bool with_energy = gh_with_energy(a), lag = gh_lag(a);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    gh_candidate(a, a.ccd_cand[k], with_energy, lag, cpt, cee, en);
  gh_flush(a, cpt, cee, en, with_energy);
}

// The GH pass's candidates without a traversal, when the kept line-search candidates hold
// every pair its culling can produce (sup_valid): the pass's DOFs lie on the segment the step's
// last CCD pass covered (the accepted step q - alpha dq, 0 <= alpha <= 1).  Each candidate is
// put to the GH pass's own culling predicate -- the exact body boxes overlap and the static
// primitive boxes overlap (culling2.py:32-79, 213-227) -- and evaluated as the traversal's
// candidates are, with its pair index from the adjacency of the point's (or lower edge's) body.
__global__ void __launch_bounds__(128) k_gh_scan(NarrowArgs a) {
  if (!*a.sup_valid || (a.dstat[DS_STATUS] & (ST_CCD_OVERFLOW | ST_PAIR_OVERFLOW))) return;
  const int n = min(a.dstat[DS_NECAND], a.cap_ecand);
  const float dhf = (float)a.prm.dhat;
  const double dhh = 0.5 * a.prm.dhat;
  int cpt = 0, cee = 0;
  XSum en;
  xs_zero(en);
  const bool with_energy = gh_with_energy(a), lag = gh_lag(a);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int4 c = a.ecand[k];
    const int type = c.x, pa = c.y, pb = c.z;
    int ids[4];
    cand_vertices(a, type, pa, pb, ids);
    const int I = __ldg(&a.vbody[ids[0]]), J = __ldg(&a.vbody[ids[type == 0 ? 1 : 2]]);
    if (!overlap(load_box(&a.body_box[I]), load_box(&a.body_box[J]))) continue;
    const bool hit = type == 0 ? overlap(point_box(a.y0, nullptr, pa, dhf), tri_leaf_box(a.tris, a.y0, nullptr, pb))
                               : overlap(edge_leaf_box(a.edges, a.y0, nullptr, pa, dhh),
                                         edge_leaf_box(a.edges, a.y0, nullptr, pb, dhh));
    if (!hit) continue;
    // row I of the adjacency lists its neighbours in increasing order
    int lo = a.row_ptr[I], hi = min(a.row_ptr[I + 1], a.cap_adj) - 1, pr = -1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1, col = a.adj_col[mid];
      if (col == J) {
        pr = a.adj_pair[mid];
        break;
      }
      if (col < J) lo = mid + 1;
      else hi = mid - 1;
    }
    if (pr < 0) continue;  // (the body boxes overlap, so the pair is listed)
    const int swap = (type == 0 && I > J) ? 1 : 0;
    gh_candidate(a, make_int4(pr, type | (swap << 1), pa, pb), with_energy, lag, cpt, cee, en);
  }
  gh_flush(a, cpt, cee, en, with_energy);
}

// ---------------------------------------------------------------------------------------
// per-body kernels
// ---------------------------------------------------------------------------------------
struct BodyArgs {
  abd_params prm;
  int n;
  const int* voff;
  const double *x0, *mass, *I0;
  const int* fixed;
  abd_states st;
  const double *A, *p, *y, *y1;
  const Box* body_box;
  const int *row_ptr, *adj_pair, *pair_active;
  const int2* ij;
  const double *pdiag, *pgrad;
  double *diag, *g;
  int* dstat;
  int* vg_list;
  int cap_vg;
  XSum* energy;  // or null; the pass's exact energy (GH: inertia + vertex-ground terms, added here)
  const int* energy_gate;  // device loop: the energy is summed only while this counter is 0
  int exact;     // the adjoint's system: the vertex-ground Hessian with its 2 B' term
  int* highlight;  // [n] or null: the body takes part in an active PT / EE / vertex-ground contact
};

__device__ inline void tilde(const BodyArgs& a, int b, double At[9], double pt[3]) {
  tilde_of(a.prm, a.st, b, At, pt);
}
__device__ inline bool vg_candidate(const BodyArgs& a, const Box& bb, const double* y0, const double* y1, int v) {
  return vg_candidate_of(a.prm, bb, y0, y1, v);
}

constexpr int BT = 160;

__global__ void __launch_bounds__(BT) k_body_gh(BodyArgs a) {
  const int b = blockIdx.x, t = threadIdx.x;
  XSum* const energy = (a.energy && (!a.energy_gate || *a.energy_gate == 0)) ? a.energy : nullptr;
  const bool fixed = a.fixed[b] != 0;
  const double dt = a.prm.dt, ks = a.prm.stiffness;
  const double* A = a.A + 9 * b;
  double val = 0.0;
  // vertex-ground sums, exact: g (4 y-components) and H (4x4 yy-components); vx[20]: the
  // body's energy (vertex-ground barriers of every body, inertia + orthogonality of a free one)
  __shared__ XSum vx[21];
  __shared__ int vg_hit;  // an active vertex-ground contact (d^2 < dhat^2)
  const bool vg_any = a.prm.ground_enabled && a.prm.enable_vg, vg_on = vg_any && !fixed;
  for (int e = t; e < 21 * (kXD + 1); e += BT) reinterpret_cast<long long*>(vx)[e] = 0;
  if (t == 0) vg_hit = 0;
  __syncthreads();
  if (energy && t == 128 && !fixed)
    xs_add_atomic(&vx[20], inertia_energy(a.prm, a.st, a.mass, a.I0, b, a.A + 9 * b, a.p + 3 * b));
  if (vg_any && t < 128) {
    const Box bb = load_box(&a.body_box[b]);
    int cnt = 0;  // the culling's vertex-ground pairs, fixed bodies included (culling.py:54-82)
    for (int v = a.voff[b] + t; v < a.voff[b + 1]; v += 128) {
      if (!vg_candidate(a, bb, a.y, nullptr, v)) continue;
      ++cnt;
      const double d = a.y[3 * v + 1] - a.prm.ground;
      if (d * d < a.prm.d2hat) vg_hit = 1;
      if (energy) {
        const double e = barrier(d * d, a.prm);
        if (e != 0.0) xs_add_atomic(&vx[20], e);
      }
      if (!vg_on) continue;
      const double d2b = barrier_d2(d * d, a.prm), db = barrier_d1(d * d, a.prm);
      const double th[4] = {1.0, a.x0[3 * v], a.x0[3 * v + 1], a.x0[3 * v + 2]};
#pragma unroll
      for (int ii = 0; ii < 4; ++ii) {
        xs_add_atomic(&vx[ii], ((d * 2.0) * th[ii]) * db);
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
          xs_add_atomic(&vx[4 + 4 * ii + jj], (((th[ii] * th[jj]) * d2b) * 4.0) * d * d);
          if (a.exact) xs_add_atomic(&vx[4 + 4 * ii + jj], (th[ii] * th[jj]) * (2.0 * db));
        }
      }
    }
    if (cnt) atomicAdd(&a.dstat[DS_VG_COUNT], cnt);
  }
  __syncthreads();
  if (energy && t <= kXD) {
    const long long v = reinterpret_cast<const long long*>(&vx[20])[t];
    long long* d = reinterpret_cast<long long*>(energy);
    if (v) {
      if (t < kXD) atomicAdd((unsigned long long*)&d[t], (unsigned long long)v);
      else atomicOr((unsigned long long*)&d[t], (unsigned long long)v);
    }
  }
  // contact flags (abd.py:238): any active contact of the body's pairs, or vertex-ground
  if (a.highlight && t == 156) {
    int on = vg_hit;
    const int k1 = (a.dstat[DS_STATUS] & ST_PAIR_OVERFLOW) ? a.row_ptr[b] : a.row_ptr[b + 1];
    for (int k = a.row_ptr[b]; k < k1 && !on; ++k) on = a.pair_active[a.adj_pair[k]] > 0;
    a.highlight[b] = on;
  }
  if (t >= 156) return;
  if (!fixed) {
    double At[9], pt[3];
    tilde(a, b, At, pt);
    if (t < 144) {
      const int r = t / 12, c = t % 12, ii = r / 3, jj = c / 3, rr = r % 3, cc = c % 3;
      const double m = (ii != jj) ? 0.0 : (ii == 0 ? a.mass[b] : a.I0[b]);
      double dh = rr == cc ? m : 0.0;
      if (ii > 0 && jj > 0) {
        const int i = ii - 1, j = jj - 1;
        double h;
        if (i == j) {
          h = 0.0;
          for (int k = 0; k < 3; ++k) h += A[3 * k + rr] * A[3 * k + cc];
          const double ti = (A[3 * i] * A[3 * i] + A[3 * i + 1] * A[3 * i + 1] + A[3 * i + 2] * A[3 * i + 2]) - 1.0;
          h += (A[3 * i + rr] * A[3 * i + cc] + (rr == cc ? ti : 0.0));
        } else {
          const double tj = A[3 * j] * A[3 * i] + A[3 * j + 1] * A[3 * i + 1] + A[3 * j + 2] * A[3 * i + 2];
          h = A[3 * j + rr] * A[3 * i + cc] + (rr == cc ? tj : 0.0);
        }
        dh = dh + ((h * 4.0) * ks) * dt * dt;
      }
      val = dh;
    } else {
      const int k = t - 144, m = k / 3, comp = k % 3;
      if (m == 0) {
        val = 0.0 + (a.p[3 * b + comp] - pt[comp]) * a.mass[b];
      } else {
        const int i = m - 1;
        double gr = -A[3 * i + comp];
        for (int j = 0; j < 3; ++j) {
          const double dj = A[3 * i] * A[3 * j] + A[3 * i + 1] * A[3 * j + 1] + A[3 * i + 2] * A[3 * j + 2];
          gr = gr + dj * A[3 * j + comp];
        }
        gr = (gr * 4.0) * ks;
        gr = (dt * dt) * gr;
        val = gr + (A[3 * i + comp] - At[3 * i + comp]) * a.I0[b];
      }
    }
    // entry = inertia + vertex-ground terms + the pair contributions (adjacency order; the sum
    // is exact, so the order does not matter), rounded once
    XSum acc;
    xs_zero(acc);
    xs_add(acc, val);
    if (vg_on) {
      if (t < 144) {
        const int r = t / 12, c = t % 12;
        if (r % 3 == 1 && c % 3 == 1) xs_merge(acc, vx[4 + 4 * (r / 3) + c / 3]);
      } else if ((t - 144) % 3 == 1) {
        xs_merge(acc, vx[(t - 144) / 3]);
      }
    }
    // skipped when the pair lists of this pass overflowed (the host reruns the pass)
    const int k1 = (a.dstat[DS_STATUS] & ST_PAIR_OVERFLOW) ? a.row_ptr[b] : a.row_ptr[b + 1];
    for (int k = a.row_ptr[b]; k < k1; ++k) {
      const int pr = a.adj_pair[k];
      if (a.pair_active[pr] <= 0) continue;
      const int side = a.ij[pr].x == b ? 0 : 1;
      xs_add(acc, t < 144 ? a.pdiag[(size_t)pr * 288 + side * 144 + t] : a.pgrad[(size_t)pr * 24 + side * 12 + (t - 144)]);
    }
    val = xs_round(acc);
    if (!isfinite(val)) atomicOr(&a.dstat[DS_STATUS], ST_NAN);
  } else {
    val = (t < 144 && (t % 13) == 0) ? 1.0 : 0.0;
  }
  if (t < 144) a.diag[(size_t)b * 144 + t] = val;
  else a.g[(size_t)b * 12 + (t - 144)] = val;
}

__global__ void k_vg_list(BodyArgs a) {
  const int b = blockIdx.x;
  const Box bb = load_box(&a.body_box[b]);
  for (int v = a.voff[b] + threadIdx.x; v < a.voff[b + 1]; v += blockDim.x) {
    if (!vg_candidate(a, bb, a.y, a.y1, v)) continue;
    const int pos = atomicAdd(&a.dstat[DS_VG_COUNT], 1);
    if (pos < a.cap_vg) {
      a.vg_list[2 * pos] = b;
      a.vg_list[2 * pos + 1] = v;
    } else {
      atomicOr(&a.dstat[DS_STATUS], ST_VG_OVERFLOW);
    }
  }
}

// exported blocks follow the solver's view: pairs without active contacts or touching a fixed
// (Dirichlet) body have no coupling block
__global__ void k_export_off(int np, const int* pair_active, const int* fixed, const double* offdiag, const int2* ij,
                             double* out, int* ijout, int cap) {
  const int p = blockIdx.x;
  if (p >= np || p >= cap) return;
  const bool live = pair_active[p] > 0 && !fixed[ij[p].x] && !fixed[ij[p].y];
  for (int e = threadIdx.x; e < 144; e += blockDim.x) out[(size_t)p * 144 + e] = live ? offdiag[(size_t)p * 288 + e] : 0.0;
  if (threadIdx.x == 0 && ijout) {
    ijout[2 * p] = ij[p].x;
    ijout[2 * p + 1] = ij[p].y;
  }
}

// (Ao, po) = (A, p) - alpha dq (alpha_dev: the step length on the device); also into (Ao2, po2)
// when given
__global__ void k_update_dofs(int n, const double* A, const double* p, const double* dq, double alpha, double* Ao,
                              double* po, const double* alpha_dev, double* Ao2, double* po2) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  update_body_dofs(b, A, p, dq, alpha_dev ? *alpha_dev : alpha, Ao, po, Ao2, po2);
}

__global__ void k_finish(int n, double dt, abd_states st) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  for (int k = 0; k < 3; ++k) {
    st.pdot[3 * b + k] = (st.p[3 * b + k] - st.p0[3 * b + k]) / dt;
    st.p0[3 * b + k] = st.p[3 * b + k];
  }
  for (int k = 0; k < 9; ++k) {
    st.Adot[9 * b + k] = (st.A[9 * b + k] - st.A0[9 * b + k]) / dt;
    st.A0[9 * b + k] = st.A[9 * b + k];
  }
}

// Exact dot products a.b and c.d (c may be null) on a fixed grid of kRedDot CTAs; the last CTA
// to finish sums the partials and writes the rounded results to out[0], out[1].
constexpr int kRedDot = 64;
__global__ void __launch_bounds__(256) k_dots(int N, const double* a, const double* b, const double* c,
                                              const double* d, XSum* part, int* count, double* out) {
  __shared__ XSum sh[8];
  __shared__ bool last;
  XSum x0, x1;
  xs_zero(x0);
  xs_zero(x1);
  for (int i = blockIdx.x * 256 + threadIdx.x; i < N; i += kRedDot * 256) {
    xs_add(x0, a[i] * b[i]);
    if (c) xs_add(x1, c[i] * d[i]);
  }
  xs_block_sum(x0, sh);
  xs_block_sum(x1, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = x0;
    part[kRedDot + blockIdx.x] = x1;
    __threadfence();
    last = atomicAdd(count, 1) == kRedDot - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = 0; k < (c ? 2 : 1); ++k) {
    XSum t;
    xs_zero(t);
    for (int i = threadIdx.x; i < kRedDot; i += 256) {
      const long long* q = reinterpret_cast<const long long*>(part + k * kRedDot + i);
#pragma unroll
      for (int j = 0; j < kXD; ++j) t.d[j] += __ldcg(q + j);
      t.flags |= __ldcg(q + kXD);
    }
    xs_block_sum(t, sh);
    if (threadIdx.x == 0) out[k] = xs_round(t);
  }
  if (threadIdx.x == 0) *count = 0;
}

NarrowArgs narrow_args(Sim& s, int mode, const double* A, const double* p, const double* A1, const double* p1,
                       const double* y0, const double* y1, const abd_states* st) {
  NarrowArgs a;
  a.A = A;
  a.p = p;
  a.A1 = A1;
  a.p1 = p1;
  a.affine = A && p && (!y1 || (A1 && p1));
  a.mode = mode;
  a.prm = s.prm;
  a.n = s.n;
  a.cap_adj = s.cap_adj;
  a.ij = s.ij;
  a.row_ptr = s.row_ptr;
  a.adj_col = s.adj_col;
  a.row_cnt = s.row_cnt;
  a.pair_mask = s.pair_mask;
  a.pair_wpre = s.pair_wpre;
  a.nbr = s.nbr;
  a.fdof = s.fdof;
  a.chunk_box = s.chunk_box;
  a.vperm = s.vperm;
  a.W = s.W;
  a.body_box = s.body_box;
  a.chunk = s.chunk;
  a.nch = s.nch;
  a.chunk_act = s.chunk_act;
  a.energy = s.energy_acc;
  a.prof = s.prof_on == 2;
  a.prof_rows = &s.box->prof[0][0];
  a.adj_pair = s.adj_pair;
  a.cap_ccd = s.cap_ccd;
  a.ccd_cand = s.ccd_cand;
  a.body_sup = s.body_sup;
  a.gh_energy = s.gh_energy;
  a.energy_gate = s.energy_gate;
  a.gtime = s.prof_events < 0 ? &s.box->step.t0 : nullptr;
  a.sup_valid = s.dint + kSupValid;
  a.cap_act = s.cap_act;
  a.act_pairs = s.act_pairs;
  const bool fr = s.prm.friction_mu > 0.0;
  a.fric = fr ? s.fric : nullptr;
  a.cap_fric = s.cap_fric;
  a.fric_mask = fr ? s.fric_mask : nullptr;
  a.fric_lag = fr ? (s.energy_gate ? 1 : s.fric_lag) : 0;
  a.vbody = s.vbody;
  a.cap_ecand = s.cap_ecand;
  a.ecand = s.ecand;
  a.cap_contacts = s.cap_contacts;
  a.contacts = s.contacts;
  a.contacts_by_pair = s.contacts_by_pair;
  a.toi_key = s.dmin;
  a.ls_energy = s.box->ls_energy;
  a.st = st ? *st : abd_states{};
  a.mass = s.mass;
  a.I0 = s.I0;
  a.fixed = s.fixed;
  a.voff = s.voff;
  a.toff = s.toff;
  a.eoff = s.eoff;
  a.tris = s.tris;
  a.edges = s.edges;
  a.y0 = y0;
  a.y1 = y1;
  a.x0 = s.x0;
  a.tri = s.tri_tree;
  a.edge = s.edge_tree;
  a.pt_list = s.pt_list;
  a.ee_list = s.ee_list;
  a.cap_pt = s.cap_pt;
  a.cap_ee = s.cap_ee;
  a.pair_cand = s.pair_cand;
  a.dstat = s.dstat;
  a.offdiag = s.offdiag;
  a.pdiag = s.pdiag;
  a.pgrad = s.pgrad;
  a.pair_val = s.pair_val;
  a.pair_active = s.pair_active;
  return a;
}

BodyArgs body_args(Sim& s, const abd_states* st, const double* A, const double* p, const double* y, const double* y1) {
  BodyArgs a;
  a.prm = s.prm;
  a.n = s.n;
  a.voff = s.voff;
  a.x0 = s.x0;
  a.mass = s.mass;
  a.I0 = s.I0;
  a.fixed = s.fixed;
  if (st) a.st = *st;
  else a.st = abd_states{};
  a.A = A;
  a.p = p;
  a.y = y;
  a.y1 = y1;
  a.body_box = s.body_box;
  a.row_ptr = s.row_ptr;
  a.adj_pair = s.adj_pair;
  a.pair_active = s.pair_active;
  a.ij = s.ij;
  a.pdiag = s.pdiag;
  a.pgrad = s.pgrad;
  a.diag = s.diag;
  a.g = s.g;
  a.dstat = s.dstat;
  a.vg_list = s.vg_list;
  a.cap_vg = s.cap_vg;
  a.energy = s.gh_energy ? s.energy_acc : nullptr;
  a.energy_gate = s.energy_gate;
  a.exact = s.exact_hessian;
  a.highlight = s.highlight;
  return a;
}

// A chunk pass: the chunk filter, then the chunk kernel over the chunks with work (a grid of
// every chunk; the CTAs past the count return at once).  Counts the filter's launch.
template <int MODE>
cudaError_t chunk_pass(Sim& s, const NarrowArgs& a) {
  // (the body-box kernel of the pass cleared the filter's count)
  constexpr int per = KA / 32;
  k_chunk_active<MODE><<<(s.nch + per - 1) / per, KA, 0, s.stream>>>(a);
  k_chunk_narrow<MODE><<<s.nch, CT, 0, s.stream>>>(a);
  ++s.launches;
  return cudaGetLastError();
}

}  // namespace

cudaError_t narrow(Sim& s, int mode, const double* A, const double* p, const double* A1, const double* p1,
                   const double* y0, const double* y1, const abd_states* st) {
  const NarrowArgs a = narrow_args(s, mode, A, p, A1, p1, y0, y1, st);
  if (mode == NARROW_ENERGY || mode == NARROW_CCD || mode == NARROW_CCD_LS || mode == NARROW_GH) {
    // energy, CCD and GH always run at DOFs; the energy needs the states (inertia terms)
    if (!a.affine || (mode == NARROW_ENERGY && !(st && st->A0 && st->Adot && st->p0 && st->pdot)))
      return cudaErrorInvalidValue;
    if (s.nch == 0) return cudaSuccess;
    if (mode == NARROW_ENERGY) {
      if (cudaError_t e = chunk_pass<NARROW_ENERGY>(s, a)) return e;
      if (a.fric) {  // the friction potential of the step's lagged contacts
        k_fric_energy<<<kRedBlocks, 128, 0, s.stream>>>(a);
        ++s.launches;
      }
    } else if (mode == NARROW_CCD || mode == NARROW_CCD_LS) {
      // (the body-box kernel of the pass cleared DS_NCCD and DS_NECAND)
      cudaError_t e = cudaSuccess;
      if (mode == NARROW_CCD_LS) {
        if (!a.y1) return cudaErrorInvalidValue;
        if (s.prof_events > 0 && record_event(s.prof_ev[0], s.stream))
          return cudaErrorUnknown;
        if ((e = chunk_pass<NARROW_CCD_LS>(s, a)) != cudaSuccess) return e;
        if (s.prof_events > 0 && record_event(s.prof_ev[1], s.stream))
          return cudaErrorUnknown;
        k_ccd_eval<true><<<kRedBlocks, 128, 0, s.stream>>>(a);
      } else {
        if ((e = chunk_pass<NARROW_CCD>(s, a)) != cudaSuccess) return e;
        k_ccd_eval<false><<<kRedBlocks, 128, 0, s.stream>>>(a);
      }
      ++s.launches;
    } else {
      // (the pass's pair scan cleared the per-pair contact counts, DS_NCONTACT, DS_NCCD and
      // DS_NACTP; the contact scan sets the offsets and scatter counters)
      cudaError_t e = cudaSuccess;
      if (s.gh_if_on) {
        // captured: the traversal and the evaluation of its candidates in an IF node
        // (k_sup_check sets its condition); the kernels in the body are not counted among the
        // pass's launches (they rarely run)
        s.gh_if_on = false;
        cudaGraph_t body = nullptr;
        if (add_conditional(s.stream, s.gh_if, cudaGraphCondTypeIf, &body) != ABD_OK) return cudaErrorUnknown;
        const int r = capture_body(s, body, s.cap_stream5, [&]() -> int {
          if (chunk_pass<NARROW_GH>(s, a) != cudaSuccess) return ABD_ERR_CUDA;
          k_gh_eval<<<kRedBlocks, 128, 0, s.stream>>>(a);
          return ABD_OK;
        });
        if (r != ABD_OK) return cudaErrorUnknown;
        s.launches -= 2;
      } else {
        if ((e = chunk_pass<NARROW_GH>(s, a)) != cudaSuccess) return e;
        k_gh_eval<<<kRedBlocks, 128, 0, s.stream>>>(a);
        ++s.launches;
      }
      k_gh_scan<<<kRedBlocks, 128, 0, s.stream>>>(a);
      ++s.launches;
      if (a.fric) {
        k_fric_pairs<<<kRedBlocks, 128, 0, s.stream>>>(a);
        ++s.launches;
      }
      const bool one_cta = s.cap_contacts <= kScanScatter;
      k_contact_scan<<<1, 1024, 0, s.stream>>>(s.cap_pairs, s.pair_cand, s.dstat, s.cap_contacts,
                                               one_cta ? s.contacts : nullptr, s.contacts_by_pair);
      if (!one_cta) {
        k_contact_scatter<<<blocks(s.cap_contacts, 256), 256, 0, s.stream>>>(s.cap_contacts, s.contacts,
                                                                             s.pair_cand, s.contacts_by_pair, s.dstat);
        ++s.launches;
      }
      constexpr int smem = NOUT * (int)sizeof(XSum);  // 40 KB, under the 48 KB default
      static_assert(smem + sizeof(double) * PT_WARPS * 5 * 24 + 256 <= 48 * 1024, "pair assembly shared memory");
      const int grid = s.cap_pairs < 4 * 148 ? s.cap_pairs : 4 * 148;
      if (s.exact_hessian && s.prm.ipc_full)
        k_pair_assemble<kAsmFullExact><<<grid, PT_THREADS, kExactSmem, s.stream>>>(a);
      else if (s.exact_hessian)
        k_pair_assemble<kAsmExact><<<grid, PT_THREADS, kExactSmem, s.stream>>>(a);
      else if (s.prm.ipc_full)
        k_pair_assemble<kAsmFull><<<grid, PT_THREADS, kExactSmem, s.stream>>>(a);
      else
        k_pair_assemble<kAsmRef><<<grid, PT_THREADS, smem, s.stream>>>(a);
      s.launches += 2;
    }
  } else {
    if (s.cap_pairs == 0) return cudaSuccess;
    k_pair_lists<<<s.cap_pairs, NT, 0, s.stream>>>(a);
  }
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t prepare_narrow(Sim& s) {
  (void)s;
  cudaError_t e = cudaFuncSetAttribute(k_pair_assemble<kAsmExact>, cudaFuncAttributeMaxDynamicSharedMemorySize, kExactSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_pair_assemble<kAsmFull>, cudaFuncAttributeMaxDynamicSharedMemorySize, kExactSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_pair_assemble<kAsmFullExact>, cudaFuncAttributeMaxDynamicSharedMemorySize, kExactSmem);
  return e;
}

cudaError_t gh_superset_check(Sim& s, const abd_states* st, int mode) {
  // a device-loop step's capture: a handle for the IF node narrow() puts around the GH tree
  // traversal
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s.stream, &cs);
  if (e != cudaSuccess) return e;
  s.gh_if_on = false;
  if (s.in_device_loop && cs == cudaStreamCaptureStatusActive) {
    if (make_handle(s.stream, &s.gh_if) != ABD_OK) return cudaErrorUnknown;
    s.gh_if_on = true;
  }
  k_sup_check<<<1, 1024, 0, s.stream>>>(s.n, st ? st->A0 : nullptr, st ? st->p0 : nullptr, s.q_last,
                                         s.dint + kSupHave, s.dint + kSupValid, st ? mode : 0, &s.box->step.it,
                                         s.gh_if, s.gh_if_on ? 1 : 0);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t body_gh(Sim& s, const abd_states& st, const double* A, const double* p, const double* y) {
  k_body_gh<<<s.n, BT, 0, s.stream>>>(body_args(s, &st, A, p, y, nullptr));
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t vg_list(Sim& s, const double* y0) {
  if (!(s.prm.ground_enabled && s.prm.enable_vg)) return cudaSuccess;
  k_vg_list<<<s.n, 128, 0, s.stream>>>(body_args(s, nullptr, nullptr, nullptr, y0, nullptr));
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t vg_list_swept(Sim& s, const double* y0, const double* y1) {
  if (!(s.prm.ground_enabled && s.prm.enable_vg)) return cudaSuccess;
  k_vg_list<<<s.n, 128, 0, s.stream>>>(body_args(s, nullptr, nullptr, nullptr, y0, y1));
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t export_system(Sim& s, double* off_dev, int* ij_dev, int cap) {
  const int np = s.n_pairs < cap ? s.n_pairs : cap;
  if (np == 0) return cudaSuccess;
  k_export_off<<<np, 128, 0, s.stream>>>(s.n_pairs, s.pair_active, s.fixed, s.offdiag, s.ij, off_dev, ij_dev, cap);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t update_dofs(Sim& s, const double* A, const double* p, const double* dq, double alpha, double* Aout,
                        double* pout) {
  k_update_dofs<<<blocks(s.n, 128), 128, 0, s.stream>>>(s.n, A, p, dq, alpha, Aout, pout, nullptr, nullptr, nullptr);
  ++s.launches;
  return cudaGetLastError();
}


// k_finish, unless the device loop stopped for a rerun (the states are then left as they
// were); the DOFs it ended with are kept for the next step's first GH pass
__global__ void k_finish_dev(int n, double dt, abd_states st, const int* dstat, double* q_last, int* sup_have) {
  if (dstat[DS_STATUS] & kRerunMask) return;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) {
    for (int k = 0; k < 3; ++k) {
      st.pdot[3 * b + k] = (st.p[3 * b + k] - st.p0[3 * b + k]) / dt;
      st.p0[3 * b + k] = st.p[3 * b + k];
      q_last[9 * (size_t)n + 3 * b + k] = st.p[3 * b + k];
    }
    for (int k = 0; k < 9; ++k) {
      st.Adot[9 * b + k] = (st.A[9 * b + k] - st.A0[9 * b + k]) / dt;
      st.A0[9 * b + k] = st.A[9 * b + k];
      q_last[9 * b + k] = st.A[9 * b + k];
    }
  }
  if (b == 0) *sup_have = 1;
}

cudaError_t finish_step_dev(Sim& s, const abd_states& st, double* xview) {
  k_finish_dev<<<blocks(s.n, 128), 128, 0, s.stream>>>(s.n, s.prm.dt, st, s.dstat, s.q_last, s.dint + kSupHave);
  ++s.launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !xview) return e;
  return transform(s, st.A0, st.p0, xview);
}

cudaError_t finish_step(Sim& s, const abd_states& st, double* xview) {
  k_finish<<<blocks(s.n, 128), 128, 0, s.stream>>>(s.n, s.prm.dt, st);
  ++s.launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !xview) return e;
  return transform(s, st.A0, st.p0, xview);
}

cudaError_t dots(Sim& s, const double* a, const double* b, const double* c, const double* d, double* out_dev,
                 cudaStream_t st) {
  static_assert(2 * kRedDot <= 2 * kRedBlocks, "dot partials fit two reduction slots");
  k_dots<<<kRedDot, 256, 0, st ? st : s.stream>>>(12 * s.n, a, b, c, d, s.partials + 10 * (size_t)kRedBlocks,
                                        s.red_count + 10, out_dev);
  ++s.launches;
  return cudaGetLastError();
}

}  // namespace abd
