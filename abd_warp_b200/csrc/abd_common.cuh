// Internal declarations shared by the CUDA translation units of libabd_b200.so.
//
// Build flags: -gencode arch=compute_100a,code=sm_100a -fmad=false.  Contraction of
// multiply-add into FMA is off so that the FP64 elementwise arithmetic rounds exactly
// like the CPU oracle; the heavy stages are memory- or latency-bound, not FMA-bound.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/abd_b200.h"
#include "abd_exact.cuh"

namespace abd {

// The last failed CUDA call of this thread, as "file:line: error name: description"
// (abd_error_detail returns it); note_error records one and returns e.
cudaError_t note_error(cudaError_t e, const char* file, int line);
const char* error_detail();
#define ABD_NOTE(x) ::abd::note_error((x), __FILE__, __LINE__)

// ---------------------------------------------------------------------------------------
// status bits written by kernels into the simulator's device status word
// ---------------------------------------------------------------------------------------
enum : int {
  ST_PT_OVERFLOW = 1,      // PT candidate list capacity exceeded (host grows and reruns)
  ST_EE_OVERFLOW = 2,      // EE candidate list capacity exceeded
  ST_PAIR_OVERFLOW = 4,    // body-pair capacity exceeded
  ST_STACK_OVERFLOW = 8,   // BVH traversal stack exceeded (should not happen)
  ST_SOLVER_NOCONV = 16,   // Krylov solve hit cg_max_iter
  ST_NAN = 32,             // non-finite value in the Newton system
  ST_VG_OVERFLOW = 64,     // VG list capacity exceeded
  ST_ACT_OVERFLOW = 128,   // active-pair list capacity exceeded (host grows and reruns)
  ST_CONTACT_OVERFLOW = 256,  // active-contact list capacity exceeded (host grows and reruns)
  ST_CCD_OVERFLOW = 512,   // CCD candidate list capacity exceeded (host grows and reruns)
  ST_ECAND_OVERFLOW = 1024,  // line-search candidate list capacity exceeded (grow and rerun)
  ST_LS_MORE = 2048,       // a line search needs more trials than one batch (the host finishes)
  ST_FRIC_OVERFLOW = 4096, // lagged friction contact capacity exceeded (host grows and reruns)
};
// the status bits after which the device-driven Newton loop stops and the host reruns the step
constexpr int kRerunMask = ST_PT_OVERFLOW | ST_EE_OVERFLOW | ST_PAIR_OVERFLOW | ST_VG_OVERFLOW | ST_ACT_OVERFLOW |
                           ST_CONTACT_OVERFLOW | ST_CCD_OVERFLOW | ST_ECAND_OVERFLOW | ST_LS_MORE |
                           ST_FRIC_OVERFLOW;

constexpr int kTraversalStack = 64;
constexpr int kNoChild = (int)0x80000000;  // unused slot of a node's child table

// ---------------------------------------------------------------------------------------
// small vector helpers (FP64)
// ---------------------------------------------------------------------------------------
struct d3 {
  double x, y, z;
};
__host__ __device__ inline d3 mk(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
__host__ __device__ inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline d3 cross(d3 a, d3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline d3 ld3(const double* p) { return {p[0], p[1], p[2]}; }

// f32 axis-aligned box, 32 B (one sector)
struct __align__(16) Box {
  float lo[3];
  float pad0;
  float hi[3];
  float pad1;
};

__device__ inline bool overlap(const Box& a, const Box& b) {
  return !(a.lo[0] > b.hi[0] || b.lo[0] > a.hi[0] || a.lo[1] > b.hi[1] || b.lo[1] > a.hi[1] ||
           a.lo[2] > b.hi[2] || b.lo[2] > a.hi[2]);
}

__device__ inline Box load_box(const Box* p) {
  const float4* q = reinterpret_cast<const float4*>(p);
  float4 a = __ldg(q), b = __ldg(q + 1);
  Box r;
  r.lo[0] = a.x; r.lo[1] = a.y; r.lo[2] = a.z; r.pad0 = 0.f;
  r.hi[0] = b.x; r.hi[1] = b.y; r.hi[2] = b.z; r.pad1 = 0.f;
  return r;
}
// L1-bypassing load for boxes written by other CTAs of the same kernel (refit)
__device__ inline Box load_box_cg(const Box* p) {
  const float4* q = reinterpret_cast<const float4*>(p);
  float4 a = __ldcg(q), b = __ldcg(q + 1);
  Box r;
  r.lo[0] = a.x; r.lo[1] = a.y; r.lo[2] = a.z; r.pad0 = 0.f;
  r.hi[0] = b.x; r.hi[1] = b.y; r.hi[2] = b.z; r.pad1 = 0.f;
  return r;
}
__device__ inline void store_box(Box* p, const Box& b) {
  float4* q = reinterpret_cast<float4*>(p);
  q[0] = make_float4(b.lo[0], b.lo[1], b.lo[2], 0.f);
  q[1] = make_float4(b.hi[0], b.hi[1], b.hi[2], 0.f);
}

// Leaf boxes with the reference's rounding (culling2.py:32-79, 229-280): edges take the FP64
// min / max of their end points, dilate by dhat/2 in FP64 and round to FP32; triangles are
// not dilated.  Swept boxes (y1 != null) add the undilated FP32 box at y1.
__device__ inline Box edge_leaf_box(const int* __restrict__ edges, const double* __restrict__ y0,
                                    const double* __restrict__ y1, int e, double dhh) {
  const int i0 = __ldg(&edges[2 * e]), i1 = __ldg(&edges[2 * e + 1]);
  Box B;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double u = y0[3 * i0 + k], w = y0[3 * i1 + k];
    B.lo[k] = (float)(fmin(u, w) - dhh);
    B.hi[k] = (float)(fmax(u, w) + dhh);
    if (y1) {
      const double u1 = y1[3 * i0 + k], w1 = y1[3 * i1 + k];
      B.lo[k] = fminf(B.lo[k], (float)fmin(u1, w1));
      B.hi[k] = fmaxf(B.hi[k], (float)fmax(u1, w1));
    }
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}
__device__ inline Box tri_leaf_box(const int* __restrict__ tris, const double* __restrict__ y0,
                                   const double* __restrict__ y1, int t) {
  const int i0 = __ldg(&tris[3 * t]), i1 = __ldg(&tris[3 * t + 1]), i2 = __ldg(&tris[3 * t + 2]);
  Box B;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double u = y0[3 * i0 + k], w = y0[3 * i1 + k], q = y0[3 * i2 + k];
    B.lo[k] = (float)(fmin(fmin(u, w), q) - 0.0);
    B.hi[k] = (float)(fmax(fmax(u, w), q) + 0.0);
    if (y1) {
      const double u1 = y1[3 * i0 + k], w1 = y1[3 * i1 + k], q1 = y1[3 * i2 + k];
      B.lo[k] = fminf(B.lo[k], (float)fmin(fmin(u1, w1), q1));
      B.hi[k] = fmaxf(B.hi[k], (float)fmax(fmax(u1, w1), q1));
    }
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}
// Point boxes: the FP32 position dilated by FP32 dhat (culling2.py:32-45); swept adds y1.
__device__ inline Box point_box(const double* y0, const double* y1, int v, float dhf) {
  Box B;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float c = (float)y0[3 * v + k];
    B.lo[k] = c - dhf;
    B.hi[k] = c + dhf;
    if (y1) {
      const float c1 = (float)y1[3 * v + k];
      B.lo[k] = fminf(B.lo[k], c1);
      B.hi[k] = fmaxf(B.hi[k], c1);
    }
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}

// the GPU's global nanosecond timer (kernel timing inside graphs, where events cannot go)
__device__ inline unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// order-preserving encoding of a non-negative double for atomicMin on 64-bit integers
__device__ inline unsigned long long dkey(double v) { return (unsigned long long)__double_as_longlong(v); }

// ---------------------------------------------------------------------------------------
// LBVH over the primitives of every body (one tree per primitive kind; each body's
// primitives form a subtree whose root is body_root[b])
// ---------------------------------------------------------------------------------------
struct Tree {
  int N = 0;              // leaves (primitives)
  int* child = nullptr;   // [N-1][2] node ids: internal 0..N-2, leaf = N-1+sorted position
  int* parent = nullptr;  // [2N-1]
  int* leaf_prim = nullptr;   // [N] sorted position -> primitive index
  int* prim_leaf = nullptr;   // [N] primitive index -> sorted position
  int* body_root = nullptr;   // [n] node id of the body's subtree, -1 if the body has none
  Box* box = nullptr;         // [2N-1] world boxes: internal nodes (refit), then leaves
  // [2N-1] node boxes in the body's rest frame (the refit of the rest positions: internal
  // nodes, then leaves); when the positions are x = A^T r + p, a node's world box is bounded
  // by the affine image of its rest box, which the traversal computes from the body's DOFs
  // instead of a refit
  Box* rest = nullptr;
  // per internal node, its up to four descendants one or two levels down (its children that
  // are leaves and the children of its internal children) as the traversal needs them, so
  // that one visit is one round of independent loads and the walk is half as deep: their
  // rest boxes [N-1][4] and codes [N-1] (node id if internal, ~primitive if a leaf,
  // kNoChild for an unused slot)
  Box* crest = nullptr;
  int4* ccode = nullptr;
  // per-body bottom-up refit schedule: the internal nodes of body b's subtree grouped by
  // height, order[lvl[body_lvl[b] + h - 1] .. lvl[body_lvl[b] + h]) for h = 1..heights
  int* order = nullptr;       // [N-1]
  int* lvl = nullptr;         // [sum over bodies of (heights + 1)]
  int* body_lvl = nullptr;    // [n+1]
  int max_height = 0;         // internal levels of the deepest body subtree (host)
};

// ---------------------------------------------------------------------------------------
// the simulator
// ---------------------------------------------------------------------------------------
struct Mailbox;

constexpr int kMaxCluster = 12;  // bodies per preconditioner cluster: 144 x 144 doubles fit in
                                 // shared memory

// scratch of the clustering kernel, [n] each
struct ClusterWork {
  int *label = nullptr, *size = nullptr, *to = nullptr, *cidx = nullptr, *fill = nullptr;
  unsigned long long* best = nullptr;
};
inline size_t cluster_work_bytes(int n) { return (5 * sizeof(int) + sizeof(unsigned long long)) * (size_t)n; }
inline ClusterWork cluster_work_at(void* base, int n) {
  ClusterWork w;
  w.best = static_cast<unsigned long long*>(base);
  int* q = reinterpret_cast<int*>(w.best + n);
  w.label = q;
  w.size = q + n;
  w.to = q + 2 * (size_t)n;
  w.cidx = q + 3 * (size_t)n;
  w.fill = q + 4 * (size_t)n;
  return w;
}

// A lagged friction contact: the step start's closest-point weights w, tangent basis P (3x2,
// row-major) and normal force lam, the four points there (xt) and their vertex ids; the first
// group (the point; edge a) moves with body I.
struct FricRec {
  double w[4], P[6], lam;
  double xt[12];
  int ids[4];
  int I, J, kind, pad;
};

// one captured pass (see abd_graph.cuh)
struct GraphSlot {
  cudaGraphExec_t exec = nullptr;
  uint64_t key = 0;
  long long nlaunch = 0;  // kernels per replay
};

struct Sim {
  cudaStream_t stream = 0;
  abd_params prm{};
  int n = 0, V = 0, T = 0, E = 0;
  int max_body_v = 0, max_body_t = 0, max_body_e = 0;
  long long launches = 0;
  int host_status = 0;   // status bits raised on the host (solver non-convergence)

  // mesh (device)
  int *voff = nullptr, *toff = nullptr, *eoff = nullptr;
  int *vbody = nullptr, *tbody = nullptr, *ebody = nullptr;
  int *tris = nullptr, *edges = nullptr;
  double *x0 = nullptr, *mass = nullptr, *I0 = nullptr;
  int* fixed = nullptr;
  Tree tri_tree, edge_tree;

  // positions
  double *x = nullptr, *xk = nullptr;
  Box* body_box = nullptr;  // [n] FP32 body boxes of the last pass (written by the pair mask)
  Box* body_rest = nullptr; // [n] rest-frame box of each body's vertices
  // [n] boxes holding the body's box at every DOF set between the two of a swept pass (the
  // line-search candidate pass culls its body pairs with them)
  Box* body_sup = nullptr;
  unsigned long long* body_bnd = nullptr;  // [n][12] exact bounds as max-keys (broad phase)
  int swept = 0;            // the last broad phase was swept

  // body pairs
  int W = 0;                       // mask words per row
  uint32_t* pair_mask = nullptr;   // [n][W]
  int* pair_wpre = nullptr;        // [n][W] popcounts, then per-row exclusive prefix
  int *row_ptr = nullptr, *upper_ptr = nullptr;  // [n+1]
  int cap_pairs = 0, cap_adj = 0;
  int2* ij = nullptr;              // [cap_pairs]
  int *adj_col = nullptr, *adj_pair = nullptr;   // [cap_adj]
  int n_pairs = 0, n_adj = 0;      // host copies, valid after a read of dstat
  // active pairs (contacts, both bodies free) with their coupling weight, for the
  // preconditioner's clustering on the device: int4 (pair, I, J, weight bits)
  int cap_act = 0;
  int4* act_pairs = nullptr;       // device [cap_act]

  // per-body work chunks of the energy / CCD narrow passes: (body, first item) with items
  // [0, nV) the body's points and [nV, nV + nE) its edges, kChunk items per chunk
  int nch = 0;
  int2* chunk = nullptr;           // [nch]
  int* chunk_act = nullptr;        // [nch + 1] the chunks of a narrow pass with work, then their count
  // CTAs of the solver's kernels, at most kRedBlocks (their dot products are exact sums of
  // per-CTA partials, the same for any grid): the row kernels one per 8 body rows (a warp per
  // row), the cluster kernels one per 4 bodies (a warp per cluster, at most one each)
  int red_grid = 1, cl_grid = 1;
  // lagged friction (friction_mu > 0): the step's contacts, and its body pairs as bits of the
  // overlap matrix that every GH pass of the step adds; fric_lag: the host loop's first GH pass
  // of a step (the device loop lags at its first Newton iteration)
  FricRec* fric = nullptr;
  int cap_fric = 0;
  uint32_t* fric_mask = nullptr;   // [n][W]
  int fric_lag = 0;
  Box* chunk_box = nullptr;        // [nch] rest-frame box of each chunk's items
  int* vperm = nullptr;            // [V] vertices of each body in Morton order (chunk items)
  // vertex slices of the line-search bounds: (body, first vertex, count), count <= kSlice
  int nslice = 0;
  int4* slice = nullptr;
  XSum* energy_acc = nullptr;      // = &box->energy
  // everything the host reads after a pass, in one device block (one copy per sync)
  Mailbox* box = nullptr;          // device
  Mailbox* hbox = nullptr;         // pinned host mirror
  int* row_cnt = nullptr;          // [n] neighbours of each body (pair mask)
  int* nbr = nullptr;              // [n][kNbList] first neighbours of each body (pair mask)
  float* fdof = nullptr;           // [n][2][12] FP32 DOFs of the last broad phase
  int* upper_cnt = nullptr;        // [n] neighbours J > I
  // device pass parameters: [0] trial step, [1] = 1, [kParK] trials of a line-search batch,
  // [kParAlpha + k] their step lengths
  double* dpar = nullptr;
  // device integers: [0] preconditioner clusters, [kSupHave] the line-search candidates of the
  // last step's last CCD pass are kept, [kSupValid] they hold the current GH pass's candidates
  int* dint = nullptr;
  double* q_last = nullptr;        // [12 n] the DOFs (A, then p) the last step ended with
  int* highlight = nullptr;        // [n] contact flags of the last GH pass (k_body_gh)
  // captured passes: CCD bound (with events for profiling), GH, the Krylov solve, line-search
  // batches (step lengths from the host or from the CCD pass on the device)
  cudaStream_t cap_stream = nullptr;
  cudaStream_t cap_stream2 = nullptr;  // captures the bodies of conditional (loop) nodes
  GraphSlot g_ccd, g_ccd_ev, g_gh, g_gh0, g_kinit, g_ls, g_ls_dev;
  GraphSlot g_step;                // a whole time step as a device loop
  GraphSlot g_kadj;                // the adjoint's Krylov solve
  double* adj_x = nullptr;         // [12 n] the adjoint solve's unknown lambda
  cudaStream_t cap_stream3 = nullptr, cap_stream4 = nullptr;  // capture the loop's bodies
  // side branches of a pass (the GH pass's clustering, the CCD pass's dot products): a stream
  // joins the capture it forks from until that capture ends, so the device loop gives each
  // capture scope its own (fork_a: the Newton body, fork_b: its IF body); null: cap_stream2
  cudaStream_t fork_a = nullptr, fork_b = nullptr, side = nullptr;
  // A device-loop step (in_device_loop: its capture is in progress) puts the passes that most
  // Newton iterations skip in IF nodes: the GH pass's tree traversal (needed only when the
  // kept line-search candidates do not cover the pass; the superset check sets the condition)
  // and the inverse of clusters of more than one body.  (The host loop launches them, and they
  // return at once.)  gh_if_on: the GH handle belongs to the capture in progress
  cudaStream_t cap_stream5 = nullptr;  // captures those IF nodes' bodies
  cudaGraphConditionalHandle gh_if = 0;
  bool in_device_loop = false, gh_if_on = false;
  double* dq_save = nullptr;       // [12 n] dq at the start of a device-loop step (for a rerun)
  long long step_launch[3] = {0, 0, 0};  // kernels of a step graph: outside the loops, per
                                         // Newton iteration, per Krylov iteration
  int gh_energy = 0;               // the GH pass also sums the energy at its DOFs
  int exact_hessian = 0;           // the GH pass assembles the exact Hessian (the adjoint's)
  const int* energy_gate = nullptr;  // device loop: the GH pass sums the energy only while this
                                     // device counter (the Newton iteration) is 0
  unsigned prm_version = 0;        // bumped by set_params (parameters are kernel arguments)
  unsigned cap_gen = 0;            // bumped by every capacity growth (buffers are kernel arguments)
  // kernel profiling of the line-search candidate pass's narrow kernel: CUDA events around
  // it (recorded as graph nodes), its duration and algorithmic bytes accumulated per pass
  int prof_on = 0;                 // 0 off, 1 time every kProfEvery-th pass, 2 time and count all
  int prof_events = 0;             // this pass records the events
  long long prof_tick = 0;
  cudaEvent_t prof_ev[2] = {nullptr, nullptr};
  // fork / join of a side branch in a captured pass (the CCD pass's dot products)
  cudaEvent_t fork_ev[2] = {nullptr, nullptr};
  bool fork_open = false;
  double prof_ms = 0.0, prof_bytes = 0.0;
  long long prof_launches = 0;
  double* hpar = nullptr;          // pinned staging of dpar

  // candidate lists
  int cap_pt = 0, cap_ee = 0, cap_vg = 0;
  int *pt_list = nullptr, *ee_list = nullptr, *vg_list = nullptr;  // [cap][5], [cap][5], [cap][2]
  int* pair_cand = nullptr;        // [cap_pairs][4] PT base, PT count, EE base, EE count

  // per-pair scratch of the contact assembly
  double *offdiag = nullptr;       // [cap_pairs][2][144]: H_IJ, H_JI
  double *pdiag = nullptr;         // [cap_pairs][2][144]: contributions to diag I, diag J
  double *pgrad = nullptr;         // [cap_pairs][2][12]
  int* pair_active = nullptr;      // [cap_pairs] active contacts of the pair
  // active contacts of the GH pass: int4 (pair, type | swap << 1, primitive a, primitive b),
  // appended in any order, then grouped by pair (pair_cand[4p]: offset, count, fill)
  int cap_contacts = 0;
  int4 *contacts = nullptr, *contacts_by_pair = nullptr;
  int cap_ccd = 0;
  int4* ccd_cand = nullptr;        // CCD candidates (type, primitive a, primitive b)
  // line-search candidates of the last CCD pass: every PT / EE pair that can be in the
  // culled set at some DOFs between its two sets (type, primitive a, primitive b)
  int cap_ecand = 0;
  int4* ecand = nullptr;
  int list_counts[4] = {0, 0, 0, 0};  // pairs, PT, EE, VG of the last list culling
  double* pair_val = nullptr;      // [cap_pairs] energy or toi per pair


  // Newton system
  double *g = nullptr, *dq = nullptr, *diag = nullptr;  // [n][12], [n][12], [n][144]
  // Krylov work vectors [n][12]
  double *r = nullptr, *rh = nullptr, *pv = nullptr, *v = nullptr, *y = nullptr, *s = nullptr, *z = nullptr,
         *t = nullptr;
  // preconditioner clusters (contact-coupled bodies, <= cluster_max each), formed on the
  // device: the tables live in one device block (ClusterTables layout)
  int cl_smem = 0;                               // dynamic shared memory opted in for the inverse
  ClusterWork cl_work;                           // the clustering kernel's scratch ([n] each)
  void* cl_work_buf = nullptr;
  void* cl_tab = nullptr;
  int *cl_ptr = nullptr, *cl_body = nullptr;     // [ncl+1], [n]
  int *body_cl = nullptr, *ncl_dev = nullptr;    // [n], [1]
  long long* cl_off = nullptr;                   // [ncl+1] offsets into cl_inv (doubles)
  double* cl_inv = nullptr;                      // dense inverses of the cluster systems
                                                 // (144 kMaxCluster n doubles: the most any
                                                 // clustering needs)
  XSum* partials = nullptr; // exact reduction partials [kRedSlots][kRedBlocks]
  int* red_count = nullptr;        // [kRedSlots] CTAs done per reduction (last CTA finishes)
  double* scal = nullptr;          // solver scalars
  int* dstat = nullptr;            // = box->dstat: [0] status, [1..] counters
  int* hstat = nullptr;            // pinned: [0, 16) mirror of dstat, [16, 32) host scratch
  double* hval = nullptr;          // pinned host scalars
  unsigned long long* dmin = nullptr;  // = &box->toi_key
};

// Records ev on st: while st is capturing, as a graph node that records it on every replay
// (which the host can wait for), else directly
inline cudaError_t record_event(cudaEvent_t ev, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const cudaError_t e = cudaStreamIsCapturing(st, &cs);
  if (e != cudaSuccess) return e;
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
                                             : cudaEventRecord(ev, st);
}

// The preconditioner's cluster tables, laid out the same in the pinned staging block and on
// the device so that one copy moves them: the cluster count, cl_ptr [n+1], cl_body [n] and
// body_cl [n] (ints), then cl_off [n+1] (long longs, 8-byte aligned)
struct ClusterTables {
  int *ncl, *cl_ptr, *cl_body, *body_cl;
  long long* cl_off;
  size_t off_bytes;  // byte offset of cl_off
  size_t bytes_through(int ncl_) const { return off_bytes + sizeof(long long) * ((size_t)ncl_ + 1); }
};
inline size_t cluster_tables_bytes(int n) {
  return ((sizeof(int) * (3 * (size_t)n + 3) + 7) & ~(size_t)7) + sizeof(long long) * ((size_t)n + 1);
}
inline ClusterTables cluster_tables_at(void* base, int n) {
  ClusterTables t;
  int* b = static_cast<int*>(base);
  t.ncl = b;
  t.cl_ptr = b + 2;
  t.cl_body = b + 3 + n;
  t.body_cl = b + 3 + 2 * (size_t)n;
  t.off_bytes = (sizeof(int) * (3 * (size_t)n + 3) + 7) & ~(size_t)7;
  t.cl_off = reinterpret_cast<long long*>(static_cast<char*>(base) + t.off_bytes);
  return t;
}

constexpr int kRedBlocks = 296;   // 2 x 148 SMs: fixed grid of every reduction kernel
constexpr int kChunk = 128;       // items per chunk of the energy / CCD narrow passes
constexpr int kNbList = 32;       // neighbours per body listed by the pair mask
constexpr int kRedSlots = 12;
constexpr int kLsMax = 16;        // line-search trials evaluated per batch
constexpr int kSupHave = 1;       // dint slots (see Sim::dint)
constexpr int kSupValid = 2;
constexpr int kSlice = 96;        // vertices per warp of k_vertex_broad (three per lane)
constexpr int kParK = 4;          // dpar slot of a batch's trial count
constexpr int kParAlpha = 5;      // dpar slots of its step lengths
constexpr int kParAcc = kParAlpha + kLsMax;  // dpar slot of the accepted step length
constexpr int kNPar = kParAcc + 1;

// dstat layout
enum : int {
  DS_STATUS = 0,
  DS_PT_COUNT = 1,
  DS_EE_COUNT = 2,
  DS_VG_COUNT = 3,
  DS_ACTIVE = 4,
  DS_KRYLOV_RUNS = 5,  // Krylov loop body executions of the current solve (a watchdog)
  DS_SOLVER_ITERS = 6,
  DS_NPAIRS = 7,     // body pairs of the last culling pass
  DS_NADJ = 8,       // adjacency entries (2 x pairs)
  DS_NACTP = 9,      // active pairs appended by the pair assembly
  DS_NCONTACT = 12,  // active contacts appended by the GH pass
  DS_IT = 13,        // Krylov iteration counter (device-side, for replayed blocks)
  DS_NCCD = 14,      // CCD candidates appended by the CCD pass
  DS_NECAND = 15,    // line-search candidates appended by the CCD pass
  DS_NFRIC = 16,     // lagged friction contacts of the step (its first GH pass appends them)
  DS_NSLOTS = 17
};


// Counters of a time step run as a device loop (the step info, kept on the device), and the
// kernel timing of the CCD pass's narrow kernel by the GPU's global timer.
struct StepDev {
  int it;            // Newton iterations done (the loop's counter)
  int lin, ls;       // Krylov iterations, line-search trials
  int n_pt, n_ee, n_vg, n_ij, n_active;
  double E0;         // energy of the current iterate
  double alpha, toi; // the last accepted step length and raw time of impact
  unsigned long long t0, t1;       // first start and last end (ns) of the current narrow launch
  unsigned long long prof_ns, prof_n;  // their accumulated durations and launches
  double prof_bytes;               // algorithmic bytes of those launches (profiling mode 2)
};

// The host's view of a pass: status word and counters, the exact energy, the minimum time of
// impact and the Newton dot products, contiguous so that one copy brings them all.
struct Mailbox {
  int dstat[DS_NSLOTS];
  XSum energy;
  unsigned long long toi_key;  // complemented bits of the minimum time of impact (0: none)
  double dots[2];              // dq.g, g.g
  XSum ls_energy[kLsMax];      // exact energies of a line-search batch's trials
  // work counters of the line-search candidate pass's narrow kernel (kernel profiling only),
  // spread over 32 rows against atomic contention: [row][PF_*]
  unsigned long long prof[32][8];
  StepDev step;
};

// counters of the line-search candidate pass's narrow kernel (kernel profiling): the data it
// reads and writes, per kind of access
enum : int {
  PF_POINT = 0,      // point queries: FP64 rest position (24 B)
  PF_EDGE = 1,       // edge queries: leaf position + rest box (36 B)
  PF_NEIGHBOUR = 2,  // (chunk, neighbour) records: body box, FP32 DOFs of both sets, roots (140 B)
  PF_NODE = 3,       // internal tree entries tested: rest box + child code (36 B)
  PF_TRI = 4,        // triangle leaf entries tested: rest box + code (36 B)
  PF_EDGELEAF = 5,   // edge leaf entries tested: rest box + code (36 B)
  PF_CAND = 6,       // candidates appended (16 B written)
  PF_N = 7
};
constexpr double kProfBytes[PF_N] = {24.0, 36.0, 140.0, 36.0, 36.0, 36.0, 16.0};


// ---------------------------------------------------------------------------------------
// launchers (each returns cudaError_t of the launch)
// ---------------------------------------------------------------------------------------
// lbvh.cu
cudaError_t build_tree(Sim& s, Tree& tr, int N, const int* prim_body_dev, const double* centroid_dev,
                       const int* prim_off_host);
cudaError_t radix_sort_pairs(Sim& s, unsigned long long* keys, int* vals, unsigned long long* keys_tmp,
                             int* vals_tmp, int N, int key_bits);

// broad.cu
cudaError_t transform(Sim& s, const double* A, const double* p, double* x);
// DOFs of a pass: (A, p) as given, or, when dq is set, (A, p) - alpha dq with alpha read from
// device memory, written to (Aout, pout) by the broad phase (update_qk, abd.py:154-157)
struct Dofs {
  const double *A = nullptr, *p = nullptr;
  const double* dq = nullptr;
  const double* alpha = nullptr;  // device scalar
  double *Aout = nullptr, *pout = nullptr;
  const double* Aeff() const { return dq ? Aout : A; }
  const double* peff() const { return dq ? pout : p; }
};

// Broad phase.  With DOFs (d0, and d1 for swept boxes): y0 = x(d0) (and y1 = x(d1)), one
// thread per vertex, and the exact body bounds; the traversal bounds internal nodes by the
// affine images of their rest boxes.  Without (d0 == null): y0 / y1 are given positions, the
// leaf boxes are stored and the body subtrees refit level by level.
cudaError_t body_broad(Sim& s, const Dofs* d0, const Dofs* d1, double* y0, double* y1);
// (dhh: the edge dilation, default dhat / 2)
cudaError_t body_broad(Sim& s, const double* A, const double* p, const double* A1, const double* p1, double* y0,
                       double* y1, double dhh = -1.0);
// body pairs: full (mask, scan, fill: the sorted pair list and the adjacency with pair
// indices) or mask only (row counts and the bit matrix, all the energy and CCD passes need)
// sup: cull with the boxes over every DOF set between the two of a swept pass (body_sup)
// forced: [n][W] bits added to the overlap matrix (the step's friction pairs), or null;
// ccd: a CCD pass follows (its candidate counters are cleared)
cudaError_t body_pairs(Sim& s, bool full, bool sup = false, const uint32_t* forced = nullptr, bool ccd = false);
// rest-frame internal node boxes of both trees (once, at creation)
cudaError_t rest_boxes(Sim& s);

// narrow.cu
// CCD_LS: the CCD pass that also collects the line-search candidates (ecand)
enum NarrowMode { NARROW_GH = 0, NARROW_ENERGY = 1, NARROW_CCD = 2, NARROW_LISTS = 3, NARROW_CCD_LS = 4 };
// A != null: internal node boxes are the affine images of the rest boxes under (A, p) (united
// with (A1, p1) when swept); A == null: the refit boxes.  y0 / y1 are the positions.
// ENERGY (at DOFs A, p; st for the inertia terms) adds the pass's whole energy -- contacts,
// vertex-ground and inertia -- to energy_acc; CCD (at DOFs) maximises dmin[0] with the
// complemented bits of every time of impact below 1 (contacts and vertex-ground).
cudaError_t narrow(Sim& s, int mode, const double* A, const double* p, const double* A1, const double* p1,
                   const double* y0, const double* y1, const abd_states* st = nullptr);
cudaError_t body_gh(Sim& s, const abd_states& st, const double* A, const double* p, const double* y);
cudaError_t prepare_narrow(Sim& s);  // kernel attributes (once, at creation)
// Whether the next GH pass may take its candidates from the kept line-search candidates
// (dint[kSupValid]): mode 0 no, 2 yes (a later Newton iteration of the step), 1 when they
// were kept (dint[kSupHave]) and the step starts from the DOFs the last step ended with.
cudaError_t gh_superset_check(Sim& s, const abd_states* st, int mode);
// mode 3 (the device loop): 1 at the step's first Newton iteration, else 2
cudaError_t vg_list(Sim& s, const double* y0);
cudaError_t export_system(Sim& s, double* off_dev, int* ij_dev, int cap);
cudaError_t update_dofs(Sim& s, const double* A, const double* p, const double* dq, double alpha, double* Aout,
                        double* pout);
cudaError_t finish_step(Sim& s, const abd_states& st, double* xview);
// exact dot products a.b (and c.d when c != null) of [n][12] vectors into out_dev[0], [1]
// (reduction slots 10 and 11), on stream st (the pass's stream when null)
cudaError_t dots(Sim& s, const double* a, const double* b, const double* c, const double* d, double* out_dev,
                 cudaStream_t st = nullptr);

// linesearch.cu
// Energies at (A, p) - alpha_k dq for the dpar[kParK] step lengths dpar[kParAlpha + k] in
// [0, 1], from the candidates of the last CCD_LS pass between (A, p) and (A, p) - dq, into
// the mailbox's ls_energy[k].  from_ccd: directly after that pass, which cleared ls_energy;
// the trials then come from its time of impact and are written to dpar.
cudaError_t ls_energies(Sim& s, const abd_states& st, const double* A, const double* p, bool from_ccd);

// solver.cu
// The preconditioner: cluster_tables forms the clusters on the device from the last GH pass's
// active-pair list (on stream st, the pass's stream when null); cluster_inverse inverts each
// cluster's system; build_preconditioner does both.  The last two return an ABD status.
cudaError_t cluster_tables(Sim& s, cudaStream_t st);
int cluster_inverse(Sim& s);
int build_preconditioner(Sim& s);
int prepare_solver(Sim& s);
// returns ABD status; iters == null: enqueue only (krylov_outcome after the next mailbox read)
int krylov_solve(Sim& s, double* x, int* iters, GraphSlot* slot = nullptr);
int krylov_outcome(Sim& s);                       // iterations of the last solve
// Enqueues a solve (its set-up kernel and the WHILE node of its iterations) into the graph
// being captured on s.stream, for the device-driven Newton loop; the solve adds its outcome to
// the mailbox's step counters where it ends.
int krylov_issue(Sim& s, double* x);

// newton.cu: the kernels of the device-driven Newton loop (abd_step when the parameters'
// newton_loop is 0).  Each enqueues on s.stream.
// the step's start: q and the line-search origin from q0, the warm start kept for a rerun,
// the step's counters cleared, the Newton loop's condition set
cudaError_t step_begin(Sim& s, const abd_states& st, cudaGraphConditionalHandle h);
cudaError_t gate_no_overflow(Sim& s, cudaGraphConditionalHandle h);
cudaError_t ls_accept(Sim& s);
// the loop's end: (A, p) -= alpha dq with the accepted alpha on the device, also into (Ak, pk),
// then the convergence test
cudaError_t newton_end(Sim& s, const abd_states& st, cudaGraphConditionalHandle h);
cudaError_t finish_step_dev(Sim& s, const abd_states& st, double* xview);
// the adjoint step (abd_adjoint_step): its right-hand side into g, its outputs from lambda
cudaError_t adjoint_rhs(Sim& s, const double* qb, const double* qdb);
cudaError_t adjoint_out(Sim& s, const double* lam, const double* qdb, double* qb_out, double* qdb_out);

}  // namespace abd
