// Broad phase: vertex transform, primitive / body boxes and body pairs.
//
// Replaces update_mesh_vertex (abd/abd.py:305-324, a host NumPy loop in the reference),
// the AABB kernels bvh_points / bvh_edges / bvh_triangles and their trajectory versions
// (abd/culling2.py:32-79, 229-280), the host-side body boxes (culling2.py:278-334) and the
// body-pair query intersection_bodies (culling2.py:337-351) with its append list
// (simulator/fenwick.py:108-170).
//
// Box rounding follows the reference exactly: points are converted to float32 and then
// dilated by float32(dhat); edges, triangles and bodies take the float64 min/max, dilate in
// float64 (dhat/2, 0, dhat/2) and round to float32.  Swept boxes unite the dilated boxes at
// y0 with the undilated float32 boxes at y1.
#include <cuda_runtime.h>

#include "abd_body.cuh"

namespace abd {

namespace {

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_transform(int V, const int* __restrict__ vbody, const double* __restrict__ x0,
                            const double* __restrict__ A, const double* __restrict__ p, double* __restrict__ x) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const int b = vbody[v];
  const double r0 = x0[3 * v], r1 = x0[3 * v + 1], r2 = x0[3 * v + 2];
  const double* a = A + 9 * b;
#pragma unroll
  for (int j = 0; j < 3; ++j) x[3 * v + j] = ((a[j] * r0 + a[3 + j] * r1) + a[6 + j] * r2) + p[3 * b + j];
}

struct VertexArgs {
  int V, n;
  const int* vbody;
  const double* x0;
  Dofs d[2];   // d[1] used when swept
  int swept;
  double *y0, *y1;
  unsigned long long* bnd;
  float* fdof;   // [n][2][12] FP32 DOFs (A row-major, p) of each set
  Mailbox* box;  // accumulators of the pass, cleared here
  int nslice;
  const int4* slice;  // vertex slices: (body, first vertex, count <= kSlice)
};

// DOFs of body b in set k: as given, or (A, p) - alpha dq (same arithmetic as k_update_dofs)
__device__ inline void body_dofs(const Dofs& d, int b, double M[12]) {
  if (!d.dq) {
#pragma unroll
    for (int k = 0; k < 9; ++k) M[k] = d.A[9 * b + k];
#pragma unroll
    for (int k = 0; k < 3; ++k) M[9 + k] = d.p[3 * b + k];
    return;
  }
  dofs_at(d.A, d.p, d.dq, b, *d.alpha, M);
}

// Warp-wide maximum of the 64-bit keys of all lanes: the maximum high word first, then the
// maximum low word among the lanes that hold it.
__device__ inline unsigned long long warp_max_key(unsigned long long key) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned hm = __reduce_max_sync(0xffffffffu, hi);
  const unsigned lm = __reduce_max_sync(0xffffffffu, hi == hm ? lo : 0u);
  return ((unsigned long long)hm << 32) | lm;
}

// One warp per vertex slice (at most kSlice vertices of one body, kSlice / 32 per lane):
// y0 = x(d[0]) (and y1 = x(d[1])) with the arithmetic of k_transform, and the body bounds:
// each lane takes the min / max of its vertices' coordinates, the warp reduces their
// order-preserving keys (the maximum key is the exact min / max) and lane 0 updates the
// body's keys atomically.  Then one thread per body: the body's DOFs of each set (written
// out when updated, and as FP32 copies for the traversal's node boxes).  Block 0 clears the
// pass's accumulators.
__global__ void __launch_bounds__(256, 4) k_vertex_broad(VertexArgs a) {
  const int w = (int)((blockIdx.x * 256 + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (blockIdx.x == 0) {
    if (threadIdx.x <= kXD) reinterpret_cast<long long*>(&a.box->energy)[threadIdx.x] = 0;
    if (threadIdx.x == 32) a.box->toi_key = 0;
    static_assert(sizeof(a.box->prof) / sizeof(unsigned long long) == 256, "one counter per thread");
    (&a.box->prof[0][0])[threadIdx.x] = 0;
  }
  const int nset = a.swept ? 2 : 1;
  if (w < a.nslice) {
    const int4 sl = a.slice[w];  // body, first vertex, vertices
    const int b = sl.x;
    constexpr int VPL = kSlice / 32;
    bool has[VPL];
    double r[VPL][3];
#pragma unroll
    for (int h = 0; h < VPL; ++h) {
      has[h] = lane + 32 * h < sl.z;
#pragma unroll
      for (int j = 0; j < 3; ++j) r[h][j] = has[h] ? a.x0[3 * (sl.y + lane + 32 * h) + j] : 0.0;
    }
    for (int k = 0; k < nset; ++k) {
      double M[12];
      body_dofs(a.d[k], b, M);
      double* y = k ? a.y1 : a.y0;
      unsigned long long* kb = a.bnd + 12 * (size_t)b + 6 * k;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double lo = INFINITY, hi = -INFINITY;
#pragma unroll
        for (int h = 0; h < VPL; ++h)
          if (has[h]) {
            const double c = xform(M, r[h][0], r[h][1], r[h][2], j);
            y[3 * (sl.y + lane + 32 * h) + j] = c;
            lo = fmin(lo, c);
            hi = fmax(hi, c);
          }
        const unsigned long long mlo = warp_max_key(max_key(-lo)), mhi = warp_max_key(max_key(hi));
        if (lane == 0) {
          atomicMax(&kb[j], mlo);
          atomicMax(&kb[3 + j], mhi);
        }
      }
    }
    return;
  }
  const int t = 32 * (w - a.nslice) + lane;
  if (t < a.n) {
    for (int k = 0; k < nset; ++k) {
      double M[12];
      body_dofs(a.d[k], t, M);
      if (a.d[k].dq) {
#pragma unroll
        for (int i = 0; i < 9; ++i) a.d[k].Aout[9 * t + i] = M[i];
#pragma unroll
        for (int i = 0; i < 3; ++i) a.d[k].pout[3 * t + i] = M[9 + i];
      }
      float4* f = reinterpret_cast<float4*>(a.fdof + 24 * (size_t)t + 12 * k);
      f[0] = make_float4((float)M[0], (float)M[1], (float)M[2], (float)M[3]);
      f[1] = make_float4((float)M[4], (float)M[5], (float)M[6], (float)M[7]);
      f[2] = make_float4((float)M[8], (float)M[9], (float)M[10], (float)M[11]);
    }
  }
}

// FP32 body boxes from the bounds (one thread per body), which are cleared for the next pass.
// With body_sup: also the affine images of the body's rest box under both DOF sets, dilated
// by dhat / 2, which hold the body's box at every DOF set between the two.
// Also clears, for the narrow pass that follows, its chunk filter's count (chunk_count) and,
// in a CCD pass, its candidate counters (cand_count: DS_NCCD, DS_NECAND).
__global__ void k_body_boxes(int n, unsigned long long* bnd, int swept, double dhh, Box* body_box,
                             const Box* body_rest, const float* fdof, Box* body_sup, int* chunk_count,
                             int* cand_count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  if (b == 0) {
    *chunk_count = 0;
    if (cand_count) cand_count[0] = cand_count[1] = 0;
  }
  unsigned long long k[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    k[i] = bnd[12 * (size_t)b + i];
    bnd[12 * (size_t)b + i] = 0ULL;
  }
  store_box(&body_box[b], body_box_of(k, swept, dhh));
  if (body_sup) {
    const float* m = fdof + 24 * (size_t)b;
    store_box(&body_sup[b], affine_box2(load_box(&body_rest[b]), m, swept ? m + 12 : nullptr, __double2float_ru(dhh)));
  }
}

// ---------------------------------------------------------------------------------------
// body pairs: overlap bit matrix, per-row prefix counts, then O(1) placement of every pair
// ---------------------------------------------------------------------------------------
constexpr int PR_THREADS = 128;  // one CTA per row of the overlap matrix, its 4 warps share the words
constexpr int PR_WORDS = 128;    // words of a row per round (one scan)

// Row I of the overlap matrix, one CTA: word w (J in [32 w, 32 w + 32)) is one warp's ballot
// of the box tests of its lanes (lane l tests J = 32 w + l, a coalesced load of the boxes),
// the CTA's warps taking the row's words in turn.  A block scan of the words' popcounts gives
// the per-row exclusive prefix (wpre); the CTA also writes the row counts -- all neighbours
// (rcnt) and neighbours J > I (ucnt) -- and the first kNbList neighbours in increasing order
// (nbr).  forced (or null): bits added to the row (the step's friction pairs).
__global__ void __launch_bounds__(PR_THREADS) k_pair_mask(int n, int W, const Box* __restrict__ body_box,
                                                          const uint32_t* __restrict__ forced, uint32_t* mask,
                                                          int* wpre, int* rcnt, int* ucnt, int* nbr) {
  __shared__ uint32_t sb[PR_WORDS];
  __shared__ int wsum[PR_THREADS / 32];
  __shared__ int slow;
  const int I = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const Box a = load_box(&body_box[I]);
  if (tid == 0) slow = 0;
  int carry = 0;
  for (int w0 = 0; w0 < W; w0 += PR_WORDS) {
    const int nw = min(PR_WORDS, W - w0);
#pragma unroll 4
    for (int wl = warp; wl < nw; wl += PR_THREADS / 32) {
      const int J = 32 * (w0 + wl) + lane;
      const bool hit = J < n && J != I && overlap(a, load_box(&body_box[J]));
      const uint32_t bits = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) sb[wl] = forced ? bits | forced[(size_t)I * W + w0 + wl] : bits;
    }
    __syncthreads();
    // exclusive scan of the words' popcounts (thread t: word w0 + t)
    const uint32_t bits = tid < nw ? sb[tid] : 0u;
    const int pc = __popc(bits);
    int incl = pc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = 0, total = 0;
#pragma unroll
    for (int k = 0; k < PR_THREADS / 32; ++k) {
      before += k < warp ? wsum[k] : 0;
      total += wsum[k];
    }
    if (tid < nw) {
      const int w = w0 + tid, pre = carry + before + incl - pc;
      mask[(size_t)I * W + w] = bits;
      wpre[(size_t)I * W + w] = pre;
      for (uint32_t m = bits; m && pre + (pc - __popc(m)) < kNbList; m &= m - 1)
        nbr[(size_t)I * kNbList + pre + (pc - __popc(m))] = 32 * w + __ffs(m) - 1;
      if (w == (I >> 5)) slow = pre + __popc(bits & ((1u << (I & 31)) - 1u));
    }
    carry += total;
    __syncthreads();  // sb and wsum are reused
  }
  if (tid == 0) {
    rcnt[I] = carry;
    ucnt[I] = carry - slow;  // bit I itself is never set
  }
}

// Single CTA: exclusive scans of the row counts into row_ptr / upper_ptr (index n gets the
// totals).  Totals land in dstat; capacities that are short raise ST_PAIR_OVERFLOW (the host
// grows and reruns).  Also clears the counters of the list / GH passes that follow.
__global__ void __launch_bounds__(1024) k_pair_scan(int n, const int* rcnt, const int* ucnt, int* row_ptr,
                                                    int* upper_ptr, int cap_pairs, int cap_adj, int* pair_cand,
                                                    int* dstat) {
  __shared__ int sh[2][33];
  __shared__ int carry[2];
  if (threadIdx.x == 0) carry[0] = carry[1] = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < n; c0 += 1024) {
    const int I = c0 + threadIdx.x;
    const int full = I < n ? rcnt[I] : 0, upper = I < n ? ucnt[I] : 0;
    int xf = full, xu = upper;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int yf = __shfl_up_sync(0xffffffffu, xf, o), yu = __shfl_up_sync(0xffffffffu, xu, o);
      if (lane >= o) {
        xf += yf;
        xu += yu;
      }
    }
    if (lane == 31) {
      sh[0][warp] = xf;
      sh[1][warp] = xu;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      int acc = carry[threadIdx.x];
      for (int w = 0; w < 32; ++w) {
        const int v = sh[threadIdx.x][w];
        sh[threadIdx.x][w] = acc;
        acc += v;
      }
      sh[threadIdx.x][32] = acc;
    }
    __syncthreads();
    if (I < n) {
      row_ptr[I] = sh[0][warp] + xf - full;
      upper_ptr[I] = sh[1][warp] + xu - upper;
    }
    __syncthreads();
    if (threadIdx.x < 2) carry[threadIdx.x] = sh[threadIdx.x][32];
    __syncthreads();
  }
  const int npairs = carry[1];
  for (int p = threadIdx.x; p < min(npairs, cap_pairs); p += 1024) pair_cand[4 * p + 1] = 0;
  if (threadIdx.x == 0) {
    row_ptr[n] = carry[0];
    upper_ptr[n] = npairs;
    dstat[DS_NADJ] = carry[0];
    dstat[DS_NPAIRS] = npairs;
    dstat[DS_PT_COUNT] = dstat[DS_EE_COUNT] = dstat[DS_VG_COUNT] = dstat[DS_ACTIVE] = 0;
    dstat[DS_NCONTACT] = 0;
    dstat[DS_NCCD] = 0;   // the GH pass's candidates
    dstat[DS_NACTP] = 0;  // its active pairs
    if (npairs > cap_pairs || carry[0] > cap_adj) atomicOr(&dstat[DS_STATUS], ST_PAIR_OVERFLOW);
  }
}

// number of set bits of row R in columns [0, c)
__device__ inline int bits_before(const uint32_t* mask, const int* wpre, int W, int R, int c) {
  const size_t w = (size_t)R * W + (c >> 5);
  const int b = c & 31;
  return wpre[w] + (b ? __popc(mask[w] & ((1u << b) - 1u)) : 0);
}

// one thread per mask word: every set bit J of row I lands at its sorted adjacency slot, and
// pairs I < J at their sorted pair index
__global__ void k_pair_fill(int n, int W, const uint32_t* __restrict__ mask, const int* __restrict__ wpre,
                            const int* __restrict__ row_ptr, const int* __restrict__ upper_ptr, int cap_pairs,
                            int cap_adj, int2* ij, int* adj_col, int* adj_pair) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * W) return;
  const int I = (int)(t / W), w = (int)(t % W);
  uint32_t m = mask[t];
  if (!m) return;
  int pos = row_ptr[I] + wpre[t];
  const int lowI = bits_before(mask, wpre, W, I, I);  // neighbours of I below I
  while (m) {
    const int bit = __ffs(m) - 1;
    m &= m - 1;
    const int J = 32 * w + bit;
    int pr;
    if (J > I) {
      pr = upper_ptr[I] + (pos - row_ptr[I]) - lowI;
      if (pr < cap_pairs) ij[pr] = make_int2(I, J);
    } else {
      pr = upper_ptr[J] + bits_before(mask, wpre, W, J, I) - bits_before(mask, wpre, W, J, J);
    }
    if (pos < cap_adj) {
      adj_col[pos] = J;
      adj_pair[pos] = pr;
    }
    ++pos;
  }
}

// ---------------------------------------------------------------------------------------
// fused per-body broad phase: one CTA per body
// ---------------------------------------------------------------------------------------
constexpr int BB = 256;

struct BroadArgs {
  int n, V, T, E;
  const int *voff, *toff, *eoff, *tris, *edges;
  const double* x0;
  const double *A, *p, *A1, *p1;
  double *y0, *y1;
  double dhh;
  unsigned long long* bnd;
  const int *tri_leaf, *edge_leaf;
  Box *tri_box, *edge_box;
  const int *tri_child, *edge_child, *tri_order, *edge_order, *tri_lvl, *edge_lvl, *tri_blvl, *edge_blvl;
  int refit;  // given positions: refit the internal boxes of the body subtrees
};

__device__ inline void refit_level(const int* child, const int* order, int k0, int k1, Box* box) {
  for (int k = k0 + (int)threadIdx.x; k < k1; k += BB) {
    const int node = order[k];
    const Box a = load_box_cg(&box[child[2 * node]]);
    const Box b = load_box_cg(&box[child[2 * node + 1]]);
    Box u;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u.lo[c] = fminf(a.lo[c], b.lo[c]);
      u.hi[c] = fmaxf(a.hi[c], b.hi[c]);
    }
    store_box(&box[node], u);
  }
}

__global__ void __launch_bounds__(BB) k_body_broad(BroadArgs a) {
  const int b = blockIdx.x;
  __shared__ double red[12][BB / 32];
  const int v0 = a.voff[b], v1 = a.voff[b + 1];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  double lo1[3] = {INFINITY, INFINITY, INFINITY}, hi1[3] = {-INFINITY, -INFINITY, -INFINITY};
  const bool swept = a.y1 != nullptr;
  // vertices: transform (same arithmetic as k_transform) and bounds
  for (int v = v0 + threadIdx.x; v < v1; v += BB) {
    double y[3], z[3];
    if (a.A) {
      const double r0 = a.x0[3 * v], r1 = a.x0[3 * v + 1], r2 = a.x0[3 * v + 2];
      const double* m = a.A + 9 * b;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        y[j] = ((m[j] * r0 + m[3 + j] * r1) + m[6 + j] * r2) + a.p[3 * b + j];
        a.y0[3 * v + j] = y[j];
      }
      if (swept && a.A1) {
        const double* m1 = a.A1 + 9 * b;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          z[j] = ((m1[j] * r0 + m1[3 + j] * r1) + m1[6 + j] * r2) + a.p1[3 * b + j];
          a.y1[3 * v + j] = z[j];
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < 3; ++j) y[j] = a.y0[3 * v + j];
    }
    if (swept && !a.A1) {
#pragma unroll
      for (int j = 0; j < 3; ++j) z[j] = a.y1[3 * v + j];
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      lo[j] = fmin(lo[j], y[j]);
      hi[j] = fmax(hi[j], y[j]);
      if (swept) {
        lo1[j] = fmin(lo1[j], z[j]);
        hi1[j] = fmax(hi1[j], z[j]);
      }
    }
  }
  // body box: warp then CTA reduction of the float64 bounds (min/max are exact)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[j] = fmin(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
      hi[j] = fmax(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
      lo1[j] = fmin(lo1[j], __shfl_xor_sync(0xffffffffu, lo1[j], o));
      hi1[j] = fmax(hi1[j], __shfl_xor_sync(0xffffffffu, hi1[j], o));
    }
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      red[j][warp] = lo[j];
      red[3 + j][warp] = hi[j];
      red[6 + j][warp] = lo1[j];
      red[9 + j][warp] = hi1[j];
    }
  __syncthreads();  // also makes this CTA's y0 / y1 writes visible to all its threads
  if (threadIdx.x == 0 && v1 > v0) {
    for (int j = 0; j < 3; ++j) {
      double l = red[j][0], h = red[3 + j][0], l1 = red[6 + j][0], h1 = red[9 + j][0];
      for (int w = 1; w < BB / 32; ++w) {
        l = fmin(l, red[j][w]);
        h = fmax(h, red[3 + j][w]);
        l1 = fmin(l1, red[6 + j][w]);
        h1 = fmax(h1, red[9 + j][w]);
      }
      a.bnd[12 * b + j] = max_key(-l);
      a.bnd[12 * b + 3 + j] = max_key(h);
      if (swept) {
        a.bnd[12 * b + 6 + j] = max_key(-l1);
        a.bnd[12 * b + 9 + j] = max_key(h1);
      }
    }
  }
  // given positions only: leaf boxes (the narrow phase computes them on the fly otherwise)
  if (!a.refit) return;
  for (int e = a.eoff[b] + threadIdx.x; e < a.eoff[b + 1]; e += BB)
    store_box(&a.edge_box[(a.E - 1) + a.edge_leaf[e]], edge_leaf_box(a.edges, a.y0, a.y1, e, a.dhh));
  for (int t = a.toff[b] + threadIdx.x; t < a.toff[b + 1]; t += BB)
    store_box(&a.tri_box[(a.T - 1) + a.tri_leaf[t]], tri_leaf_box(a.tris, a.y0, a.y1, t));
  __syncthreads();
  // refit the body's subtrees of both trees in global memory, one height level at a time
  const int te0 = a.tri_blvl[b], te1 = a.tri_blvl[b + 1];
  const int ee0 = a.edge_blvl[b], ee1 = a.edge_blvl[b + 1];
  const int ht = te1 - te0 - 1, he = ee1 - ee0 - 1;
  const int H = ht > he ? ht : he;
  for (int h = 1; h <= H; ++h) {
    if (h <= ht) refit_level(a.tri_child, a.tri_order, a.tri_lvl[te0 + h - 1], a.tri_lvl[te0 + h], a.tri_box);
    if (h <= he) refit_level(a.edge_child, a.edge_order, a.edge_lvl[ee0 + h - 1], a.edge_lvl[ee0 + h], a.edge_box);
    __syncthreads();
  }
}

}  // namespace

cudaError_t body_broad(Sim& s, const double* A, const double* p, const double* A1, const double* p1, double* y0,
                       double* y1, double dhh) {
  BroadArgs a;
  a.n = s.n;
  a.V = s.V;
  a.T = s.T;
  a.E = s.E;
  a.voff = s.voff;
  a.toff = s.toff;
  a.eoff = s.eoff;
  a.tris = s.tris;
  a.edges = s.edges;
  a.x0 = s.x0;
  a.A = A;
  a.p = p;
  a.A1 = A1;
  a.p1 = p1;
  a.y0 = y0;
  a.y1 = y1;
  a.dhh = dhh >= 0.0 ? dhh : s.prm.dhat * 0.5;
  a.bnd = s.body_bnd;
  a.tri_leaf = s.tri_tree.prim_leaf;
  a.edge_leaf = s.edge_tree.prim_leaf;
  a.tri_box = s.tri_tree.box;
  a.edge_box = s.edge_tree.box;
  a.tri_child = s.tri_tree.child;
  a.edge_child = s.edge_tree.child;
  a.tri_order = s.tri_tree.order;
  a.edge_order = s.edge_tree.order;
  a.tri_lvl = s.tri_tree.lvl;
  a.edge_lvl = s.edge_tree.lvl;
  a.tri_blvl = s.tri_tree.body_lvl;
  a.edge_blvl = s.edge_tree.body_lvl;
  a.refit = 1;
  s.swept = y1 != nullptr;
  if (A && (!y1 || A1)) {  // DOFs given: the vertex-parallel path
    Dofs d0, d1;
    d0.A = A;
    d0.p = p;
    d1.A = A1;
    d1.p = p1;
    return body_broad(s, &d0, y1 ? &d1 : nullptr, y0, y1);
  }
  k_body_broad<<<s.n, BB, 0, s.stream>>>(a);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t body_broad(Sim& s, const Dofs* d0, const Dofs* d1, double* y0, double* y1) {
  VertexArgs a;
  a.V = s.V;
  a.n = s.n;
  a.vbody = s.vbody;
  a.x0 = s.x0;
  a.d[0] = *d0;
  if (d1) a.d[1] = *d1;
  a.swept = d1 != nullptr;
  a.y0 = y0;
  a.y1 = y1;
  a.bnd = s.body_bnd;
  a.fdof = s.fdof;
  a.box = s.box;
  a.nslice = s.nslice;
  a.slice = s.slice;
  s.swept = a.swept;
  const long long warps = (long long)s.nslice + (s.n + 31) / 32;
  k_vertex_broad<<<blocks(32 * warps, 256), 256, 0, s.stream>>>(a);
  ++s.launches;
  return cudaGetLastError();
}

// child tables of the traversal (one thread per internal node): the node's children that
// are leaves and the children of its internal children, up to four
__global__ void k_child_tables(int N, const int* child, const int* leaf_prim, const Box* rest, Box* crest,
                               int4* ccode) {
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N - 1) return;
  const int L0 = N - 1;
  int code[4] = {kNoChild, kNoChild, kNoChild, kNoChild}, m = 0;
  Box zero{};
  for (int h = 0; h < 2; ++h) {
    const int c = child[2 * node + h];
    if (c >= L0) {
      store_box(&crest[4 * node + m], load_box(&rest[c]));
      code[m++] = ~leaf_prim[c - L0];
    } else {
      for (int g = 0; g < 2; ++g) {
        const int cc = child[2 * c + g];
        store_box(&crest[4 * node + m], load_box(&rest[cc]));
        code[m++] = cc >= L0 ? ~leaf_prim[cc - L0] : cc;
      }
    }
  }
  for (int i = m; i < 4; ++i) store_box(&crest[4 * node + i], zero);
  ccode[node] = make_int4(code[0], code[1], code[2], code[3]);
}

// Rest-frame boxes of all nodes: the undilated leaf boxes and refit of the rest positions,
// copied aside, and the traversal's child tables.  (The traversal dilates the boxes' world
// images by what each kind of primitive box needs.)
cudaError_t rest_boxes(Sim& s) {
  cudaError_t e = body_broad(s, nullptr, nullptr, nullptr, nullptr, s.x0, nullptr, 0.0);
  for (Tree* t : {&s.tri_tree, &s.edge_tree})
    if (e == cudaSuccess && t->N > 0)
      e = cudaMemcpyAsync(t->rest, t->box, sizeof(Box) * (size_t)(2 * t->N - 1), cudaMemcpyDeviceToDevice,
                          s.stream);
  for (Tree* t : {&s.tri_tree, &s.edge_tree})
    if (e == cudaSuccess && t->N > 1) {
      if ((e = cudaMalloc(&t->crest, sizeof(Box) * 4 * (size_t)(t->N - 1))) != cudaSuccess ||
          (e = cudaMalloc(&t->ccode, sizeof(int4) * (size_t)(t->N - 1))) != cudaSuccess)
        break;
      k_child_tables<<<blocks(t->N - 1, 256), 256, 0, s.stream>>>(t->N, t->child, t->leaf_prim, t->rest, t->crest,
                                                                   t->ccode);
      ++s.launches;
      e = cudaGetLastError();
    }
  // no pair pass follows: clear the bounds here (the pair mask clears them otherwise)
  if (e == cudaSuccess) e = cudaMemsetAsync(s.body_bnd, 0, sizeof(unsigned long long) * 12 * (size_t)s.n, s.stream);
  return e;
}

cudaError_t transform(Sim& s, const double* A, const double* p, double* x) {
  if (s.V == 0) return cudaSuccess;
  k_transform<<<blocks(s.V, 256), 256, 0, s.stream>>>(s.V, s.vbody, s.x0, A, p, x);
  ++s.launches;
  return cudaGetLastError();
}

// Body pairs I < J with overlapping boxes: the bit matrix and row counts, and when `full` the
// sorted ij list and the symmetric CSR adjacency (row I: neighbours in increasing J, with
// the pair index of {I, J}).  Counts stay on the device (dstat DS_NPAIRS / DS_NADJ); a short
// capacity raises ST_PAIR_OVERFLOW and leaves the lists incomplete, for the host to grow and
// rerun at its next read of dstat.
cudaError_t body_pairs(Sim& s, bool full, bool sup, const uint32_t* forced, bool ccd) {
  const int n = s.n, W = s.W;
  static_assert(DS_NECAND == DS_NCCD + 1, "candidate counters");
  k_body_boxes<<<blocks(n, 128), 128, 0, s.stream>>>(n, s.body_bnd, s.swept, 0.5 * s.prm.dhat, s.body_box,
                                                     s.body_rest, s.fdof, sup ? s.body_sup : nullptr,
                                                     s.chunk_act + s.nch, ccd ? s.dstat + DS_NCCD : nullptr);
  k_pair_mask<<<n, PR_THREADS, 0, s.stream>>>(n, W, sup ? s.body_sup : s.body_box, forced, s.pair_mask,
                                               s.pair_wpre, s.row_cnt, s.upper_cnt, s.nbr);
  s.launches += 2;
  if (full) {
    k_pair_scan<<<1, 1024, 0, s.stream>>>(n, s.row_cnt, s.upper_cnt, s.row_ptr, s.upper_ptr, s.cap_pairs, s.cap_adj,
                                          s.pair_cand, s.dstat);
    k_pair_fill<<<blocks((long long)n * W, 256), 256, 0, s.stream>>>(n, W, s.pair_mask, s.pair_wpre, s.row_ptr,
                                                                     s.upper_ptr, s.cap_pairs, s.cap_adj, s.ij,
                                                                     s.adj_col, s.adj_pair);
    s.launches += 2;
  }
  return cudaGetLastError();
}

}  // namespace abd
