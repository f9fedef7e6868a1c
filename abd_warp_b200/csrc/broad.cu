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

#include "abd_common.cuh"
#include "abd_scan.cuh"

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

__global__ void k_edge_boxes(int E, const int* __restrict__ edges, const double* __restrict__ y0,
                             const double* __restrict__ y1, double dhh, const int* __restrict__ prim_leaf, Box* box) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const int a = edges[2 * e], b = edges[2 * e + 1];
  Box B;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double u = y0[3 * a + k], w = y0[3 * b + k];
    B.lo[k] = (float)(fmin(u, w) - dhh);
    B.hi[k] = (float)(fmax(u, w) + dhh);
    if (y1) {
      const double u1 = y1[3 * a + k], w1 = y1[3 * b + k];
      B.lo[k] = fminf(B.lo[k], (float)fmin(u1, w1));
      B.hi[k] = fmaxf(B.hi[k], (float)fmax(u1, w1));
    }
  }
  store_box(&box[(E - 1) + prim_leaf[e]], B);
}

__global__ void k_tri_boxes(int T, const int* __restrict__ tris, const double* __restrict__ y0,
                            const double* __restrict__ y1, const int* __restrict__ prim_leaf, Box* box) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const int a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
  Box B;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double u = y0[3 * a + k], w = y0[3 * b + k], q = y0[3 * c + k];
    B.lo[k] = (float)(fmin(fmin(u, w), q) - 0.0);
    B.hi[k] = (float)(fmax(fmax(u, w), q) + 0.0);
    if (y1) {
      const double u1 = y1[3 * a + k], w1 = y1[3 * b + k], q1 = y1[3 * c + k];
      B.lo[k] = fminf(B.lo[k], (float)fmin(fmin(u1, w1), q1));
      B.hi[k] = fmaxf(B.hi[k], (float)fmax(fmax(u1, w1), q1));
    }
  }
  store_box(&box[(T - 1) + prim_leaf[t]], B);
}

// one CTA per body: float64 min/max over its vertices (exact, order independent)
__global__ void k_body_boxes(int n, const int* __restrict__ voff, const double* __restrict__ y0,
                             const double* __restrict__ y1, double dhh, Box* body_box) {
  const int b = blockIdx.x;
  __shared__ double red[12][128];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  double lo1[3] = {INFINITY, INFINITY, INFINITY}, hi1[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int v = voff[b] + threadIdx.x; v < voff[b + 1]; v += blockDim.x)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double c = y0[3 * v + k];
      lo[k] = fmin(lo[k], c);
      hi[k] = fmax(hi[k], c);
      if (y1) {
        const double c1 = y1[3 * v + k];
        lo1[k] = fmin(lo1[k], c1);
        hi1[k] = fmax(hi1[k], c1);
      }
    }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    red[k][threadIdx.x] = lo[k];
    red[3 + k][threadIdx.x] = hi[k];
    red[6 + k][threadIdx.x] = lo1[k];
    red[9 + k][threadIdx.x] = hi1[k];
  }
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (threadIdx.x < s)
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        red[k][threadIdx.x] = fmin(red[k][threadIdx.x], red[k][threadIdx.x + s]);
        red[3 + k][threadIdx.x] = fmax(red[3 + k][threadIdx.x], red[3 + k][threadIdx.x + s]);
        red[6 + k][threadIdx.x] = fmin(red[6 + k][threadIdx.x], red[6 + k][threadIdx.x + s]);
        red[9 + k][threadIdx.x] = fmax(red[9 + k][threadIdx.x], red[9 + k][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    Box B;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      B.lo[k] = (float)(red[k][0] - dhh);
      B.hi[k] = (float)(red[3 + k][0] + dhh);
      if (y1) {
        B.lo[k] = fminf(B.lo[k], (float)red[6 + k][0]);
        B.hi[k] = fmaxf(B.hi[k], (float)red[9 + k][0]);
      }
    }
    store_box(&body_box[b], B);
  }
}

// bit (I, J) of the overlap matrix, word w covers J in [32w, 32w + 32)
__global__ void k_pair_mask(int n, int W, const Box* __restrict__ body_box, uint32_t* mask) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * W) return;
  const int I = (int)(t / W), w = (int)(t % W);
  const Box a = load_box(&body_box[I]);
  uint32_t bits = 0;
  const int j0 = 32 * w, j1 = min(n, j0 + 32);
  for (int J = j0; J < j1; ++J) {
    if (J == I) continue;
    const Box b = load_box(&body_box[J]);
    if (overlap(a, b)) bits |= 1u << (J - j0);
  }
  mask[t] = bits;
}

__global__ void k_row_counts(int n, int W, const uint32_t* __restrict__ mask, int* row_cnt, int* upper_cnt) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= n) return;
  int full = 0, upper = 0;
  const int wI = I >> 5;
  for (int w = 0; w < W; ++w) {
    const uint32_t m = mask[(size_t)I * W + w];
    full += __popc(m);
    if (w > wI) upper += __popc(m);
    else if (w == wI) upper += __popc(m & ~((2u << (I & 31)) - 1u));
  }
  row_cnt[I] = full;
  upper_cnt[I] = upper;
}

// number of set bits of row J in columns (J, I), J < I
__device__ inline int bits_between(const uint32_t* row, int J, int I) {
  int c = 0;
  const int lo = J + 1, hi = I;  // [lo, hi)
  for (int w = lo >> 5; w <= ((hi - 1) >> 5); ++w) {
    uint32_t m = row[w];
    const int b0 = 32 * w;
    if (lo > b0) m &= ~((1u << (lo - b0)) - 1u);
    if (hi < b0 + 32) m &= (1u << (hi - b0)) - 1u;
    c += __popc(m);
  }
  return c;
}

__global__ void k_fill_adj(int n, int W, const uint32_t* __restrict__ mask, const int* __restrict__ row_ptr,
                           const int* __restrict__ upper_ptr, int cap_pairs, int cap_adj, int2* ij, int* adj_col,
                           int* adj_pair) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= n) return;
  int pos = row_ptr[I];
  int up = upper_ptr[I];
  const uint32_t* row = mask + (size_t)I * W;
  for (int w = 0; w < W; ++w) {
    uint32_t m = row[w];
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1;
      const int J = 32 * w + bit;
      int pr;
      if (J > I) {
        pr = up++;
        if (pr < cap_pairs) ij[pr] = make_int2(I, J);
      } else {
        pr = upper_ptr[J] + bits_between(mask + (size_t)J * W, J, I);
      }
      if (pos < cap_adj) {
        adj_col[pos] = J;
        adj_pair[pos] = pr;
      }
      ++pos;
    }
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
  Box* body_box;
  const int *tri_leaf, *edge_leaf;
  Box *tri_box, *edge_box;
  const int *tri_child, *edge_child, *tri_order, *edge_order, *tri_lvl, *edge_lvl, *tri_blvl, *edge_blvl;
  int smem_refit;
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

// Refit one body's subtree in shared memory: leaves [s0, s0 + cnt) are loaded from global,
// internal nodes (global ids in [s0, s0 + cnt)) are combined level by level with local ids,
// then written back.  Local ids: internal id - s0, leaf cnt + position - s0.
__device__ inline void refit_smem(const int* child, const int* order, const int* lvl, int l0, int l1, int s0,
                                  int cnt, int N, Box* box, float* sb) {
  if (cnt <= 1) return;  // a single leaf is its own root
  const int L0 = N - 1;
  for (int k = threadIdx.x; k < cnt; k += BB) {
    const Box B = load_box_cg(&box[L0 + s0 + k]);
    float* d = sb + 6 * (size_t)(cnt + k);
    d[0] = B.lo[0]; d[1] = B.lo[1]; d[2] = B.lo[2];
    d[3] = B.hi[0]; d[4] = B.hi[1]; d[5] = B.hi[2];
  }
  __syncthreads();
  const int H = l1 - l0 - 1;
  for (int h = 1; h <= H; ++h) {
    for (int k = lvl[l0 + h - 1] + (int)threadIdx.x; k < lvl[l0 + h]; k += BB) {
      const int node = order[k];
      int c0 = child[2 * node], c1 = child[2 * node + 1];
      c0 = c0 >= L0 ? cnt + (c0 - L0 - s0) : c0 - s0;
      c1 = c1 >= L0 ? cnt + (c1 - L0 - s0) : c1 - s0;
      const float* p = sb + 6 * (size_t)c0;
      const float* q = sb + 6 * (size_t)c1;
      float* d = sb + 6 * (size_t)(node - s0);
      d[0] = fminf(p[0], q[0]); d[1] = fminf(p[1], q[1]); d[2] = fminf(p[2], q[2]);
      d[3] = fmaxf(p[3], q[3]); d[4] = fmaxf(p[4], q[4]); d[5] = fmaxf(p[5], q[5]);
    }
    __syncthreads();
  }
  for (int k = lvl[l0] + (int)threadIdx.x; k < lvl[l1 - 1]; k += BB) {
    const int node = order[k];
    const float* d = sb + 6 * (size_t)(node - s0);
    Box B;
    B.lo[0] = d[0]; B.lo[1] = d[1]; B.lo[2] = d[2];
    B.hi[0] = d[3]; B.hi[1] = d[4]; B.hi[2] = d[5];
    store_box(&box[node], B);
  }
  __syncthreads();
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
  if (threadIdx.x == 0) {
    Box B;
    for (int j = 0; j < 3; ++j) {
      double l = red[j][0], h = red[3 + j][0], l1 = red[6 + j][0], h1 = red[9 + j][0];
      for (int w = 1; w < BB / 32; ++w) {
        l = fmin(l, red[j][w]);
        h = fmax(h, red[3 + j][w]);
        l1 = fmin(l1, red[6 + j][w]);
        h1 = fmax(h1, red[9 + j][w]);
      }
      B.lo[j] = (float)(l - a.dhh);
      B.hi[j] = (float)(h + a.dhh);
      if (swept) {
        B.lo[j] = fminf(B.lo[j], (float)l1);
        B.hi[j] = fmaxf(B.hi[j], (float)h1);
      }
    }
    store_box(&a.body_box[b], B);
  }
  // leaf boxes (same rounding as k_edge_boxes / k_tri_boxes)
  for (int e = a.eoff[b] + threadIdx.x; e < a.eoff[b + 1]; e += BB) {
    const int i0 = a.edges[2 * e], i1 = a.edges[2 * e + 1];
    Box B;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double u = a.y0[3 * i0 + k], w = a.y0[3 * i1 + k];
      B.lo[k] = (float)(fmin(u, w) - a.dhh);
      B.hi[k] = (float)(fmax(u, w) + a.dhh);
      if (swept) {
        const double u1 = a.y1[3 * i0 + k], w1 = a.y1[3 * i1 + k];
        B.lo[k] = fminf(B.lo[k], (float)fmin(u1, w1));
        B.hi[k] = fmaxf(B.hi[k], (float)fmax(u1, w1));
      }
    }
    store_box(&a.edge_box[(a.E - 1) + a.edge_leaf[e]], B);
  }
  for (int t = a.toff[b] + threadIdx.x; t < a.toff[b + 1]; t += BB) {
    const int i0 = a.tris[3 * t], i1 = a.tris[3 * t + 1], i2 = a.tris[3 * t + 2];
    Box B;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double u = a.y0[3 * i0 + k], w = a.y0[3 * i1 + k], q = a.y0[3 * i2 + k];
      B.lo[k] = (float)(fmin(fmin(u, w), q) - 0.0);
      B.hi[k] = (float)(fmax(fmax(u, w), q) + 0.0);
      if (swept) {
        const double u1 = a.y1[3 * i0 + k], w1 = a.y1[3 * i1 + k], q1 = a.y1[3 * i2 + k];
        B.lo[k] = fminf(B.lo[k], (float)fmin(fmin(u1, w1), q1));
        B.hi[k] = fmaxf(B.hi[k], (float)fmax(fmax(u1, w1), q1));
      }
    }
    store_box(&a.tri_box[(a.T - 1) + a.tri_leaf[t]], B);
  }
  __syncthreads();
  if (a.smem_refit) {
    extern __shared__ float sbox[];  // [2 * cnt][6]: internal nodes, then leaves (local ids)
    refit_smem(a.edge_child, a.edge_order, a.edge_lvl, a.edge_blvl[b], a.edge_blvl[b + 1], a.eoff[b],
               a.eoff[b + 1] - a.eoff[b], a.E, a.edge_box, sbox);
    refit_smem(a.tri_child, a.tri_order, a.tri_lvl, a.tri_blvl[b], a.tri_blvl[b + 1], a.toff[b],
               a.toff[b + 1] - a.toff[b], a.T, a.tri_box, sbox);
    return;
  }
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
                       double* y1) {
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
  a.dhh = s.prm.dhat * 0.5;
  a.body_box = s.body_box;
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
  // shared-memory refit when the largest body subtree fits (2 boxes of 24 B per primitive)
  const int maxp = s.max_body_t > s.max_body_e ? s.max_body_t : s.max_body_e;
  const size_t smem = 2 * sizeof(float) * 6 * (size_t)maxp;
  a.smem_refit = smem <= 200 * 1024;
  if (a.smem_refit && smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_body_broad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_body_broad<<<s.n, BB, a.smem_refit ? smem : 0, s.stream>>>(a);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t transform(Sim& s, const double* A, const double* p, double* x) {
  if (s.V == 0) return cudaSuccess;
  k_transform<<<blocks(s.V, 256), 256, 0, s.stream>>>(s.V, s.vbody, s.x0, A, p, x);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t prim_boxes(Sim& s, const double* y0, const double* y1) {
  const double dhh = s.prm.dhat * 0.5;
  if (s.E > 0) {
    k_edge_boxes<<<blocks(s.E, 256), 256, 0, s.stream>>>(s.E, s.edges, y0, y1, dhh, s.edge_tree.prim_leaf,
                                                         s.edge_tree.box);
    ++s.launches;
  }
  if (s.T > 0) {
    k_tri_boxes<<<blocks(s.T, 256), 256, 0, s.stream>>>(s.T, s.tris, y0, y1, s.tri_tree.prim_leaf, s.tri_tree.box);
    ++s.launches;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if ((e = refit(s, s.edge_tree)) != cudaSuccess) return e;
  return refit(s, s.tri_tree);
}

cudaError_t body_boxes(Sim& s, const double* y0, const double* y1) {
  k_body_boxes<<<s.n, 128, 0, s.stream>>>(s.n, s.voff, y0, y1, s.prm.dhat * 0.5, s.body_box);
  ++s.launches;
  return cudaGetLastError();
}

// Body pairs I < J with overlapping boxes (the ij list, sorted) and the symmetric CSR
// adjacency (row I: neighbours in increasing J, with the pair index of {I, J}).
// Synchronises the stream to read the counts; *overflow is set when a capacity is short.
cudaError_t body_pairs(Sim& s, bool* overflow) {
  const int n = s.n, W = s.W;
  k_pair_mask<<<blocks((long long)n * W, 256), 256, 0, s.stream>>>(n, W, s.body_box, s.pair_mask);
  k_row_counts<<<blocks(n, 256), 256, 0, s.stream>>>(n, W, s.pair_mask, s.row_ptr, s.upper_ptr);
  k_scan_excl<<<1, 1024, 0, s.stream>>>(s.row_ptr, n, s.row_ptr + n);
  k_scan_excl<<<1, 1024, 0, s.stream>>>(s.upper_ptr, n, s.upper_ptr + n);
  k_fill_adj<<<blocks(n, 128), 128, 0, s.stream>>>(n, W, s.pair_mask, s.row_ptr, s.upper_ptr, s.cap_pairs, s.cap_adj,
                                                   s.ij, s.adj_col, s.adj_pair);
  s.launches += 5;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  cudaMemcpyAsync(s.hstat + 16, s.upper_ptr + n, sizeof(int), cudaMemcpyDeviceToHost, s.stream);
  cudaMemcpyAsync(s.hstat + 17, s.row_ptr + n, sizeof(int), cudaMemcpyDeviceToHost, s.stream);
  if ((e = cudaStreamSynchronize(s.stream)) != cudaSuccess) return e;
  s.n_pairs = s.hstat[16];
  s.n_adj = s.hstat[17];
  *overflow = s.n_pairs > s.cap_pairs || s.n_adj > s.cap_adj;
  return cudaSuccess;
}

}  // namespace abd
