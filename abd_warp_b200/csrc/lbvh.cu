// Linear BVH over the primitives of all bodies: Morton codes, LSD radix sort, Karras build,
// bottom-up refit.  Replaces the reference's per-body wp.Bvh build / refit
// (abd/culling2.py:83-210, abd/abd.py:74-93).
//
// Keys are (body << 30) | morton30(rest-space centroid normalised to the body's rest box).
// Sorting by body first makes every body's primitives a contiguous key range, and in a
// binary radix tree the keys sharing the body prefix form one subtree: body_root[b].
// Affine motion keeps the rest-space hierarchy spatially coherent, so the topology is built
// once.  The rest-frame boxes of the internal nodes are computed once as well (rest_boxes,
// broad.cu); under motion by DOFs a node's world box is bounded by their affine image.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "abd_common.cuh"
#include "abd_scan.cuh"

namespace abd {

namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;

__device__ inline unsigned int expand10(unsigned int v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_body_bounds(int n, const int* off, const double* cen, float* lohi) {
  const int b = blockIdx.x;
  if (b >= n) return;
  __shared__ float red[6][128];
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = off[b] + threadIdx.x; i < off[b + 1]; i += blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const float c = (float)cen[3 * i + k];
      lo[k] = fminf(lo[k], c);
      hi[k] = fmaxf(hi[k], c);
    }
  for (int k = 0; k < 3; ++k) {
    red[k][threadIdx.x] = lo[k];
    red[3 + k][threadIdx.x] = hi[k];
  }
  __syncthreads();
  for (int s = 64; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 3; ++k) {
        red[k][threadIdx.x] = fminf(red[k][threadIdx.x], red[k][threadIdx.x + s]);
        red[3 + k][threadIdx.x] = fmaxf(red[3 + k][threadIdx.x], red[3 + k][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) lohi[6 * b + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_morton(int N, const int* body, const double* cen, const float* lohi, unsigned long long* keys,
                         int* vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int b = body[i];
  unsigned int m = 0;
  unsigned int q[3];
  for (int k = 0; k < 3; ++k) {
    const float lo = lohi[6 * b + k], hi = lohi[6 * b + 3 + k];
    const float ext = hi - lo;
    float u = ext > 0.f ? ((float)cen[3 * i + k] - lo) / ext : 0.5f;
    u = fminf(fmaxf(u, 0.f), 1.f);
    q[k] = min((unsigned int)(u * 1024.f), 1023u);
  }
  m = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
  keys[i] = ((unsigned long long)b << 30) | (unsigned long long)m;
  vals[i] = i;
}

// ---- radix sort (stable LSD, 8-bit digits) ----
__global__ void k_rs_hist(const unsigned long long* keys, int N, int shift, int tiles, int* hist) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * RS_TILE;
  for (int i = 0; i < RS_ITEMS; ++i) {
    const int idx = base + i * RS_THREADS + threadIdx.x;
    if (idx < N) atomicAdd(&cnt[(int)((keys[idx] >> shift) & 255ull)], 1);
  }
  __syncthreads();
  hist[threadIdx.x * tiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void k_rs_scatter(const unsigned long long* kin, const int* vin, unsigned long long* kout, int* vout, int N,
                             int shift, int tiles, const int* hist) {
  __shared__ int base[256];
  __shared__ int running[256];
  __shared__ int wcnt[RS_THREADS / 32][256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  base[tid] = hist[tid * tiles + blockIdx.x];
  running[tid] = 0;
  for (int w = 0; w < RS_THREADS / 32; ++w) wcnt[w][tid] = 0;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int i = 0; i < RS_ITEMS; ++i) {
    const int idx = blockIdx.x * RS_TILE + i * RS_THREADS + tid;
    const bool valid = idx < N;
    unsigned long long key = valid ? kin[idx] : 0ull;
    const int val = valid ? vin[idx] : 0;
    const int d = valid ? (int)((key >> shift) & 255ull) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & lt);
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      int acc = running[tid];
      for (int w = 0; w < RS_THREADS / 32; ++w) {
        const int c = wcnt[w][tid];
        wcnt[w][tid] = acc;
        acc += c;
      }
      running[tid] = acc;
    }
    __syncthreads();
    if (valid) {
      const int pos = base[d] + wcnt[warp][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    for (int w = 0; w < RS_THREADS / 32; ++w) wcnt[w][tid] = 0;
    __syncthreads();
  }
}

// ---- Karras 2012 binary radix tree ----
__device__ inline int kdelta(const unsigned long long* keys, int N, int i, int j) {
  if (j < 0 || j > N - 1) return -1;
  const unsigned long long a = keys[i], b = keys[j];
  if (a == b) return 64 + __clz(i ^ j);
  return __clzll(a ^ b);
}

__global__ void k_karras(int N, const unsigned long long* keys, int* child, int* parent, int* lo_hi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N - 1) return;
  const int d = (kdelta(keys, N, i, i + 1) - kdelta(keys, N, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = kdelta(keys, N, i, i - d);
  int lmax = 2;
  while (kdelta(keys, N, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (kdelta(keys, N, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = kdelta(keys, N, i, j);
  int s = 0;
  for (int div = 2;; div <<= 1) {
    const int t = (l + div - 1) / div;
    if (kdelta(keys, N, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int left = (lo == gamma) ? (N - 1 + gamma) : gamma;
  const int right = (hi == gamma + 1) ? (N - 1 + gamma + 1) : gamma + 1;
  child[2 * i] = left;
  child[2 * i + 1] = right;
  parent[left] = i;
  parent[right] = i;
  lo_hi[2 * i] = lo;
  lo_hi[2 * i + 1] = hi;
}

__global__ void k_body_roots(int N, int n, const int* off, const int* lo_hi, int* body_root) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N - 1) {
    // binary search the body of sorted position lo_hi[2i]
    const int lo = lo_hi[2 * i], hi = lo_hi[2 * i + 1];
    int a = 0, b = n - 1;
    while (a < b) {
      const int m = (a + b + 1) >> 1;
      if (off[m] <= lo) a = m;
      else b = m - 1;
    }
    if (off[a] == lo && off[a + 1] - 1 == hi) body_root[a] = i;
  }
  if (i < n) {
    const int cnt = off[i + 1] - off[i];
    if (cnt == 1) body_root[i] = N - 1 + off[i];
    if (cnt == 0) body_root[i] = -1;
  }
}

__global__ void k_inverse_perm(int N, const int* leaf_prim, int* prim_leaf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) prim_leaf[leaf_prim[i]] = i;
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t radix_sort_pairs(Sim& s, unsigned long long* keys, int* vals, unsigned long long* keys_tmp, int* vals_tmp,
                             int N, int key_bits) {
  if (N <= 1) return cudaSuccess;
  const int tiles = (N + RS_TILE - 1) / RS_TILE;
  int* hist = nullptr;
  cudaError_t e = cudaMallocAsync(&hist, sizeof(int) * 256 * (size_t)tiles, s.stream);
  if (e != cudaSuccess) return e;
  unsigned long long *ka = keys, *kb = keys_tmp;
  int *va = vals, *vb = vals_tmp;
  const int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_rs_hist<<<tiles, RS_THREADS, 0, s.stream>>>(ka, N, shift, tiles, hist);
    k_scan_excl<<<1, 1024, 0, s.stream>>>(hist, 256 * tiles, nullptr);
    k_rs_scatter<<<tiles, RS_THREADS, 0, s.stream>>>(ka, va, kb, vb, N, shift, tiles, hist);
    s.launches += 3;
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    cudaMemcpyAsync(keys, ka, sizeof(unsigned long long) * N, cudaMemcpyDeviceToDevice, s.stream);
    cudaMemcpyAsync(vals, va, sizeof(int) * N, cudaMemcpyDeviceToDevice, s.stream);
  }
  cudaFreeAsync(hist, s.stream);
  return cudaGetLastError();
}

cudaError_t build_tree(Sim& s, Tree& tr, int N, const int* prim_body, const double* cen, const int* prim_off_host) {
  (void)prim_off_host;
  tr.N = N;
  const int n = s.n;
  cudaError_t e;
  const size_t nodes = N > 0 ? 2 * (size_t)N - 1 : 1;
#define TRY(x)                    \
  do {                            \
    e = (x);                      \
    if (e != cudaSuccess) return e; \
  } while (0)
  TRY(cudaMalloc(&tr.child, sizeof(int) * 2 * (size_t)(N > 1 ? N - 1 : 1)));
  TRY(cudaMalloc(&tr.parent, sizeof(int) * nodes));
  TRY(cudaMalloc(&tr.leaf_prim, sizeof(int) * (size_t)(N > 0 ? N : 1)));
  TRY(cudaMalloc(&tr.prim_leaf, sizeof(int) * (size_t)(N > 0 ? N : 1)));
  TRY(cudaMalloc(&tr.body_root, sizeof(int) * (size_t)n));
  TRY(cudaMalloc(&tr.rest, sizeof(Box) * (size_t)(N > 0 ? 2 * N - 1 : 1)));
  TRY(cudaMalloc(&tr.box, sizeof(Box) * nodes));
  TRY(cudaMemsetAsync(tr.body_root, 0xff, sizeof(int) * n, s.stream));
  TRY(cudaMemsetAsync(tr.parent, 0xff, sizeof(int) * nodes, s.stream));
  if (N == 0) {
    std::vector<int> zeros(2 * (size_t)n + 1, 0), bl(n + 1);
    for (int b = 0; b <= n; ++b) bl[b] = 2 * b;  // every body: an empty schedule [0, 0]
    TRY(cudaMalloc(&tr.order, sizeof(int)));
    TRY(cudaMalloc(&tr.lvl, sizeof(int) * zeros.size()));
    TRY(cudaMalloc(&tr.body_lvl, sizeof(int) * bl.size()));
    TRY(cudaMemcpy(tr.lvl, zeros.data(), sizeof(int) * zeros.size(), cudaMemcpyHostToDevice));
    TRY(cudaMemcpy(tr.body_lvl, bl.data(), sizeof(int) * bl.size(), cudaMemcpyHostToDevice));
    return cudaSuccess;
  }
  const int* off = (prim_body == s.tbody) ? s.toff : s.eoff;
  float* lohi = nullptr;
  unsigned long long *keys = nullptr, *ktmp = nullptr;
  int *vtmp = nullptr, *lo_hi = nullptr;
  TRY(cudaMallocAsync(&lohi, sizeof(float) * 6 * n, s.stream));
  TRY(cudaMallocAsync(&keys, sizeof(unsigned long long) * N, s.stream));
  TRY(cudaMallocAsync(&ktmp, sizeof(unsigned long long) * N, s.stream));
  TRY(cudaMallocAsync(&vtmp, sizeof(int) * N, s.stream));
  TRY(cudaMallocAsync(&lo_hi, sizeof(int) * 2 * (size_t)(N > 1 ? N - 1 : 1), s.stream));
  k_body_bounds<<<n, 128, 0, s.stream>>>(n, off, cen, lohi);
  k_morton<<<blocks(N, 256), 256, 0, s.stream>>>(N, prim_body, cen, lohi, keys, tr.leaf_prim);
  s.launches += 2;
  int body_bits = 1;
  while ((1 << body_bits) < n) ++body_bits;
  TRY(radix_sort_pairs(s, keys, tr.leaf_prim, ktmp, vtmp, N, 30 + body_bits));
  if (N > 1) {
    k_karras<<<blocks(N - 1, 256), 256, 0, s.stream>>>(N, keys, tr.child, tr.parent, lo_hi);
    ++s.launches;
  }
  k_body_roots<<<blocks((N > n ? N : n), 256), 256, 0, s.stream>>>(N, n, off, lo_hi, tr.body_root);
  k_inverse_perm<<<blocks(N, 256), 256, 0, s.stream>>>(N, tr.leaf_prim, tr.prim_leaf);
  s.launches += 2;
  // per-body refit schedule (host, once): node heights, then each body's internal nodes
  // grouped by height.  Karras node i spans [i, j] or [j, i], so a body's subtree nodes are
  // exactly the internal nodes whose span lies inside the body's leaf range.
  {
    const int M = N - 1;
    std::vector<int> child(2 * (size_t)(M > 0 ? M : 1)), span(2 * (size_t)(M > 0 ? M : 1)), offh(n + 1);
    if (M > 0) {
      TRY(cudaMemcpyAsync(child.data(), tr.child, sizeof(int) * 2 * M, cudaMemcpyDeviceToHost, s.stream));
      TRY(cudaMemcpyAsync(span.data(), lo_hi, sizeof(int) * 2 * M, cudaMemcpyDeviceToHost, s.stream));
    }
    TRY(cudaMemcpyAsync(offh.data(), off, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s.stream));
    TRY(cudaStreamSynchronize(s.stream));
    std::vector<int> byspan(M), height(M, 0), owner(M, -1);
    for (int i = 0; i < M; ++i) byspan[i] = i;
    std::sort(byspan.begin(), byspan.end(), [&](int a, int b) {
      return span[2 * a + 1] - span[2 * a] < span[2 * b + 1] - span[2 * b];
    });
    for (int i : byspan) {
      int h = 0;
      for (int c = 0; c < 2; ++c) {
        const int ch = child[2 * i + c];
        if (ch < M) h = std::max(h, height[ch]);
      }
      height[i] = h + 1;
      const int lo = span[2 * i], hi = span[2 * i + 1];
      const int b = int(std::upper_bound(offh.begin(), offh.end(), lo) - offh.begin()) - 1;
      if (b >= 0 && b < n && hi < offh[b + 1]) owner[i] = b;
    }
    std::vector<int> order, lvl, body_lvl(n + 1, 0);
    std::vector<std::vector<int>> per(n);
    tr.max_height = 0;
    for (int i = 0; i < M; ++i)
      if (owner[i] >= 0) {
        per[owner[i]].push_back(i);
        tr.max_height = std::max(tr.max_height, height[i]);
      }
    for (int b = 0; b < n; ++b) {
      std::vector<int>& v = per[b];
      std::stable_sort(v.begin(), v.end(), [&](int a, int c) { return height[a] < height[c]; });
      body_lvl[b] = (int)lvl.size();
      lvl.push_back((int)order.size());
      int h = 1;
      for (size_t k = 0; k < v.size(); ++k) {
        while (height[v[k]] > h) {
          lvl.push_back((int)order.size());
          ++h;
        }
        order.push_back(v[k]);
      }
      lvl.push_back((int)order.size());
    }
    body_lvl[n] = (int)lvl.size();
    TRY(cudaMalloc(&tr.order, sizeof(int) * std::max<size_t>(1, order.size())));
    TRY(cudaMalloc(&tr.lvl, sizeof(int) * lvl.size()));
    TRY(cudaMalloc(&tr.body_lvl, sizeof(int) * body_lvl.size()));
    if (!order.empty())
      TRY(cudaMemcpyAsync(tr.order, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, s.stream));
    TRY(cudaMemcpyAsync(tr.lvl, lvl.data(), sizeof(int) * lvl.size(), cudaMemcpyHostToDevice, s.stream));
    TRY(cudaMemcpyAsync(tr.body_lvl, body_lvl.data(), sizeof(int) * body_lvl.size(), cudaMemcpyHostToDevice,
                        s.stream));
    TRY(cudaStreamSynchronize(s.stream));
  }
  cudaFreeAsync(lohi, s.stream);
  cudaFreeAsync(keys, s.stream);
  cudaFreeAsync(ktmp, s.stream);
  cudaFreeAsync(vtmp, s.stream);
  cudaFreeAsync(lo_hi, s.stream);
#undef TRY
  return cudaGetLastError();
}

}  // namespace abd
