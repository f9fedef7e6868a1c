// CPU FP64 oracle: a restatement of the reference ABD implicit contact step.
//
// TEST INFRASTRUCTURE ONLY.  Loaded by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg as the checker; the product path (abd_warp_b200/, libabd_b200.so) never
// links or calls it.
//
// Follows, function by function (citations are to the reference project's files):
//   step / line search / ccd driver ........ abd/abd.py:124-362
//   inertia + orthogonality ................ abd/orthogonal_energy.py:24-135
//   barrier ................................ abd/ipcsk/barrier.py:3-49
//   PT / EE / VG gradient + Hessian ........ abd/ipcsk/pt_ipc.py:111-287, ee_ipc.py:13-218,
//                                            vg_ipc.py:4-34, put.py:25-66
//   contact energy ......................... abd/ipcsk/energy.py:9-48
//   distance geometry + eigensystem ........ abd/psd/vf.py:3-71, psd/ee.py:5-163,
//                                            psd/hl.py:15-39,155-195
//   CCD .................................... abd/ccd.py:9-195, abd/cubic_roots.py:6-193
//   culling (intended cull_ semantics) ..... abd/culling.py:32-99, abd/culling2.py:32-280
// with the corrections of the reference's evident defects: PT/EE lists used consistently,
// per-body-pair culling instead of the hard-wired pair (0,1), the full coupled Hessian,
// capacity-free lists, per-body mass / I0, fixed (Dirichlet) bodies, and the Armijo sign
// selectable (armijo_sign = -1 correct, +1 the reference's form).
//
// Parity pin: the per-pair math is checked against oracle/np_ref.py and the reference's
// known-answer fixtures (tests/golden).  Whole-step trajectories cannot be checked
// against the reference itself (it does not run without Warp and abdtk): the step-level
// parity of this oracle is unpinned with respect to the reference's own execution.
//
// Build: oracle/Makefile  (g++ -O2 -fopenmp -ffp-contract=off).  No FMA contraction, so
// elementwise arithmetic matches the CUDA build (nvcc -fmad=false) bit for bit where the
// operation order is the same.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

// The full IPC model's per-contact arithmetic, shared with the CUDA library (plain C++): the
// oracle's full mode evaluates it so that whole steps can be compared bit for bit, and checks
// it against its own forward-mode restatement below (full_energy_d / full_terms).
#include "../abd_warp_b200/csrc/abd_ipc_full.cuh"

namespace {

struct Params {
  double dt, dhat, d2hat, kappa, stiffness, gravity, tol, c1, alpha_min, ground, cg_tol, refine_tol;
  double ls_noise_floor;
  int max_iter, armijo_sign, ground_enabled, psd_ee, enable_pt, enable_ee, enable_vg, solver,
      cg_max_iter, precision, contact_psd, precond, cluster_max;
  int min_capacity;  // the CUDA library's capacity injection (the oracle has no capacities)
  int newton_loop;   // the CUDA library's choice of Newton loop (the oracle has one)
  int ipc_full;      // the full contact model (the oracle's own switch, Oracle::ipc_full, decides)
  double friction_mu;     // lagged friction (with the full model): coefficient, 0 = off
  double friction_epsv;   // its slip velocity (eps = friction_epsv dt)
};

struct V3 {
  double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

struct Box {
  float lo[3], hi[3];
};
inline bool overlap(const Box& a, const Box& b) {
  for (int k = 0; k < 3; ++k)
    if (a.lo[k] > b.hi[k] || b.lo[k] > a.hi[k]) return false;
  return true;
}

struct Cand {
  int I, J, pair, pi, pj;  // vec5i (I, J, ij index, prim of I, prim of J)
};

// ---------------------------------------------------------------------------------------
// Exact summation.  Every reduction of the step is the exact sum of its FP64 terms, each
// truncated to a multiple of 2^-192, rounded to FP64 once (to nearest, ties to even).  The
// sum does not depend on the order of the terms, so it is fixed by the terms alone; the
// CUDA product sums the same way (32-bit digits in 64-bit limbs).
// ---------------------------------------------------------------------------------------
constexpr int kXD = 10, kXB0 = -192;

struct XSum {
  long long d[kXD] = {};
  int flags = 0;  // 1 NaN, 2 +inf, 4 -inf, 8 out of range

  void add(double x) {
    uint64_t bits;
    std::memcpy(&bits, &x, 8);
    const int ex = (int)((bits >> 52) & 0x7ff);
    const uint64_t frac = bits & 0xfffffffffffffULL;
    const bool neg = (bits >> 63) != 0;
    if (ex == 0x7ff) {
      flags |= frac ? 1 : (neg ? 4 : 2);
      return;
    }
    uint64_t m = ex ? (frac | (1ULL << 52)) : frac;
    int sft = (ex ? ex : 1) - 1075 - kXB0;
    if (sft < 0) {
      if (sft <= -64) return;
      m >>= -sft;
      sft = 0;
    }
    if (!m) return;
    const int j = sft >> 5;
    const unsigned __int128 v = (unsigned __int128)m << (sft & 31);
    const uint64_t u[3] = {(uint64_t)v & 0xffffffffULL, (uint64_t)(v >> 32) & 0xffffffffULL, (uint64_t)(v >> 64)};
    const int top = u[2] ? 2 : (u[1] ? 1 : 0);
    if (j + top >= kXD) {
      flags |= 8;
      return;
    }
    for (int k = 0; k < 3 && j + k < kXD; ++k) d[j + k] += neg ? -(long long)u[k] : (long long)u[k];
  }
  void merge(const XSum& o) {
    for (int i = 0; i < kXD; ++i) d[i] += o.d[i];
    flags |= o.flags;
  }
  double round() const {
    if (flags & (1 | 8)) return std::nan("");
    if (flags & 2) return (flags & 4) ? std::nan("") : INFINITY;
    if (flags & 4) return -INFINITY;
    long long e[kXD + 1];
    for (int i = 0; i < kXD; ++i) e[i] = d[i];
    e[kXD] = 0;
    auto carry = [&]() {
      for (int i = 0; i < kXD; ++i) {
        const long long c = e[i] >> 32;  // floor division by 2^32
        e[i] -= c * 4294967296LL;
        e[i + 1] += c;
      }
    };
    carry();
    const bool neg = e[kXD] < 0;
    if (neg) {
      for (int i = 0; i <= kXD; ++i) e[i] = -e[i];
      carry();
    }
    int h = -1;
    for (int i = 0; i <= kXD; ++i)
      if (e[i] != 0) h = i;
    if (h < 0) return 0.0;
    const uint64_t t2 = (uint64_t)e[h], t1 = h >= 1 ? (uint64_t)e[h - 1] : 0, t0 = h >= 2 ? (uint64_t)e[h - 2] : 0;
    bool sticky = false;
    for (int i = 0; i < h - 2; ++i) sticky = sticky || e[i] != 0;
    const unsigned __int128 w = ((unsigned __int128)t2 << 64) | ((unsigned __int128)t1 << 32) | t0;
    const int msb = 127 - __builtin_clzll(t2);  // t2 != 0
    const int drop = msb - 52;
    uint64_t mant = (uint64_t)(w >> drop);
    const unsigned __int128 rem = w & ((((unsigned __int128)1) << drop) - 1);
    const unsigned __int128 half = ((unsigned __int128)1) << (drop - 1);
    if (rem > half || (rem == half && (sticky || (mant & 1)))) ++mant;
    const double r = std::ldexp((double)mant, drop + 32 * (h - 2) + kXB0);
    return neg ? -r : r;
  }
};

// Natural logarithm from IEEE-exact operations only, so that it returns the same bits as
// the CUDA product's: x = (1 + f) 2^k with 1 + f in [sqrt(1/2), sqrt(2)), f exact;
// log(1 + f) = 2 atanh(s), s = f / (2 + f), = f - s (f - R) with R = sum_{i=1..11}
// 2 s^(2i) / (2i + 1) in Horner form (the atanh reduction as in J.-M. Muller, "Elementary
// Functions", ch. 11), and log 2 split in a 40-bit head and a tail.
inline double abd_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -INFINITY : std::nan("");
  if (std::isinf(x)) return x;
  int k;
  double m = std::frexp(x, &k);
  if (m < 0.70710678118654752) {
    m = m * 2.0;
    k -= 1;
  }
  const double f = m - 1.0;
  const double s = f / (2.0 + f);
  const double z = s * s;
  const double c[10] = {2.0 / 21.0, 2.0 / 19.0, 2.0 / 17.0, 2.0 / 15.0, 2.0 / 13.0,
                        2.0 / 11.0, 2.0 / 9.0,  2.0 / 7.0,  2.0 / 5.0,  2.0 / 3.0};
  double r = 2.0 / 23.0;
  for (int i = 0; i < 10; ++i) r = r * z + c[i];
  r = r * z;
  const double ln2_hi = 0.6931471805592082, ln2_lo = 7.371002565167799e-13;  // ln2_hi: 40 bits
  return (double)k * ln2_hi + (f - (s * (f - r) - (double)k * ln2_lo));
}

struct Oracle {
  int n, V, T, E;
  std::vector<int> voff, toff, eoff, tris, edges, fixed;
  std::vector<double> x0, mass, I0;
  Params prm;
  // states, [n][9] row-major A (row k = a_k) and [n][3] p
  std::vector<double> A, p, Ak, pk, Adot, pdot, A0, p0;
  std::vector<double> dq, g;  // [n][12]
  std::vector<double> x, xk, xview;
  // assembled system
  std::vector<double> diag;       // [n][144]
  std::vector<double> off;        // [npairs][144], block (I,J) with I<J
  std::vector<int> ij;            // [npairs][2]
  std::vector<int> pact;          // [npairs] active contacts
  std::vector<int> adj_ptr, adj;  // per body (neighbour, pair, side), neighbours increasing
  std::vector<int> highlight;     // [n] body in an active PT / EE / vertex-ground contact (abd.py:238)
  // stats
  int stat_newton = 0, stat_lin = 0, stat_ls = 0, stat_pt = 0, stat_ee = 0, stat_vg = 0, stat_ij = 0,
      stat_active = 0, stat_refine = 0;
  int last_sweeps = 0;  // refinement sweeps of the last mixed-precision solve
  bool ipc_full = false;  // full IPC contact model (closest-feature types, mollifier)
  bool ipc_independent = false;  // full model in the oracle's own arithmetic (else the header's)
  // lagged friction (with the full model): coefficient, slip velocity, and the contacts that
  // the step fixed at its start
  double fr_mu = 0.0, fr_epsv = 1e-3;
  struct Fric {
    int I, J, kind;  // the first group (point / edge a) moves with I
    double w[4], P[6], lam, xt[12], rs[12];
    int ids[4];
    abd::ipc::FrictionLag hl;  // the header's lagged quantities (the default arithmetic)
  };
  std::vector<Fric> fric;
  double stat_alpha = 0, stat_toi = 0, stat_energy = 0;
};

// ---------------------------------------------------------------------------------------
// transform + boxes (abd.py:305-324, culling2.py:32-79, 229-280)
// ---------------------------------------------------------------------------------------
void transform(const Oracle& o, const double* A, const double* p, double* out) {
#pragma omp parallel for schedule(static)
  for (int b = 0; b < o.n; ++b) {
    const double* a = A + 9 * b;
    for (int v = o.voff[b]; v < o.voff[b + 1]; ++v) {
      const double r0 = o.x0[3 * v], r1 = o.x0[3 * v + 1], r2 = o.x0[3 * v + 2];
      for (int j = 0; j < 3; ++j)
        out[3 * v + j] = ((a[0 * 3 + j] * r0 + a[1 * 3 + j] * r1) + a[2 * 3 + j] * r2) + p[3 * b + j];
    }
  }
}

struct Boxes {
  std::vector<Box> pt, ed, tr, body;
};

void static_boxes(const Oracle& o, const double* y, Boxes& bx) {
  const double dh = o.prm.dhat, dhh = o.prm.dhat * 0.5;
  bx.pt.resize(o.V);
  bx.ed.resize(o.E);
  bx.tr.resize(o.T);
  bx.body.resize(o.n);
  const float dhf = (float)dh;
#pragma omp parallel for schedule(static)
  for (int v = 0; v < o.V; ++v)
    for (int k = 0; k < 3; ++k) {
      float c = (float)y[3 * v + k];
      bx.pt[v].lo[k] = c - dhf;
      bx.pt[v].hi[k] = c + dhf;
    }
#pragma omp parallel for schedule(static)
  for (int e = 0; e < o.E; ++e) {
    const int a = o.edges[2 * e], b = o.edges[2 * e + 1];
    for (int k = 0; k < 3; ++k) {
      double lo = std::min(y[3 * a + k], y[3 * b + k]);
      double hi = std::max(y[3 * a + k], y[3 * b + k]);
      bx.ed[e].lo[k] = (float)(lo - dhh);
      bx.ed[e].hi[k] = (float)(hi + dhh);
    }
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < o.T; ++t) {
    const int a = o.tris[3 * t], b = o.tris[3 * t + 1], c = o.tris[3 * t + 2];
    for (int k = 0; k < 3; ++k) {
      double lo = std::min(std::min(y[3 * a + k], y[3 * b + k]), y[3 * c + k]);
      double hi = std::max(std::max(y[3 * a + k], y[3 * b + k]), y[3 * c + k]);
      bx.tr[t].lo[k] = (float)(lo - 0.0);
      bx.tr[t].hi[k] = (float)(hi + 0.0);
    }
  }
#pragma omp parallel for schedule(static)
  for (int b = 0; b < o.n; ++b) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int v = o.voff[b]; v < o.voff[b + 1]; ++v)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], y[3 * v + k]);
        hi[k] = std::max(hi[k], y[3 * v + k]);
      }
    for (int k = 0; k < 3; ++k) {
      bx.body[b].lo[k] = (float)(lo[k] - dhh);
      bx.body[b].hi[k] = (float)(hi[k] + dhh);
    }
  }
}

// swept boxes: the static (dilated) boxes at x united with the undilated boxes at xk
void swept_boxes(const Oracle& o, const double* x, const double* xk, Boxes& bx) {
  static_boxes(o, x, bx);
  auto grow = [](Box& b, int k, double lo, double hi) {
    b.lo[k] = std::min(b.lo[k], (float)lo);
    b.hi[k] = std::max(b.hi[k], (float)hi);
  };
#pragma omp parallel for schedule(static)
  for (int v = 0; v < o.V; ++v)
    for (int k = 0; k < 3; ++k) grow(bx.pt[v], k, xk[3 * v + k], xk[3 * v + k]);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < o.E; ++e) {
    const int a = o.edges[2 * e], b = o.edges[2 * e + 1];
    for (int k = 0; k < 3; ++k)
      grow(bx.ed[e], k, std::min(xk[3 * a + k], xk[3 * b + k]), std::max(xk[3 * a + k], xk[3 * b + k]));
  }
#pragma omp parallel for schedule(static)
  for (int t = 0; t < o.T; ++t) {
    const int a = o.tris[3 * t], b = o.tris[3 * t + 1], c = o.tris[3 * t + 2];
    for (int k = 0; k < 3; ++k)
      grow(bx.tr[t], k, std::min(std::min(xk[3 * a + k], xk[3 * b + k]), xk[3 * c + k]),
           std::max(std::max(xk[3 * a + k], xk[3 * b + k]), xk[3 * c + k]));
  }
#pragma omp parallel for schedule(static)
  for (int b = 0; b < o.n; ++b) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int v = o.voff[b]; v < o.voff[b + 1]; ++v)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], xk[3 * v + k]);
        hi[k] = std::max(hi[k], xk[3 * v + k]);
      }
    for (int k = 0; k < 3; ++k) grow(bx.body[b], k, lo[k], hi[k]);
  }
}

// ---------------------------------------------------------------------------------------
// culling: body pairs (culling2.py:213-227), primitive pairs (culling.py:85-99),
// vertex-ground (culling.py:64-82)
// ---------------------------------------------------------------------------------------
struct Lists {
  std::vector<int> ij;      // [m][2], I < J
  std::vector<Cand> pt, ee;
  std::vector<int> vg;      // [k][2] (body, global vertex)
};

void cull(const Oracle& o, const Boxes& bx, Lists& L) {
  L.ij.clear();
  for (int I = 0; I < o.n; ++I)
    for (int J = I + 1; J < o.n; ++J)
      if (overlap(bx.body[I], bx.body[J])) {
        L.ij.push_back(I);
        L.ij.push_back(J);
      }
  const int m = (int)L.ij.size() / 2;
  std::vector<std::vector<Cand>> ptp(m), eep(m);
#pragma omp parallel for schedule(dynamic, 1)
  for (int q = 0; q < m; ++q) {
    const int I = L.ij[2 * q], J = L.ij[2 * q + 1];
    // primitives of each body that can touch the other body's box (exact prefilter:
    // every primitive box lies inside its body box)
    auto near = [&](const std::vector<Box>& bs, int lo, int hi, const Box& other) {
      std::vector<int> r;
      for (int i = lo; i < hi; ++i)
        if (overlap(bs[i], other)) r.push_back(i);
      return r;
    };
    // a point box (+-dhat) is not inside its body box (+-dhat/2): triangles are
    // prefiltered by the union of the near points' boxes instead
    auto unite = [&](const std::vector<int>& ids) {
      Box u;
      for (int k = 0; k < 3; ++k) {
        u.lo[k] = INFINITY;
        u.hi[k] = -INFINITY;
      }
      for (int i : ids)
        for (int k = 0; k < 3; ++k) {
          u.lo[k] = std::min(u.lo[k], bx.pt[i].lo[k]);
          u.hi[k] = std::max(u.hi[k], bx.pt[i].hi[k]);
        }
      return u;
    };
    if (o.prm.enable_pt) {
      std::vector<int> pI = near(bx.pt, o.voff[I], o.voff[I + 1], bx.body[J]);
      if (!pI.empty()) {
        std::vector<int> tJ = near(bx.tr, o.toff[J], o.toff[J + 1], unite(pI));
        for (int a : pI)
          for (int t : tJ)
            if (overlap(bx.pt[a], bx.tr[t])) ptp[q].push_back({I, J, q, a - o.voff[I], t - o.toff[J]});
      }
      std::vector<int> pJ = near(bx.pt, o.voff[J], o.voff[J + 1], bx.body[I]);
      if (!pJ.empty()) {
        std::vector<int> tI = near(bx.tr, o.toff[I], o.toff[I + 1], unite(pJ));
        for (int a : pJ)
          for (int t : tI)
            if (overlap(bx.pt[a], bx.tr[t])) ptp[q].push_back({J, I, q, a - o.voff[J], t - o.toff[I]});
      }
    }
    if (o.prm.enable_ee) {
      std::vector<int> eI = near(bx.ed, o.eoff[I], o.eoff[I + 1], bx.body[J]);
      std::vector<int> eJ = near(bx.ed, o.eoff[J], o.eoff[J + 1], bx.body[I]);
      for (int a : eI)
        for (int b : eJ)
          if (overlap(bx.ed[a], bx.ed[b])) eep[q].push_back({I, J, q, a - o.eoff[I], b - o.eoff[J]});
    }
  }
  L.pt.clear();
  L.ee.clear();
  for (int q = 0; q < m; ++q) {
    L.pt.insert(L.pt.end(), ptp[q].begin(), ptp[q].end());
    L.ee.insert(L.ee.end(), eep[q].begin(), eep[q].end());
  }
  L.vg.clear();
  if (o.prm.ground_enabled && o.prm.enable_vg) {
    const float g32 = (float)o.prm.ground;
    Box gq;
    gq.lo[0] = gq.lo[1] = gq.lo[2] = -1e3f;
    gq.hi[0] = 1e3f;
    gq.hi[1] = g32;
    gq.hi[2] = 1e3f;
    for (int b = 0; b < o.n; ++b) {
      if (!((double)bx.body[b].lo[1] < 0.5 * o.prm.dhat + o.prm.ground)) continue;
      for (int v = o.voff[b]; v < o.voff[b + 1]; ++v)
        if (overlap(bx.pt[v], gq)) {
          L.vg.push_back(b);
          L.vg.push_back(v);
        }
    }
  }
}

// ---------------------------------------------------------------------------------------
// per-primitive geometry (psd/vf.py, psd/ee.py, psd/hl.py, ccd.py:44-54)
// ---------------------------------------------------------------------------------------
inline void solve22(V3 e0, V3 e1, V3 e2, double& beta, double& gamma) {
  const double a = dot(e0, e0), b = dot(e0, e1), d = dot(e1, e1);
  const double det = a * d - b * b;
  const double s = 1.0 / det;
  const double i00 = d * s, i01 = -b * s, i10 = -b * s, i11 = a * s;
  const double r0 = dot(e0, e2), r1 = dot(e1, e2);
  beta = i00 * r0 + i01 * r1;
  gamma = i10 * r0 + i11 * r1;
}

struct Geo {
  V3 e0, e1p, e2p;
  double alpha, beta, gamma;
};

// type 0: point-triangle (x0 point; x1,x2,x3 triangle); type 1: edge-edge
inline Geo geometry(int type, V3 x0, V3 x1, V3 x2, V3 x3) {
  Geo G;
  V3 e0, e1, e2;
  if (type == 0) {
    e0 = x1 - x2;
    e1 = x3 - x2;
    e2 = x0 - x2;
  } else {
    e0 = x1 - x0;
    e1 = x3 - x2;
    e2 = x2 - x0;
  }
  G.alpha = dot(e0, e1) / dot(e0, e0);
  G.e0 = e0;
  G.e1p = e1 - G.alpha * e0;
  solve22(e0, e1, e2, G.beta, G.gamma);
  G.e2p = (e2 - G.beta * e0) - G.gamma * e1;
  return G;
}

inline bool valid_root(int type, double beta, double gamma) {
  if (type == 0) return 0.0 < beta && beta < 1.0 && 0.0 < gamma && gamma < 1.0 && 0.0 < beta + gamma &&
                        beta + gamma < 1.0;
  return 0.0 < beta && beta < 1.0 && 0.0 < -gamma && -gamma < 1.0;
}

inline double signed_distance(V3 e0p, V3 e1p, V3 e2p) {
  V3 n = cross(e0p, e1p);
  return dot(e2p, n) / std::sqrt(dot(n, n));
}

inline double barrier(double d, const Params& P) {
  if (d < P.d2hat) {
    const double s = d / P.d2hat;
    const double t = s - 1.0;  // pow(s - 1, 2.0) as its correctly rounded value
    return P.kappa * -(t * t) * abd_log(s);
  }
  return 0.0;
}
inline double barrier_d1(double d, const Params& P) {
  if (d < P.d2hat)
    return P.kappa * (P.d2hat - d) * (2.0 * abd_log(d / P.d2hat) + (d - P.d2hat) / d) / (P.d2hat * P.d2hat);
  return 0.0;
}
inline double barrier_d2(double d, const Params& P) {
  if (d < P.d2hat)
    return -P.kappa *
           (2.0 * abd_log(d / P.d2hat) + (d - P.d2hat) / d + (d - P.d2hat) * (2.0 / d + P.d2hat / (d * d))) /
           (P.d2hat * P.d2hat);
  return 0.0;
}

// Contact gradient (24) and Hessian blocks (3 x 12x12) of one PT/EE pair
// (pt_ipc.py:111-185, 194-246; ee_ipc.py:381-475).  Returns false when inactive.
bool contact_gh(int type, const V3 xs[4], const V3 rs[4], const Params& P, double& d2out, double g24[24],
                double Hi[144], double Hj[144], double Hij[144]) {
  Geo G = geometry(type, xs[0], xs[1], xs[2], xs[3]);
  const bool valid = valid_root(type, G.beta, G.gamma);
  double d2;
  if (type == 0) {
    const double l = signed_distance(G.e0, G.e1p, G.e2p);
    d2 = l * l;
  } else {
    d2 = dot(G.e2p, G.e2p);
  }
  d2out = d2;
  if (!(d2 < P.d2hat && valid)) return false;
  const double l = signed_distance(G.e0, G.e1p, G.e2p);
  const double e0pn = dot(G.e0, G.e0), e1pn = dot(G.e1p, G.e1p), e2pn = dot(G.e2p, G.e2p);
  const double f12 = std::sqrt(1.0 + 4.0 * (e1pn / e2pn));
  const double f02 = std::sqrt(1.0 + 4.0 * (e0pn / e2pn));
  double lam[5];
  lam[0] = -l / (2.0 * e1pn) * (1.0 + f12);
  lam[1] = -l / (2.0 * e1pn) * (1.0 - f12);
  lam[2] = -l / (2.0 * e0pn) * (1.0 + f02);
  lam[3] = -l / (2.0 * e0pn) * (1.0 - f02);
  double om[4];
  for (int k = 0; k < 4; ++k) om[k] = lam[k] / (lam[k] - l / e2pn);
  double Q[5][9];
  std::memset(Q, 0, sizeof(Q));
  for (int k = 0; k < 2; ++k) {
    V3 t = om[k] * G.e1p;
    Q[k][3] = G.e2p.x; Q[k][4] = G.e2p.y; Q[k][5] = G.e2p.z;
    Q[k][6] = t.x; Q[k][7] = t.y; Q[k][8] = t.z;
  }
  for (int k = 2; k < 4; ++k) {
    V3 t = om[k] * G.e0;
    Q[k][0] = G.e2p.x; Q[k][1] = G.e2p.y; Q[k][2] = G.e2p.z;
    Q[k][6] = t.x; Q[k][7] = t.y; Q[k][8] = t.z;
  }
  {
    V3 gl2 = G.e2p * l;
    gl2 = {gl2.x / e2pn, gl2.y / e2pn, gl2.z / e2pn};
    V3 q4 = (gl2 * 2.0) * l;
    Q[4][6] = q4.x; Q[4][7] = q4.y; Q[4][8] = q4.z;
  }
  for (int k = 0; k < 4; ++k) lam[k] = lam[k] * 2.0 * l;
  lam[4] = 2.0;
  const double Bp = barrier_d1(d2, P), Bpp = barrier_d2(d2, P);
  double q4n = 0.0;
  for (int i = 0; i < 9; ++i) q4n += Q[4][i] * Q[4][i];
  if (P.contact_psd == 1) {
    // projected barrier Hessian: eigenvalues of B' Hc + B'' q4 q4^T on the (orthogonal)
    // eigenvectors q_k, clamped at zero; the B'' term is folded into the fifth pair
    for (int k = 0; k < 4; ++k) lam[k] = std::max(Bp * lam[k], 0.0);
    lam[4] = std::max(Bp * 2.0 + Bpp * q4n, 0.0);
  } else if (type == 0 || P.psd_ee) {
    for (int k = 0; k < 4; ++k) lam[k] = std::max(lam[k], 0.0);
  }
  // D (3x4): dcvfdx_s / dceedx_s
  double D[3][4];
  if (type == 0) {
    const double al = G.alpha, be = G.beta, ga = G.gamma;
    double t[3][4] = {{0.0, 1.0, -1.0, 0.0}, {0.0, -al, al - 1.0, 1.0}, {1.0, -be, be + ga - 1.0, -ga}};
    std::memcpy(D, t, sizeof(D));
  } else {
    const double al = G.alpha, be = G.beta, ga = G.gamma;
    double t[3][4] = {{-1.0, 1.0, 0.0, 0.0}, {al, -al, -1.0, 1.0}, {be - 1.0, -be, ga + 1.0, -ga}};
    std::memcpy(D, t, sizeof(D));
  }
  // Hc = Q diag(lam) diag(1/|q|^2) Q^T   (QLQinv)
  double qn[5];
  for (int k = 0; k < 5; ++k) {
    double s = 0.0;
    for (int i = 0; i < 9; ++i) s += Q[k][i] * Q[k][i];
    qn[k] = 1.0 / s;
  }
  double Hc[9][9];
  for (int a = 0; a < 9; ++a)
    for (int b = 0; b < 9; ++b) {
      double s = 0.0;
      for (int k = 0; k < 5; ++k) s += (Q[k][a] * lam[k]) * (qn[k] * Q[k][b]);
      Hc[a][b] = s;
    }
  // Hx = (D kron I)^T Hc (D kron I)  (dcTHldc), g12 = (D kron I)^T q4
  double Hx[12][12], g12[12];
  for (int j = 0; j < 4; ++j)
    for (int a = 0; a < 3; ++a) {
      double s = 0.0;
      for (int i = 0; i < 3; ++i) s += D[i][j] * Q[4][3 * i + a];
      g12[3 * j + a] = s;
    }
  {
    double T1[9][12];  // Hc (D kron I)
    for (int a = 0; a < 9; ++a)
      for (int l2 = 0; l2 < 4; ++l2)
        for (int b = 0; b < 3; ++b) {
          double s = 0.0;
          for (int k = 0; k < 3; ++k) s += Hc[a][3 * k + b] * D[k][l2];
          T1[a][3 * l2 + b] = s;
        }
    for (int j = 0; j < 4; ++j)
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 12; ++c) {
          double s = 0.0;
          for (int i = 0; i < 3; ++i) s += D[i][j] * T1[3 * i + a][c];
          Hx[3 * j + a][c] = s;
        }
  }
  double H12[12][12];
  for (int a = 0; a < 12; ++a)
    for (int b = 0; b < 12; ++b)
      H12[a][b] = (P.contact_psd == 1) ? Hx[a][b] : Hx[a][b] * Bp + g12[a] * g12[b] * Bpp;
  // body Jacobians: vertex v -> weights w_v = (1, r_v); PT: v0 in I, v1..3 in J;
  // EE: v0,v1 in I, v2,v3 in J
  const int nI = (type == 0) ? 1 : 2;
  double w[4][4];
  for (int v = 0; v < 4; ++v) {
    w[v][0] = 1.0;
    w[v][1] = rs[v].x;
    w[v][2] = rs[v].y;
    w[v][3] = rs[v].z;
  }
  // gradient: g_I[3m+a] = sum_{v in I} w_v[m] g12[3v+a] * B'
  for (int m = 0; m < 4; ++m)
    for (int a = 0; a < 3; ++a) {
      double sI = 0.0, sJ = 0.0;
      for (int v = 0; v < nI; ++v) sI += w[v][m] * g12[3 * v + a];
      for (int v = nI; v < 4; ++v) sJ += w[v][m] * g12[3 * v + a];
      g24[3 * m + a] = sI * Bp;
      g24[12 + 3 * m + a] = sJ * Bp;
    }
  for (int m = 0; m < 4; ++m)
    for (int a = 0; a < 3; ++a)
      for (int n2 = 0; n2 < 4; ++n2)
        for (int b = 0; b < 3; ++b) {
          double sII = 0.0, sJJ = 0.0, sIJ = 0.0;
          for (int u = 0; u < 4; ++u)
            for (int v = 0; v < 4; ++v) {
              const double h = w[u][m] * H12[3 * u + a][3 * v + b] * w[v][n2];
              const bool uI = u < nI, vI = v < nI;
              if (uI && vI) sII += h;
              else if (!uI && !vI) sJJ += h;
              else if (uI && !vI) sIJ += h;
            }
          Hi[(3 * m + a) * 12 + 3 * n2 + b] = sII;
          Hj[(3 * m + a) * 12 + 3 * n2 + b] = sJJ;
          Hij[(3 * m + a) * 12 + 3 * n2 + b] = sIJ;
        }
  return true;
}

// The same contact's gradient and Hessian as 5 rank-one terms (the form the assembly sums):
//   H = sum_k coef[k] u_k u_k^T,  g = B' u_4,
// u_k (24: the pair's first body, then its second) = W^T (D kron I3)^T q_k with q_k the
// eigenvectors of the c-space Hessian of l^2 (q_4 = grad l^2), D = dc/dx (3x4, frozen
// alpha, beta, gamma) and W the vertex weights [1, r_v].  Mathematically identical to
// contact_gh (which follows the reference's matrix products); the assembly uses this form
// and its operation order.  `swap`: the candidate's first vertex group (point / first edge)
// belongs to the pair's second body.  out[456]: H_IJ (144), H_II (144), H_JJ (144), g (24).
bool contact_terms(int type, const V3 xs[4], const V3 rs[4], int swap, const Params& P, double out[456]) {
  Geo G = geometry(type, xs[0], xs[1], xs[2], xs[3]);
  const bool valid = valid_root(type, G.beta, G.gamma);
  double d2;
  if (type == 0) {
    const double l = signed_distance(G.e0, G.e1p, G.e2p);
    d2 = l * l;
  } else {
    d2 = dot(G.e2p, G.e2p);
  }
  if (!(d2 < P.d2hat && valid)) return false;
  const double l = signed_distance(G.e0, G.e1p, G.e2p);
  const double e0pn = dot(G.e0, G.e0), e1pn = dot(G.e1p, G.e1p), e2pn = dot(G.e2p, G.e2p);
  const double f12 = std::sqrt(1.0 + 4.0 * (e1pn / e2pn));
  const double f02 = std::sqrt(1.0 + 4.0 * (e0pn / e2pn));
  double lam[5];
  lam[0] = -l / (2.0 * e1pn) * (1.0 + f12);
  lam[1] = -l / (2.0 * e1pn) * (1.0 - f12);
  lam[2] = -l / (2.0 * e0pn) * (1.0 + f02);
  lam[3] = -l / (2.0 * e0pn) * (1.0 - f02);
  double om[4];
  for (int k = 0; k < 4; ++k) om[k] = lam[k] / (lam[k] - l / e2pn);
  double q[5][9];
  std::memset(q, 0, sizeof(q));
  for (int k = 0; k < 2; ++k) {
    V3 t = om[k] * G.e1p;
    q[k][3] = G.e2p.x; q[k][4] = G.e2p.y; q[k][5] = G.e2p.z;
    q[k][6] = t.x; q[k][7] = t.y; q[k][8] = t.z;
  }
  for (int k = 2; k < 4; ++k) {
    V3 t = om[k] * G.e0;
    q[k][0] = G.e2p.x; q[k][1] = G.e2p.y; q[k][2] = G.e2p.z;
    q[k][6] = t.x; q[k][7] = t.y; q[k][8] = t.z;
  }
  {
    V3 gl2 = G.e2p * l;
    gl2 = {gl2.x / e2pn, gl2.y / e2pn, gl2.z / e2pn};
    V3 q4 = (gl2 * 2.0) * l;
    q[4][6] = q4.x; q[4][7] = q4.y; q[4][8] = q4.z;
  }
  for (int k = 0; k < 4; ++k) lam[k] = lam[k] * 2.0 * l;
  lam[4] = 2.0;
  double qn[5];
  for (int k = 0; k < 5; ++k) {
    double sq = 0.0;
    for (int i = 0; i < 9; ++i) sq += q[k][i] * q[k][i];
    qn[k] = sq;
  }
  const double Bp = barrier_d1(d2, P), Bpp = barrier_d2(d2, P);
  double coef[5];
  if (P.contact_psd == 1) {
    for (int k = 0; k < 4; ++k) coef[k] = std::fmax(Bp * lam[k], 0.0) / qn[k];
    coef[4] = std::fmax(Bp * 2.0 + Bpp * qn[4], 0.0) / qn[4];
  } else {
    const bool clamp = (type == 0) || P.psd_ee;
    for (int k = 0; k < 4; ++k) coef[k] = Bp * (clamp ? std::fmax(lam[k], 0.0) : lam[k]) / qn[k];
    coef[4] = Bp * 2.0 / qn[4] + Bpp;
  }
  const double al = G.alpha, be = G.beta, ga = G.gamma;
  double D[3][4];
  if (type == 0) {
    const double t[3][4] = {{0.0, 1.0, -1.0, 0.0}, {0.0, -al, al - 1.0, 1.0}, {1.0, -be, be + ga - 1.0, -ga}};
    std::memcpy(D, t, sizeof(D));
  } else {
    const double t[3][4] = {{-1.0, 1.0, 0.0, 0.0}, {al, -al, -1.0, 1.0}, {be - 1.0, -be, ga + 1.0, -ga}};
    std::memcpy(D, t, sizeof(D));
  }
  double u[5][24];
  for (int e = 0; e < 24; ++e) {
    const int side = e / 12, m = (e % 12) / 3, c = e % 3;
    const int group = side ^ swap;
    const int v0 = type == 0 ? (group ? 1 : 0) : (group ? 2 : 0);
    const int v1 = type == 0 ? (group ? 4 : 1) : (group ? 4 : 2);
    double dw[3];
    for (int i = 0; i < 3; ++i) {
      double sacc = 0.0;
      for (int v = v0; v < v1; ++v) {
        const double w = m == 0 ? 1.0 : (m == 1 ? rs[v].x : (m == 2 ? rs[v].y : rs[v].z));
        sacc += D[i][v] * w;
      }
      dw[i] = sacc;
    }
    for (int k = 0; k < 5; ++k) u[k][e] = dw[0] * q[k][c] + dw[1] * q[k][3 + c] + dw[2] * q[k][6 + c];
  }
  for (int e = 0; e < 456; ++e) {
    double v = 0.0;
    if (e < 432) {
      const int blk = e / 144, r = (e % 144) / 12, c = e % 12;
      const int ra = blk == 2 ? 12 + r : r;
      const int cb = blk == 1 ? c : 12 + c;
      for (int k = 0; k < 5; ++k) v += coef[k] * (u[k][ra] * u[k][cb]);
    } else {
      v = Bp * u[4][e - 432];
    }
    out[e] = v;
  }
  return true;
}

inline void fetch(const Oracle& o, const double* y, const Cand& c, int type, V3 xs[4], V3 rs[4]) {
  int ids[4];
  if (type == 0) {
    ids[0] = o.voff[c.I] + c.pi;
    const int t = o.toff[c.J] + c.pj;
    ids[1] = o.tris[3 * t];
    ids[2] = o.tris[3 * t + 1];
    ids[3] = o.tris[3 * t + 2];
  } else {
    const int ea = o.eoff[c.I] + c.pi, eb = o.eoff[c.J] + c.pj;
    ids[0] = o.edges[2 * ea];
    ids[1] = o.edges[2 * ea + 1];
    ids[2] = o.edges[2 * eb];
    ids[3] = o.edges[2 * eb + 1];
  }
  for (int k = 0; k < 4; ++k) {
    xs[k] = {y[3 * ids[k]], y[3 * ids[k] + 1], y[3 * ids[k] + 2]};
    rs[k] = {o.x0[3 * ids[k]], o.x0[3 * ids[k] + 1], o.x0[3 * ids[k] + 2]};
  }
}

// contact energy of one candidate (ipcsk/energy.py:9-48)
inline double contact_energy(int type, const V3 xs[4], const Params& P) {
  Geo G = geometry(type, xs[0], xs[1], xs[2], xs[3]);
  if (!valid_root(type, G.beta, G.gamma)) return 0.0;
  double d2;
  if (type == 0) {
    d2 = dot(G.e2p, G.e2p);
  } else {
    const double d = signed_distance(G.e0, G.e1p, G.e2p);
    d2 = d * d;
  }
  return barrier(d2, P);
}

// ---------------------------------------------------------------------------------------
// Full IPC contact model (opt-in, Oracle::ipc_full): the closest feature pair of a PT or EE
// candidate (point-triangle / point-edge / point-point; line-line / point-edge /
// point-point), the barrier on its squared distance, the edge-edge mollifier below
// e_x = 1e-3 |a_rest|^2 |b_rest|^2, and the local 12x12 Hessian projected to PSD per contact
// (Li et al., "Incremental Potential Contact", SIGGRAPH 2020).  The reference evaluates only
// the interior cases (ipcsk/energy.py:20-22, 46-48; ccd.py:44-54).  Derivatives: forward-mode
// automatic differentiation carrying the full gradient and Hessian through every operation.
// ---------------------------------------------------------------------------------------
struct D12 {
  double v;
  double g[12];
  double H[144];
};
inline D12 d12_const(double x) {
  D12 r;
  r.v = x;
  std::memset(r.g, 0, sizeof(r.g));
  std::memset(r.H, 0, sizeof(r.H));
  return r;
}
inline D12 d12_var(double x, int i) {
  D12 r = d12_const(x);
  r.g[i] = 1.0;
  return r;
}
inline D12 operator+(const D12& a, const D12& b) {
  D12 r;
  r.v = a.v + b.v;
  for (int i = 0; i < 12; ++i) r.g[i] = a.g[i] + b.g[i];
  for (int i = 0; i < 144; ++i) r.H[i] = a.H[i] + b.H[i];
  return r;
}
inline D12 operator-(const D12& a, const D12& b) {
  D12 r;
  r.v = a.v - b.v;
  for (int i = 0; i < 12; ++i) r.g[i] = a.g[i] - b.g[i];
  for (int i = 0; i < 144; ++i) r.H[i] = a.H[i] - b.H[i];
  return r;
}
inline D12 operator*(const D12& a, const D12& b) {
  D12 r;
  r.v = a.v * b.v;
  for (int i = 0; i < 12; ++i) r.g[i] = a.v * b.g[i] + b.v * a.g[i];
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j)
      r.H[12 * i + j] = a.v * b.H[12 * i + j] + b.v * a.H[12 * i + j] + a.g[i] * b.g[j] + b.g[i] * a.g[j];
  return r;
}
inline D12 scale(const D12& a, double s) {
  D12 r;
  r.v = a.v * s;
  for (int i = 0; i < 12; ++i) r.g[i] = a.g[i] * s;
  for (int i = 0; i < 144; ++i) r.H[i] = a.H[i] * s;
  return r;
}
// f(a) from f, f', f'' at a.v (chain rule)
inline D12 apply(const D12& a, double f, double f1, double f2) {
  D12 r;
  r.v = f;
  for (int i = 0; i < 12; ++i) r.g[i] = f1 * a.g[i];
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) r.H[12 * i + j] = f1 * a.H[12 * i + j] + f2 * a.g[i] * a.g[j];
  return r;
}
inline D12 operator/(const D12& a, const D12& b) {
  const double q = 1.0 / b.v;
  return a * apply(b, q, -q * q, 2.0 * q * q * q);
}
struct V3D {
  D12 x, y, z;
};
inline V3D vsub(const V3D& a, const V3D& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D12 vdot(const V3D& a, const V3D& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3D vcross(const V3D& a, const V3D& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// closest-feature types (triangle edges E0 = t0t1, E1 = t1t2, E2 = t2t0; edge a = x0x1,
// edge b = x2x3)
enum { F_PT = 0, F_PE0, F_PE1, F_PE2, F_PV0, F_PV1, F_PV2 };
enum { F_EE = 0, F_A0B, F_A1B, F_AB0, F_AB1, F_A0B0, F_A0B1, F_A1B0, F_A1B1 };

// clamped parameter of the point of segment [a, b] nearest p, and the squared distance
inline double seg_param(V3 p, V3 a, V3 b, double& d2) {
  const V3 e = b - a;
  const double ee = dot(e, e);
  double s = ee > 0.0 ? dot(p - a, e) / ee : 0.0;
  s = std::min(1.0, std::max(0.0, s));
  const V3 c = a + e * s;
  d2 = dot(p - c, p - c);
  return s;
}

// Point-triangle: the interior when the point's projection has non-negative barycentric
// coordinates (from sub-triangle areas); else the nearest edge as a segment (an edge or one
// of its end points), ties to the first of E0, E1, E2.
int full_pt_type(const V3 x[4]) {
  const V3 p = x[0], t0 = x[1], t1 = x[2], t2 = x[3];
  const V3 n = cross(t1 - t0, t2 - t0);
  const double nn = dot(n, n);
  if (nn > 0.0) {
    const V3 q = p - n * (dot(p - t0, n) / nn);
    const double u = dot(cross(t1 - q, t2 - q), n), v = dot(cross(t2 - q, t0 - q), n),
                 w = dot(cross(t0 - q, t1 - q), n);
    if (u >= 0.0 && v >= 0.0 && w >= 0.0) return F_PT;
  }
  const V3 tv[3] = {t0, t1, t2};
  int best = 0;
  double bd = 0.0, bs = 0.0;
  for (int k = 0; k < 3; ++k) {
    double d2;
    const double s = seg_param(p, tv[k], tv[(k + 1) % 3], d2);
    if (k == 0 || d2 < bd) {
      best = k;
      bd = d2;
      bs = s;
    }
  }
  if (bs <= 0.0) return F_PV0 + best;
  if (bs >= 1.0) return F_PV0 + (best + 1) % 3;
  return F_PE0 + best;
}

// Edge-edge: line-line when the stationary point of the two lines' distance lies inside
// both segments; else the nearest end point to segment distance (a0, a1 to b; b0, b1 to a),
// ties to the first.
int full_ee_type(const V3 x[4]) {
  const V3 u = x[1] - x[0], v = x[3] - x[2], w = x[0] - x[2];
  const double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), e = dot(v, w);
  const double D = a * c - b * b;
  if (D > 0.0) {
    const double s = (b * e - c * d) / D, t = (a * e - b * d) / D;
    if (s > 0.0 && s < 1.0 && t > 0.0 && t < 1.0) return F_EE;
  }
  double d2[4], s[4];
  s[0] = seg_param(x[0], x[2], x[3], d2[0]);
  s[1] = seg_param(x[1], x[2], x[3], d2[1]);
  s[2] = seg_param(x[2], x[0], x[1], d2[2]);
  s[3] = seg_param(x[3], x[0], x[1], d2[3]);
  int k = 0;
  for (int m = 1; m < 4; ++m)
    if (d2[m] < d2[k]) k = m;
  const int edge[4] = {F_A0B, F_A1B, F_AB0, F_AB1}, at0[4] = {F_A0B0, F_A1B0, F_A0B0, F_A0B1},
            at1[4] = {F_A0B1, F_A1B1, F_A1B0, F_A1B1};
  return s[k] <= 0.0 ? at0[k] : (s[k] >= 1.0 ? at1[k] : edge[k]);
}

inline D12 full_d2_point_line(const V3D& p, const V3D& a, const V3D& b) {
  const V3D c = vcross(vsub(a, p), vsub(b, p)), e = vsub(b, a);
  return vdot(c, c) / vdot(e, e);
}
inline D12 full_d2_pp(const V3D& p, const V3D& q) {
  const V3D d = vsub(p, q);
  return vdot(d, d);
}
inline D12 full_d2_plane(const V3D& p, const V3D& o, const V3D& n) {
  const D12 s = vdot(vsub(p, o), n);
  return (s * s) / vdot(n, n);
}

// squared distance of feature pair `type` (kind 0 PT, 1 EE) on AD variables
D12 full_d2(int kind, int type, const V3D X[4]) {
  if (kind == 0) {
    switch (type) {
      case F_PT: return full_d2_plane(X[0], X[1], vcross(vsub(X[2], X[1]), vsub(X[3], X[1])));
      case F_PE0: return full_d2_point_line(X[0], X[1], X[2]);
      case F_PE1: return full_d2_point_line(X[0], X[2], X[3]);
      case F_PE2: return full_d2_point_line(X[0], X[3], X[1]);
      default: return full_d2_pp(X[0], X[1 + type - F_PV0]);
    }
  }
  switch (type) {
    case F_EE: return full_d2_plane(X[2], X[0], vcross(vsub(X[1], X[0]), vsub(X[3], X[2])));
    case F_A0B: return full_d2_point_line(X[0], X[2], X[3]);
    case F_A1B: return full_d2_point_line(X[1], X[2], X[3]);
    case F_AB0: return full_d2_point_line(X[2], X[0], X[1]);
    case F_AB1: return full_d2_point_line(X[3], X[0], X[1]);
    case F_A0B0: return full_d2_pp(X[0], X[2]);
    case F_A0B1: return full_d2_pp(X[0], X[3]);
    case F_A1B0: return full_d2_pp(X[1], X[2]);
    default: return full_d2_pp(X[1], X[3]);
  }
}

// energy of one candidate with its derivatives in the four points' coordinates; false when
// the classified distance is not below dhat^2
bool full_energy_d(int kind, const V3 xs[4], const V3 rs[4], const Params& P, D12& E, double* d2out = nullptr) {
  const int type = kind == 0 ? full_pt_type(xs) : full_ee_type(xs);
  V3D X[4];
  for (int k = 0; k < 4; ++k) X[k] = {d12_var(xs[k].x, 3 * k), d12_var(xs[k].y, 3 * k + 1), d12_var(xs[k].z, 3 * k + 2)};
  const D12 d = full_d2(kind, type, X);
  if (d2out) *d2out = d.v;
  if (!(d.v < P.d2hat)) return false;
  // b(d) = -kappa (d / dh - 1)^2 log(d / dh) and its first two derivatives in d
  const double dh = P.d2hat, s = d.v / dh, l = std::log(s);
  const double f = -P.kappa * (s - 1.0) * (s - 1.0) * l;
  const double f1 = -P.kappa * (2.0 * (s - 1.0) * l + (s - 1.0) * (s - 1.0) / s) / dh;
  const double f2 = -P.kappa * (2.0 * l + 4.0 * (s - 1.0) / s - (s - 1.0) * (s - 1.0) / (s * s)) / (dh * dh);
  E = apply(d, f, f1, f2);
  if (kind == 1) {  // mollifier m(c) = (2 - c / e_x) c / e_x below e_x, c = |a x b|^2
    const V3 ra = rs[1] - rs[0], rb = rs[3] - rs[2];
    const double ex = 1e-3 * dot(ra, ra) * dot(rb, rb);
    const V3D nv = vcross(vsub(X[1], X[0]), vsub(X[3], X[2]));
    const D12 c = vdot(nv, nv);
    if (c.v < ex) E = E * apply(c, (2.0 - c.v / ex) * c.v / ex, 2.0 / ex - 2.0 * c.v / (ex * ex), -2.0 / (ex * ex));
  }
  return true;
}

// symmetric 12x12 matrix onto the PSD cone (cyclic Jacobi, negative eigenvalues dropped)
void psd12(double* H) {
  double A[12][12], Q[12][12];
  double fro = 0.0;
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) {
      A[i][j] = 0.5 * (H[12 * i + j] + H[12 * j + i]);
      Q[i][j] = i == j ? 1.0 : 0.0;
      fro += A[i][j] * A[i][j];
    }
  if (!(fro > 0.0)) return;
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < 12; ++i)
      for (int j = 0; j < 12; ++j)
        if (i != j) off += A[i][j] * A[i][j];
    if (off <= 1e-30 * fro) break;
    for (int p = 0; p < 12; ++p)
      for (int q = p + 1; q < 12; ++q) {
        if (A[p][q] == 0.0) continue;
        const double th = 0.5 * std::atan2(2.0 * A[p][q], A[q][q] - A[p][p]);
        const double c = std::cos(th), s = std::sin(th);
        for (int k = 0; k < 12; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 12; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 12; ++k) {
          const double qkp = Q[k][p], qkq = Q[k][q];
          Q[k][p] = c * qkp - s * qkq;
          Q[k][q] = s * qkp + c * qkq;
        }
      }
  }
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 12; ++k)
        if (A[k][k] > 0.0) acc += Q[i][k] * A[k][k] * Q[j][k];
      H[12 * i + j] = acc;
    }
}

// The pair terms of one candidate under the full model, in contact_terms' layout: out[456] =
// H_IJ, H_II, H_JJ, g (the pair's first body, then its second); `swap`: the candidate's
// first group (point / edge a) belongs to the pair's second body.
bool full_terms(int kind, const V3 xs[4], const V3 rs[4], int swap, const Params& P, double out[456]) {
  D12 E;
  if (!full_energy_d(kind, xs, rs, P, E)) return false;
  double H[144];
  std::memcpy(H, E.H, sizeof(H));
  psd12(H);
  const int nI = kind == 0 ? 1 : 2;  // points of the first group
  // x_a = p_a + sum_k r_k A_ka: weights (1, r) of DOF group m for point v
  double w[4][4];
  for (int v = 0; v < 4; ++v) {
    w[v][0] = 1.0;
    w[v][1] = rs[v].x;
    w[v][2] = rs[v].y;
    w[v][3] = rs[v].z;
  }
  double G[2][12], B[2][2][144];
  std::memset(G, 0, sizeof(G));
  std::memset(B, 0, sizeof(B));
  for (int u = 0; u < 4; ++u)
    for (int m = 0; m < 4; ++m)
      for (int a = 0; a < 3; ++a) {
        const int gu = u < nI ? 0 : 1;
        G[gu][3 * m + a] += w[u][m] * E.g[3 * u + a];
        for (int v = 0; v < 4; ++v)
          for (int n2 = 0; n2 < 4; ++n2)
            for (int b = 0; b < 3; ++b)
              B[gu][v < nI ? 0 : 1][12 * (3 * m + a) + 3 * n2 + b] += w[u][m] * H[12 * (3 * u + a) + 3 * v + b] * w[v][n2];
      }
  const int I = swap ? 1 : 0, J = 1 - I;  // groups of the pair's first and second body
  for (int e = 0; e < 144; ++e) {
    out[e] = B[I][J][e];
    out[144 + e] = B[I][I][e];
    out[288 + e] = B[J][J][e];
  }
  for (int e = 0; e < 12; ++e) {
    out[432 + e] = G[I][e];
    out[444 + e] = G[J][e];
  }
  return true;
}

double full_energy(int kind, const V3 xs[4], const V3 rs[4], const Params& P) {
  D12 E;
  return full_energy_d(kind, xs, rs, P, E) ? E.v : 0.0;
}

// The full model in the CUDA library's arithmetic (abd_ipc_full.cuh with the shared log): the
// energy, and a contact's 456 affine terms as the pair assembly forms them -- the local Hessian
// and gradient from hyper-dual entries, projected onto the PSD cone, then each affine entry
// summed over the contact's vertices in the kernel's order (vertex u, then w)
inline void pts12(const V3 v[4], double x[12]) {
  for (int k = 0; k < 4; ++k) {
    x[3 * k] = v[k].x;
    x[3 * k + 1] = v[k].y;
    x[3 * k + 2] = v[k].z;
  }
}
double full_energy_hd(int kind, const V3 xs[4], const V3 rs[4], const Params& P) {
  double x[12], r[12];
  pts12(xs, x);
  pts12(rs, r);
  abd::ipc::V3<double> v[4];
  abd::ipc::load(x, v);
  const int ty = abd::ipc::contact_type(kind, x);
  const double d2 = kind == 0 ? abd::ipc::pt_d2(ty, v) : abd::ipc::ee_d2(ty, v);
  if (!(d2 < P.d2hat)) return 0.0;
  return abd::ipc::local_energy(kind, ty, v, kind == 1 ? abd::ipc::ee_eps_x(r) : 0.0, P.d2hat, P.kappa,
                                [](double u) { return abd_log(u); });
}
void affine_map_hd(int kind, const double r[12], int swap, const double* H, const double* g, double out[456]);
bool full_terms_hd(int kind, const V3 xs[4], const V3 rs[4], int swap, const Params& P, double out[456]) {
  double x[12], r[12], H[144], g[12], E, d2;
  int ty;
  pts12(xs, x);
  pts12(rs, r);
  if (!abd::ipc::local_gh(kind, x, r, P.d2hat, P.kappa, [](double u) { return abd_log(u); }, &ty, &d2, &E, g, H))
    return false;
  abd::ipc::project_psd12(H);
  affine_map_hd(kind, r, swap, H, g, out);
  return true;
}

// A contact's point-coordinate gradient g[12] and Hessian H[144] as the pair terms out[456]
// (H_IJ, H_II, H_JJ, g_I, g_J) of its two bodies' affine DOFs, with the CUDA library's
// summation order: the first nI points (the point; edge a) move with the first group's body,
// which is the pair's first body unless swapped; r: the points' rest positions.
void affine_map_hd(int kind, const double r[12], int swap, const double* H, const double* g, double out[456]) {
  const int nI = kind == 0 ? 1 : 2;
  auto side = [&](int v) { return (v < nI ? 0 : 1) ^ swap; };
  auto wt = [&](int v, int m) { return m == 0 ? 1.0 : r[3 * v + m - 1]; };
  for (int e = 0; e < 456; ++e) {
    double val = 0.0;
    if (e < 432) {
      const int blk = e / 144, rw = (e % 144) / 12, c = e % 12;
      const int rsd = blk == 2 ? 1 : 0, csd = blk == 1 ? 0 : 1;
      const int m = rw / 3, ra = rw % 3, n = c / 3, cb = c % 3;
      for (int u = 0; u < 4; ++u) {
        if (side(u) != rsd) continue;
        for (int w = 0; w < 4; ++w)
          if (side(w) == csd) val += (wt(u, m) * H[12 * (3 * u + ra) + 3 * w + cb]) * wt(w, n);
      }
    } else {
      const int k = e - 432, sd = k / 12, m = (k % 12) / 3, comp = k % 3;
      for (int u = 0; u < 4; ++u)
        if (side(u) == sd) val += wt(u, m) * g[3 * u + comp];
    }
    out[e] = val;
  }
}

// ---------------------------------------------------------------------------------------
// Lagged friction (Li et al. 2020, section 5), with the full contact model: at the step start
// each contact within dhat fixes the weights w of its closest points (c_a - c_b =
// sum_v w_v x_v), a basis P of the plane orthogonal to c_a - c_b, and its normal force
// lambda = -dE/dd.  D(x) = mu lambda f0(|P^T sum_v w_v (x_v - x^t_v)|), f0' = 2y/eps -
// y^2/eps^2 below eps = eps_v dt, 1 above.
// ---------------------------------------------------------------------------------------
void fric_weights(int kind, int type, const V3 x[4], double w[4]) {
  for (int k = 0; k < 4; ++k) w[k] = 0.0;
  w[0] = 1.0;
  if (kind == 0) {
    const V3 p = x[0], t0 = x[1], t1 = x[2], t2 = x[3];
    if (type == F_PT) {  // barycentric coordinates of the projection from sub-triangle areas
      const V3 n = cross(t1 - t0, t2 - t0);
      const double nn = dot(n, n);
      const V3 q = p - n * (dot(p - t0, n) / nn);
      w[1] = -dot(cross(t1 - q, t2 - q), n) / nn;
      w[2] = -dot(cross(t2 - q, t0 - q), n) / nn;
      w[3] = -dot(cross(t0 - q, t1 - q), n) / nn;
    } else if (type <= F_PE2) {
      const int a = type - F_PE0, b = (a + 1) % 3;
      double d2;
      const double s = seg_param(p, x[1 + a], x[1 + b], d2);
      w[1 + a] = -(1.0 - s);
      w[1 + b] = -s;
    } else {
      w[1 + type - F_PV0] = -1.0;
    }
    return;
  }
  double s = 0.0, t = 0.0, d2;
  if (type == F_EE) {
    const V3 u = x[1] - x[0], v = x[3] - x[2], q = x[0] - x[2];
    const double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, q), e = dot(v, q);
    const double D = a * c - b * b;
    s = (b * e - c * d) / D;
    t = (a * e - b * d) / D;
  } else if (type == F_A0B) {
    t = seg_param(x[0], x[2], x[3], d2);
  } else if (type == F_A1B) {
    s = 1.0;
    t = seg_param(x[1], x[2], x[3], d2);
  } else if (type == F_AB0) {
    s = seg_param(x[2], x[0], x[1], d2);
  } else if (type == F_AB1) {
    s = seg_param(x[3], x[0], x[1], d2);
    t = 1.0;
  } else {
    s = (type == F_A1B0 || type == F_A1B1) ? 1.0 : 0.0;
    t = (type == F_A0B1 || type == F_A1B1) ? 1.0 : 0.0;
  }
  w[0] = 1.0 - s;
  w[1] = s;
  w[2] = -(1.0 - t);
  w[3] = -t;
}

// the lagged quantities of one candidate at its step-start positions xs (rest positions rs);
// false when it is not within dhat there
bool make_fric(int kind, const V3 xs[4], const V3 rs[4], const Params& P, Oracle::Fric& f) {
  const int type = kind == 0 ? full_pt_type(xs) : full_ee_type(xs);
  fric_weights(kind, type, xs, f.w);
  V3 n = {0.0, 0.0, 0.0};
  for (int k = 0; k < 4; ++k) n = n + xs[k] * f.w[k];
  const double d2 = dot(n, n);
  if (!(d2 < P.d2hat) || !(d2 > 0.0)) return false;
  const double d = std::sqrt(d2);
  n = n * (1.0 / d);
  // basis: the coordinate axis least aligned with n, made orthogonal to it
  const double an[3] = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
  const int ax = an[0] <= an[1] && an[0] <= an[2] ? 0 : (an[1] <= an[2] ? 1 : 2);
  const V3 e = {ax == 0 ? 1.0 : 0.0, ax == 1 ? 1.0 : 0.0, ax == 2 ? 1.0 : 0.0};
  V3 t1 = cross(n, e);
  t1 = t1 * (1.0 / std::sqrt(dot(t1, t1)));
  const V3 t2 = cross(n, t1);
  const double B[6] = {t1.x, t2.x, t1.y, t2.y, t1.z, t2.z};
  std::memcpy(f.P, B, sizeof(B));
  double m = 1.0;
  if (kind == 1) {
    const V3 ra = rs[1] - rs[0], rb = rs[3] - rs[2];
    const double ex = 1e-3 * dot(ra, ra) * dot(rb, rb);
    const V3 c = cross(xs[1] - xs[0], xs[3] - xs[2]);
    const double cc = dot(c, c);
    if (cc < ex) m = (2.0 - cc / ex) * cc / ex;
  }
  f.lam = -2.0 * d * m * barrier_d1(d2, P);
  f.kind = kind;
  for (int k = 0; k < 4; ++k) {
    f.xt[3 * k] = xs[k].x, f.xt[3 * k + 1] = xs[k].y, f.xt[3 * k + 2] = xs[k].z;
    f.rs[3 * k] = rs[k].x, f.rs[3 * k + 1] = rs[k].y, f.rs[3 * k + 2] = rs[k].z;
  }
  return true;
}

// the contacts within dhat at DOFs (A0, p0), with their lagged quantities
void friction_lag(Oracle& o) {
  o.fric.clear();
  if (!(o.fr_mu > 0.0) || !o.ipc_full) return;
  std::vector<double> xt(3 * (size_t)o.V);
  transform(o, o.A0.data(), o.p0.data(), xt.data());
  Boxes bx;
  Lists L;
  static_boxes(o, xt.data(), bx);
  cull(o, bx, L);
  for (int kind = 0; kind < 2; ++kind)
    for (const Cand& cd : kind == 0 ? L.pt : L.ee) {
      V3 xs[4], rs[4];
      fetch(o, xt.data(), cd, kind, xs, rs);
      Oracle::Fric f;
      if (o.ipc_independent) {
        if (!make_fric(kind, xs, rs, o.prm, f)) continue;
      } else {  // the header's (the CUDA library's arithmetic)
        double x12[12], r12[12];
        pts12(xs, x12);
        pts12(rs, r12);
        if (!abd::ipc::friction_lag(kind, x12, r12, o.prm.d2hat, o.prm.kappa, [](double u) { return abd_log(u); },
                                    &f.hl))
          continue;
        f.kind = kind;
        std::memcpy(f.xt, x12, sizeof(x12));
        std::memcpy(f.rs, r12, sizeof(r12));
      }
      f.I = cd.I;
      f.J = cd.J;
      // the vertex ids, for reading the current positions
      if (kind == 0) {
        f.ids[0] = o.voff[cd.I] + cd.pi;
        const int t = o.toff[cd.J] + cd.pj;
        for (int k = 0; k < 3; ++k) f.ids[1 + k] = o.tris[3 * t + k];
      } else {
        const int ea = o.eoff[cd.I] + cd.pi, eb = o.eoff[cd.J] + cd.pj;
        f.ids[0] = o.edges[2 * ea];
        f.ids[1] = o.edges[2 * ea + 1];
        f.ids[2] = o.edges[2 * eb];
        f.ids[3] = o.edges[2 * eb + 1];
      }
      o.fric.push_back(f);
    }
}

// D, gradient g[12] and Hessian H[144] of one lagged contact at positions y (all vertices)
double friction_gh(double mu, double eps, const Oracle::Fric& f, const double* y, double* g, double* H) {
  const double c = mu * f.lam;
  double dx[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) dx[a] += f.w[k] * (y[3 * f.ids[k] + a] - f.xt[3 * k + a]);
  const double u0 = f.P[0] * dx[0] + f.P[2] * dx[1] + f.P[4] * dx[2];
  const double u1 = f.P[1] * dx[0] + f.P[3] * dx[1] + f.P[5] * dx[2];
  const double yy = std::sqrt(u0 * u0 + u1 * u1);
  double f0, f1y, M[3];
  if (yy >= eps) {
    f0 = yy;
    f1y = 1.0 / yy;
    M[0] = f1y * (1.0 - u0 * u0 / (yy * yy));
    M[1] = -f1y * u0 * u1 / (yy * yy);
    M[2] = f1y * (1.0 - u1 * u1 / (yy * yy));
  } else {
    f0 = -yy * yy * yy / (3.0 * eps * eps) + yy * yy / eps + eps / 3.0;
    f1y = 2.0 / eps - yy / (eps * eps);
    const double k = yy > 0.0 ? 1.0 / (eps * eps * yy) : 0.0;
    M[0] = f1y - k * u0 * u0;
    M[1] = -k * u0 * u1;
    M[2] = f1y - k * u1 * u1;
  }
  if (g && H) {
    for (int v = 0; v < 4; ++v)
      for (int a = 0; a < 3; ++a) {
        g[3 * v + a] = c * f.w[v] * f1y * (f.P[2 * a] * u0 + f.P[2 * a + 1] * u1);
        for (int q = 0; q < 4; ++q)
          for (int b = 0; b < 3; ++b) {
            const double pmp = f.P[2 * a] * (M[0] * f.P[2 * b] + M[1] * f.P[2 * b + 1]) +
                               f.P[2 * a + 1] * (M[1] * f.P[2 * b] + M[2] * f.P[2 * b + 1]);
            H[12 * (3 * v + a) + 3 * q + b] = c * f.w[v] * f.w[q] * pmp;
          }
      }
  }
  return c * f0;
}

// point-coordinate gradient / Hessian of a contact (first nI points with the first group's
// body) as the pair terms out[456] = H_IJ, H_II, H_JJ, g; swap as in contact_terms
void affine_terms(const double rs12[12], int nI, const double* g12, const double* H12, int swap, double out[456]) {
  double w[4][4];
  for (int v = 0; v < 4; ++v) {
    w[v][0] = 1.0;
    for (int m = 1; m < 4; ++m) w[v][m] = rs12[3 * v + m - 1];
  }
  double G[2][12], B[2][2][144];
  std::memset(G, 0, sizeof(G));
  std::memset(B, 0, sizeof(B));
  for (int u = 0; u < 4; ++u)
    for (int m = 0; m < 4; ++m)
      for (int a = 0; a < 3; ++a) {
        const int gu = u < nI ? 0 : 1;
        G[gu][3 * m + a] += w[u][m] * g12[3 * u + a];
        for (int v = 0; v < 4; ++v)
          for (int n2 = 0; n2 < 4; ++n2)
            for (int b = 0; b < 3; ++b)
              B[gu][v < nI ? 0 : 1][12 * (3 * m + a) + 3 * n2 + b] += w[u][m] * H12[12 * (3 * u + a) + 3 * v + b] * w[v][n2];
      }
  const int I = swap ? 1 : 0, J = 1 - I;
  for (int e = 0; e < 144; ++e) {
    out[e] = B[I][J][e];
    out[144 + e] = B[I][I][e];
    out[288 + e] = B[J][J][e];
  }
  for (int e = 0; e < 12; ++e) {
    out[432 + e] = G[I][e];
    out[444 + e] = G[J][e];
  }
}

// one lagged contact's friction potential at positions y (all vertices)
double friction_energy(const Oracle& o, const Oracle::Fric& f, const double* y) {
  if (o.ipc_independent) return friction_gh(o.fr_mu, o.fr_epsv * o.prm.dt, f, y, nullptr, nullptr);
  double x12[12], g12[12], H12[144];
  for (int k = 0; k < 12; ++k) x12[k] = y[3 * f.ids[k / 3] + k % 3];
  return abd::ipc::friction_gh(f.hl, x12, f.xt, o.fr_mu, o.fr_epsv * o.prm.dt, g12, H12);
}

// the body pairs of the lagged contacts join the culled pairs (a contact may outlast the
// overlap of its bodies' boxes during the step)
void add_friction_pairs(const Oracle& o, Lists& L) {
  for (const Oracle::Fric& f : o.fric) {
    const int a = std::min(f.I, f.J), b = std::max(f.I, f.J);
    bool have = false;
    for (size_t q = 0; q + 1 < L.ij.size() && !have; q += 2) have = L.ij[q] == a && L.ij[q + 1] == b;
    if (!have) {
      L.ij.push_back(a);
      L.ij.push_back(b);
    }
  }
}

// ---------------------------------------------------------------------------------------
// inertia + orthogonality (orthogonal_energy.py:24-135)
// ---------------------------------------------------------------------------------------
inline V3 row(const double* A, int k) { return {A[3 * k], A[3 * k + 1], A[3 * k + 2]}; }

void tilde(const Oracle& o, int b, double At[9], double pt[3]) {
  const double dt = o.prm.dt;
  for (int k = 0; k < 9; ++k) At[k] = o.A0[9 * b + k] + dt * o.Adot[9 * b + k];
  const double gv[3] = {0.0, o.prm.gravity, 0.0};
  for (int k = 0; k < 3; ++k) pt[k] = (o.p0[3 * b + k] + dt * o.pdot[3 * b + k]) + (dt * dt) * gv[k];
}

double inertia_energy(const Oracle& o, int b, const double* Ak, const double* pk) {
  double At[9], pt[3];
  tilde(o, b, At, pt);
  const double* a = Ak + 9 * b;
  double eo = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double t = dot(row(a, i), row(a, j)) - (i == j ? 1.0 : 0.0);
      eo += t * t;
    }
  eo = eo * o.prm.stiffness;
  V3 d0 = V3{pk[3 * b], pk[3 * b + 1], pk[3 * b + 2]} - V3{pt[0], pt[1], pt[2]};
  V3 d1 = row(a, 0) - row(At, 0), d2 = row(a, 1) - row(At, 1), d3 = row(a, 2) - row(At, 2);
  const double nm = dot(d0, d0) * o.mass[b] + (dot(d1, d1) + dot(d2, d2) + dot(d3, d3)) * o.I0[b];
  return eo * o.prm.dt * o.prm.dt + 0.5 * nm;
}

void inertia_gh(const Oracle& o, int b, double g12[12], double H[144]) {
  const double dt = o.prm.dt, ks = o.prm.stiffness;
  const double* a = o.A.data() + 9 * b;
  double At[9], pt[3];
  tilde(o, b, At, pt);
  for (int k = 0; k < 3; ++k) g12[k] = 0.0;
  for (int ii = 1; ii < 4; ++ii) {
    const int i = ii - 1;
    V3 gr = V3{-a[3 * i], -a[3 * i + 1], -a[3 * i + 2]};
    for (int j = 0; j < 3; ++j) gr = gr + dot(row(a, i), row(a, j)) * row(a, j);
    gr = (gr * 4.0) * ks;
    gr = (dt * dt) * gr;
    g12[3 * ii] = gr.x;
    g12[3 * ii + 1] = gr.y;
    g12[3 * ii + 2] = gr.z;
  }
  const double m = o.mass[b], I0 = o.I0[b];
  for (int k = 0; k < 3; ++k) g12[k] += (o.p[3 * b + k] - pt[k]) * m;
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) g12[3 * (r + 1) + k] += (a[3 * r + k] - At[3 * r + k]) * I0;
  std::memset(H, 0, sizeof(double) * 144);
  for (int ii = 0; ii < 4; ++ii)
    for (int jj = 0; jj < 4; ++jj) {
      double dh[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      const double mm = (ii != jj) ? 0.0 : (ii == 0 ? m : I0);
      for (int k = 0; k < 3; ++k) dh[k][k] = mm;
      if (ii > 0 && jj > 0) {
        const int i = ii - 1, j = jj - 1;
        double h[3][3];
        if (i == j) {
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) h[r][c] = 0.0;
          for (int k = 0; k < 3; ++k)
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) h[r][c] += a[3 * k + r] * a[3 * k + c];
          const double ti = dot(row(a, i), row(a, i)) - 1.0;
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) h[r][c] += (a[3 * i + r] * a[3 * i + c] + (r == c ? ti : 0.0));
        } else {
          const double tj = dot(row(a, j), row(a, i));
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) h[r][c] = a[3 * j + r] * a[3 * i + c] + (r == c ? tj : 0.0);
        }
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) dh[r][c] = dh[r][c] + ((h[r][c] * 4.0) * ks) * dt * dt;
      }
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) H[(3 * ii + r) * 12 + 3 * jj + c] = dh[r][c];
    }
}

// ---------------------------------------------------------------------------------------
// assembly: g, diagonal blocks, off-diagonal blocks per body pair (put.py:25-66)
// ---------------------------------------------------------------------------------------
void assemble(Oracle& o, const double* y, const Boxes& bx, const Lists& L) {
  const int n = o.n, m = (int)L.ij.size() / 2;
  o.ij = L.ij;
  o.g.assign(12 * n, 0.0);
  o.diag.assign(144 * n, 0.0);
  o.off.assign(144 * (size_t)m, 0.0);
  o.pact.assign(m, 0);
  // adjacency: body -> (neighbour, pair, side), neighbours increasing
  o.adj_ptr.assign(n + 1, 0);
  for (int q = 0; q < m; ++q) {
    ++o.adj_ptr[L.ij[2 * q] + 1];
    ++o.adj_ptr[L.ij[2 * q + 1] + 1];
  }
  for (int b = 0; b < n; ++b) o.adj_ptr[b + 1] += o.adj_ptr[b];
  o.adj.assign(3 * (size_t)o.adj_ptr[n], 0);
  {
    std::vector<std::vector<std::array<int, 3>>> rows(n);
    for (int q = 0; q < m; ++q) {
      const int I = L.ij[2 * q], J = L.ij[2 * q + 1];
      rows[I].push_back({J, q, 0});
      rows[J].push_back({I, q, 1});
    }
    for (int b = 0; b < n; ++b) {
      std::sort(rows[b].begin(), rows[b].end());
      for (size_t k = 0; k < rows[b].size(); ++k)
        for (int t = 0; t < 3; ++t) o.adj[3 * (size_t)(o.adj_ptr[b] + k) + t] = rows[b][k][t];
    }
  }
  // contact terms of every active candidate
  struct Act {
    int pair;
    double v[456];
  };
  std::vector<Act> acts;
  int active = 0;
  for (int type = 0; type < 2; ++type) {
    const std::vector<Cand>& C = type == 0 ? L.pt : L.ee;
    const int nc = (int)C.size();
    std::vector<Act> R(nc);
    std::vector<char> on(nc, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < nc; ++i) {
      V3 xs[4], rs[4];
      fetch(o, y, C[i], type, xs, rs);
      const int swap = C[i].I != L.ij[2 * C[i].pair];
      on[i] = (o.ipc_full ? (o.ipc_independent ? full_terms(type, xs, rs, swap, o.prm, R[i].v)
                                               : full_terms_hd(type, xs, rs, swap, o.prm, R[i].v))
                          : contact_terms(type, xs, rs, swap, o.prm, R[i].v))
                  ? 1
                  : 0;
      R[i].pair = C[i].pair;
    }
    for (int i = 0; i < nc; ++i)
      if (on[i]) {
        acts.push_back(R[i]);
        ++o.pact[R[i].pair];
        ++active;
      }
  }
  for (const Oracle::Fric& f : o.fric) {  // lagged friction: terms of the contact's body pair
    const int a = std::min(f.I, f.J), b = std::max(f.I, f.J);
    int q = -1;
    for (int k = 0; k < m && q < 0; ++k)
      if (L.ij[2 * k] == a && L.ij[2 * k + 1] == b) q = k;
    if (q < 0) continue;
    double g12[12], H12[144];
    Act act;
    act.pair = q;
    if (o.ipc_independent) {
      friction_gh(o.fr_mu, o.fr_epsv * o.prm.dt, f, y, g12, H12);
      affine_terms(f.rs, f.kind == 0 ? 1 : 2, g12, H12, f.I != L.ij[2 * q], act.v);
    } else {
      double x12[12];
      for (int k = 0; k < 12; ++k) x12[k] = y[3 * f.ids[k / 3] + k % 3];
      abd::ipc::friction_gh(f.hl, x12, f.xt, o.fr_mu, o.fr_epsv * o.prm.dt, g12, H12);
      affine_map_hd(f.kind, f.rs, f.I != L.ij[2 * q], H12, g12, act.v);
    }
    acts.push_back(act);
    ++o.pact[q];
  }
  // per pair: exact sums of its contacts, rounded (H_IJ, contributions to diag I / J, g I / J)
  std::vector<double> pdiag(288 * (size_t)m, 0.0), pgrad(24 * (size_t)m, 0.0);
  {
    std::vector<std::vector<int>> by_pair(m);
    for (size_t k = 0; k < acts.size(); ++k) by_pair[acts[k].pair].push_back((int)k);
#pragma omp parallel for schedule(dynamic, 16)
    for (int q = 0; q < m; ++q) {
      if (by_pair[q].empty()) continue;
      std::vector<XSum> acc(456);
      for (int k : by_pair[q])
        for (int e = 0; e < 456; ++e) acc[e].add(acts[k].v[e]);
      for (int e = 0; e < 456; ++e) {
        const double v = acc[e].round();
        if (e < 144) o.off[144 * (size_t)q + e] = v;
        else if (e < 432) pdiag[288 * (size_t)q + (e - 144)] = v;
        else pgrad[24 * (size_t)q + (e - 432)] = v;
      }
    }
  }
  // per body: inertia + vertex-ground terms + the rounded pair contributions, summed exactly
  std::vector<std::vector<int>> vg_of(n);
  for (size_t k = 0; k + 1 < L.vg.size(); k += 2) vg_of[L.vg[k]].push_back(L.vg[k + 1]);
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < n; ++b) {
    if (o.fixed[b]) {
      for (int k = 0; k < 12; ++k) o.g[12 * b + k] = 0.0;
      for (int k = 0; k < 144; ++k) o.diag[144 * b + k] = (k % 13 == 0) ? 1.0 : 0.0;
      continue;
    }
    std::vector<XSum> acc(156);
    double gb[12], Hb[144];
    inertia_gh(o, b, gb, Hb);
    for (int k = 0; k < 144; ++k) acc[k].add(Hb[k]);
    for (int k = 0; k < 12; ++k) acc[144 + k].add(gb[k]);
    if (o.prm.ground_enabled && o.prm.enable_vg)  // vertex-ground terms (vg_ipc.py:4-34)
      for (int v : vg_of[b]) {
        const double d = y[3 * v + 1] - o.prm.ground;
        const double d2b = barrier_d2(d * d, o.prm), db = barrier_d1(d * d, o.prm);
        const double th[4] = {1.0, o.x0[3 * v], o.x0[3 * v + 1], o.x0[3 * v + 2]};
        for (int ii = 0; ii < 4; ++ii) {
          acc[144 + 3 * ii + 1].add(((d * 2.0) * th[ii]) * db);
          for (int jj = 0; jj < 4; ++jj) acc[(3 * ii + 1) * 12 + 3 * jj + 1].add((((th[ii] * th[jj]) * d2b) * 4.0) * d * d);
        }
      }
    for (int k = o.adj_ptr[b]; k < o.adj_ptr[b + 1]; ++k) {
      const int q = o.adj[3 * (size_t)k + 1], side = o.adj[3 * (size_t)k + 2];
      if (o.pact[q] <= 0) continue;
      for (int e = 0; e < 144; ++e) acc[e].add(pdiag[288 * (size_t)q + 144 * side + e]);
      for (int e = 0; e < 12; ++e) acc[144 + e].add(pgrad[24 * (size_t)q + 12 * side + e]);
    }
    for (int k = 0; k < 144; ++k) o.diag[144 * b + k] = acc[k].round();
    for (int k = 0; k < 12; ++k) o.g[12 * b + k] = acc[144 + k].round();
  }
  // contact flags (abd.py:238; ipc.py:59-60 keeps only EE, here PT, EE and vertex-ground all
  // count, for both bodies of a contact)
  o.highlight.assign(n, 0);
  for (int q = 0; q < m; ++q)
    if (o.pact[q] > 0) o.highlight[L.ij[2 * q]] = o.highlight[L.ij[2 * q + 1]] = 1;
  if (o.prm.ground_enabled && o.prm.enable_vg)
    for (size_t k = 0; k + 1 < L.vg.size(); k += 2) {
      const double d = y[3 * L.vg[k + 1] + 1] - o.prm.ground;
      if (d * d < o.prm.d2hat) o.highlight[L.vg[k]] = 1;
    }
  // pairs touching a fixed (Dirichlet) body have no coupling block
  for (int q = 0; q < m; ++q)
    if (o.fixed[L.ij[2 * q]] || o.fixed[L.ij[2 * q + 1]])
      std::fill(o.off.begin() + 144 * (size_t)q, o.off.begin() + 144 * (size_t)(q + 1), 0.0);
  o.stat_active = active;
}

// ---------------------------------------------------------------------------------------
// linear solve H dq = g: block-Jacobi preconditioned BiCGSTAB (reference solver choice,
// abd.py:244) or PCG
// ---------------------------------------------------------------------------------------
double ddot(const std::vector<double>& a, const std::vector<double>& b) {
  // exact sum of the products (order-independent), rounded once
  const long N = (long)a.size();
  XSum total;
#pragma omp parallel
  {
    XSum part;
#pragma omp for schedule(static) nowait
    for (long i = 0; i < N; ++i) part.add(a[i] * b[i]);
#pragma omp critical
    total.merge(part);
  }
  return total.round();
}

// y = H x, block row by block row: the row of body b sums its diagonal block and the blocks
// of its active pairs with free neighbours in increasing neighbour order, columns 0..5 and
// 6..11 separately, then adds the two halves (the CUDA product's per-row order).
void spmv(const Oracle& o, const std::vector<double>& xv, std::vector<double>& yv) {
  const int n = o.n;
  yv.assign(12 * n, 0.0);
#pragma omp parallel for schedule(static)
  for (int b = 0; b < n; ++b)
    for (int r = 0; r < 12; ++r) {
      double acc[2];
      for (int h = 0; h < 2; ++h) {
        double a = 0.0;
        for (int c = 0; c < 6; ++c) a += o.diag[144 * b + r * 12 + 6 * h + c] * xv[12 * b + 6 * h + c];
        if (!o.fixed[b])
          for (int k = o.adj_ptr[b]; k < o.adj_ptr[b + 1]; ++k) {
            const int J = o.adj[3 * (size_t)k], q = o.adj[3 * (size_t)k + 1], side = o.adj[3 * (size_t)k + 2];
            if (o.pact[q] <= 0 || o.fixed[J]) continue;
            const double* B = &o.off[144 * (size_t)q];
            for (int c = 0; c < 6; ++c) {
              const int col = 6 * h + c;
              const double O = side == 0 ? B[r * 12 + col] : B[col * 12 + r];
              a += O * xv[12 * J + col];
            }
          }
        acc[h] = a;
      }
      yv[12 * b + r] = acc[0] + acc[1];
    }
}

// inverse of a 12x12 block by Gauss-Jordan with partial pivoting
void inv12(const double* Ain, double* out) {
  double a[12][24];
  for (int r = 0; r < 12; ++r)
    for (int c = 0; c < 12; ++c) {
      a[r][c] = Ain[r * 12 + c];
      a[r][12 + c] = (r == c) ? 1.0 : 0.0;
    }
  for (int c = 0; c < 12; ++c) {
    int piv = c;
    for (int r = c + 1; r < 12; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 24; ++k) std::swap(a[c][k], a[piv][k]);
    const double inv = 1.0 / a[c][c];
    for (int k = 0; k < 24; ++k) a[c][k] *= inv;
    for (int r = 0; r < 12; ++r) {
      if (r == c) continue;
      const double f = a[r][c];
      if (f != 0.0)
        for (int k = 0; k < 24; ++k) a[r][k] -= f * a[c][k];
    }
  }
  for (int r = 0; r < 12; ++r)
    for (int c = 0; c < 12; ++c) out[r * 12 + c] = a[r][12 + c];
}

// In-place Gauss-Jordan inverse without pivoting of an SPD matrix (row-major N x N), in the
// arithmetic of T (double; float for the mixed-precision preconditioner).
template <class T>
void inv_spd_inplace(std::vector<T>& a, int N) {
  for (int k = 0; k < N; ++k) {
    const T p = a[(size_t)k * N + k];
    a[(size_t)k * N + k] = T(1);
    const T ip = T(1) / p;
    for (int j = 0; j < N; ++j) a[(size_t)k * N + j] *= ip;
    for (int i = 0; i < N; ++i) {
      if (i == k) continue;
      const T f = a[(size_t)i * N + k];
      a[(size_t)i * N + k] = T(0);
      if (f != T(0))
        for (int j = 0; j < N; ++j) a[(size_t)i * N + j] -= f * a[(size_t)k * N + j];
    }
  }
}

// Contact clusters for the preconditioner (the preconditioner is this project's, not the
// reference's, whose bicgstab runs unpreconditioned): free body pairs with active contacts,
// weighted by the Frobenius norm of their coupling block (as float), merged in rounds.  In a
// round every cluster picks its strongest admissible pair to another cluster -- weight, then
// the lower pair index; admissible: the two clusters together within cluster_max bodies --
// and two clusters that pick the same pair merge, under the lower label (the lower first
// body).  Rounds repeat until none merges.  Every decision of a round uses the labels and
// sizes from its start, so the rule has the same result in any order of evaluation (the GPU
// forms the clusters this way in parallel).  Clusters list their bodies in increasing order
// and are ordered by their first body.
void build_clusters(const Oracle& o, std::vector<int>& cl_ptr, std::vector<int>& cl_body) {
  const int n = o.n, m = (int)o.ij.size() / 2;
  struct Edge {
    unsigned long long key;
    int I, J;
  };
  std::vector<Edge> w;
  for (int q = 0; q < m; ++q) {
    const int I = o.ij[2 * q], J = o.ij[2 * q + 1];
    if (o.fixed[I] || o.fixed[J] || o.pact[q] <= 0) continue;
    double f = 0.0;
    for (int k = 0; k < 144; ++k) f += o.off[144 * (size_t)q + k] * o.off[144 * (size_t)q + k];
    const float wf = (float)std::sqrt(f);
    if (!(wf > 0.f)) continue;
    unsigned wb;
    std::memcpy(&wb, &wf, 4);
    w.push_back({((unsigned long long)wb << 32) | (0xffffffffULL - (unsigned)q), I, J});
  }
  const int cap = o.prm.precond == 1 ? std::max(1, o.prm.cluster_max) : 1;
  std::vector<int> label(n), size(n, 1), to(n);
  for (int b = 0; b < n; ++b) label[b] = b;
  std::vector<unsigned long long> best(n);
  for (bool merged = cap > 1; merged;) {
    merged = false;
    std::fill(best.begin(), best.end(), 0ULL);
    for (const Edge& e : w) {
      const int a = label[e.I], b = label[e.J];
      if (a == b || size[a] + size[b] > cap) continue;
      best[a] = std::max(best[a], e.key);
      best[b] = std::max(best[b], e.key);
    }
    for (int b = 0; b < n; ++b) to[b] = b;
    for (const Edge& e : w) {
      const int a = label[e.I], b = label[e.J];
      if (a == b || best[a] != e.key || best[b] != e.key) continue;
      const int r = std::min(a, b), q = std::max(a, b);
      to[q] = r;
      size[r] += size[q];
      merged = true;
    }
    for (int b = 0; b < n; ++b) label[b] = to[label[b]];
  }
  std::vector<int> first(n, -1);
  std::vector<std::vector<int>> members;
  for (int b = 0; b < n; ++b) {
    const int r = label[b];
    if (first[r] < 0) {
      first[r] = (int)members.size();
      members.push_back({});
    }
    members[first[r]].push_back(b);
  }
  cl_ptr.assign(1, 0);
  cl_body.clear();
  for (auto& mb : members) {
    cl_body.insert(cl_body.end(), mb.begin(), mb.end());
    cl_ptr.push_back((int)cl_body.size());
  }
}

// Refinement (precision == 2, kept as a measured negative result): FP64 iterative refinement
// around an FP32 PCG.  Each sweep
// takes the FP64 residual r = b - H x and its preconditioned norm; the solve stops when that
// norm meets the FP64 target (rz <= thr2, the FP64 solve's test), else an FP32 PCG solves
// H e = r from e = 0 -- FP32 copies of the blocks and of the cluster inverses, FP32 vector
// arithmetic in the FP64 solve's operation order, exact dot products of the FP32 products,
// FP64 scalars -- until its own preconditioned norm falls by refine_tol, and x += e in FP64.
// At most kMaxSweeps sweeps; cg_max_iter bounds the FP32 iterations of the whole solve.
constexpr int kMaxSweeps = 16;
template <class Prec>
int solve_mixed(Oracle& o, const std::vector<double>& Kinv, const std::vector<size_t>& cl_off,
                const std::vector<int>& cl_ptr, const std::vector<int>& cl_body, Prec&& prec, double thr2) {
  const int n = o.n, N = 12 * n, ncl = (int)cl_ptr.size() - 1;
  std::vector<float> d32(o.diag.size()), f32(o.off.size()), K32(Kinv.size());
  for (size_t i = 0; i < d32.size(); ++i) d32[i] = (float)o.diag[i];
  for (size_t i = 0; i < f32.size(); ++i) f32[i] = (float)o.off[i];
  for (size_t i = 0; i < K32.size(); ++i) K32[i] = (float)Kinv[i];
  // y = H32 x in the order of spmv
  auto spmv32 = [&](const std::vector<float>& xv, std::vector<float>& yv) {
    yv.assign(N, 0.f);
#pragma omp parallel for schedule(static)
    for (int b = 0; b < n; ++b)
      for (int r = 0; r < 12; ++r) {
        float acc[2];
        for (int h = 0; h < 2; ++h) {
          float a = 0.f;
          for (int c = 0; c < 6; ++c) a += d32[144 * b + r * 12 + 6 * h + c] * xv[12 * b + 6 * h + c];
          if (!o.fixed[b])
            for (int k = o.adj_ptr[b]; k < o.adj_ptr[b + 1]; ++k) {
              const int J = o.adj[3 * (size_t)k], q = o.adj[3 * (size_t)k + 1], side = o.adj[3 * (size_t)k + 2];
              if (o.pact[q] <= 0 || o.fixed[J]) continue;
              const float* B = &f32[144 * (size_t)q];
              for (int c = 0; c < 6; ++c) {
                const int col = 6 * h + c;
                const float O = side == 0 ? B[r * 12 + col] : B[col * 12 + r];
                a += O * xv[12 * J + col];
              }
            }
          acc[h] = a;
        }
        yv[12 * b + r] = acc[0] + acc[1];
      }
  };
  // out = M32^-1 v in the order of prec
  auto prec32 = [&](const std::vector<float>& v, std::vector<float>& out) {
    out.assign(N, 0.f);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < ncl; ++c) {
      const int sz = cl_ptr[c + 1] - cl_ptr[c], D = 12 * sz;
      const float* K = &K32[cl_off[c]];
      for (int i = 0; i < D; ++i) {
        float acc = 0.f;
        for (int j = 0; j < D; ++j) acc += K[(size_t)i * D + j] * v[12 * cl_body[cl_ptr[c] + j / 12] + j % 12];
        out[12 * cl_body[cl_ptr[c] + i / 12] + i % 12] = acc;
      }
    }
  };
  // exact sum of the FP32 products, rounded once to FP64
  auto dot32 = [&](const std::vector<float>& a, const std::vector<float>& b) {
    XSum total;
#pragma omp parallel
    {
      XSum part;
#pragma omp for schedule(static) nowait
      for (int i = 0; i < N; ++i) part.add((double)(a[i] * b[i]));
#pragma omp critical
      total.merge(part);
    }
    return total.round();
  };
  std::vector<double>& x = o.dq;
  const std::vector<double>& bvec = o.g;
  std::vector<double> r(N), Ax, z;
  std::vector<float> r32(N), e32(N), z32, p32, Ap32;
  int its = 0, sweeps = 0;
  for (;;) {
    spmv(o, x, Ax);
    for (int i = 0; i < N; ++i) r[i] = bvec[i] - Ax[i];
    prec(r, z);
    if (ddot(r, z) <= thr2 || sweeps >= kMaxSweeps || its >= o.prm.cg_max_iter) break;
    ++sweeps;
    for (int i = 0; i < N; ++i) {
      r32[i] = (float)r[i];
      e32[i] = 0.f;
    }
    prec32(r32, z32);
    double rz = dot32(r32, z32);
    const double ithr = o.prm.refine_tol * o.prm.refine_tol * rz;
    p32 = z32;
    while (its < o.prm.cg_max_iter) {
      spmv32(p32, Ap32);
      const double pAp = dot32(p32, Ap32);
      if (!(pAp > 0.0)) break;
      ++its;
      const float af = (float)(rz / pAp);
      for (int i = 0; i < N; ++i) {
        e32[i] = e32[i] + af * p32[i];
        r32[i] = r32[i] - af * Ap32[i];
      }
      prec32(r32, z32);
      const double rzn = dot32(r32, z32);
      if (rzn <= ithr) break;
      const float bf = (float)(rzn / rz);
      for (int i = 0; i < N; ++i) p32[i] = z32[i] + bf * p32[i];
      rz = rzn;
    }
    for (int i = 0; i < N; ++i) x[i] = x[i] + (double)e32[i];
  }
  o.last_sweeps = sweeps;
  return its;
}

int solve(Oracle& o) {
  const int n = o.n, N = 12 * n, m = (int)o.ij.size() / 2;
  o.last_sweeps = 0;
  // preconditioner: dense inverse of every cluster's block system
  std::vector<int> cl_ptr, cl_body;
  build_clusters(o, cl_ptr, cl_body);
  const int ncl = (int)cl_ptr.size() - 1;
  std::vector<size_t> cl_off(ncl + 1, 0);
  for (int c = 0; c < ncl; ++c) {
    const size_t s = cl_ptr[c + 1] - cl_ptr[c];
    cl_off[c + 1] = cl_off[c] + 144 * s * s;
  }
  // precision 1: the cluster systems rounded to FP32 and inverted in FP32 arithmetic; the
  // preconditioner is then applied in FP32 (the Krylov iteration itself stays FP64)
  const bool p32 = o.prm.precision == 1;
  std::vector<double> Kinv(p32 ? 0 : cl_off[ncl]);
  std::vector<float> Kinv32(p32 ? cl_off[ncl] : 0);
  std::vector<int> where(n, -1);
  for (int c = 0; c < ncl; ++c)
    for (int k = cl_ptr[c]; k < cl_ptr[c + 1]; ++k) where[cl_body[k]] = k - cl_ptr[c];
  std::vector<int> body_cl(n);
  for (int c = 0; c < ncl; ++c)
    for (int k = cl_ptr[c]; k < cl_ptr[c + 1]; ++k) body_cl[cl_body[k]] = c;
#pragma omp parallel for schedule(dynamic, 1)
  for (int c = 0; c < ncl; ++c) {
    const int s = cl_ptr[c + 1] - cl_ptr[c], D = 12 * s;
    std::vector<double> K((size_t)D * D, 0.0);
    for (int a = 0; a < s; ++a) {
      const int b = cl_body[cl_ptr[c] + a];
      for (int r = 0; r < 12; ++r)
        for (int cc = 0; cc < 12; ++cc) K[(size_t)(12 * a + r) * D + 12 * a + cc] = o.diag[144 * b + r * 12 + cc];
    }
    if (s > 1)
      for (int q = 0; q < m; ++q) {
        const int I = o.ij[2 * q], J = o.ij[2 * q + 1];
        if (body_cl[I] != c || body_cl[J] != c) continue;
        const int a = where[I], b = where[J];
        for (int r = 0; r < 12; ++r)
          for (int cc = 0; cc < 12; ++cc) {
            const double v = o.off[144 * (size_t)q + r * 12 + cc];
            K[(size_t)(12 * a + r) * D + 12 * b + cc] = v;
            K[(size_t)(12 * b + cc) * D + 12 * a + r] = v;
          }
      }
    if (p32) {
      std::vector<float> K32(K.size());
      for (size_t e = 0; e < K.size(); ++e) K32[e] = (float)K[e];
      inv_spd_inplace(K32, D);
      std::copy(K32.begin(), K32.end(), Kinv32.begin() + cl_off[c]);
    } else {
      inv_spd_inplace(K, D);
      std::copy(K.begin(), K.end(), Kinv.begin() + cl_off[c]);
    }
  }
  // out = M^-1 v: FP64, or (precision 1) the FP32 inverse times v rounded to FP32, summed in
  // FP32 and widened
  auto prec = [&](const std::vector<double>& v, std::vector<double>& out) {
    out.assign(N, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < ncl; ++c) {
      const int s = cl_ptr[c + 1] - cl_ptr[c], D = 12 * s;
      if (p32) {
        const float* K = &Kinv32[cl_off[c]];
        for (int i = 0; i < D; ++i) {
          float acc = 0.f;
          for (int j = 0; j < D; ++j)
            acc += K[(size_t)i * D + j] * (float)v[12 * cl_body[cl_ptr[c] + j / 12] + j % 12];
          out[12 * cl_body[cl_ptr[c] + i / 12] + i % 12] = (double)acc;
        }
        continue;
      }
      const double* K = &Kinv[cl_off[c]];
      for (int i = 0; i < D; ++i) {
        double acc = 0.0;
        for (int j = 0; j < D; ++j) acc += K[(size_t)i * D + j] * v[12 * cl_body[cl_ptr[c] + j / 12] + j % 12];
        out[12 * cl_body[cl_ptr[c] + i / 12] + i % 12] = acc;
      }
    }
  };
  std::vector<double>& x = o.dq;
  const std::vector<double>& bvec = o.g;
  std::vector<double> zb;
  prec(bvec, zb);
  const double bz = ddot(bvec, zb);
  if (!(bz > 0.0)) {
    std::fill(x.begin(), x.end(), 0.0);
    return 0;
  }
  const double thr2 = o.prm.cg_tol * o.prm.cg_tol * bz;
  if (o.prm.precision == 2) return solve_mixed(o, Kinv, cl_off, cl_ptr, cl_body, prec, thr2);
  std::vector<double> r(N), Ax;
  spmv(o, x, Ax);
  for (int i = 0; i < N; ++i) r[i] = bvec[i] - Ax[i];
  int it = 0;
  if (o.prm.solver == 1) {  // PCG, converged when r^T M^-1 r <= tol^2 b^T M^-1 b
    // precision 1: flexible CG (Polak-Ribiere beta = z_new.(r_new - r_old) / z_old.r_old), which
    // tolerates the FP32 preconditioner's rounding (not exactly a symmetric linear map)
    std::vector<double> z, pv, Ap, rold;
    prec(r, z);
    double rz = ddot(r, z);
    if (rz <= thr2) return 0;
    pv = z;
    for (it = 1; it <= o.prm.cg_max_iter; ++it) {
      spmv(o, pv, Ap);
      const double pAp = ddot(pv, Ap);
      if (!(pAp > 0.0)) {  // non-positive curvature: stop before this iteration's update
        --it;
        break;
      }
      const double alpha = rz / pAp;
      if (p32) rold = r;
      for (int i = 0; i < N; ++i) {
        x[i] += alpha * pv[i];
        r[i] -= alpha * Ap[i];
      }
      prec(r, z);
      const double rzn = ddot(r, z);
      if (rzn <= thr2) break;
      const double beta = p32 ? (rzn - ddot(rold, z)) / rz : rzn / rz;
      for (int i = 0; i < N; ++i) pv[i] = z[i] + beta * pv[i];
      rz = rzn;
    }
    return std::min(it, o.prm.cg_max_iter);
  }
  // BiCGSTAB, right preconditioned; converged in the preconditioned norm of s / r
  std::vector<double> rh = r, pv(N, 0.0), v(N, 0.0), y, s(N), z, t, zz;
  prec(r, zz);
  if (ddot(r, zz) <= thr2) return 0;
  double rho_old = 1.0, alpha = 1.0, omega = 1.0;
  for (it = 1; it <= o.prm.cg_max_iter; ++it) {
    const double rho = ddot(rh, r);
    if (rho == 0.0 || !std::isfinite(rho)) {  // breakdown: stop before this iteration
      --it;
      break;
    }
    if (it == 1) {
      pv = r;
    } else {
      const double beta = (rho / rho_old) * (alpha / omega);
      for (int i = 0; i < N; ++i) pv[i] = r[i] + beta * (pv[i] - omega * v[i]);
    }
    prec(pv, y);
    spmv(o, y, v);
    alpha = rho / ddot(rh, v);
    for (int i = 0; i < N; ++i) s[i] = r[i] - alpha * v[i];
    prec(s, z);
    if (ddot(s, z) <= thr2) {
      for (int i = 0; i < N; ++i) x[i] += alpha * y[i];
      break;
    }
    spmv(o, z, t);
    omega = ddot(t, s) / ddot(t, t);
    for (int i = 0; i < N; ++i) {
      x[i] += alpha * y[i] + omega * z[i];
      r[i] = s[i] - omega * t[i];
    }
    prec(r, zz);
    if (ddot(r, zz) <= thr2) break;
    rho_old = rho;
  }
  return std::min(it, o.prm.cg_max_iter);
}

// ---------------------------------------------------------------------------------------
// CCD (ccd.py:56-195, cubic_roots.py:6-193)
// ---------------------------------------------------------------------------------------
const double X_ERROR = 1e-10;
inline double evaluate(const double c[4], double x) { return c[0] + x * (c[1] + x * (c[2] + x * c[3])); }
inline double multi_sign(double a, double b) { return b < 0.0 ? -a : a; }
inline bool diff_sign(double y0, double yr) { return y0 * yr < 0.0; }

double find_closed(const double coef[4], const double deriv[4], double x0, double x1, double y0, double y1) {
  (void)y1;
  double xr = (x0 + x1) / 2.0;
  double yr = evaluate(coef, xr);
  double xb0 = x0, xb1 = x1;
  if (x1 - x0 <= X_ERROR * 2.0) return xr;
  for (int guard = 0; guard < 4096; ++guard) {
    if (diff_sign(y0, yr)) xb1 = xr;
    else xb0 = xr;
    const double dy = evaluate(deriv, xr);
    const double dx = yr / dy;
    const double xn = xr - dx;
    if (xn > xb0 && xn < xb1) {
      const double step = std::fabs(xr - xn);
      xr = xn;
      if (step > X_ERROR) yr = evaluate(coef, xr);
      else break;
    } else {
      xr = (xb0 + xb1) / 2.0;
      yr = evaluate(coef, xr);
      if (xb0 == xr || xb1 == xr || xb1 - xb0 <= 2.0 * X_ERROR) break;
    }
  }
  return xr;
}

int quadratic_roots(const double coef[3], double x0, double x1, double roots[2]) {
  roots[0] = roots[1] = 0.0;
  const double c = coef[0], b = coef[1], a = coef[2];
  const double delta = b * b - 4.0 * a * c;
  int ret = 0;
  if (delta > 0.0) {
    const double d = std::sqrt(delta);
    const double q = -(b + multi_sign(d, b)) * 0.5;
    const double rv0 = q / a, rv1 = c / q;
    const double xa = rv0 < rv1 ? rv0 : rv1, xb = rv0 > rv1 ? rv0 : rv1;
    if (xa >= x0 && xa <= x1) roots[ret++] = xa;
    if (xb >= x0 && xb <= x1) roots[ret++] = xb;
  } else if (delta < 0.0) {
    ret = 0;
  } else {
    const double r0 = -0.5 * b / a;
    roots[0] = r0;
    if (r0 >= x0 && r0 <= x1) ret = 1;
  }
  return ret;
}

int cubic_roots(const double coef[4], double x0, double x1, double roots[3]) {
  roots[0] = roots[1] = roots[2] = 0.0;
  const double y0 = evaluate(coef, x0), y1 = evaluate(coef, x1);
  const double a = coef[3] * 3.0, b_2 = coef[2], c = coef[1];
  const double deriv[4] = {c, 2.0 * b_2, a, 0.0};
  const double delta_4 = b_2 * b_2 - a * c;
  auto deflate_solve = [&](double lo) {
    double dp[3];
    dp[2] = coef[3];
    for (int i = 2; i > 0; --i) dp[i - 1] = coef[i] + roots[0] * dp[i];
    double qr[2];
    const int r = quadratic_roots(dp, lo, x1, qr);
    roots[1] = qr[0];
    roots[2] = qr[1];
    return r + 1;
  };
  if (delta_4 > 0.0) {
    const double d_2 = std::sqrt(delta_4);
    const double q = -(b_2 + multi_sign(d_2, b_2));
    const double rv0 = q / a, rv1 = c / q;
    const double xa = rv0 < rv1 ? rv0 : rv1, xb = rv0 > rv1 ? rv0 : rv1;
    if (diff_sign(y0, y1)) {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) {
        roots[0] = find_closed(coef, deriv, x0, x1, y0, y1);
        return 1;
      }
    } else {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) return 0;
    }
    if (xa > x0) {
      const double ya = evaluate(coef, xa);
      if (diff_sign(y0, ya)) {
        roots[0] = find_closed(coef, deriv, x0, xa, y0, ya);
        if (diff_sign(ya, y1) || (xb < x1 && diff_sign(ya, evaluate(coef, xb)))) return deflate_solve(xa);
        return 1;
      }
      if (xb < x1) {
        const double yb = evaluate(coef, xb);
        if (diff_sign(ya, yb)) {
          roots[0] = find_closed(coef, deriv, xa, xb, ya, yb);
          if (diff_sign(yb, y1)) return deflate_solve(xb);
          return 1;
        }
        if (diff_sign(yb, y1)) {
          roots[0] = find_closed(coef, deriv, xb, x1, yb, y1);
          return 1;
        }
      } else if (diff_sign(ya, y1)) {
        roots[0] = find_closed(coef, deriv, xa, x1, ya, y1);
        return 1;
      }
    } else {
      const double yb = evaluate(coef, xb);
      if (diff_sign(y0, yb)) {
        roots[0] = find_closed(coef, deriv, x0, xb, y0, yb);
        if (diff_sign(yb, y1)) return deflate_solve(xb);
        return 1;
      }
      if (diff_sign(yb, y1)) {
        roots[0] = find_closed(coef, deriv, xb, x1, yb, y1);
        return 1;
      }
    }
    return 0;
  }
  if (diff_sign(y0, y1)) {
    roots[0] = find_closed(coef, deriv, x0, x1, y0, y1);
    return 1;
  }
  return 0;
}

inline void cubic_binomial(const double a[3], const double b[3], double out[4]) {
  out[0] = b[0] * b[1] * b[2];
  out[1] = a[0] * b[1] * b[2] + b[0] * b[1] * a[2] + b[0] * a[1] * b[2];
  out[2] = a[0] * a[1] * b[2] + a[0] * b[1] * a[2] + b[0] * a[1] * a[2];
  out[3] = a[0] * a[1] * a[2];
}

// det(b + t a) of 3x3 matrices (row-major m[r][c])
void det_polynomial(const double a[3][3], const double b[3][3], double out[4]) {
  static const int P[6][3][2] = {{{0, 0}, {1, 1}, {2, 2}}, {{0, 1}, {1, 2}, {2, 0}}, {{0, 2}, {1, 0}, {2, 1}},
                                 {{0, 0}, {1, 2}, {2, 1}}, {{0, 1}, {1, 0}, {2, 2}}, {{0, 2}, {1, 1}, {2, 0}}};
  double pos[4] = {0, 0, 0, 0}, neg[4] = {0, 0, 0, 0};
  for (int t = 0; t < 6; ++t) {
    double av[3], bv[3], cb[4];
    for (int k = 0; k < 3; ++k) {
      av[k] = a[P[t][k][0]][P[t][k][1]];
      bv[k] = b[P[t][k][0]][P[t][k][1]];
    }
    cubic_binomial(av, bv, cb);
    double* dst = t < 3 ? pos : neg;
    for (int k = 0; k < 4; ++k) dst[k] = dst[k] + cb[k];
  }
  for (int k = 0; k < 4; ++k) out[k] = pos[k] - neg[k];
}

// columns = the three points (wp.mat33(v0, v1, v2) is column-wise)
inline void cols(V3 p, V3 q, V3 r, double m[3][3]) {
  m[0][0] = p.x; m[1][0] = p.y; m[2][0] = p.z;
  m[0][1] = q.x; m[1][1] = q.y; m[2][1] = q.z;
  m[0][2] = r.x; m[1][2] = r.y; m[2][2] = r.z;
}

// inclusive: a root also counts on the closed triangle / segments (edge and vertex hits, which
// the full contact model resolves), within 1e-9 of their parameter bounds
double collision_time(int type, const V3 a0[4], const V3 a1[4], bool inclusive = false) {
  double A[4][3][3], B[4][3][3];
  const int sel[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  for (int k = 0; k < 4; ++k) {
    cols(a1[sel[k][0]], a1[sel[k][1]], a1[sel[k][2]], A[k]);
    cols(a0[sel[k][0]], a0[sel[k][1]], a0[sel[k][2]], B[k]);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) A[k][r][c] -= B[k][r][c];
  }
  double d[4][4];
  for (int k = 0; k < 4; ++k) det_polynomial(A[k], B[k], d[k]);
  double coef[4];
  for (int k = 0; k < 4; ++k) coef[k] = ((d[0][k] - d[1][k]) + d[2][k]) - d[3][k];
  double roots[3];
  const int nr = cubic_roots(coef, 0.0, 1.0, roots);
  double root = 1.0;
  bool ok = false;
  for (int i = 0; i < nr; ++i) {
    root = roots[i];
    V3 pt[4];
    for (int k = 0; k < 4; ++k) pt[k] = a0[k] * (1.0 - root) + a1[k] * root;  // wp.lerp
    Geo G = geometry(type, pt[0], pt[1], pt[2], pt[3]);
    if (inclusive) {
      const double t = 1e-9, b = G.beta, c = type == 0 ? G.gamma : -G.gamma;
      ok = b >= -t && c >= -t && (type == 0 ? b + c <= 1.0 + t : (b <= 1.0 + t && c <= 1.0 + t));
    } else {
      ok = valid_root(type, G.beta, G.gamma);
    }
    if (ok) break;
  }
  return ok ? root : 1.0;
}

// ---------------------------------------------------------------------------------------
// driver (abd.py:124-362)
// ---------------------------------------------------------------------------------------
void update_qk(Oracle& o, double alpha) {
  for (int b = 0; b < o.n; ++b) {
    for (int k = 0; k < 3; ++k) o.pk[3 * b + k] = o.p[3 * b + k] - o.dq[12 * b + k] * alpha;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) o.Ak[9 * b + 3 * r + k] = o.A[9 * b + 3 * r + k] - o.dq[12 * b + 3 * (r + 1) + k] * alpha;
  }
}

void update_q(Oracle& o, double alpha) {
  for (int b = 0; b < o.n; ++b) {
    for (int k = 0; k < 3; ++k) o.p[3 * b + k] = o.p[3 * b + k] - o.dq[12 * b + k] * alpha;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) o.A[9 * b + 3 * r + k] = o.A[9 * b + 3 * r + k] - o.dq[12 * b + 3 * (r + 1) + k] * alpha;
  }
}

// barrier energies of the candidates and the vertex-ground pairs plus inertia, summed
// exactly (compute_energy, abd.py:133-141)
double energy_at(Oracle& o, const double* y, const double* Akp, const double* pkp) {
  Boxes bx;
  Lists L;
  static_boxes(o, y, bx);
  cull(o, bx, L);
  XSum total;
  for (int type = 0; type < 2; ++type) {
    const std::vector<Cand>& C = type == 0 ? L.pt : L.ee;
    const int nc = (int)C.size();
#pragma omp parallel
    {
      XSum part;
#pragma omp for schedule(static) nowait
      for (int i = 0; i < nc; ++i) {
        V3 xs[4], rs[4];
        fetch(o, y, C[i], type, xs, rs);
        part.add(o.ipc_full ? (o.ipc_independent ? full_energy(type, xs, rs, o.prm) : full_energy_hd(type, xs, rs, o.prm))
                            : contact_energy(type, xs, o.prm));
      }
#pragma omp critical
      total.merge(part);
    }
  }
  for (size_t k = 0; k + 1 < L.vg.size(); k += 2) {
    const double d = y[3 * L.vg[k + 1] + 1] - o.prm.ground;
    total.add(barrier(d * d, o.prm));
  }
  for (const Oracle::Fric& f : o.fric) total.add(friction_energy(o, f, y));
  for (int b = 0; b < o.n; ++b)
    if (!o.fixed[b]) total.add(inertia_energy(o, b, Akp, pkp));
  return total.round();
}

double compute_energy(Oracle& o, double alpha) {
  update_qk(o, alpha);
  transform(o, o.Ak.data(), o.pk.data(), o.xk.data());
  return energy_at(o, o.xk.data(), o.Ak.data(), o.pk.data());
}

double ccd_toi(Oracle& o, const double* x, const double* xk, double* raw) {
  Boxes bx;
  Lists L;
  swept_boxes(o, x, xk, bx);
  cull(o, bx, L);
  double toi = 1.0;
  for (size_t k = 0; k + 1 < L.vg.size(); k += 2) {
    const int v = L.vg[k + 1];
    const double d1 = xk[3 * v + 1] - o.prm.ground;
    double t = 1.0;
    if (d1 < 0) {
      const double d0 = x[3 * v + 1] - o.prm.ground;
      t = d0 / (d0 - d1);
    }
    if (t < 1.0) toi = std::min(toi, t);
  }
  for (int type = 0; type < 2; ++type) {
    const std::vector<Cand>& C = type == 0 ? L.pt : L.ee;
    const int nc = (int)C.size();
    double tmin = 1.0;
#pragma omp parallel for schedule(dynamic, 64) reduction(min : tmin)
    for (int i = 0; i < nc; ++i) {
      V3 a0[4], a1[4], rs[4];
      fetch(o, x, C[i], type, a0, rs);
      fetch(o, xk, C[i], type, a1, rs);
      const double t = collision_time(type, a0, a1, o.ipc_full);
      if (t < 1.0) tmin = std::min(tmin, t);
    }
    toi = std::min(toi, tmin);
  }
  if (raw) *raw = toi;
  double t = std::max(0.0, std::min(1.0, toi));
  if (t < 1.0) t *= 0.9;
  return t;
}

void step(Oracle& o) {
  const int n = o.n;
  o.A = o.A0;
  o.p = o.p0;
  o.Ak = o.A0;
  o.pk = o.p0;
  friction_lag(o);
  double E0 = compute_energy(o, 0.0);
  int it = 0, lin = 0, ls = 0, sweeps = 0;
  for (;;) {
    transform(o, o.A.data(), o.p.data(), o.x.data());
    o.xk = o.x;
    Boxes bx;
    Lists L;
    static_boxes(o, o.x.data(), bx);
    cull(o, bx, L);
    if (it == 0) {
      o.stat_pt = (int)L.pt.size();
      o.stat_ee = (int)L.ee.size();
      o.stat_vg = (int)L.vg.size() / 2;
      o.stat_ij = (int)L.ij.size() / 2;
    }
    add_friction_pairs(o, L);
    assemble(o, o.x.data(), bx, L);
    lin += solve(o);
    sweeps += o.last_sweeps;
    // CCD (abd.py:278-303)
    update_qk(o, 1.0);
    transform(o, o.Ak.data(), o.pk.data(), o.xk.data());
    const double alpha_cap = ccd_toi(o, o.x.data(), o.xk.data(), &o.stat_toi);
    // line search (abd.py:146-160)
    const double qTg = ddot(o.dq, o.g);
    double alpha = alpha_cap, E1;
    for (;;) {
      E1 = compute_energy(o, alpha);
      ++ls;
      const bool wolfe = E1 < E0 + o.prm.armijo_sign * o.prm.c1 * alpha * qTg ||
                         std::fabs(E1 - E0) <= o.prm.ls_noise_floor * std::fabs(E0);
      if (wolfe || alpha < o.prm.alpha_min) break;
      alpha *= 0.5;
    }
    E0 = E1;
    update_q(o, alpha);
    ++it;
    o.stat_alpha = alpha;
    const double gTg = ddot(o.g, o.g);
    if (gTg < o.prm.tol || it >= o.prm.max_iter) break;
  }
  for (int b = 0; b < n; ++b) {
    for (int k = 0; k < 3; ++k) {
      o.pdot[3 * b + k] = (o.p[3 * b + k] - o.p0[3 * b + k]) / o.prm.dt;
      o.p0[3 * b + k] = o.p[3 * b + k];
    }
    for (int k = 0; k < 9; ++k) {
      o.Adot[9 * b + k] = (o.A[9 * b + k] - o.A0[9 * b + k]) / o.prm.dt;
      o.A0[9 * b + k] = o.A[9 * b + k];
    }
  }
  transform(o, o.A0.data(), o.p0.data(), o.xview.data());
  o.stat_newton = it;
  o.stat_lin = lin;
  o.stat_refine = sweeps;
  o.stat_ls = ls;
  o.stat_energy = E0;
}

}  // namespace

// =======================================================================================
// C ABI for the tests (ctypes)
// =======================================================================================
extern "C" {

struct orc_info {
  int newton_iters, linear_iters, ls_trials, n_pt, n_ee, n_vg, n_ij, n_active;
  double alpha, toi, energy;
  int refine_iters;  // precision == 1: FP64 refinement sweeps of the step
};

void* orc_create(int n, const int* voff, const int* toff, const int* eoff, const double* x0, const int* tris,
                 const int* edges, const double* mass, const double* I0, const int* fixed, const Params* prm) {
  Oracle* o = new Oracle();
  o->n = n;
  o->voff.assign(voff, voff + n + 1);
  o->toff.assign(toff, toff + n + 1);
  o->eoff.assign(eoff, eoff + n + 1);
  o->V = o->voff[n];
  o->T = o->toff[n];
  o->E = o->eoff[n];
  o->x0.assign(x0, x0 + 3 * (size_t)o->V);
  o->tris.assign(tris, tris + 3 * (size_t)o->T);
  o->edges.assign(edges, edges + 2 * (size_t)o->E);
  o->mass.assign(mass, mass + n);
  o->I0.assign(I0, I0 + n);
  o->fixed.assign(fixed, fixed + n);
  o->prm = *prm;
  o->ipc_full = prm->ipc_full != 0;
  if (prm->friction_mu > 0.0) {
    o->fr_mu = prm->friction_mu;
    o->fr_epsv = prm->friction_epsv;
  }
  for (auto* v : {&o->A, &o->Ak, &o->Adot, &o->A0}) v->assign(9 * (size_t)n, 0.0);
  for (auto* v : {&o->p, &o->pk, &o->pdot, &o->p0}) v->assign(3 * (size_t)n, 0.0);
  o->dq.assign(12 * (size_t)n, 0.0);
  o->g.assign(12 * (size_t)n, 0.0);
  o->x.assign(3 * (size_t)o->V, 0.0);
  o->xk = o->x;
  o->xview = o->x;
  return o;
}

void orc_destroy(void* h) { delete (Oracle*)h; }
// contact flags of the last assembly (the step's last Newton iteration, or orc_gh)
void orc_get_highlight(void* h, int* out) {
  const Oracle& o = *(Oracle*)h;
  for (int b = 0; b < o.n; ++b) out[b] = (int)o.highlight.size() == o.n ? o.highlight[b] : 0;
}
void orc_set_params(void* h, const Params* prm) {
  Oracle* o = (Oracle*)h;
  o->prm = *prm;
  if (prm->ipc_full) o->ipc_full = true;
  if (prm->friction_mu > 0.0) {
    o->fr_mu = prm->friction_mu;
    o->fr_epsv = prm->friction_epsv;
  }
}
// on: 0 the reference's model, 1 the full model in the CUDA library's arithmetic, 2 the full
// model in the oracle's own
void orc_set_ipc_full(void* h, int on) {
  ((Oracle*)h)->ipc_full = on != 0;
  ((Oracle*)h)->ipc_independent = on == 2;
}
// lagged friction with coefficient mu and slip velocity eps_v (needs the full contact model)
// one candidate's lagged friction: fixed at step-start positions xt12 (rest rs12), evaluated at
// x12 with coefficient mu and threshold eps (displacement); returns 0 when not within dhat
int orc_friction_contact(int kind, const double* xt12, const double* rs12, const Params* prm, double mu, double eps,
                         const double* x12, double* D, double* g12, double* H144, double* w, double* lam) {
  V3 xs[4], rs[4];
  for (int k = 0; k < 4; ++k) {
    xs[k] = {xt12[3 * k], xt12[3 * k + 1], xt12[3 * k + 2]};
    rs[k] = {rs12[3 * k], rs12[3 * k + 1], rs12[3 * k + 2]};
  }
  Oracle::Fric f;
  if (!make_fric(kind, xs, rs, *prm, f)) return 0;
  for (int k = 0; k < 4; ++k) f.ids[k] = k;
  *D = friction_gh(mu, eps, f, x12, g12, H144);
  for (int k = 0; k < 4; ++k) w[k] = f.w[k];
  *lam = f.lam;
  return 1;
}

void orc_set_friction(void* h, double mu, double eps_v) {
  ((Oracle*)h)->fr_mu = mu;
  ((Oracle*)h)->fr_epsv = eps_v;
}

// full-model pair terms of one candidate (swap as in the assembly): out[456] = H_IJ, H_II,
// H_JJ, g; *E the energy, *d2 the classified squared distance, *type its feature pair
int orc_full_terms(int kind, const double* xs12, const double* rs12, const Params* prm, int swap, double* out,
                   double* E, double* d2, int* type) {
  V3 xs[4], rs[4];
  for (int k = 0; k < 4; ++k) {
    xs[k] = {xs12[3 * k], xs12[3 * k + 1], xs12[3 * k + 2]};
    rs[k] = {rs12[3 * k], rs12[3 * k + 1], rs12[3 * k + 2]};
  }
  *type = kind == 0 ? full_pt_type(xs) : full_ee_type(xs);
  D12 e;
  const bool on = full_energy_d(kind, xs, rs, *prm, e, d2);
  *E = on ? e.v : 0.0;
  return on && full_terms(kind, xs, rs, swap, *prm, out) ? 1 : 0;
}
void orc_set_threads(int t) { omp_set_num_threads(t); }
int orc_max_threads() { return omp_get_max_threads(); }

void orc_set_state(void* h, const double* A0, const double* p0, const double* Adot, const double* pdot,
                   const double* dq) {
  Oracle* o = (Oracle*)h;
  std::copy(A0, A0 + 9 * o->n, o->A0.begin());
  std::copy(p0, p0 + 3 * o->n, o->p0.begin());
  std::copy(Adot, Adot + 9 * o->n, o->Adot.begin());
  std::copy(pdot, pdot + 3 * o->n, o->pdot.begin());
  o->A = o->A0;
  o->p = o->p0;
  if (dq) std::copy(dq, dq + 12 * o->n, o->dq.begin());
  else std::fill(o->dq.begin(), o->dq.end(), 0.0);
}

void orc_get_state(void* h, double* A0, double* p0, double* Adot, double* pdot, double* dq, double* xview) {
  Oracle* o = (Oracle*)h;
  if (A0) std::copy(o->A0.begin(), o->A0.end(), A0);
  if (p0) std::copy(o->p0.begin(), o->p0.end(), p0);
  if (Adot) std::copy(o->Adot.begin(), o->Adot.end(), Adot);
  if (pdot) std::copy(o->pdot.begin(), o->pdot.end(), pdot);
  if (dq) std::copy(o->dq.begin(), o->dq.end(), dq);
  if (xview) std::copy(o->xview.begin(), o->xview.end(), xview);
}

int orc_step(void* h, orc_info* info) {
  Oracle* o = (Oracle*)h;
  step(*o);
  if (info) {
    info->newton_iters = o->stat_newton;
    info->linear_iters = o->stat_lin;
    info->ls_trials = o->stat_ls;
    info->n_pt = o->stat_pt;
    info->n_ee = o->stat_ee;
    info->n_vg = o->stat_vg;
    info->n_ij = o->stat_ij;
    info->n_active = o->stat_active;
    info->alpha = o->stat_alpha;
    info->toi = o->stat_toi;
    info->energy = o->stat_energy;
    info->refine_iters = o->stat_refine;
  }
  return 0;
}

void orc_transform(void* h, const double* A, const double* p, double* x) { transform(*(Oracle*)h, A, p, x); }

// Culling lists.  mode 0: static boxes at y0; mode 1: swept boxes y0 -> y1.
// Returns the counts in counts[4] = {ij, pt, ee, vg}; lists are written up to their caps.
void orc_collision_set(void* h, int mode, const double* y0, const double* y1, int* ij, int* pt, int* ee, int* vg,
                       int cap, int* counts) {
  Oracle* o = (Oracle*)h;
  Boxes bx;
  Lists L;
  if (mode == 0) static_boxes(*o, y0, bx);
  else swept_boxes(*o, y0, y1, bx);
  cull(*o, bx, L);
  counts[0] = (int)L.ij.size() / 2;
  counts[1] = (int)L.pt.size();
  counts[2] = (int)L.ee.size();
  counts[3] = (int)L.vg.size() / 2;
  for (int i = 0; i < std::min(cap, counts[0]); ++i) {
    ij[2 * i] = L.ij[2 * i];
    ij[2 * i + 1] = L.ij[2 * i + 1];
  }
  for (int i = 0; i < std::min(cap, counts[1]); ++i) std::memcpy(pt + 5 * i, &L.pt[i], 5 * sizeof(int));
  for (int i = 0; i < std::min(cap, counts[2]); ++i) std::memcpy(ee + 5 * i, &L.ee[i], 5 * sizeof(int));
  for (int i = 0; i < std::min(cap, counts[3]); ++i) {
    vg[2 * i] = L.vg[2 * i];
    vg[2 * i + 1] = L.vg[2 * i + 1];
  }
}

// Gradient and Hessian at the state set by orc_set_state with A, p overridden.  Outputs
// g [n*12], diag [n*144], off [cap*144] (block (I,J) of ij pair q, I<J), ij [cap*2];
// returns the number of body pairs.
int orc_gh(void* h, const double* A, const double* p, double* g, double* diag, double* off, int* ij, int cap,
           int* n_active) {
  Oracle* o = (Oracle*)h;
  std::copy(A, A + 9 * o->n, o->A.begin());
  std::copy(p, p + 3 * o->n, o->p.begin());
  transform(*o, o->A.data(), o->p.data(), o->x.data());
  Boxes bx;
  Lists L;
  static_boxes(*o, o->x.data(), bx);
  cull(*o, bx, L);
  add_friction_pairs(*o, L);  // as the step's GH passes (no-op without friction)
  assemble(*o, o->x.data(), bx, L);
  std::copy(o->g.begin(), o->g.end(), g);
  std::copy(o->diag.begin(), o->diag.end(), diag);
  const int m = (int)L.ij.size() / 2;
  for (int q = 0; q < std::min(m, cap); ++q) {
    std::copy(o->off.begin() + 144 * (size_t)q, o->off.begin() + 144 * (size_t)(q + 1), off + 144 * (size_t)q);
    ij[2 * q] = L.ij[2 * q];
    ij[2 * q + 1] = L.ij[2 * q + 1];
  }
  if (n_active) *n_active = o->stat_active;
  return m;
}

// The exact Hessian of the step's energy at DOFs (A, p), dense [12n][12n] in the DOF order
// [p, A row 0, row 1, row 2] per body, for the adjoint of a converged step: inertia and
// orthogonality (exact in the assembly already) plus every candidate's unprojected
// full-model contact Hessian.  Needs the full contact model (set_ipc_full).  Rows and columns
// of fixed bodies are left zero.  Returns the number of active contacts, -1 without the model.
// Exact, unprojected Hessian of the step's energy at (A, p), dense [12n][12n].  model 1: the
// full contact model (needs ipc_full); model 0: the reference's model -- the interior PT /
// EE contacts the reference evaluates (d^2 < dhat^2 and a valid closest-point configuration,
// pt_ipc.py:111-118, ee_ipc.py:93-97), each the barrier of the point-plane or line-line
// squared distance with its full second derivative (the terms with the derivatives of the
// closest-point coefficients that the reference's Newton Hessian leaves out, psd/vf.py:150-176,
// psd/ee.py:94-116), and the vertex-ground barriers with their 2 B' term (vg_ipc.py:28-33
// leaves it out).
int orc_full_hessian(void* h, const double* A, const double* p, double* Hd, int model) {
  Oracle* o = (Oracle*)h;
  if (model == 1 && !o->ipc_full) return -1;
  const int n = o->n;
  const size_t N = 12 * (size_t)n;
  std::fill(Hd, Hd + N * N, 0.0);
  std::copy(A, A + 9 * n, o->A.begin());
  std::copy(p, p + 3 * n, o->p.begin());
  for (int b = 0; b < n; ++b) {
    if (o->fixed[b]) continue;
    double gb[12], Hb[144];
    inertia_gh(*o, b, gb, Hb);
    for (int r = 0; r < 12; ++r)
      for (int c = 0; c < 12; ++c) Hd[(12 * (size_t)b + r) * N + 12 * (size_t)b + c] += Hb[12 * r + c];
  }
  transform(*o, o->A.data(), o->p.data(), o->x.data());
  Boxes bx;
  Lists L;
  static_boxes(*o, o->x.data(), bx);
  cull(*o, bx, L);
  // vertex-ground barriers, exact: d = y - ground, d2E/dy2 = 2 B'(d^2) + 4 d^2 B''(d^2)
  if (o->prm.ground_enabled && o->prm.enable_vg)
    for (size_t q = 0; q + 1 < L.vg.size(); q += 2) {
      const int b = L.vg[q], v = L.vg[q + 1];
      if (o->fixed[b]) continue;
      const double d = o->x[3 * (size_t)v + 1] - o->prm.ground;
      const double hy = 2.0 * barrier_d1(d * d, o->prm) + 4.0 * d * d * barrier_d2(d * d, o->prm);
      const double th[4] = {1.0, o->x0[3 * v], o->x0[3 * v + 1], o->x0[3 * v + 2]};
      for (int m = 0; m < 4; ++m)
        for (int n2 = 0; n2 < 4; ++n2)
          Hd[(12 * (size_t)b + 3 * m + 1) * N + 12 * (size_t)b + 3 * n2 + 1] += th[m] * th[n2] * hy;
    }
  int active = 0;
  for (int kind = 0; kind < 2; ++kind) {
    const std::vector<Cand>& C = kind == 0 ? L.pt : L.ee;
    for (const Cand& cd : C) {
      V3 xs[4], rs[4];
      fetch(*o, o->x.data(), cd, kind, xs, rs);
      D12 E;
      if (model == 1) {
        if (!full_energy_d(kind, xs, rs, o->prm, E)) continue;
      } else {
        double terms[456];
        if (!contact_terms(kind, xs, rs, 0, o->prm, terms)) continue;  // the reference's activity
        V3D X[4];
        for (int k = 0; k < 4; ++k)
          X[k] = {d12_var(xs[k].x, 3 * k), d12_var(xs[k].y, 3 * k + 1), d12_var(xs[k].z, 3 * k + 2)};
        const D12 d = full_d2(kind, kind == 0 ? (int)F_PT : (int)F_EE, X);
        const double dh = o->prm.d2hat, sv = d.v / dh, l = std::log(sv);
        const double f = -o->prm.kappa * (sv - 1.0) * (sv - 1.0) * l;
        const double f1 = -o->prm.kappa * (2.0 * (sv - 1.0) * l + (sv - 1.0) * (sv - 1.0) / sv) / dh;
        const double f2 =
            -o->prm.kappa * (2.0 * l + 4.0 * (sv - 1.0) / sv - (sv - 1.0) * (sv - 1.0) / (sv * sv)) / (dh * dh);
        E = apply(d, f, f1, f2);
      }
      ++active;
      const int nI = kind == 0 ? 1 : 2;
      const int body[2] = {cd.I, cd.J};  // the candidate's first group moves with cd.I
      for (int u = 0; u < 4; ++u)
        for (int v = 0; v < 4; ++v) {
          const int bu = body[u < nI ? 0 : 1], bv = body[v < nI ? 0 : 1];
          if (o->fixed[bu] || o->fixed[bv]) continue;
          const double wu[4] = {1.0, rs[u].x, rs[u].y, rs[u].z}, wv[4] = {1.0, rs[v].x, rs[v].y, rs[v].z};
          for (int m = 0; m < 4; ++m)
            for (int a = 0; a < 3; ++a)
              for (int n2 = 0; n2 < 4; ++n2)
                for (int b2 = 0; b2 < 3; ++b2)
                  Hd[(12 * (size_t)bu + 3 * m + a) * N + 12 * (size_t)bv + 3 * n2 + b2] +=
                      wu[m] * E.H[12 * (3 * u + a) + 3 * v + b2] * wv[n2];
        }
    }
  }
  return active;
}

// Energy at trial DOFs (Ak, pk) against the state set by orc_set_state.
double orc_energy(void* h, const double* Ak, const double* pk) {
  Oracle* o = (Oracle*)h;
  std::vector<double> y(3 * (size_t)o->V);
  transform(*o, Ak, pk, y.data());
  return energy_at(*o, y.data(), Ak, pk);
}

// CCD step bound between DOFs (A, p) and (A1, p1): returns the capped alpha; raw toi too.
double orc_ccd(void* h, const double* A, const double* p, const double* A1, const double* p1, double* raw) {
  Oracle* o = (Oracle*)h;
  std::vector<double> x(3 * (size_t)o->V), xk(3 * (size_t)o->V);
  transform(*o, A, p, x.data());
  transform(*o, A1, p1, xk.data());
  return ccd_toi(*o, x.data(), xk.data(), raw);
}

// Per-pair contact terms for KATs: type 0 PT, 1 EE.  Returns active flag.
int orc_contact_gh(int type, const double* xs12, const double* rs12, const Params* prm, double* d2, double* g24,
                   double* Hi, double* Hj, double* Hij) {
  V3 xs[4], rs[4];
  for (int k = 0; k < 4; ++k) {
    xs[k] = {xs12[3 * k], xs12[3 * k + 1], xs12[3 * k + 2]};
    rs[k] = {rs12[3 * k], rs12[3 * k + 1], rs12[3 * k + 2]};
  }
  return contact_gh(type, xs, rs, *prm, *d2, g24, Hi, Hj, Hij) ? 1 : 0;
}

// rank-one form of the same pair's terms (swap = 0): out[456] = H_IJ, H_II, H_JJ, g
int orc_contact_terms(int type, const double* xs12, const double* rs12, const Params* prm, double* out) {
  V3 xs[4], rs[4];
  for (int k = 0; k < 4; ++k) {
    xs[k] = {xs12[3 * k], xs12[3 * k + 1], xs12[3 * k + 2]};
    rs[k] = {rs12[3 * k], rs12[3 * k + 1], rs12[3 * k + 2]};
  }
  return contact_terms(type, xs, rs, 0, *prm, out) ? 1 : 0;
}

double orc_log(double x) { return abd_log(x); }

// exact sum of n values, rounded once
double orc_exact_sum(const double* v, long n) {
  XSum s;
  for (long i = 0; i < n; ++i) s.add(v[i]);
  return s.round();
}

// Inertia + orthogonality energy of n free-standing bodies (orthogonal_energy.py:24-32, the
// per-body term of inertia_energy above) at trial DOFs (Ak, pk) with the prediction from
// (A0, p0, Adot, pdot), summed exactly; fixed bodies contribute nothing.  Checks the library's
// allocation-free energy on synthetic states of any size.
double orc_inertia_energy_sum(int n, const Params* prm, const double* Ak, const double* pk, const double* A0,
                              const double* p0, const double* Adot, const double* pdot, const double* mass,
                              const double* I0, const int* fixed) {
  XSum total;
  const double dt = prm->dt;
  for (int b = 0; b < n; ++b) {
    if (fixed[b]) continue;
    double At[9], pt[3];
    for (int k = 0; k < 9; ++k) At[k] = A0[9 * b + k] + dt * Adot[9 * b + k];
    const double gv[3] = {0.0, prm->gravity, 0.0};
    for (int k = 0; k < 3; ++k) pt[k] = (p0[3 * b + k] + dt * pdot[3 * b + k]) + (dt * dt) * gv[k];
    const double* a = Ak + 9 * b;
    double eo = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const double t = dot(row(a, i), row(a, j)) - (i == j ? 1.0 : 0.0);
        eo += t * t;
      }
    eo = eo * prm->stiffness;
    V3 d0 = V3{pk[3 * b], pk[3 * b + 1], pk[3 * b + 2]} - V3{pt[0], pt[1], pt[2]};
    V3 d1 = row(a, 0) - row(At, 0), d2 = row(a, 1) - row(At, 1), d3 = row(a, 2) - row(At, 2);
    const double nm = dot(d0, d0) * mass[b] + (dot(d1, d1) + dot(d2, d2) + dot(d3, d3)) * I0[b];
    total.add(eo * dt * dt + 0.5 * nm);
  }
  return total.round();
}

double orc_contact_energy(int type, const double* xs12, const Params* prm) {
  V3 xs[4];
  for (int k = 0; k < 4; ++k) xs[k] = {xs12[3 * k], xs12[3 * k + 1], xs12[3 * k + 2]};
  return contact_energy(type, xs, *prm);
}

double orc_collision_time(int type, const double* p0_12, const double* p1_12) {
  V3 a0[4], a1[4];
  for (int k = 0; k < 4; ++k) {
    a0[k] = {p0_12[3 * k], p0_12[3 * k + 1], p0_12[3 * k + 2]};
    a1[k] = {p1_12[3 * k], p1_12[3 * k + 1], p1_12[3 * k + 2]};
  }
  return collision_time(type, a0, a1);
}

int orc_cubic_roots(const double* coef, double x0, double x1, double* roots) {
  return cubic_roots(coef, x0, x1, roots);
}

// Solve with the system assembled by the last orc_gh; dq is the warm start, overwritten.
int orc_solve(void* h, double* dq) {
  Oracle* o = (Oracle*)h;
  std::copy(dq, dq + 12 * o->n, o->dq.begin());
  const int it = solve(*o);
  std::copy(o->dq.begin(), o->dq.end(), dq);
  return it;
}

}  // extern "C"
