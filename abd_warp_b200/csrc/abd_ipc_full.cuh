// Full IPC contact model for one point-triangle (PT) or edge-edge (EE) candidate: the closest
// feature pair is classified (point-triangle, point-edge and point-point for PT; line-line,
// point-edge and point-point for EE), the barrier acts on the squared distance of that
// feature pair, and EE contacts are mollified as the edges turn parallel.  This is the
// robustness gap of the reference's contact model, which evaluates only the interior cases
// (ipcsk/energy.py:20-22, 46-48 leave the other feature pairs out; ccd.py:44-54 masks them).
//
// The model follows Li et al., "Incremental Potential Contact" (SIGGRAPH 2020): distance
// types by closest features, the log barrier on squared distance, the edge-edge mollifier
// e_x = 1e-3 |a_rest|^2 |b_rest|^2, and a per-contact PSD projection of the local Hessian.
// Derivatives are exact to rounding: the local energy is evaluated on hyper-dual numbers
// (Fike and Alonso 2011), one evaluation per Hessian entry.  The projection is the cyclic
// Jacobi eigenvalue method in round-robin (parallel) order (Golub and Van Loan, Matrix
// Computations, 8.5).
//
// Friction follows the same paper's lagged dissipative potential (section 5).
//
// Everything here is plain arithmetic callable from host and device code.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define ABD_HD __host__ __device__
#else
#define ABD_HD
#endif

namespace abd {
namespace ipc {

// closest-feature types of a point-triangle pair (triangle edges E0 = t0t1, E1 = t1t2,
// E2 = t2t0)
enum PtType { PT_P_T = 0, PT_P_E0, PT_P_E1, PT_P_E2, PT_P_V0, PT_P_V1, PT_P_V2 };
// closest-feature types of an edge-edge pair (edge a = a0a1, edge b = b0b1)
enum EeType {
  EE_EA_EB = 0,
  EE_EA0_EB, EE_EA1_EB, EE_EA_EB0, EE_EA_EB1,
  EE_EA0_EB0, EE_EA0_EB1, EE_EA1_EB0, EE_EA1_EB1
};

// hyper-dual number v + a e1 + b e2 + ab e1 e2 with e1^2 = e2^2 = 0: with e1 on coordinate i
// and e2 on coordinate j, f(x) carries df/dx_i in a, df/dx_j in b and d2f/dx_i dx_j in ab
struct HD {
  double v, a, b, ab;
};
ABD_HD inline HD hd(double v) { return {v, 0.0, 0.0, 0.0}; }
ABD_HD inline HD operator+(HD x, HD y) { return {x.v + y.v, x.a + y.a, x.b + y.b, x.ab + y.ab}; }
ABD_HD inline HD operator-(HD x, HD y) { return {x.v - y.v, x.a - y.a, x.b - y.b, x.ab - y.ab}; }
ABD_HD inline HD operator-(HD x) { return {-x.v, -x.a, -x.b, -x.ab}; }
ABD_HD inline HD operator*(HD x, HD y) {
  return {x.v * y.v, x.v * y.a + x.a * y.v, x.v * y.b + x.b * y.v, x.v * y.ab + x.a * y.b + x.b * y.a + x.ab * y.v};
}
ABD_HD inline HD operator*(HD x, double s) { return {x.v * s, x.a * s, x.b * s, x.ab * s}; }
ABD_HD inline HD operator*(double s, HD x) { return x * s; }
ABD_HD inline HD operator+(HD x, double s) { return {x.v + s, x.a, x.b, x.ab}; }
ABD_HD inline HD operator-(HD x, double s) { return {x.v - s, x.a, x.b, x.ab}; }
ABD_HD inline HD operator-(double s, HD x) { return {s - x.v, -x.a, -x.b, -x.ab}; }
ABD_HD inline HD recip(HD x) {
  const double r = 1.0 / x.v, r2 = r * r;
  return {r, -x.a * r2, -x.b * r2, -x.ab * r2 + 2.0 * x.a * x.b * r2 * r};
}
ABD_HD inline HD operator/(HD x, HD y) { return x * recip(y); }
ABD_HD inline double value(double x) { return x; }
ABD_HD inline double value(const HD& x) { return x.v; }
ABD_HD inline double recip(double x) { return 1.0 / x; }
// the constant v as a number of x's kind
ABD_HD inline double constant_like(double, double v) { return v; }
ABD_HD inline HD constant_like(const HD&, double v) { return hd(v); }
// log with the value from lg (so host and device can share one log): d log u = du / u
template <class LogFn>
ABD_HD inline double log_of(double x, LogFn lg) { return lg(x); }
template <class LogFn>
ABD_HD inline HD log_of(HD x, LogFn lg) {
  const double r = 1.0 / x.v;
  return {lg(x.v), x.a * r, x.b * r, x.ab * r - x.a * x.b * r * r};
}

template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
ABD_HD inline V3<T> sub(const V3<T>& p, const V3<T>& q) {
  return {p.x - q.x, p.y - q.y, p.z - q.z};
}
template <class T>
ABD_HD inline T dot(const V3<T>& p, const V3<T>& q) {
  return (p.x * q.x + p.y * q.y) + p.z * q.z;
}
template <class T>
ABD_HD inline V3<T> cross(const V3<T>& p, const V3<T>& q) {
  return {p.y * q.z - p.z * q.y, p.z * q.x - p.x * q.z, p.x * q.y - p.y * q.x};
}

// squared distances of the feature pairs
template <class T>
ABD_HD inline T d2_point_point(const V3<T>& p, const V3<T>& q) {
  const V3<T> d = sub(p, q);
  return dot(d, d);
}
// point to the line through e0, e1: |(e0 - p) x (e1 - p)|^2 / |e1 - e0|^2
template <class T>
ABD_HD inline T d2_point_line(const V3<T>& p, const V3<T>& e0, const V3<T>& e1) {
  const V3<T> c = cross(sub(e0, p), sub(e1, p));
  const V3<T> e = sub(e1, e0);
  return dot(c, c) / dot(e, e);
}
// point to the plane through t0, t1, t2: ((p - t0) . n)^2 / |n|^2, n = (t1 - t0) x (t2 - t0)
template <class T>
ABD_HD inline T d2_point_plane(const V3<T>& p, const V3<T>& t0, const V3<T>& t1, const V3<T>& t2) {
  const V3<T> n = cross(sub(t1, t0), sub(t2, t0));
  const T s = dot(sub(p, t0), n);
  return s * s / dot(n, n);
}
// line through a0, a1 to the line through b0, b1: ((b0 - a0) . n)^2 / |n|^2, n = a x b
template <class T>
ABD_HD inline T d2_line_line(const V3<T>& a0, const V3<T>& a1, const V3<T>& b0, const V3<T>& b1) {
  const V3<T> n = cross(sub(a1, a0), sub(b1, b0));
  const T s = dot(sub(b0, a0), n);
  return s * s / dot(n, n);
}

// closest point of segment [a, b] to p as its clamped parameter s in [0, 1], and the squared
// distance to it
ABD_HD inline double point_segment(const V3<double>& p, const V3<double>& a, const V3<double>& b, double* d2) {
  const V3<double> e = sub(b, a);
  const double ee = dot(e, e);
  double s = ee > 0.0 ? dot(sub(p, a), e) / ee : 0.0;
  s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
  const V3<double> c = {a.x + s * e.x, a.y + s * e.y, a.z + s * e.z};
  *d2 = d2_point_point(p, c);
  return s;
}

// Point-triangle type: the interior when the point's projection lies in the closed triangle
// (the distance is convex in the barycentric parameters, so that minimum is global), else
// the nearest of the three edges as a segment, which is an edge or one of its end points.
// Ties go to the first in the order E0, E1, E2.
ABD_HD inline int pt_type(const V3<double>& p, const V3<double>& t0, const V3<double>& t1, const V3<double>& t2) {
  const V3<double> e1 = sub(t1, t0), e2 = sub(t2, t0), w = sub(p, t0);
  const double a = dot(e1, e1), b = dot(e1, e2), c = dot(e2, e2), d = dot(e1, w), e = dot(e2, w);
  const double det = a * c - b * b;
  if (det > 0.0) {
    const double beta = (c * d - b * e) / det, gamma = (a * e - b * d) / det;
    if (beta >= 0.0 && gamma >= 0.0 && beta + gamma <= 1.0) return PT_P_T;
  }
  const V3<double> tv[3] = {t0, t1, t2};
  int best = -1;
  double bd = 0.0, bs = 0.0;
  for (int k = 0; k < 3; ++k) {
    double d2;
    const double s = point_segment(p, tv[k], tv[(k + 1) % 3], &d2);
    if (best < 0 || d2 < bd) {
      best = k;
      bd = d2;
      bs = s;
    }
  }
  if (bs <= 0.0) return PT_P_V0 + best;
  if (bs >= 1.0) return PT_P_V0 + (best + 1) % 3;
  return PT_P_E0 + best;
}

// Edge-edge type: line-line when the closest points of the two lines lie inside both segments
// (the distance is convex in the two parameters), else the nearest of the four end point to
// segment distances (a0 and a1 to edge b, then b0 and b1 to edge a; ties go to the first).
// Parallel edges have no interior solution and fall to the end points.
ABD_HD inline int ee_type(const V3<double>& a0, const V3<double>& a1, const V3<double>& b0, const V3<double>& b1) {
  const V3<double> u = sub(a1, a0), v = sub(b1, b0), w = sub(a0, b0);
  const double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), e = dot(v, w);
  const double det = a * c - b * b;
  if (det > 0.0) {
    const double s = (b * e - c * d) / det, t = (a * e - b * d) / det;
    if (s > 0.0 && s < 1.0 && t > 0.0 && t < 1.0) return EE_EA_EB;
  }
  double d2[4], s[4];
  s[0] = point_segment(a0, b0, b1, &d2[0]);
  s[1] = point_segment(a1, b0, b1, &d2[1]);
  s[2] = point_segment(b0, a0, a1, &d2[2]);
  s[3] = point_segment(b1, a0, a1, &d2[3]);
  int k = 0;
  for (int m = 1; m < 4; ++m)
    if (d2[m] < d2[k]) k = m;
  // end point k against the other edge: its interior, or one of its end points
  const int kEdge[4] = {EE_EA0_EB, EE_EA1_EB, EE_EA_EB0, EE_EA_EB1};
  const int kAt0[4] = {EE_EA0_EB0, EE_EA1_EB0, EE_EA0_EB0, EE_EA0_EB1};
  const int kAt1[4] = {EE_EA0_EB1, EE_EA1_EB1, EE_EA1_EB0, EE_EA1_EB1};
  if (s[k] <= 0.0) return kAt0[k];
  if (s[k] >= 1.0) return kAt1[k];
  return kEdge[k];
}

// squared distance of a classified pair; x[0] point, x[1..3] triangle (PT) or x[0], x[1]
// edge a, x[2], x[3] edge b (EE)
template <class T>
ABD_HD inline T pt_d2(int type, const V3<T> x[4]) {
  switch (type) {
    case PT_P_T: return d2_point_plane(x[0], x[1], x[2], x[3]);
    case PT_P_E0: return d2_point_line(x[0], x[1], x[2]);
    case PT_P_E1: return d2_point_line(x[0], x[2], x[3]);
    case PT_P_E2: return d2_point_line(x[0], x[3], x[1]);
    case PT_P_V0: return d2_point_point(x[0], x[1]);
    case PT_P_V1: return d2_point_point(x[0], x[2]);
    default: return d2_point_point(x[0], x[3]);
  }
}
template <class T>
ABD_HD inline T ee_d2(int type, const V3<T> x[4]) {
  switch (type) {
    case EE_EA_EB: return d2_line_line(x[0], x[1], x[2], x[3]);
    case EE_EA0_EB: return d2_point_line(x[0], x[2], x[3]);
    case EE_EA1_EB: return d2_point_line(x[1], x[2], x[3]);
    case EE_EA_EB0: return d2_point_line(x[2], x[0], x[1]);
    case EE_EA_EB1: return d2_point_line(x[3], x[0], x[1]);
    case EE_EA0_EB0: return d2_point_point(x[0], x[2]);
    case EE_EA0_EB1: return d2_point_point(x[0], x[3]);
    case EE_EA1_EB0: return d2_point_point(x[1], x[2]);
    default: return d2_point_point(x[1], x[3]);
  }
}

// edge-edge mollifier threshold from the rest positions: 1e-3 |a_rest|^2 |b_rest|^2
ABD_HD inline double ee_eps_x(const double r[12]) {
  const V3<double> a = {r[3] - r[0], r[4] - r[1], r[5] - r[2]};
  const V3<double> b = {r[9] - r[6], r[10] - r[7], r[11] - r[8]};
  return 1e-3 * dot(a, a) * dot(b, b);
}
// m(x) = (2 - x / e_x) x / e_x below e_x, else 1, with x = |a x b|^2
template <class T>
ABD_HD inline T ee_mollifier(const V3<T> x[4], double eps_x) {
  const V3<T> n = cross(sub(x[1], x[0]), sub(x[3], x[2]));
  const T c = dot(n, n);
  if (!(value(c) < eps_x)) return constant_like(c, 1.0);
  const T q = c * (1.0 / eps_x);
  return (2.0 - q) * q;
}

// log barrier on squared distance d below dhat^2 = dh: -kappa (d / dh - 1)^2 log(d / dh)
template <class T, class LogFn>
ABD_HD inline T barrier_of(const T& d, double dh, double kappa, LogFn lg) {
  const T s = d * (1.0 / dh);
  const T t = s - 1.0;
  return -kappa * (t * t) * log_of(s, lg);
}

// contact energy of a classified pair (kind 0 PT, 1 EE)
template <class T, class LogFn>
ABD_HD inline T local_energy(int kind, int type, const V3<T> x[4], double eps_x, double dh, double kappa,
                             LogFn lg) {
  if (kind == 0) return barrier_of(pt_d2(type, x), dh, kappa, lg);
  return ee_mollifier(x, eps_x) * barrier_of(ee_d2(type, x), dh, kappa, lg);
}

ABD_HD inline void load(const double x[12], V3<double> v[4]) {
  for (int k = 0; k < 4; ++k) v[k] = {x[3 * k], x[3 * k + 1], x[3 * k + 2]};
}

// the pair's type (kind 0 PT, 1 EE) at positions x[12]
ABD_HD inline int contact_type(int kind, const double x[12]) {
  V3<double> v[4];
  load(x, v);
  return kind == 0 ? pt_type(v[0], v[1], v[2], v[3]) : ee_type(v[0], v[1], v[2], v[3]);
}

// Energy, gradient g[12] and Hessian H[144] (row-major) of one contact in the coordinates of
// its four points x[12]; r[12] the rest positions (for the mollifier).  Returns false, with
// nothing written but *type and *d2, when the pair is not within dhat.
template <class LogFn>
ABD_HD inline bool local_gh(int kind, const double x[12], const double r[12], double dh, double kappa, LogFn lg,
                            int* type, double* d2, double* E, double g[12], double H[144]) {
  V3<double> v[4];
  load(x, v);
  const int ty = kind == 0 ? pt_type(v[0], v[1], v[2], v[3]) : ee_type(v[0], v[1], v[2], v[3]);
  const double dd = kind == 0 ? pt_d2(ty, v) : ee_d2(ty, v);
  *type = ty;
  *d2 = dd;
  if (!(dd < dh)) return false;
  const double ex = kind == 1 ? ee_eps_x(r) : 0.0;
  for (int i = 0; i < 12; ++i)
    for (int j = i; j < 12; ++j) {
      V3<HD> h[4];
      for (int k = 0; k < 4; ++k) {
        HD c[3];
        for (int m = 0; m < 3; ++m) {
          const int q = 3 * k + m;
          c[m] = {x[q], q == i ? 1.0 : 0.0, q == j ? 1.0 : 0.0, 0.0};
        }
        h[k] = {c[0], c[1], c[2]};
      }
      const HD e = local_energy(kind, ty, h, ex, dh, kappa, lg);
      H[12 * i + j] = H[12 * j + i] = e.ab;
      if (j == i) g[i] = e.a;
      if (i == 0 && j == 0) *E = e.v;
    }
  return true;
}

// Eigen-decomposition of a symmetric 12x12 matrix H = V diag(lam) V^T (V's columns the
// eigenvectors, row-major) by Jacobi rotations in round-robin order: each sweep is 11 rounds
// of 6 rotations on disjoint index pairs (index 0 fixed, the others shifted one place per
// round).  A round takes its 6 angles from the matrix as it enters the round, then applies the
// 6 column updates, then the 6 row updates: the order a warp follows when its lanes share one
// round.  Stops when the off-diagonal part is below 1e-30 of the whole, or after 32 sweeps.
ABD_HD inline void eig_sym12(const double H[144], double lam[12], double V[144]) {
  double A[144];
  double total = 0.0;
  for (int k = 0; k < 144; ++k) {
    A[k] = H[k];
    V[k] = (k / 12 == k % 12) ? 1.0 : 0.0;
    total += H[k] * H[k];
  }
  int pos[12];
  for (int k = 0; k < 12; ++k) pos[k] = k;
  for (int sweep = 0; sweep < 32 && total > 0.0; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 12; ++p)
      for (int q = p + 1; q < 12; ++q) off += 2.0 * A[12 * p + q] * A[12 * p + q];
    if (!(off > 1e-30 * total)) break;
    for (int round = 0; round < 11; ++round) {
      int P[6], Q[6];
      double C[6], S[6];
      for (int k = 0; k < 6; ++k) {
        const int a = pos[k], b = pos[11 - k];
        P[k] = a < b ? a : b;
        Q[k] = a < b ? b : a;
        const double apq = A[12 * P[k] + Q[k]];
        if (apq == 0.0) {
          C[k] = 1.0;
          S[k] = 0.0;
          continue;
        }
        const double theta = (A[12 * Q[k] + Q[k]] - A[12 * P[k] + P[k]]) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        C[k] = 1.0 / sqrt(t * t + 1.0);
        S[k] = t * C[k];
      }
      for (int k = 0; k < 6; ++k)  // A <- A J, V <- V J (columns P, Q)
        for (int r = 0; r < 12; ++r) {
          const double ap = A[12 * r + P[k]], aq = A[12 * r + Q[k]];
          A[12 * r + P[k]] = C[k] * ap - S[k] * aq;
          A[12 * r + Q[k]] = S[k] * ap + C[k] * aq;
          const double vp = V[12 * r + P[k]], vq = V[12 * r + Q[k]];
          V[12 * r + P[k]] = C[k] * vp - S[k] * vq;
          V[12 * r + Q[k]] = S[k] * vp + C[k] * vq;
        }
      for (int k = 0; k < 6; ++k)  // A <- J^T A (rows P, Q)
        for (int c = 0; c < 12; ++c) {
          const double ap = A[12 * P[k] + c], aq = A[12 * Q[k] + c];
          A[12 * P[k] + c] = C[k] * ap - S[k] * aq;
          A[12 * Q[k] + c] = S[k] * ap + C[k] * aq;
        }
      const int last = pos[11];  // next round: shift indices 1..11 by one place
      for (int k = 11; k > 1; --k) pos[k] = pos[k - 1];
      pos[1] = last;
    }
  }
  for (int k = 0; k < 12; ++k) lam[k] = A[13 * k];
}

// Projects a symmetric 12x12 matrix onto the positive semidefinite cone: its eigenpairs
// (eig_sym12) with negative eigenvalues set to 0, the matrix rebuilt from them.
ABD_HD inline void project_psd12(double H[144]) {
  double lam[12], Vm[144];
  eig_sym12(H, lam, Vm);
  for (int k = 0; k < 12; ++k) lam[k] = lam[k] > 0.0 ? lam[k] : 0.0;
  for (int i = 0; i < 12; ++i)
    for (int j = i; j < 12; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 12; ++k) acc += Vm[12 * i + k] * lam[k] * Vm[12 * j + k];
      H[12 * i + j] = H[12 * j + i] = acc;
    }
}

// A point-coordinate vector v[12] as a vector over the two bodies' affine DOFs u[24] (the
// first body's 12, then the second's), with the weights of to_affine: a rank-one term
// c v v^T of the projected contact Hessian becomes c u u^T in the DOFs.
ABD_HD inline void to_affine_vec(const double v[12], const double r[12], int nI, double u[24]) {
  for (int k = 0; k < 24; ++k) u[k] = 0.0;
  for (int p = 0; p < 4; ++p) {
    const int off = p < nI ? 0 : 12;
    const double w[4] = {1.0, r[3 * p], r[3 * p + 1], r[3 * p + 2]};
    for (int m = 0; m < 4; ++m)
      for (int a = 0; a < 3; ++a) u[off + 3 * m + a] += w[m] * v[3 * p + a];
  }
}

// Maps a contact's gradient and Hessian in point coordinates to the affine DOFs of its two
// bodies (x = A^T r + p, DOFs [p, A row 0, row 1, row 2]).  Points 0 .. nI-1 move with the
// first body (PT: the point, nI = 1; EE: edge a, nI = 2), the rest with the second.
// g24: the first body's 12 DOFs, then the second's; Hi, Hj the diagonal blocks, Hij the
// coupling block (first body's rows, second body's columns).
ABD_HD inline void to_affine(const double gx[12], const double Hx[144], const double r[12], int nI, double g24[24],
                             double Hi[144], double Hj[144], double Hij[144]) {
  double w[4][4];  // w[v][m]: weight of DOF group m (1, r_v) for point v
  for (int v = 0; v < 4; ++v) {
    w[v][0] = 1.0;
    for (int m = 1; m < 4; ++m) w[v][m] = r[3 * v + m - 1];
  }
  for (int m = 0; m < 4; ++m)
    for (int a = 0; a < 3; ++a) {
      double sI = 0.0, sJ = 0.0;
      for (int v = 0; v < 4; ++v) (v < nI ? sI : sJ) += w[v][m] * gx[3 * v + a];
      g24[3 * m + a] = sI;
      g24[12 + 3 * m + a] = sJ;
    }
  for (int m = 0; m < 4; ++m)
    for (int a = 0; a < 3; ++a)
      for (int n = 0; n < 4; ++n)
        for (int b = 0; b < 3; ++b) {
          double sII = 0.0, sJJ = 0.0, sIJ = 0.0;
          for (int u = 0; u < 4; ++u)
            for (int v = 0; v < 4; ++v) {
              const double h = w[u][m] * Hx[12 * (3 * u + a) + 3 * v + b] * w[v][n];
              if (u < nI && v < nI) sII += h;
              else if (u >= nI && v >= nI) sJJ += h;
              else if (u < nI) sIJ += h;
            }
          Hi[12 * (3 * m + a) + 3 * n + b] = sII;
          Hj[12 * (3 * m + a) + 3 * n + b] = sJJ;
          Hij[12 * (3 * m + a) + 3 * n + b] = sIJ;
        }
}

// ---------------------------------------------------------------------------------------
// Lagged friction (Li et al. 2020, section 5): at the step start x^t each contact fixes the
// weights w of its closest points (c_a - c_b = sum_v w_v x_v: + for the first group, - for
// the second), a tangent basis P (3x2) orthogonal to the separation n = c_a - c_b, and the
// normal force lambda = -dE/dd of its barrier (mollified for EE).  The friction potential is
// D(x) = mu lambda f0(|u|), u = P^T sum_v w_v (x_v - x^t_v) the tangential displacement over
// the step, with f0' = f1(y) = 2 y / eps - y^2 / eps^2 below eps (static friction, eps =
// eps_v dt) and 1 above (sliding).  Its Hessian is positive semidefinite by construction.
// ---------------------------------------------------------------------------------------
struct FrictionLag {
  double w[4];    // closest-point weights of the four points
  double P[6];    // tangent basis, row-major 3x2
  double lambda;  // normal force
};

// closest-point weights of a classified pair at positions v[4]
ABD_HD inline void closest_weights(int kind, int type, const V3<double> v[4], double w[4]) {
  for (int k = 0; k < 4; ++k) w[k] = 0.0;
  w[0] = 1.0;
  if (kind == 0) {
    if (type == PT_P_T) {
      const V3<double> e1 = sub(v[2], v[1]), e2 = sub(v[3], v[1]), q = sub(v[0], v[1]);
      const double a = dot(e1, e1), b = dot(e1, e2), c = dot(e2, e2), d = dot(e1, q), e = dot(e2, q);
      const double det = a * c - b * b, s = (c * d - b * e) / det, t = (a * e - b * d) / det;
      w[1] = -(1.0 - s - t);
      w[2] = -s;
      w[3] = -t;
    } else if (type <= PT_P_E2) {
      const int i = 1 + (type - PT_P_E0), j = 1 + (type - PT_P_E0 + 1) % 3;
      double d2;
      const double s = point_segment(v[0], v[i], v[j], &d2);
      w[i] = -(1.0 - s);
      w[j] = -s;
    } else {
      w[1 + type - PT_P_V0] = -1.0;
    }
    return;
  }
  const V3<double> u = sub(v[1], v[0]), e = sub(v[3], v[2]), q = sub(v[0], v[2]);
  double s = 0.0, t = 0.0, d2;
  switch (type) {
    case EE_EA_EB: {
      const double a = dot(u, u), b = dot(u, e), c = dot(e, e), d = dot(u, q), f = dot(e, q);
      const double det = a * c - b * b;
      s = (b * f - c * d) / det;
      t = (a * f - b * d) / det;
      break;
    }
    case EE_EA0_EB: t = point_segment(v[0], v[2], v[3], &d2); break;
    case EE_EA1_EB: s = 1.0; t = point_segment(v[1], v[2], v[3], &d2); break;
    case EE_EA_EB0: s = point_segment(v[2], v[0], v[1], &d2); break;
    case EE_EA_EB1: s = point_segment(v[3], v[0], v[1], &d2); t = 1.0; break;
    case EE_EA0_EB0: break;
    case EE_EA0_EB1: t = 1.0; break;
    case EE_EA1_EB0: s = 1.0; break;
    default: s = 1.0; t = 1.0; break;
  }
  w[0] = 1.0 - s;
  w[1] = s;
  w[2] = -(1.0 - t);
  w[3] = -t;
}

// The lagged quantities of one contact at the step start xt[12] (rest positions r for the
// EE mollifier); false when the pair is not within dhat there.
template <class LogFn>
ABD_HD inline bool friction_lag(int kind, const double xt[12], const double r[12], double dh, double kappa, LogFn lg,
                                FrictionLag* L) {
  V3<double> v[4];
  load(xt, v);
  const int type = kind == 0 ? pt_type(v[0], v[1], v[2], v[3]) : ee_type(v[0], v[1], v[2], v[3]);
  const double d2 = kind == 0 ? pt_d2(type, v) : ee_d2(type, v);
  if (!(d2 < dh) || !(d2 > 0.0)) return false;
  closest_weights(kind, type, v, L->w);
  V3<double> n = {0.0, 0.0, 0.0};
  for (int k = 0; k < 4; ++k) {
    n.x += L->w[k] * v[k].x;
    n.y += L->w[k] * v[k].y;
    n.z += L->w[k] * v[k].z;
  }
  const double nl = sqrt(dot(n, n));
  n = {n.x / nl, n.y / nl, n.z / nl};
  // tangent basis: the coordinate axis least aligned with n, made orthogonal to it
  const double ax = fabs(n.x), ay = fabs(n.y), az = fabs(n.z);
  const V3<double> axis = (ax <= ay && ax <= az) ? V3<double>{1.0, 0.0, 0.0}
                          : (ay <= az)            ? V3<double>{0.0, 1.0, 0.0}
                                                  : V3<double>{0.0, 0.0, 1.0};
  V3<double> t1 = cross(n, axis);
  const double tl = sqrt(dot(t1, t1));
  t1 = {t1.x / tl, t1.y / tl, t1.z / tl};
  const V3<double> t2 = cross(n, t1);
  L->P[0] = t1.x, L->P[1] = t2.x, L->P[2] = t1.y, L->P[3] = t2.y, L->P[4] = t1.z, L->P[5] = t2.z;
  // lambda = -dE/dd, E = m b(d^2): -2 d m b'(d^2) with b'(d^2) from the barrier's derivative
  const double d = sqrt(d2);
  HD dd = {d, 1.0, 0.0, 0.0};
  const HD e = barrier_of(dd * dd, dh, kappa, lg);
  const double m = kind == 1 ? ee_mollifier(v, ee_eps_x(r)) : 1.0;
  L->lambda = -m * e.a;
  return true;
}

// friction potential, gradient g[12] and Hessian H[144] at positions x (step start xt)
ABD_HD inline double friction_gh(const FrictionLag& L, const double x[12], const double xt[12], double mu,
                                 double eps, double g[12], double H[144]) {
  double dx[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) dx[a] += L.w[k] * (x[3 * k + a] - xt[3 * k + a]);
  const double u0 = L.P[0] * dx[0] + L.P[2] * dx[1] + L.P[4] * dx[2];
  const double u1 = L.P[1] * dx[0] + L.P[3] * dx[1] + L.P[5] * dx[2];
  const double y = sqrt(u0 * u0 + u1 * u1), c = mu * L.lambda;
  double f0, f1y, M00, M01, M11;  // f1(y) / y and the 2x2 Hessian of f0(|u|)
  if (y >= eps) {
    f0 = y;
    f1y = 1.0 / y;
    const double h0 = u0 / y, h1 = u1 / y;
    M00 = f1y * (1.0 - h0 * h0);
    M01 = -f1y * h0 * h1;
    M11 = f1y * (1.0 - h1 * h1);
  } else {
    f0 = -y * y * y / (3.0 * eps * eps) + y * y / eps + eps / 3.0;
    f1y = 2.0 / eps - y / (eps * eps);
    const double k = y > 0.0 ? 1.0 / (eps * eps * y) : 0.0;  // -(f1' - f1 / y) / y^2
    M00 = f1y - k * u0 * u0;
    M01 = -k * u0 * u1;
    M11 = f1y - k * u1 * u1;
  }
  // per point v: d u / d x_v = w_v P^T, so g_v = c w_v P (f1 / y) u, H_vw = c w_v w_w P M P^T
  const double gu0 = f1y * u0, gu1 = f1y * u1;
  double PMP[9];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      PMP[3 * a + b] = L.P[2 * a] * (M00 * L.P[2 * b] + M01 * L.P[2 * b + 1]) +
                       L.P[2 * a + 1] * (M01 * L.P[2 * b] + M11 * L.P[2 * b + 1]);
  for (int v = 0; v < 4; ++v)
    for (int a = 0; a < 3; ++a) {
      g[3 * v + a] = c * L.w[v] * (L.P[2 * a] * gu0 + L.P[2 * a + 1] * gu1);
      for (int q = 0; q < 4; ++q)
        for (int b = 0; b < 3; ++b) H[12 * (3 * v + a) + 3 * q + b] = c * L.w[v] * L.w[q] * PMP[3 * a + b];
    }
  return c * f0;
}

// the friction potential alone, with friction_gh's arithmetic (the same value, bit for bit)
ABD_HD inline double friction_d(const FrictionLag& L, const double x[12], const double xt[12], double mu, double eps) {
  double dx[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) dx[a] += L.w[k] * (x[3 * k + a] - xt[3 * k + a]);
  const double u0 = L.P[0] * dx[0] + L.P[2] * dx[1] + L.P[4] * dx[2];
  const double u1 = L.P[1] * dx[0] + L.P[3] * dx[1] + L.P[5] * dx[2];
  const double y = sqrt(u0 * u0 + u1 * u1), c = mu * L.lambda;
  const double f0 = y >= eps ? y : -y * y * y / (3.0 * eps * eps) + y * y / eps + eps / 3.0;
  return c * f0;
}

}  // namespace ipc
}  // namespace abd
