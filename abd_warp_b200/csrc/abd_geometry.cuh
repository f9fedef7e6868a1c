// Per-primitive-pair device math: distance geometry, barrier, the analytic eigensystem of
// the distance Hessian ("psd method") and the FP64 cubic continuous collision detection.
//
// Reference formulas (files of Luke-Skycrawler/abd-warp):
//   c-coordinates, alpha/beta/gamma ........... abd/psd/vf.py:3-41, abd/psd/ee.py:5-31,118-132
//   dc/dx with frozen alpha, beta, gamma ...... abd/psd/vf.py:43-71, abd/psd/ee.py:134-163
//   signed distance, gradient ................. abd/psd/hl.py:15-17, 36-39
//   eigensystem of 2 l Hl ..................... abd/psd/hl.py:155-195, pt_ipc.py:258-280
//   interior tests ............................ abd/ccd.py:44-54
//   barrier and derivatives ................... abd/ipcsk/barrier.py:3-49
//   contact energy ............................ abd/ipcsk/energy.py:9-48
//   coplanarity cubic and roots ............... abd/ccd.py:56-195, abd/cubic_roots.py:6-193
// Operation order follows those files so that, with FMA contraction off, results round
// like the CPU oracle.  pow(x, 2.0) is evaluated as x * x (its correctly rounded value).
#pragma once

#include "abd_common.cuh"
#include "abd_exact.cuh"
#include "abd_ipc_full.cuh"

namespace abd {

struct Geo {
  d3 e0, e1p, e2p;
  double alpha, beta, gamma;
};

// type 0: point-triangle (x0 point, x1..x3 triangle); type 1: edge-edge (x0x1, x2x3)
__device__ inline Geo geometry(int type, d3 x0, d3 x1, d3 x2, d3 x3) {
  Geo G;
  d3 e0, e1, e2;
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
  // [beta, gamma] = inverse([[e0.e0, e0.e1], [e0.e1, e1.e1]]) [e0.e2, e1.e2]
  const double a = dot(e0, e0), b = dot(e0, e1), d = dot(e1, e1);
  const double det = a * d - b * b;
  const double sc = 1.0 / det;
  const double i00 = d * sc, i01 = -b * sc, i10 = -b * sc, i11 = a * sc;
  const double r0 = dot(e0, e2), r1 = dot(e1, e2);
  G.beta = i00 * r0 + i01 * r1;
  G.gamma = i10 * r0 + i11 * r1;
  G.e2p = (e2 - G.beta * e0) - G.gamma * e1;
  return G;
}

__device__ inline bool valid_root(int type, double beta, double gamma) {
  if (type == 0)
    return 0.0 < beta && beta < 1.0 && 0.0 < gamma && gamma < 1.0 && 0.0 < beta + gamma && beta + gamma < 1.0;
  return 0.0 < beta && beta < 1.0 && 0.0 < -gamma && -gamma < 1.0;
}

__device__ inline double signed_distance(d3 e0p, d3 e1p, d3 e2p) {
  d3 n = cross(e0p, e1p);
  return dot(e2p, n) / sqrt(dot(n, n));
}

// Natural logarithm, computed with IEEE-exact operations only (+, -, *, / correctly rounded,
// frexp exact) so that the oracle's restatement of the same steps returns the same bits.
// Method: argument reduction x = (1 + f) 2^k with 1 + f in [sqrt(1/2), sqrt(2)) (f exact by
// Sterbenz's lemma) and the series log(1 + f) = 2 atanh(s), s = f / (2 + f), |s| < 0.1716:
// 2 atanh(s) = 2s + s R(z), z = s^2, R = sum_{i=1..11} 2 z^i / (2i + 1), and 2s = f - f s,
// so log(1 + f) = f - s (f - R), whose correction term is small against the exact f (the
// classical atanh reduction, e.g. J.-M. Muller, "Elementary Functions: Algorithms and
// Implementation", ch. 11).  log 2 is split in two parts so that k log 2 adds no rounding
// error of its own.  Measured accuracy: within 1 ulp of the true logarithm.
__device__ inline double abd_log(double x) {
  if (!(x > 0.0)) return x == 0.0 ? -INFINITY : __longlong_as_double(0x7ff8000000000000LL);
  if (isinf(x)) return x;
  int k;
  double m = frexp(x, &k);  // x = m 2^k, m in [0.5, 1)
  if (m < 0.70710678118654752) {
    m = m * 2.0;
    k -= 1;
  }
  const double f = m - 1.0;
  const double s = f / (2.0 + f);
  const double z = s * s;
  double r = 2.0 / 23.0;
  r = r * z + 2.0 / 21.0;
  r = r * z + 2.0 / 19.0;
  r = r * z + 2.0 / 17.0;
  r = r * z + 2.0 / 15.0;
  r = r * z + 2.0 / 13.0;
  r = r * z + 2.0 / 11.0;
  r = r * z + 2.0 / 9.0;
  r = r * z + 2.0 / 7.0;
  r = r * z + 2.0 / 5.0;
  r = r * z + 2.0 / 3.0;
  r = r * z;
  // log 2 = kLn2Hi + kLn2Lo with kLn2Hi on 40 bits, so k * kLn2Hi is exact for |k| < 2^12
  const double kLn2Hi = 0.6931471805592082, kLn2Lo = 7.371002565167799e-13;
  return (double)k * kLn2Hi + (f - (s * (f - r) - (double)k * kLn2Lo));
}

__device__ inline double barrier(double d, const abd_params& P) {
  if (d < P.d2hat) {
    const double s = d / P.d2hat;
    const double t = s - 1.0;
    return P.kappa * -(t * t) * abd_log(s);
  }
  return 0.0;
}
__device__ inline double barrier_d1(double d, const abd_params& P) {
  if (d < P.d2hat)
    return P.kappa * (P.d2hat - d) * (2.0 * abd_log(d / P.d2hat) + (d - P.d2hat) / d) / (P.d2hat * P.d2hat);
  return 0.0;
}
__device__ inline double barrier_d2(double d, const abd_params& P) {
  if (d < P.d2hat)
    return -P.kappa *
           (2.0 * abd_log(d / P.d2hat) + (d - P.d2hat) / d + (d - P.d2hat) * (2.0 / d + P.d2hat / (d * d))) /
           (P.d2hat * P.d2hat);
  return 0.0;
}

// Energy of one candidate (ipcsk/energy.py: PT uses |e2p|^2, EE the squared signed distance)
__device__ inline double contact_energy(int type, const d3 xs[4], const abd_params& P) {
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

// Activity test of the gradient/Hessian pass (pt_ipc.py:13-22, 114; ee_ipc.py:13-23, 382):
// PT uses the squared signed distance, EE |e2p|^2.
__device__ inline bool contact_active(int type, const d3 xs[4], const abd_params& P, Geo* Gout, double* d2out) {
  Geo G = geometry(type, xs[0], xs[1], xs[2], xs[3]);
  const bool valid = valid_root(type, G.beta, G.gamma);
  double d2;
  if (type == 0) {
    const double l = signed_distance(G.e0, G.e1p, G.e2p);
    d2 = l * l;
  } else {
    d2 = dot(G.e2p, G.e2p);
  }
  *Gout = G;
  *d2out = d2;
  return d2 < P.d2hat && valid;
}

// ---------------------------------------------------------------------------------------
// The full IPC contact model (abd_params.ipc_full; abd_ipc_full.cuh): the closest feature pair
// is classified and the barrier acts on its squared distance, with the edge-edge mollifier.
// The logarithm is the shared one, so the oracle's full mode (which evaluates the same header)
// gets the same bits.
// ---------------------------------------------------------------------------------------
struct SharedLog {
  __device__ double operator()(double v) const { return abd_log(v); }
};
__device__ inline void points12(const d3 xs[4], double x[12]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[3 * k] = xs[k].x;
    x[3 * k + 1] = xs[k].y;
    x[3 * k + 2] = xs[k].z;
  }
}
// the candidate's classified squared distance (and its type): the contact is active below dhat^2
__device__ inline double full_d2(int kind, const d3 xs[4], int* type) {
  double x[12];
  points12(xs, x);
  ipc::V3<double> v[4];
  ipc::load(x, v);
  const int ty = ipc::contact_type(kind, x);
  *type = ty;
  return kind == 0 ? ipc::pt_d2(ty, v) : ipc::ee_d2(ty, v);
}
// its energy (0 beyond dhat); r: the four points' rest positions (the mollifier's scale)
__device__ inline double full_contact_energy(int kind, const d3 xs[4], const double r[12], const abd_params& P) {
  int ty;
  if (!(full_d2(kind, xs, &ty) < P.d2hat)) return 0.0;
  double x[12];
  points12(xs, x);
  ipc::V3<double> v[4];
  ipc::load(x, v);
  return ipc::local_energy(kind, ty, v, kind == 1 ? ipc::ee_eps_x(r) : 0.0, P.d2hat, P.kappa, SharedLog());
}

// Factored barrier Hessian of one active contact:
//   H = sum_k coef[k] u_k u_k^T,   g = gscale * u_4,
// where u_k (24 entries, body I DOFs then body J DOFs) = (W^T (D kron I3)^T) q_k, q_k the
// eigenvectors of the c-space Hessian of l^2 (q_4 = 2 l grad l), D the 3x4 dc/dx and W the
// per-vertex affine Jacobian rows [1, r_v] (pt_ipc.py:194-255, ee_ipc.py:449-498).
// This is the reference's (D^T Q Lambda Q^-1 D) / J^T H J product regrouped as a sum of
// rank-one terms; contact_psd selects the reference's eigenvalue treatment (0) or the PSD
// projection of the barrier Hessian (1).
struct ContactScalars {
  double q[5][9];
  double coef[5];
  double gscale;
  double D[3][4];
};

__device__ inline void contact_scalars(int type, const Geo& G, double d2, const abd_params& P,
                                       ContactScalars& C) {
  const double l = signed_distance(G.e0, G.e1p, G.e2p);
  const double e0pn = dot(G.e0, G.e0), e1pn = dot(G.e1p, G.e1p), e2pn = dot(G.e2p, G.e2p);
  const double f12 = sqrt(1.0 + 4.0 * (e1pn / e2pn));
  const double f02 = sqrt(1.0 + 4.0 * (e0pn / e2pn));
  double lam[5];
  lam[0] = -l / (2.0 * e1pn) * (1.0 + f12);
  lam[1] = -l / (2.0 * e1pn) * (1.0 - f12);
  lam[2] = -l / (2.0 * e0pn) * (1.0 + f02);
  lam[3] = -l / (2.0 * e0pn) * (1.0 - f02);
  double om[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) om[k] = lam[k] / (lam[k] - l / e2pn);
#pragma unroll
  for (int k = 0; k < 5; ++k)
#pragma unroll
    for (int i = 0; i < 9; ++i) C.q[k][i] = 0.0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    d3 t = om[k] * G.e1p;
    C.q[k][3] = G.e2p.x; C.q[k][4] = G.e2p.y; C.q[k][5] = G.e2p.z;
    C.q[k][6] = t.x; C.q[k][7] = t.y; C.q[k][8] = t.z;
  }
#pragma unroll
  for (int k = 2; k < 4; ++k) {
    d3 t = om[k] * G.e0;
    C.q[k][0] = G.e2p.x; C.q[k][1] = G.e2p.y; C.q[k][2] = G.e2p.z;
    C.q[k][6] = t.x; C.q[k][7] = t.y; C.q[k][8] = t.z;
  }
  {
    d3 gl2 = G.e2p * l;
    gl2 = mk(gl2.x / e2pn, gl2.y / e2pn, gl2.z / e2pn);
    d3 q4 = (gl2 * 2.0) * l;
    C.q[4][6] = q4.x; C.q[4][7] = q4.y; C.q[4][8] = q4.z;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) lam[k] = lam[k] * 2.0 * l;
  lam[4] = 2.0;
  double qn[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double sq = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) sq += C.q[k][i] * C.q[k][i];
    qn[k] = sq;
  }
  const double Bp = barrier_d1(d2, P), Bpp = barrier_d2(d2, P);
  if (P.contact_psd == 1) {
#pragma unroll
    for (int k = 0; k < 4; ++k) C.coef[k] = fmax(Bp * lam[k], 0.0) / qn[k];
    C.coef[4] = fmax(Bp * 2.0 + Bpp * qn[4], 0.0) / qn[4];
  } else {
    const bool clamp = (type == 0) || P.psd_ee;
#pragma unroll
    for (int k = 0; k < 4; ++k) C.coef[k] = Bp * (clamp ? fmax(lam[k], 0.0) : lam[k]) / qn[k];
    C.coef[4] = Bp * 2.0 / qn[4] + Bpp;
  }
  C.gscale = Bp;
  const double al = G.alpha, be = G.beta, ga = G.gamma;
  if (type == 0) {
    C.D[0][0] = 0.0; C.D[0][1] = 1.0; C.D[0][2] = -1.0; C.D[0][3] = 0.0;
    C.D[1][0] = 0.0; C.D[1][1] = -al; C.D[1][2] = al - 1.0; C.D[1][3] = 1.0;
    C.D[2][0] = 1.0; C.D[2][1] = -be; C.D[2][2] = be + ga - 1.0; C.D[2][3] = -ga;
  } else {
    C.D[0][0] = -1.0; C.D[0][1] = 1.0; C.D[0][2] = 0.0; C.D[0][3] = 0.0;
    C.D[1][0] = al; C.D[1][1] = -al; C.D[1][2] = -1.0; C.D[1][3] = 1.0;
    C.D[2][0] = be - 1.0; C.D[2][1] = -be; C.D[2][2] = ga + 1.0; C.D[2][3] = -ga;
  }
}

// ---------------------------------------------------------------------------------------
// CCD: earliest coplanarity time in [0, 1] whose configuration passes the interior test
// ---------------------------------------------------------------------------------------
constexpr double kXError = 1e-10;  // cubic_roots.py:4

__device__ inline double cr_eval(const double c[4], double x) { return c[0] + x * (c[1] + x * (c[2] + x * c[3])); }
__device__ inline double multi_sign(double a, double b) { return b < 0.0 ? -a : a; }
__device__ inline bool diff_sign(double y0, double yr) { return y0 * yr < 0.0; }

__device__ inline double find_closed(const double coef[4], const double deriv[4], double x0, double x1, double y0) {
  double xr = (x0 + x1) / 2.0;
  double yr = cr_eval(coef, xr);
  double xb0 = x0, xb1 = x1;
  if (x1 - x0 <= kXError * 2.0) return xr;
  // the bracket [xb0, xb1] halves at least every other iteration; 4096 bounds the loop
  for (int guard = 0; guard < 4096; ++guard) {
    if (diff_sign(y0, yr)) xb1 = xr;
    else xb0 = xr;
    const double dy = cr_eval(deriv, xr);
    const double dx = yr / dy;
    const double xn = xr - dx;
    if (xn > xb0 && xn < xb1) {
      const double step = fabs(xr - xn);
      xr = xn;
      if (step > kXError) yr = cr_eval(coef, xr);
      else break;
    } else {
      xr = (xb0 + xb1) / 2.0;
      yr = cr_eval(coef, xr);
      if (xb0 == xr || xb1 == xr || xb1 - xb0 <= 2.0 * kXError) break;
    }
  }
  return xr;
}

__device__ inline int quadratic_roots(const double coef[3], double x0, double x1, double roots[2]) {
  roots[0] = roots[1] = 0.0;
  const double c = coef[0], b = coef[1], a = coef[2];
  const double delta = b * b - 4.0 * a * c;
  int ret = 0;
  if (delta > 0.0) {
    const double d = sqrt(delta);
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

__device__ inline int deflate_solve(const double coef[4], double roots[3], double lo, double x1) {
  double dp[3];
  dp[2] = coef[3];
  for (int i = 2; i > 0; --i) dp[i - 1] = coef[i] + roots[0] * dp[i];
  double qr[2];
  const int r = quadratic_roots(dp, lo, x1, qr);
  roots[1] = qr[0];
  roots[2] = qr[1];
  return r + 1;
}

__device__ inline int cubic_roots(const double coef[4], double x0, double x1, double roots[3]) {
  roots[0] = roots[1] = roots[2] = 0.0;
  const double y0 = cr_eval(coef, x0), y1 = cr_eval(coef, x1);
  const double a = coef[3] * 3.0, b_2 = coef[2], c = coef[1];
  const double deriv[4] = {c, 2.0 * b_2, a, 0.0};
  const double delta_4 = b_2 * b_2 - a * c;
  if (delta_4 > 0.0) {
    const double d_2 = sqrt(delta_4);
    const double q = -(b_2 + multi_sign(d_2, b_2));
    const double rv0 = q / a, rv1 = c / q;
    const double xa = rv0 < rv1 ? rv0 : rv1, xb = rv0 > rv1 ? rv0 : rv1;
    if (diff_sign(y0, y1)) {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) {
        roots[0] = find_closed(coef, deriv, x0, x1, y0);
        return 1;
      }
    } else {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) return 0;
    }
    if (xa > x0) {
      const double ya = cr_eval(coef, xa);
      if (diff_sign(y0, ya)) {
        roots[0] = find_closed(coef, deriv, x0, xa, y0);
        if (diff_sign(ya, y1) || (xb < x1 && diff_sign(ya, cr_eval(coef, xb)))) return deflate_solve(coef, roots, xa, x1);
        return 1;
      }
      if (xb < x1) {
        const double yb = cr_eval(coef, xb);
        if (diff_sign(ya, yb)) {
          roots[0] = find_closed(coef, deriv, xa, xb, ya);
          if (diff_sign(yb, y1)) return deflate_solve(coef, roots, xb, x1);
          return 1;
        }
        if (diff_sign(yb, y1)) {
          roots[0] = find_closed(coef, deriv, xb, x1, yb);
          return 1;
        }
      } else if (diff_sign(ya, y1)) {
        roots[0] = find_closed(coef, deriv, xa, x1, ya);
        return 1;
      }
    } else {
      const double yb = cr_eval(coef, xb);
      if (diff_sign(y0, yb)) {
        roots[0] = find_closed(coef, deriv, x0, xb, y0);
        if (diff_sign(yb, y1)) return deflate_solve(coef, roots, xb, x1);
        return 1;
      }
      if (diff_sign(yb, y1)) {
        roots[0] = find_closed(coef, deriv, xb, x1, yb);
        return 1;
      }
    }
    return 0;
  }
  if (diff_sign(y0, y1)) {
    roots[0] = find_closed(coef, deriv, x0, x1, y0);
    return 1;
  }
  return 0;
}

__device__ inline void cubic_binomial(const double a[3], const double b[3], double out[4]) {
  out[0] = b[0] * b[1] * b[2];
  out[1] = a[0] * b[1] * b[2] + b[0] * b[1] * a[2] + b[0] * a[1] * b[2];
  out[2] = a[0] * a[1] * b[2] + a[0] * b[1] * a[2] + b[0] * a[1] * a[2];
  out[3] = a[0] * a[1] * a[2];
}

// det(b + t a) of 3x3 row-major matrices, by the Leibniz terms (ccd.py:82-119)
__device__ inline void det_polynomial(const double a[9], const double b[9], double out[4]) {
  const int P[6][3] = {{0, 4, 8}, {1, 5, 6}, {2, 3, 7}, {0, 5, 7}, {1, 3, 8}, {2, 4, 6}};
  double pos[4] = {0.0, 0.0, 0.0, 0.0}, neg[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int t = 0; t < 6; ++t) {
    double av[3] = {a[P[t][0]], a[P[t][1]], a[P[t][2]]};
    double bv[3] = {b[P[t][0]], b[P[t][1]], b[P[t][2]]};
    double cb[4];
    cubic_binomial(av, bv, cb);
    if (t < 3) {
#pragma unroll
      for (int k = 0; k < 4; ++k) pos[k] = pos[k] + cb[k];
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) neg[k] = neg[k] + cb[k];
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = pos[k] - neg[k];
}

// matrix with the three points as columns (wp.mat33(v0, v1, v2) is column-wise)
__device__ inline void cols3(d3 p, d3 q, d3 r, double m[9]) {
  m[0] = p.x; m[3] = p.y; m[6] = p.z;
  m[1] = q.x; m[4] = q.y; m[7] = q.z;
  m[2] = r.x; m[5] = r.y; m[8] = r.z;
}

// pt_collision_time / ee_collision_time (ccd.py:133-186).  inclusive (the full contact model):
// a coplanarity root also counts on the closed triangle / segments, within 1e-9
__device__ inline double collision_time(int type, const d3 a0[4], const d3 a1[4], bool inclusive = false) {
  const int sel[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  double coef[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double A[9], B[9], d[4];
    cols3(a1[sel[k][0]], a1[sel[k][1]], a1[sel[k][2]], A);
    cols3(a0[sel[k][0]], a0[sel[k][1]], a0[sel[k][2]], B);
#pragma unroll
    for (int i = 0; i < 9; ++i) A[i] -= B[i];
    det_polynomial(A, B, d);
    // ((d0 - d1) + d2) - d3
#pragma unroll
    for (int i = 0; i < 4; ++i) coef[i] = (k == 0) ? d[i] : ((k & 1) ? coef[i] - d[i] : coef[i] + d[i]);
  }
  double roots[3];
  const int nr = cubic_roots(coef, 0.0, 1.0, roots);
  double root = 1.0;
  bool ok = false;
  for (int i = 0; i < nr; ++i) {
    root = roots[i];
    d3 pt[4];
#pragma unroll
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

// the lagged quantities of a friction record, as the full-model header's type
__device__ inline ipc::FrictionLag lag_of(const FricRec& f) {
  ipc::FrictionLag L;
  for (int k = 0; k < 4; ++k) L.w[k] = f.w[k];
  for (int k = 0; k < 6; ++k) L.P[k] = f.P[k];
  L.lambda = f.lam;
  return L;
}

}  // namespace abd
