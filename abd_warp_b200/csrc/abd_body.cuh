// Device helpers shared by the broad phase, the narrow passes and the batched line search:
// the DOF update and the vertex transform, the exact body bounds and the reference's FP32
// boxes at given positions, conservative affine images of rest-frame boxes, and the
// per-body inertia / orthogonality and vertex-ground terms.
#pragma once

#include "abd_common.cuh"

namespace abd {

// DOFs of body b at (A, p) - al dq, as [A row-major (9), p (3)] (update_qk, abd.py:154-157;
// dq holds p's three components first, then the rows of A)
__device__ inline void dofs_at(const double* A, const double* p, const double* dq, int b, double al, double M[12]) {
#pragma unroll
  for (int k = 0; k < 3; ++k) M[9 + k] = p[3 * b + k] - dq[12 * b + k] * al;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) M[3 * r + k] = A[9 * b + 3 * r + k] - dq[12 * b + 3 * (r + 1) + k] * al;
}

// (Ao, po) = (A, p) - al dq for body b, also into (Ao2, po2) when given (in place when Ao is A)
__device__ inline void update_body_dofs(int b, const double* A, const double* p, const double* dq, double al,
                                        double* Ao, double* po, double* Ao2, double* po2) {
  double M[12];
  dofs_at(A, p, dq, b, al, M);
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    Ao[9 * b + k] = M[k];
    if (Ao2) Ao2[9 * b + k] = M[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    po[3 * b + k] = M[9 + k];
    if (po2) po2[3 * b + k] = M[9 + k];
  }
}

// coordinate j of x = A^T r + p (update_mesh_vertex, abd.py:305-324)
__device__ inline double xform(const double M[12], double r0, double r1, double r2, int j) {
  return ((M[j] * r0 + M[3 + j] * r1) + M[6 + j] * r2) + M[9 + j];
}

// ---------------------------------------------------------------------------------------
// body bounds as order-preserving 64-bit keys, maximised atomically (exact, any order):
// key(-lo_k), key(hi_k) for k = 0..2 (swept bounds add the same six for the end positions);
// 0 = no vertex
// ---------------------------------------------------------------------------------------
__device__ inline unsigned long long max_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ inline double key_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
  return __longlong_as_double((long long)b);
}

// The FP32 body box of the reference (culling2.py:278-334): FP64 min / max of the vertices,
// dilated by dhat / 2 in FP64 and rounded to FP32; swept boxes add the undilated FP32 box
// of the end positions.
__device__ inline Box body_box_of(const unsigned long long* k, bool swept, double dhh) {
  Box B;
  B.pad0 = B.pad1 = 0.f;
  if (k[3] == 0) {  // no vertex
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      B.lo[j] = INFINITY;
      B.hi[j] = -INFINITY;
    }
    return B;
  }
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    B.lo[j] = (float)(-key_value(k[j]) - dhh);
    B.hi[j] = (float)(key_value(k[3 + j]) + dhh);
    if (swept) {
      B.lo[j] = fminf(B.lo[j], (float)(-key_value(k[6 + j])));
      B.hi[j] = fmaxf(B.hi[j], (float)key_value(k[9 + j]));
    }
  }
  return B;
}

// The reference's static FP32 boxes at given positions (culling2.py:32-79): a point converted
// to FP32 and dilated by FP32 dhat; a triangle's FP64 min / max rounded to FP32; an edge's
// FP64 min / max dilated by dhat / 2 and rounded.  The same arithmetic as point_box,
// tri_leaf_box and edge_leaf_box without end positions.
__device__ inline Box point_box_at(const d3& x, float dhf) {
  Box B;
  const double c[3] = {x.x, x.y, x.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float f = (float)c[k];
    B.lo[k] = f - dhf;
    B.hi[k] = f + dhf;
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}
__device__ inline Box tri_box_at(const d3& a, const d3& b, const d3& c) {
  Box B;
  const double u[3] = {a.x, a.y, a.z}, w[3] = {b.x, b.y, b.z}, q[3] = {c.x, c.y, c.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    B.lo[k] = (float)(fmin(fmin(u[k], w[k]), q[k]) - 0.0);
    B.hi[k] = (float)(fmax(fmax(u[k], w[k]), q[k]) + 0.0);
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}
__device__ inline Box edge_box_at(const d3& a, const d3& b, double dhh) {
  Box B;
  const double u[3] = {a.x, a.y, a.z}, w[3] = {b.x, b.y, b.z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    B.lo[k] = (float)(fmin(u[k], w[k]) - dhh);
    B.hi[k] = (float)(fmax(u[k], w[k]) + dhh);
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}

// the box of the vertex-ground culling's half space under the plane (culling.py:64-82)
__device__ inline Box ground_box(const abd_params& P) {
  Box g;
  g.lo[0] = g.lo[1] = g.lo[2] = -1e3f;
  g.hi[0] = 1e3f;
  g.hi[1] = (float)P.ground;
  g.hi[2] = 1e3f;
  g.pad0 = g.pad1 = 0.f;
  return g;
}

// Vertex-ground culling (culling.py:64-82): the vertex's body box bb reaches below
// ground + dhat / 2 and the vertex's box q overlaps the half space under the plane.
__device__ inline bool vg_box_test(const abd_params& P, const Box& bb, const Box& q) {
  if (!((double)bb.lo[1] < 0.5 * P.dhat + P.ground)) return false;
  return overlap(q, ground_box(P));
}

// Conservative world box of a rest-frame box R of a body moving by x = A^T r + p.  Centre
// and half extents map to p + A^T c and |A|^T h.  Computed in FP32 from FP32 copies
// m = (A row-major, p) of the DOFs; every rounding error of that (operand conversion, the
// products and sums, the rest box's own rounding) stays below
// 2^-21 (|p_j| + sum_k |A_kj| max(|R.lo_k|, |R.hi_k|)), so a margin of 2^-16 of that plus the
// dilation `pad` (rounded up) keeps every box of the enclosed primitives inside the result.
// The margin also covers positions at DOFs between two sets m0, m1 (x is affine in the DOFs;
// the FP64 rounding of intermediate DOFs and positions is far below 2^-21 of the scale), so
// the union of the images under m0 and m1 holds every such position's box.
__device__ inline Box affine_box(const Box& R, const float* m, float pad) {
  float c[3], h[3], e[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    c[k] = 0.5f * (R.lo[k] + R.hi[k]);
    h[k] = 0.5f * (R.hi[k] - R.lo[k]);
    e[k] = fmaxf(fabsf(R.lo[k]), fabsf(R.hi[k]));
  }
  Box B;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float a0 = m[j], a1 = m[3 + j], a2 = m[6 + j];
    const float cw = __fmaf_rn(a2, c[2], __fmaf_rn(a1, c[1], __fmaf_rn(a0, c[0], m[9 + j])));
    const float hw = __fmaf_rn(fabsf(a2), h[2], __fmaf_rn(fabsf(a1), h[1], fabsf(a0) * h[0]));
    const float sc = __fmaf_rn(fabsf(a2), e[2], __fmaf_rn(fabsf(a1), e[1], __fmaf_rn(fabsf(a0), e[0], fabsf(m[9 + j]))));
    const float w = hw + __fmaf_rn(sc, 0x1p-16f, pad);
    B.lo[j] = cw - w;
    B.hi[j] = cw + w;
  }
  B.pad0 = B.pad1 = 0.f;
  return B;
}

// affine_box under m0, united with the image under m1 when m1 is set
__device__ inline Box affine_box2(const Box& R, const float* m0, const float* m1, float pad) {
  Box B = affine_box(R, m0, pad);
  if (m1) {
    const Box B1 = affine_box(R, m1, pad);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      B.lo[k] = fminf(B.lo[k], B1.lo[k]);
      B.hi[k] = fmaxf(B.hi[k], B1.hi[k]);
    }
  }
  return B;
}

// predicted DOFs q~ = q0 + dt qdot (+ dt^2 g for p) (orthogonal_energy.py:24-32)
__device__ inline void tilde_of(const abd_params& P, const abd_states& st, int b, double At[9], double pt[3]) {
  const double dt = P.dt;
#pragma unroll
  for (int k = 0; k < 9; ++k) At[k] = st.A0[9 * b + k] + dt * st.Adot[9 * b + k];
  const double gv[3] = {0.0, P.gravity, 0.0};
#pragma unroll
  for (int k = 0; k < 3; ++k) pt[k] = (st.p0[3 * b + k] + dt * st.pdot[3 * b + k]) + (dt * dt) * gv[k];
}

// inertia + orthogonality energy of a free body at trial DOFs K, pk (orthogonal_energy.py:24-32)
__device__ inline double inertia_energy(const abd_params& P, const abd_states& st, const double* mass,
                                        const double* I0, int b, const double* K, const double* pk) {
  double At[9], pt[3];
  tilde_of(P, st, b, At, pt);
  double eo = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const double tt =
          (K[3 * i] * K[3 * j] + K[3 * i + 1] * K[3 * j + 1] + K[3 * i + 2] * K[3 * j + 2]) - (i == j ? 1.0 : 0.0);
      eo += tt * tt;
    }
  eo = eo * P.stiffness;
  double d0[3], d1[3], d2[3], d3v[3];
  for (int k = 0; k < 3; ++k) {
    d0[k] = pk[k] - pt[k];
    d1[k] = K[k] - At[k];
    d2[k] = K[3 + k] - At[3 + k];
    d3v[k] = K[6 + k] - At[6 + k];
  }
  auto dd = [](const double* u) { return u[0] * u[0] + u[1] * u[1] + u[2] * u[2]; };
  const double nm = dd(d0) * mass[b] + (dd(d1) + dd(d2) + dd(d3v)) * I0[b];
  return eo * P.dt * P.dt + 0.5 * nm;
}

}  // namespace abd
