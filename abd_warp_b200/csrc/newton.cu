// The step's Newton iterations as a device loop (abd_step with newton_loop = 0).
//
// AffineBodySimulator.step (abd/abd.py:212-276) iterates gradient / Hessian, linear solve, CCD
// bound and backtracking line search until g.g < tol or max_iter iterations.  Run from the host,
// every iteration waits for the device twice: to read the line search's energies and to check
// the passes' list capacities.  Here one CUDA graph holds the whole step: a WHILE node over the
// Newton iterations, whose body is the GH pass, then (an IF node, taken when no list of that
// pass overflowed) the preconditioner, the Krylov solve (itself a WHILE node), the CCD pass with
// the line search's trials, the acceptance test and the DOF update; the loop's last kernel makes
// the convergence test.  The host launches it once per step and reads the step's counters with
// one copy.  When a list overflowed, the loop stops, the states are left as they were, and the
// host grows the list and runs the step again from its start (the warm start dq is restored
// from the copy the graph made).
//
// The kernels here keep the host loop's arithmetic, so both loops give the same bits: the
// energies are the exact sums rounded once on the device (the host rounds the same sums with
// the same rule), the Armijo test is evaluated in the same order, and the iteration counts
// follow the same rules.
#include <cuda_runtime.h>

#include "abd_body.cuh"

namespace abd {

static_assert(PF_N == 7 && kProfBytes[0] == 24.0 && kProfBytes[1] == 36.0 && kProfBytes[2] == 140.0 &&
                  kProfBytes[3] == 36.0 && kProfBytes[4] == 36.0 && kProfBytes[5] == 36.0 && kProfBytes[6] == 16.0,
              "k_ls_accept's copy of the profiling weights");

namespace {

// The step's start, one thread per body: q <- q0 and the line-search origin (Ak, pk) <- q0
// (abd.py:124-128), and the warm start dq kept for a rerun; thread 0 clears the step's
// counters and enters the Newton loop.
__global__ void k_step_begin(Mailbox* box, cudaGraphConditionalHandle h, int n, abd_states st, const double* dq,
                             double* dq_save) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n) {
    for (int k = 0; k < 9; ++k) st.A[9 * b + k] = st.Ak[9 * b + k] = st.A0[9 * b + k];
    for (int k = 0; k < 3; ++k) st.p[3 * b + k] = st.pk[3 * b + k] = st.p0[3 * b + k];
    for (int k = 0; k < 12; ++k) dq_save[12 * b + k] = dq[12 * b + k];
  }
  if (b != 0) return;
  StepDev& S = box->step;
  S.it = S.lin = S.ls = 0;
  S.n_pt = S.n_ee = S.n_vg = S.n_ij = S.n_active = 0;
  S.E0 = S.alpha = 0.0;
  S.toi = 1.0;
  S.t0 = ~0ULL;
  S.t1 = 0ULL;
  S.prof_ns = S.prof_n = 0ULL;
  S.prof_bytes = 0.0;
  cudaGraphSetConditional(h, 1u);
}

// The IF node after the GH pass: taken unless a list of the pass overflowed.  When it is
// taken, also the pass's outcome for the step: the active contacts of the iteration; at the
// first iteration the energy at q0 (the pass summed it: abd.py:126-128), the culling counts,
// and the kept line-search candidates are consumed (the step's CCD passes replace them).
__global__ void k_gate(Mailbox* box, cudaGraphConditionalHandle h, int* sup_have) {
  const int* ds = box->dstat;
  const bool ok = !(ds[DS_STATUS] & kRerunMask);
  cudaGraphSetConditional(h, ok ? 1u : 0u);
  if (!ok) return;
  StepDev& S = box->step;
  S.n_active = ds[DS_ACTIVE];
  if (S.it == 0) {
    S.E0 = xs_round(box->energy);
    S.n_pt = ds[DS_PT_COUNT];
    S.n_ee = ds[DS_EE_COUNT];
    S.n_vg = ds[DS_VG_COUNT];
    S.n_ij = ds[DS_NPAIRS];
    *sup_have = 0;
  }
}

// Backtracking line search (abd.py:146-160) over the trials of the batch (k_ls_eval's step
// lengths alpha, alpha / 2, ... to the first below alpha_min): the first trial that passes
// the Armijo test, or the first below alpha_min, is taken, as the sequential search takes it.
// A batch whose trials all fail while none is below alpha_min raises ST_LS_MORE (the host
// finishes that step).  Also the kernel timing of the CCD pass's narrow kernel.
__global__ void k_ls_accept(Mailbox* box, double* dpar, abd_params P, int prof_bytes) {
  StepDev& S = box->step;
  const int K = (int)dpar[kParK];
  const double E0 = S.E0, qTg = box->dots[0];
  double alpha = 0.0, E1 = E0;
  bool done = false;
  for (int k = 0; k < K && !done; ++k) {
    alpha = dpar[kParAlpha + k];
    E1 = xs_round(box->ls_energy[k]);
    ++S.ls;
    const bool wolfe = E1 < E0 + P.armijo_sign * P.c1 * alpha * qTg || fabs(E1 - E0) <= P.ls_noise_floor * fabs(E0);
    done = wolfe || alpha < P.alpha_min;
  }
  if (!done) atomicOr(&box->dstat[DS_STATUS], ST_LS_MORE);
  S.E0 = E1;
  S.alpha = alpha;
  dpar[kParAcc] = alpha;
  double toi = 1.0;
  if (const unsigned long long key = box->toi_key) toi = __longlong_as_double((long long)~key);
  S.toi = toi;
  if (S.t1 > S.t0 && S.t0 != ~0ULL) {
    S.prof_ns += S.t1 - S.t0;
    ++S.prof_n;
    if (prof_bytes) {
      // the weights of kProfBytes (bytes per counted access)
      const double w[PF_N] = {24.0, 36.0, 140.0, 36.0, 36.0, 36.0, 16.0};
      for (int row = 0; row < 32; ++row)
        for (int c = 0; c < PF_N; ++c) S.prof_bytes += w[c] * (double)box->prof[row][c];
    }
  }
  S.t0 = ~0ULL;
  S.t1 = 0ULL;
}

// The loop's last kernel, one thread per body: the accepted step q <- q - alpha dq, also
// into the line-search origin (Ak, pk) (update_qk, abd.py:154-157); then thread 0: the
// iteration count and the convergence test (abd.py:259-271: g.g < tol on the gradient the
// iteration solved with, or max_iter iterations).  A list overflow or a line search that needs
// more trials ends the loop without the update (the step is then made again from its start).
__global__ void k_newton_end(Mailbox* box, double tol, int max_iter, cudaGraphConditionalHandle h, int n,
                             abd_states st, const double* dq, const double* alpha) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < n && !(box->dstat[DS_STATUS] & kRerunMask))
    update_body_dofs(b, st.A, st.p, dq, *alpha, st.A, st.p, st.Ak, st.pk);
  if (b != 0) return;
  StepDev& S = box->step;
  ++S.it;
  const double gTg = box->dots[1];
  const bool stop = gTg < tol || S.it >= max_iter || (box->dstat[DS_STATUS] & kRerunMask);
  cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// The adjoint step's right-hand side a = qb + qdb / dt (fixed bodies: 0), into g
__global__ void k_adjoint_rhs(int n, const double* qb, const double* qdb, double dt, const int* fixed, double* g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 12 * n) return;
  g[i] = fixed[i / 12] ? 0.0 : qb[i] + qdb[i] / dt;
}

// From lambda = H^-1 a: t = M lambda, qb_t = t - qdb / dt, qdb_t = dt t (fixed bodies: 0);
// M = mass on p, I0 on the rows of A
__global__ void k_adjoint_out(int n, const double* lam, const double* mass, const double* I0, const double* qdb,
                              double dt, const int* fixed, double* qb_out, double* qdb_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 12 * n) return;
  const int b = i / 12;
  if (fixed[b]) {
    qb_out[i] = 0.0;
    qdb_out[i] = 0.0;
    return;
  }
  const double t = ((i % 12) < 3 ? mass[b] : I0[b]) * lam[i];
  const double d = qdb[i];
  qb_out[i] = t - d / dt;
  qdb_out[i] = dt * t;
}

}  // namespace

cudaError_t adjoint_rhs(Sim& s, const double* qb, const double* qdb) {
  k_adjoint_rhs<<<(12 * s.n + 255) / 256, 256, 0, s.stream>>>(s.n, qb, qdb, s.prm.dt, s.fixed, s.g);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t adjoint_out(Sim& s, const double* lam, const double* qdb, double* qb_out, double* qdb_out) {
  k_adjoint_out<<<(12 * s.n + 255) / 256, 256, 0, s.stream>>>(s.n, lam, s.mass, s.I0, qdb, s.prm.dt, s.fixed,
                                                             qb_out, qdb_out);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t step_begin(Sim& s, const abd_states& st, cudaGraphConditionalHandle h) {
  k_step_begin<<<(s.n + 127) / 128, 128, 0, s.stream>>>(s.box, h, s.n, st, s.dq, s.dq_save);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t gate_no_overflow(Sim& s, cudaGraphConditionalHandle h) {
  k_gate<<<1, 1, 0, s.stream>>>(s.box, h, s.dint + kSupHave);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t ls_accept(Sim& s) {
  k_ls_accept<<<1, 1, 0, s.stream>>>(s.box, s.dpar, s.prm, s.prof_on == 2 ? 1 : 0);
  ++s.launches;
  return cudaGetLastError();
}

cudaError_t newton_end(Sim& s, const abd_states& st, cudaGraphConditionalHandle h) {
  k_newton_end<<<(s.n + 127) / 128, 128, 0, s.stream>>>(s.box, s.prm.tol, s.prm.max_iter, h, s.n, st, s.dq,
                                                        s.dpar + kParAcc);
  ++s.launches;
  return cudaGetLastError();
}

}  // namespace abd
