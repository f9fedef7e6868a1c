// Host build of the full IPC contact model (abd_warp_b200/csrc/abd_ipc_full.cuh) for the CPU
// tests: the header's arithmetic runs unchanged on the host, and the tests compare it with
// the numpy restatement in oracle/ipc_full_ref.py.  Test infrastructure only.
#include <cmath>

#include "../../abd_warp_b200/csrc/abd_ipc_full.cuh"

namespace {
struct StdLog {
  double operator()(double x) const { return std::log(x); }
};
}  // namespace

extern "C" {

int ipcf_type(int kind, const double* x) { return abd::ipc::contact_type(kind, x); }

double ipcf_d2(int kind, int type, const double* x) {
  abd::ipc::V3<double> v[4];
  abd::ipc::load(x, v);
  return kind == 0 ? abd::ipc::pt_d2(type, v) : abd::ipc::ee_d2(type, v);
}

double ipcf_energy(int kind, const double* x, const double* r, double dh, double kappa) {
  abd::ipc::V3<double> v[4];
  abd::ipc::load(x, v);
  const int ty = abd::ipc::contact_type(kind, x);
  const double d2 = kind == 0 ? abd::ipc::pt_d2(ty, v) : abd::ipc::ee_d2(ty, v);
  if (!(d2 < dh)) return 0.0;
  const double ex = kind == 1 ? abd::ipc::ee_eps_x(r) : 0.0;
  return abd::ipc::local_energy(kind, ty, v, ex, dh, kappa, StdLog());
}

int ipcf_local_gh(int kind, const double* x, const double* r, double dh, double kappa, int* type, double* d2,
                  double* E, double* g, double* H) {
  return abd::ipc::local_gh(kind, x, r, dh, kappa, StdLog(), type, d2, E, g, H) ? 1 : 0;
}

void ipcf_project_psd12(double* H) { abd::ipc::project_psd12(H); }

void ipcf_eig_sym12(const double* H, double* lam, double* V) { abd::ipc::eig_sym12(H, lam, V); }

void ipcf_to_affine_vec(const double* v, const double* r, int nI, double* u) { abd::ipc::to_affine_vec(v, r, nI, u); }

int ipcf_friction_lag(int kind, const double* xt, const double* r, double dh, double kappa, double* w, double* P,
                      double* lambda) {
  abd::ipc::FrictionLag L;
  if (!abd::ipc::friction_lag(kind, xt, r, dh, kappa, StdLog(), &L)) return 0;
  for (int k = 0; k < 4; ++k) w[k] = L.w[k];
  for (int k = 0; k < 6; ++k) P[k] = L.P[k];
  *lambda = L.lambda;
  return 1;
}

double ipcf_friction_gh(const double* w, const double* P, double lambda, const double* x, const double* xt, double mu,
                        double eps, double* g, double* H) {
  abd::ipc::FrictionLag L;
  for (int k = 0; k < 4; ++k) L.w[k] = w[k];
  for (int k = 0; k < 6; ++k) L.P[k] = P[k];
  L.lambda = lambda;
  return abd::ipc::friction_gh(L, x, xt, mu, eps, g, H);
}

void ipcf_to_affine(const double* gx, const double* Hx, const double* r, int nI, double* g24, double* Hi, double* Hj,
                    double* Hij) {
  abd::ipc::to_affine(gx, Hx, r, nI, g24, Hi, Hj, Hij);
}

}  // extern "C"
