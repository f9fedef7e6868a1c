// Inertia + orthogonality energy of all bodies, computed without allocating device memory.
//
// Who this is for: callers that may not allocate device memory once they are running.
// Examples are a real-time control loop with a fixed memory budget, where cudaMalloc can
// stall the device and fragment memory, and a plug-in inside a host application that owns
// every device allocation through its own pool.  For them the only device memory this entry
// point uses besides the caller's inputs and output is a fixed scratch array compiled into
// the library.
//
// The scratch array holds one partial sum per CTA of 256 bodies, so a call accepts at most
// kMaxBodies = 4096 * 256 = 1,048,576 bodies and returns ABD_ERR_INVALID beyond that.  The
// array lives in every GPU that loads the library until the process exits.  All calls share
// it: two calls that overlap on the GPU (different streams, or different host threads with
// no ordering between them) race on it.  Each call writes every partial it later reads, so
// nothing has to be cleared between calls.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and remembers it for later calls; make
// that first call before any stream capture begins.  The remembered address belongs to the
// device's primary context: after cudaDeviceReset on that device it is stale, so a process
// that resets a device must not call this entry point on it afterwards.
//
// The sum: each CTA adds its 256 bodies' energies by a fixed-order tree and the last kernel
// adds the CTA partials the same way, so the result is deterministic but can differ in the
// last bits from abd_compute_energy, whose sum is exact (rounded once).
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/abd_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 4096;
constexpr long long kMaxBodies = (long long)kMaxBlocks * kThreads;
constexpr int kMaxDevices = 64;

}  // namespace

// per-CTA partial energies of the last call (device memory owned by the library image)
static __device__ __align__(256) double g_noalloc_partials[kMaxBlocks];

namespace {

struct NoAllocArgs {
  abd_params prm;
  int n;
  const double *Ak, *pk, *A0, *p0, *Adot, *pdot, *mass, *I0;
  const int* fixed;
};

// energy_inertia (orthogonal_energy.py:24-32) per body, same operation order as the
// simulator's body-energy kernel; CTA partial by a fixed-order tree
__global__ void __launch_bounds__(kThreads) k_energy_partials(NoAllocArgs a, double* partials) {
  __shared__ double red[kThreads];
  const int b = blockIdx.x * kThreads + threadIdx.x;
  double e = 0.0;
  if (b < a.n && !a.fixed[b]) {
    const double dt = a.prm.dt;
    double At[9], pt[3];
    for (int k = 0; k < 9; ++k) At[k] = a.A0[9 * b + k] + dt * a.Adot[9 * b + k];
    const double gv[3] = {0.0, a.prm.gravity, 0.0};
    for (int k = 0; k < 3; ++k) pt[k] = (a.p0[3 * b + k] + dt * a.pdot[3 * b + k]) + (dt * dt) * gv[k];
    const double* K = a.Ak + 9 * b;
    double eo = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const double t =
            (K[3 * i] * K[3 * j] + K[3 * i + 1] * K[3 * j + 1] + K[3 * i + 2] * K[3 * j + 2]) - (i == j ? 1.0 : 0.0);
        eo += t * t;
      }
    eo = eo * a.prm.stiffness;
    const double* pk = a.pk + 3 * b;
    double d0[3], d1[3], d2[3], d3[3];
    for (int k = 0; k < 3; ++k) {
      d0[k] = pk[k] - pt[k];
      d1[k] = K[k] - At[k];
      d2[k] = K[3 + k] - At[3 + k];
      d3[k] = K[6 + k] - At[6 + k];
    }
    auto dd = [](const double* u) { return u[0] * u[0] + u[1] * u[1] + u[2] * u[2]; };
    const double nm = dd(d0) * a.mass[b] + (dd(d1) + dd(d2) + dd(d3)) * a.I0[b];
    e = eo * dt * dt + 0.5 * nm;
  }
  red[threadIdx.x] = e;
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(1024) k_energy_finish(const double* partials, int nb, double* out) {
  __shared__ double red[1024];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += 1024) acc += partials[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {};

// device address of the scratch array on the current device (looked up once per device)
int scratch_address(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ABD_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return ABD_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_partials) != cudaSuccess || !p) return ABD_ERR_CUDA;
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return ABD_OK;
}

}  // namespace

extern "C" int abd_inertia_energy_noalloc(const abd_params* prm, int n_bodies, const abd_states* st,
                                          const double* Ak_dev, const double* pk_dev, const double* mass_dev,
                                          const double* I0_dev, const int* fixed_dev, double* E_dev, void* stream) {
  if (!prm || !st || !Ak_dev || !pk_dev || !mass_dev || !I0_dev || !fixed_dev || !E_dev || !st->A0 || !st->p0 ||
      !st->Adot || !st->pdot)
    return ABD_ERR_INVALID;
  if (n_bodies <= 0 || (long long)n_bodies > kMaxBodies) return ABD_ERR_INVALID;
  double* partials = nullptr;
  const int r = scratch_address(&partials);
  if (r != ABD_OK) return r;
  NoAllocArgs a;
  a.prm = *prm;
  a.n = n_bodies;
  a.Ak = Ak_dev;
  a.pk = pk_dev;
  a.A0 = st->A0;
  a.p0 = st->p0;
  a.Adot = st->Adot;
  a.pdot = st->pdot;
  a.mass = mass_dev;
  a.I0 = I0_dev;
  a.fixed = fixed_dev;
  int nb = (n_bodies + kThreads - 1) / kThreads;
  cudaStream_t s = (cudaStream_t)stream;
  // launched through cudaLaunchKernel so that each launch's own error is the one returned (an
  // error left by an unrelated earlier call is not this call's)
  void* pargs[] = {&a, &partials};
  if (cudaLaunchKernel((const void*)k_energy_partials, dim3(nb), dim3(kThreads), pargs, 0, s) != cudaSuccess)
    return ABD_ERR_CUDA;
  void* fargs[] = {&partials, &nb, &E_dev};
  if (cudaLaunchKernel((const void*)k_energy_finish, dim3(1), dim3(1024), fargs, 0, s) != cudaSuccess)
    return ABD_ERR_CUDA;
  return ABD_OK;
}
