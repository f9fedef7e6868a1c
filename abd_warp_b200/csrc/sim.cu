// Host orchestration and the C ABI (include/abd_b200.h).
//
// abd_step follows AffineBodySimulator.step (abd/abd.py:212-276) with the corrections of the
// reference's defects: PT / EE lists used consistently in the energy and in CCD, the full
// coupled Hessian (diagonal + both off-diagonal blocks of every contacting body pair),
// capacity-checked lists that grow and rerun instead of writing out of bounds, and the
// Armijo sign selectable.  Device work is issued on one stream; the host synchronises only
// to read list counts, energies, the time of impact and the solver's convergence flags.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "abd_common.cuh"
#include "abd_graph.cuh"

namespace abd {
cudaError_t vg_list_swept(Sim& s, const double* y0, const double* y1);
}

struct abd_sim {
  abd::Sim s;
};

// Independent scenes stepped together: one CUDA graph holds every scene's device-loop step as
// a branch of its own (see abd_batch_step)
struct abd_batch {
  std::vector<abd_sim*> sims;
  cudaStream_t stream = nullptr;      // the stream the steps are launched on
  cudaStream_t cap = nullptr;         // captures the graph
  std::vector<cudaStream_t> branch;   // one per scene, for the capture
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t key = 0;
  std::vector<long long> top;         // kernels of each branch outside its loops
};

namespace abd {

namespace {
thread_local char g_error_detail[256] = "";
}

const char* error_detail() { return g_error_detail; }

cudaError_t note_error(cudaError_t e, const char* file, int line) {
  if (e != cudaSuccess) {
    const char* base = std::strrchr(file, '/');
    std::snprintf(g_error_detail, sizeof(g_error_detail), "%s:%d: %s: %s", base ? base + 1 : file, line,
                  cudaGetErrorName(e), cudaGetErrorString(e));
    (void)cudaGetLastError();  // the caller gets the error here; it must not reach later calls
  }
  return e;
}

}  // namespace abd

namespace {

using abd::Sim;

#define CK(x)                                       \
  do {                                              \
    if (ABD_NOTE(x) != cudaSuccess) return ABD_ERR_CUDA; \
  } while (0)

// The exact accumulator rounded to FP64 on the host (the same rounding as the device's).
double xs_round_host(const abd::XSum& x) {
  if (x.flags & (abd::XS_NAN | abd::XS_RANGE)) return std::nan("");
  if (x.flags & abd::XS_PINF) return (x.flags & abd::XS_NINF) ? std::nan("") : INFINITY;
  if (x.flags & abd::XS_NINF) return -INFINITY;
  long long d[abd::kXD + 1];
  for (int i = 0; i < abd::kXD; ++i) d[i] = x.d[i];
  d[abd::kXD] = 0;
  auto carry = [&]() {
    for (int i = 0; i < abd::kXD; ++i) {
      const long long c = d[i] >> 32;
      d[i] -= c * 4294967296LL;
      d[i + 1] += c;
    }
  };
  carry();
  const bool neg = d[abd::kXD] < 0;
  if (neg) {
    for (int i = 0; i <= abd::kXD; ++i) d[i] = -d[i];
    carry();
  }
  int h = -1;
  for (int i = 0; i <= abd::kXD; ++i)
    if (d[i] != 0) h = i;
  if (h < 0) return 0.0;
  const unsigned long long t2 = (unsigned long long)d[h], t1 = h >= 1 ? (unsigned long long)d[h - 1] : 0ULL,
                           t0 = h >= 2 ? (unsigned long long)d[h - 2] : 0ULL;
  bool sticky = false;
  for (int i = 0; i < h - 2; ++i) sticky = sticky || d[i] != 0;
  const unsigned __int128 w = ((unsigned __int128)t2 << 64) | ((unsigned __int128)t1 << 32) | t0;
  const int msb = 127 - __builtin_clzll(t2);
  const int drop = msb - 52;
  unsigned long long mant = (unsigned long long)(w >> drop);
  const unsigned __int128 rem = w & ((((unsigned __int128)1) << drop) - 1);
  const unsigned __int128 half = ((unsigned __int128)1) << (drop - 1);
  if (rem > half || (rem == half && (sticky || (mant & 1ULL)))) ++mant;
  const double r = std::ldexp((double)mant, drop + 32 * (h - 2) + abd::kXB0);
  return neg ? -r : r;
}

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count > 0 ? count : 1));
}

template <class T>
cudaError_t upload(T** p, const T* host, size_t count, cudaStream_t st) {
  cudaError_t e = dalloc(p, count);
  if (e != cudaSuccess || count == 0) return e;
  return cudaMemcpyAsync(*p, host, sizeof(T) * count, cudaMemcpyHostToDevice, st);
}

void free_tree(abd::Tree& t) {
  for (void* q : {(void*)t.child, (void*)t.parent, (void*)t.leaf_prim, (void*)t.prim_leaf, (void*)t.body_root,
                  (void*)t.rest, (void*)t.box, (void*)t.order, (void*)t.lvl, (void*)t.body_lvl, (void*)t.crest,
                  (void*)t.ccode})
    if (q) cudaFree(q);
  t = abd::Tree{};
}

int grow_pairs(Sim& s, int need) {
  ++s.cap_gen;  // every captured pass is keyed on it
  const int cap = std::max(need + need / 2, 2 * s.cap_pairs);
  const int cap_adj = 2 * cap;
  for (void* q : {(void*)s.ij, (void*)s.adj_col, (void*)s.adj_pair, (void*)s.pair_cand, (void*)s.offdiag,
                  (void*)s.pdiag, (void*)s.pgrad, (void*)s.pair_active, (void*)s.pair_val})
    if (q) cudaFree(q);
  s.cap_pairs = cap;
  s.cap_adj = cap_adj;
  if (dalloc(&s.ij, cap) || dalloc(&s.adj_col, cap_adj) || dalloc(&s.adj_pair, cap_adj) ||
      dalloc(&s.pair_cand, 4 * (size_t)cap) || dalloc(&s.offdiag, 288 * (size_t)cap) ||
      dalloc(&s.pdiag, 288 * (size_t)cap) || dalloc(&s.pgrad, 24 * (size_t)cap) || dalloc(&s.pair_active, cap) ||
      dalloc(&s.pair_val, cap))
    return ABD_ERR_OVERFLOW;
  // zeroed so that the body ids of a pass that overflowed are still valid indices
  if (cudaMemsetAsync(s.ij, 0, sizeof(int2) * cap, s.stream) ||
      cudaMemsetAsync(s.adj_col, 0, sizeof(int) * cap_adj, s.stream) ||
      cudaMemsetAsync(s.adj_pair, 0, sizeof(int) * cap_adj, s.stream))
    return ABD_ERR_CUDA;
  return ABD_OK;
}

int grow_contacts(Sim& s, int need) {
  ++s.cap_gen;  // every captured pass is keyed on it
  if (need <= s.cap_contacts) return ABD_OK;
  if (s.contacts) cudaFree(s.contacts);
  if (s.contacts_by_pair) cudaFree(s.contacts_by_pair);
  s.contacts = s.contacts_by_pair = nullptr;
  s.cap_contacts = std::max(need + need / 2, 2 * s.cap_contacts);
  if (dalloc(&s.contacts, s.cap_contacts) || dalloc(&s.contacts_by_pair, s.cap_contacts)) return ABD_ERR_OVERFLOW;
  return ABD_OK;
}

int grow_fric(Sim& s, int need) {
  ++s.cap_gen;  // every captured pass is keyed on it
  if (need <= s.cap_fric) return ABD_OK;
  if (s.fric) cudaFree(s.fric);
  s.fric = nullptr;
  s.cap_fric = std::max(need + need / 2, 2 * s.cap_fric);
  if (dalloc(&s.fric, s.cap_fric)) return ABD_ERR_OVERFLOW;
  return ABD_OK;
}

int grow_ccd(Sim& s, int need) {
  ++s.cap_gen;  // every captured pass is keyed on it
  if (need <= s.cap_ccd) return ABD_OK;
  if (s.ccd_cand) cudaFree(s.ccd_cand);
  s.ccd_cand = nullptr;
  s.cap_ccd = std::max(need + need / 2, 2 * s.cap_ccd);
  if (dalloc(&s.ccd_cand, s.cap_ccd)) return ABD_ERR_OVERFLOW;
  return ABD_OK;
}

int grow_ecand(Sim& s, int need) {
  ++s.cap_gen;  // every captured pass is keyed on it
  if (need <= s.cap_ecand) return ABD_OK;
  if (s.ecand) cudaFree(s.ecand);
  s.ecand = nullptr;
  s.cap_ecand = std::max(need + need / 2, 2 * s.cap_ecand);
  if (dalloc(&s.ecand, s.cap_ecand)) return ABD_ERR_OVERFLOW;
  return ABD_OK;
}

int grow_act(Sim& s, int need) {
  ++s.cap_gen;  // every captured pass is keyed on it
  if (need <= s.cap_act) return ABD_OK;
  if (s.act_pairs) cudaFree(s.act_pairs);
  s.act_pairs = nullptr;
  s.cap_act = std::max(need + need / 2, 2 * s.cap_act);
  if (dalloc(&s.act_pairs, s.cap_act)) return ABD_ERR_OVERFLOW;
  return ABD_OK;
}

int grow_lists(Sim& s, int need_pt, int need_ee) {
  ++s.cap_gen;  // every captured pass is keyed on it
  if (need_pt > s.cap_pt) {
    cudaFree(s.pt_list);
    s.cap_pt = std::max(need_pt + need_pt / 2, 2 * s.cap_pt);
    if (dalloc(&s.pt_list, 5 * (size_t)s.cap_pt)) return ABD_ERR_OVERFLOW;
  }
  if (need_ee > s.cap_ee) {
    cudaFree(s.ee_list);
    s.cap_ee = std::max(need_ee + need_ee / 2, 2 * s.cap_ee);
    if (dalloc(&s.ee_list, 5 * (size_t)s.cap_ee)) return ABD_ERR_OVERFLOW;
  }
  return ABD_OK;
}

// Boxes, body pairs and the narrow pass of `mode` on positions y0 (static) or y0 -> y1
// (swept), all asynchronous: counts and overflow bits stay in the mailbox until the caller's
// next read (sync_read), after which overflow() grows what was short and asks for a rerun.
// d0 != null: y0 (and y1 when d1 != null) are computed from the DOFs by the broad phase;
// otherwise y0 / y1 are given positions.
int culling(abd_sim* h, const abd::Dofs* d0, const abd::Dofs* d1, double* y0, double* y1, int mode,
            const abd_states* st = nullptr) {
  Sim& s = h->s;
  if (d0) CK(abd::body_broad(s, d0, d1, y0, y1));
  else CK(abd::body_broad(s, nullptr, nullptr, nullptr, nullptr, y0, y1));
  const bool full = mode == abd::NARROW_GH || mode == abd::NARROW_LISTS;
  // the GH pass's pairs also hold the body pairs of the step's lagged friction contacts
  const uint32_t* forced = mode == abd::NARROW_GH && s.prm.friction_mu > 0.0 ? s.fric_mask : nullptr;
  CK(abd::body_pairs(s, full, mode == abd::NARROW_CCD_LS, forced,
                     mode == abd::NARROW_CCD || mode == abd::NARROW_CCD_LS));
  CK(abd::narrow(s, mode, d0 ? d0->Aeff() : nullptr, d0 ? d0->peff() : nullptr, d1 ? d1->Aeff() : nullptr,
                 d1 ? d1->peff() : nullptr, y0, y1, st));
  return ABD_OK;
}

abd::Dofs direct(const double* A, const double* p) {
  abd::Dofs d;
  d.A = A;
  d.p = p;
  return d;
}

// (A, p) - alpha dq into (Aout, pout), alpha = s.dpar[slot] on the device
abd::Dofs updated(Sim& s, const double* A, const double* p, int slot, double* Aout, double* pout) {
  abd::Dofs d;
  d.A = A;
  d.p = p;
  d.dq = s.dq;
  d.alpha = s.dpar + slot;
  d.Aout = Aout;
  d.pout = pout;
  return d;
}

// One synchronisation: the mailbox (status, counters, energy, time of impact, dots).
// Updates the host mirror and pair counts.
int sync_read(Sim& s) {
  CK(cudaMemcpyAsync(s.hbox, s.box, sizeof(abd::Mailbox), cudaMemcpyDeviceToHost, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  std::memcpy(s.hstat, s.hbox->dstat, sizeof(int) * abd::DS_NSLOTS);
  s.n_pairs = s.hstat[abd::DS_NPAIRS];
  s.n_adj = s.hstat[abd::DS_NADJ];
  return ABD_OK;
}

constexpr int kRerun = -1;

// After sync_read: grow every capacity whose overflow bit is set and clear those bits.
// Returns kRerun when the pass has to be rerun, 0 when it is complete, or an ABD error.
int overflow(Sim& s) {
  const int bits = s.hstat[abd::DS_STATUS];
  const int mask = abd::ST_PAIR_OVERFLOW | abd::ST_PT_OVERFLOW | abd::ST_EE_OVERFLOW | abd::ST_VG_OVERFLOW |
                   abd::ST_ACT_OVERFLOW | abd::ST_CONTACT_OVERFLOW | abd::ST_CCD_OVERFLOW |
                   abd::ST_ECAND_OVERFLOW | abd::ST_FRIC_OVERFLOW;
  if (!(bits & mask)) return 0;
  int r = ABD_OK;
  if (bits & abd::ST_PAIR_OVERFLOW) r = grow_pairs(s, std::max(s.n_pairs, s.n_adj / 2 + 1));
  else if (bits & (abd::ST_PT_OVERFLOW | abd::ST_EE_OVERFLOW))
    r = grow_lists(s, s.hstat[abd::DS_PT_COUNT], s.hstat[abd::DS_EE_COUNT]);
  if (!r && (bits & abd::ST_VG_OVERFLOW) && s.hstat[abd::DS_VG_COUNT] > s.cap_vg) {
    cudaFree(s.vg_list);
    s.vg_list = nullptr;
    ++s.cap_gen;
    s.cap_vg = 2 * s.hstat[abd::DS_VG_COUNT];
    if (dalloc(&s.vg_list, 2 * (size_t)s.cap_vg)) r = ABD_ERR_OVERFLOW;
  }
  if (!r && (bits & abd::ST_ACT_OVERFLOW)) r = grow_act(s, s.hstat[abd::DS_NACTP]);
  if (!r && (bits & abd::ST_CONTACT_OVERFLOW)) r = grow_contacts(s, s.hstat[abd::DS_NCONTACT]);
  if (!r && (bits & abd::ST_CCD_OVERFLOW)) r = grow_ccd(s, s.hstat[abd::DS_NCCD]);
  if (!r && (bits & abd::ST_ECAND_OVERFLOW)) r = grow_ecand(s, s.hstat[abd::DS_NECAND]);
  if (!r && (bits & abd::ST_FRIC_OVERFLOW)) r = grow_fric(s, s.hstat[abd::DS_NFRIC]);
  if (r) return r;
  const int clear = bits & ~mask;
  s.hstat[abd::DS_STATUS] = clear;
  CK(cudaMemcpyAsync(s.dstat + abd::DS_STATUS, &s.hstat[abd::DS_STATUS], sizeof(int), cudaMemcpyHostToDevice,
                     s.stream));
  CK(cudaStreamSynchronize(s.stream));
  return kRerun;
}

constexpr int kMaxReruns = 6;       // per pass of the host loop
constexpr int kMaxStepReruns = 48;  // per step of the device loop

uint64_t states_key(const Sim& s, const abd_states& st) {
  abd::KeyHash k;
  k.add(st.A).add(st.p).add(st.Ak).add(st.pk).add(st.A0).add(st.p0).add(st.Adot).add(st.pdot);
  k.add(s.prm_version).add(s.dq).add(s.x).add(s.xk).add(s.box).add(s.cap_gen);
  return k.h;
}

// E at the DOFs d: barrier over the culling lists + inertia (compute_energy, abd.py:133-141),
// summed exactly on the device and rounded here.  The energy pass has no capacities.
// g: replay slot for the step's trials (the DOFs then depend only on device data).
int energy_of(abd_sim* h, const abd_states& st, const abd::Dofs& d, double* E, abd::GraphSlot* g = nullptr,
              uint64_t key = 0) {
  Sim& s = h->s;
  auto issue = [&]() -> int {
    if (d.dq && cudaMemcpyAsync(s.dpar, s.hpar, sizeof(double), cudaMemcpyHostToDevice, s.stream)) return ABD_ERR_CUDA;
    int r = culling(h, &d, nullptr, s.xk, nullptr, abd::NARROW_ENERGY, &st);
    if (r) return r;
    CK(cudaMemcpyAsync(s.hbox, s.box, sizeof(abd::Mailbox), cudaMemcpyDeviceToHost, s.stream));
    return ABD_OK;
  };
  s.prof_events = 0;
  abd::KeyHash k;
  k.add(key);
  int r = g ? abd::run_graph(s, *g, k.h, issue) : issue();
  if (r) return r;
  CK(cudaStreamSynchronize(s.stream));
  std::memcpy(s.hstat, s.hbox->dstat, sizeof(int) * abd::DS_NSLOTS);
  *E = xs_round_host(s.hbox->energy);
  return ABD_OK;
}

int energy_at(abd_sim* h, const abd_states& st, const double* Ak, const double* pk, double* E) {
  return energy_of(h, st, direct(Ak, pk), E);
}


int no_post() { return ABD_OK; }

// CCD bound between DOFs d0 and d1 (ccd, abd.py:278-303); positions land in x, xk.  pre()
// enqueues work that belongs to the same pass (the step's dot products, whose results ride
// along in the mailbox), possibly on a branch it forks (s.fork_open), joined before the
// mailbox copy; post() enqueues work that follows it before the host's wait (the
// step's first line-search batch).  mode NARROW_CCD_LS also collects the line-search
// candidates between d0 and d1.
// The kernels of a CCD pass (no copy to the host); pre() as in ccd_of
template <class Pre>
int ccd_issue(abd_sim* h, const abd::Dofs& d0, const abd::Dofs& d1, int mode, Pre&& pre) {
  Sim& s = h->s;
  s.fork_open = false;
  int r = pre();
  if (r) return r;
  if ((r = culling(h, &d0, &d1, s.x, s.xk, mode))) return r;
  if (s.fork_open) {  // join the branch pre() forked
    CK(cudaStreamWaitEvent(s.stream, s.fork_ev[1], 0));
    s.fork_open = false;
  }
  return ABD_OK;
}

template <class Pre, class Post = int (*)()>
int ccd_of(abd_sim* h, const abd::Dofs& d0, const abd::Dofs& d1, double* alpha, double* raw, Pre&& pre,
           abd::GraphSlot* g = nullptr, uint64_t key = 0, int mode = abd::NARROW_CCD, Post&& post = no_post) {
  Sim& s = h->s;
  auto issue = [&]() -> int {
    if (int r = ccd_issue(h, d0, d1, mode, pre)) return r;
    CK(cudaMemcpyAsync(s.hbox, s.box, sizeof(abd::Mailbox), cudaMemcpyDeviceToHost, s.stream));
    return ABD_OK;
  };
  // kernel profiling of the line-search candidate pass's narrow kernel: events around it on
  // every kProfEvery-th pass of the step (mode 1; their graph nodes cost a few microseconds)
  // or on every pass (mode 2, which also counts its bytes)
  constexpr int kProfEvery = 4;
  const bool ls = mode == abd::NARROW_CCD_LS;
  s.prof_events = ls && (s.prof_on == 2 || (s.prof_on == 1 && (!g || s.prof_tick++ % kProfEvery == 0)));
  if (g && s.prof_events) g = &s.g_ccd_ev;
  for (int tries = 0;; ++tries) {  // the candidate lists have capacities: grow and rerun
    abd::KeyHash k;
    k.add(key).add(s.cap_ccd).add(s.ccd_cand).add(mode).add(s.cap_ecand).add(s.ecand).add(s.prof_on).add(s.prof_events);
    int r = g ? abd::run_graph(s, *g, k.h, issue) : issue();
    if (r || (r = post())) return r;
    CK(cudaStreamSynchronize(s.stream));
    std::memcpy(s.hstat, s.hbox->dstat, sizeof(int) * abd::DS_NSLOTS);
    if ((r = overflow(s)) > 0) return r;
    if (r == 0) break;
    if (tries >= kMaxReruns) return ABD_ERR_OVERFLOW;
  }
  if (s.prof_events) {  // the narrow kernel's duration and the data it moved
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, s.prof_ev[0], s.prof_ev[1]));
    s.prof_ms += ms;
    ++s.prof_launches;
    if (s.prof_on == 2)
      for (int row = 0; row < 32; ++row)
        for (int c = 0; c < abd::PF_N; ++c) s.prof_bytes += abd::kProfBytes[c] * (double)s.hbox->prof[row][c];
    s.prof_events = 0;
  }
  double toi = 1.0;
  if (const unsigned long long key2 = s.hbox->toi_key) {
    const unsigned long long bits = ~key2;
    std::memcpy(&toi, &bits, sizeof(toi));
  }
  if (raw) *raw = toi;
  double t = std::max(0.0, std::min(1.0, toi));
  if (t < 1.0) t *= 0.9;
  *alpha = t;
  return ABD_OK;
}

int ccd_at(abd_sim* h, const double* A, const double* p, const double* A1, const double* p1, double* alpha,
           double* raw) {
  return ccd_of(h, direct(A, p), direct(A1, p1), alpha, raw, []() -> int { return ABD_OK; });
}

// Enqueues the energies at (A, p) - al[k] dq, k < K <= kLsMax, 0 <= al[k] <= 1, from the
// candidates of the last CCD_LS pass between (A, p) and (A, p) - dq, with the mailbox copy: one
// replayed pass.  al == null: the step lengths follow from that pass's time of impact on the
// device (k_ls_eval derives them).  Each energy is bitwise the energy pass's at the same DOFs.
int ls_launch(abd_sim* h, const abd_states& st, const double* A, const double* p, const double* al, int K,
              uint64_t key) {
  Sim& s = h->s;
  if (al && (K < 1 || K > abd::kLsMax)) return ABD_ERR_INVALID;
  if (al) {
    s.hpar[abd::kParK] = K;
    for (int k = 0; k < abd::kLsMax; ++k) s.hpar[abd::kParAlpha + k] = k < K ? al[k] : 0.0;
  }
  auto issue = [&]() -> int {
    if (al)
      CK(cudaMemcpyAsync(s.dpar + abd::kParK, s.hpar + abd::kParK, sizeof(double) * (1 + abd::kLsMax),
                         cudaMemcpyHostToDevice, s.stream));
    CK(abd::ls_energies(s, st, A, p, !al));
    CK(cudaMemcpyAsync(s.hbox, s.box, sizeof(abd::Mailbox), cudaMemcpyDeviceToHost, s.stream));
    return ABD_OK;
  };
  abd::KeyHash kh;
  kh.add(key).add(A).add(p).add(s.cap_ecand).add(s.ecand);
  return abd::run_graph(s, al ? s.g_ls : s.g_ls_dev, kh.h, issue);
}

// The trial step lengths of a line search from the bound alpha: alpha, alpha / 2, ... up to
// the first below alpha_min, at most kLsMax (the device's k_ls_eval makes the same list)
int trial_steps(double alpha, double alpha_min, double* al) {
  int K = 0;
  for (double a_ = alpha; K < abd::kLsMax;) {
    al[K++] = a_;
    if (a_ < alpha_min) break;
    a_ *= 0.5;
  }
  return K;
}

// ls_launch with the host's wait; the energies land in E[0, K)
int ls_batch(abd_sim* h, const abd_states& st, const double* A, const double* p, const double* al, int K,
             double* E, uint64_t key) {
  Sim& s = h->s;
  int r = ls_launch(h, st, A, p, al, K, key);
  if (r) return r;
  CK(cudaStreamSynchronize(s.stream));
  std::memcpy(s.hstat, s.hbox->dstat, sizeof(int) * abd::DS_NSLOTS);
  for (int k = 0; k < K; ++k) E[k] = xs_round_host(s.hbox->ls_energy[k]);
  return ABD_OK;
}

// Gradient and Hessian blocks at (A, p), and the preconditioner's clusters: the pass forks
// after the pair assembly and forms the clusters from its active-pair list on a side branch
// while the body terms run (both on the device).
// g: replay slot for the step (its key covers every capacity the captured grids depend on).
// sup_mode (gh_superset_check): 0 the traversal finds the candidates; 1 the step's first GH
// pass, which takes them from the kept line-search candidates when the step starts where the
// last one ended; 2 a later Newton iteration's GH pass, which always does.
// The kernels of a GH pass (no copy to the host)
// The step's lagged friction contacts start empty (the first GH pass of a step fixes them)
int clear_friction(Sim& s) {
  if (!(s.prm.friction_mu > 0.0)) return ABD_OK;
  CK(cudaMemsetAsync(s.fric_mask, 0, sizeof(uint32_t) * (size_t)s.n * s.W, s.stream));
  CK(cudaMemsetAsync(s.dstat + abd::DS_NFRIC, 0, sizeof(int), s.stream));
  return ABD_OK;
}

int gh_issue(abd_sim* h, const abd_states& st, const double* A, const double* p, int sup_mode) {
  Sim& s = h->s;
  const abd::Dofs d = direct(A, p);
  if (s.fric_lag)  // the host loop's first GH pass of a step (a rerun of it starts over)
    if (int r = clear_friction(s)) return r;
  CK(abd::gh_superset_check(s, &st, sup_mode));
  int r = culling(h, &d, nullptr, s.x, nullptr, abd::NARROW_GH);
  if (r) return r;
  const cudaStream_t side = s.side ? s.side : s.cap_stream2;
  CK(cudaEventRecord(s.fork_ev[0], s.stream));
  CK(cudaStreamWaitEvent(side, s.fork_ev[0], 0));
  CK(abd::cluster_tables(s, side));
  CK(cudaEventRecord(s.fork_ev[1], side));
  CK(abd::body_gh(s, st, A, p, s.x));
  CK(cudaStreamWaitEvent(s.stream, s.fork_ev[1], 0));
  return ABD_OK;
}

int gh_of(abd_sim* h, const abd_states& st, const double* A, const double* p, int* n_active,
          abd::GraphSlot* g = nullptr, bool with_energy = false, int sup_mode = 0) {
  Sim& s = h->s;
  s.gh_energy = with_energy ? 1 : 0;  // read by the kernel arguments of this pass
  auto issue = [&]() -> int {
    if (int r = gh_issue(h, st, A, p, sup_mode)) return r;
    CK(cudaMemcpyAsync(s.hbox, s.box, sizeof(abd::Mailbox), cudaMemcpyDeviceToHost, s.stream));
    return ABD_OK;
  };
  for (int tries = 0;; ++tries) {
    int r;
    if (g) {
      abd::KeyHash k;
      k.add(states_key(s, st)).add(A).add(p).add(s.cap_pairs).add(s.cap_adj).add(s.cap_contacts).add(s.cap_act);
      k.add(s.ij).add(s.adj_col).add(s.adj_pair).add(s.contacts).add(s.contacts_by_pair).add(s.act_pairs);
      k.add(s.pair_cand).add(s.offdiag).add(s.pdiag).add(s.pgrad).add(s.pair_active);
      k.add(s.cap_ccd).add(s.ccd_cand).add(s.gh_energy).add(sup_mode).add(s.q_last).add(s.dint);
      k.add(s.cap_ecand).add(s.ecand);  // k_gh_scan reads the kept line-search candidates
      k.add(s.fric_lag);                 // the pass that fixes the step's friction contacts
      r = abd::run_graph(s, *g, k.h, issue);
    } else {
      r = issue();
    }
    if (r) return r;
    CK(cudaStreamSynchronize(s.stream));
    std::memcpy(s.hstat, s.hbox->dstat, sizeof(int) * abd::DS_NSLOTS);
    s.n_pairs = s.hstat[abd::DS_NPAIRS];
    s.n_adj = s.hstat[abd::DS_NADJ];
    if ((r = overflow(s)) > 0) return r;
    if (r == 0) break;
    if (tries >= kMaxReruns) return ABD_ERR_OVERFLOW;
  }
  if (n_active) *n_active = s.hstat[abd::DS_ACTIVE];
  return ABD_OK;
}

int gh_at(abd_sim* h, const abd_states& st, const double* A, const double* p, int* n_active) {
  return gh_of(h, st, A, p, n_active);
}

int take_status(abd_sim* h) {
  Sim& s = h->s;
  int bits = 0;
  if (cudaMemcpyAsync(s.hstat + 21, s.dstat + abd::DS_STATUS, sizeof(int), cudaMemcpyDeviceToHost, s.stream) ==
          cudaSuccess &&
      cudaStreamSynchronize(s.stream) == cudaSuccess)
    bits = s.hstat[21];
  cudaMemsetAsync(s.dstat + abd::DS_STATUS, 0, sizeof(int), s.stream);
  bits |= s.host_status;
  s.host_status = 0;
  return bits;
}

}  // namespace

extern "C" {

const char* abd_error_detail(void) { return abd::error_detail(); }

const char* abd_status_string(int code) {
  switch (code) {
    case ABD_OK: return "ok";
    case ABD_ERR_CUDA: return "CUDA runtime error";
    case ABD_ERR_INVALID: return "invalid argument";
    case ABD_ERR_OVERFLOW: return "capacity could not be grown";
    case ABD_ERR_DEVICE: return "device-side error";
    default: return "unknown status";
  }
}

// parameters the library refuses: mixed precision, negative capacities, friction without the
// full contact model or with a negative coefficient or a non-positive slip velocity
static bool bad_params(const abd_params* prm) {
  return prm->precision != 0 || prm->min_capacity < 0 || !(prm->friction_mu >= 0.0) ||
         (prm->friction_mu > 0.0 && (!prm->ipc_full || !(prm->friction_epsv > 0.0)));
}

int abd_sim_create(const abd_scene_desc* d, const abd_params* prm, void* stream, abd_sim** out) {
  if (!d || !prm || !out || d->n_bodies <= 0 || !d->vert_off || !d->tri_off || !d->edge_off || !d->x0 ||
      !d->tris || !d->edges || !d->mass || !d->I0 || !d->fixed || bad_params(prm))
    return ABD_ERR_INVALID;
  const int n = d->n_bodies;
  const int V = d->vert_off[n], T = d->tri_off[n], E = d->edge_off[n];
  if (V <= 0 || T < 0 || E < 0) return ABD_ERR_INVALID;
  if (d->vert_off[0] != 0 || d->tri_off[0] != 0 || d->edge_off[0] != 0) return ABD_ERR_INVALID;
  // every body needs a vertex: a body without one would get a point box at the origin that
  // the broad phase pairs against its neighbours
  for (int b = 0; b < n; ++b)
    if (d->vert_off[b + 1] <= d->vert_off[b] || d->tri_off[b + 1] < d->tri_off[b] ||
        d->edge_off[b + 1] < d->edge_off[b])
      return ABD_ERR_INVALID;
  // free bodies need a positive, finite mass and I0; rest positions must be finite
  for (int b = 0; b < n; ++b)
    if (!d->fixed[b] && !(d->mass[b] > 0.0 && d->I0[b] > 0.0 && std::isfinite(d->mass[b]) && std::isfinite(d->I0[b])))
      return ABD_ERR_INVALID;
  for (long k = 0; k < 3L * V; ++k)
    if (!std::isfinite(d->x0[k])) return ABD_ERR_INVALID;
  std::vector<int> vbody(V), tbody(T), ebody(E);
  int max_v = 0, max_t = 0, max_e = 0;
  for (int b = 0; b < n; ++b) {
    max_v = std::max(max_v, d->vert_off[b + 1] - d->vert_off[b]);
    max_t = std::max(max_t, d->tri_off[b + 1] - d->tri_off[b]);
    max_e = std::max(max_e, d->edge_off[b + 1] - d->edge_off[b]);
  }
  for (int b = 0; b < n; ++b) {
    for (int v = d->vert_off[b]; v < d->vert_off[b + 1]; ++v) vbody[v] = b;
    for (int t = d->tri_off[b]; t < d->tri_off[b + 1]; ++t) {
      tbody[t] = b;
      for (int k = 0; k < 3; ++k) {
        const int v = d->tris[3 * t + k];
        if (v < d->vert_off[b] || v >= d->vert_off[b + 1]) return ABD_ERR_INVALID;
      }
    }
    for (int e = d->edge_off[b]; e < d->edge_off[b + 1]; ++e) {
      ebody[e] = b;
      for (int k = 0; k < 2; ++k) {
        const int v = d->edges[2 * e + k];
        if (v < d->vert_off[b] || v >= d->vert_off[b + 1]) return ABD_ERR_INVALID;
      }
    }
  }
  abd_sim* h = new (std::nothrow) abd_sim();
  if (!h) return ABD_ERR_OVERFLOW;
  Sim& s = h->s;
  s.stream = (cudaStream_t)stream;
  s.prm = *prm;
  s.n = n;
  s.V = V;
  s.T = T;
  s.E = E;
  s.max_body_v = max_v;
  s.max_body_t = max_t;
  s.max_body_e = max_e;
  // rest-space centroids for the Morton keys
  std::vector<double> tc(3 * (size_t)T), ec(3 * (size_t)E);
  for (int t = 0; t < T; ++t)
    for (int k = 0; k < 3; ++k)
      tc[3 * t + k] = (d->x0[3 * d->tris[3 * t] + k] + d->x0[3 * d->tris[3 * t + 1] + k] +
                       d->x0[3 * d->tris[3 * t + 2] + k]) /
                      3.0;
  for (int e = 0; e < E; ++e)
    for (int k = 0; k < 3; ++k) ec[3 * e + k] = 0.5 * (d->x0[3 * d->edges[2 * e] + k] + d->x0[3 * d->edges[2 * e + 1] + k]);
  double *tcd = nullptr, *ecd = nullptr;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
    return e == cudaSuccess;
  };
  ok(upload(&s.voff, d->vert_off, n + 1, s.stream));
  ok(upload(&s.toff, d->tri_off, n + 1, s.stream));
  ok(upload(&s.eoff, d->edge_off, n + 1, s.stream));
  ok(upload(&s.vbody, vbody.data(), V, s.stream));
  ok(upload(&s.tbody, tbody.data(), T, s.stream));
  ok(upload(&s.ebody, ebody.data(), E, s.stream));
  ok(upload(&s.tris, d->tris, 3 * (size_t)T, s.stream));
  ok(upload(&s.edges, d->edges, 2 * (size_t)E, s.stream));
  ok(upload(&s.x0, d->x0, 3 * (size_t)V, s.stream));
  ok(upload(&s.mass, d->mass, n, s.stream));
  ok(upload(&s.I0, d->I0, n, s.stream));
  ok(upload(&s.fixed, d->fixed, n, s.stream));
  ok(upload(&tcd, tc.data(), tc.size(), s.stream));
  ok(upload(&ecd, ec.data(), ec.size(), s.stream));
  if (e == cudaSuccess) ok(abd::build_tree(s, s.tri_tree, T, s.tbody, tcd, d->tri_off));
  if (e == cudaSuccess) ok(abd::build_tree(s, s.edge_tree, E, s.ebody, ecd, d->edge_off));
  // a depth-first walk pops one node and pushes at most four (the node's descendants one or
  // two levels down), so a subtree of H internal levels needs at most 3 ceil(H / 2) + 1
  // stack entries; a deeper tree (many primitives sharing a Morton code) is refused
  if (e == cudaSuccess) {
    const int H = std::max(s.tri_tree.max_height, s.edge_tree.max_height);
    if (3 * ((H + 1) / 2) + 1 > abd::kTraversalStack) {
      if (tcd) cudaFree(tcd);
      if (ecd) cudaFree(ecd);
      abd_sim_destroy(h);
      return ABD_ERR_INVALID;
    }
  }
  s.W = (n + 31) / 32;
  ok(dalloc(&s.x, 3 * (size_t)V));
  ok(dalloc(&s.xk, 3 * (size_t)V));
  ok(dalloc(&s.body_box, n));
  ok(dalloc(&s.body_bnd, 12 * (size_t)n));
  ok(dalloc(&s.pair_mask, (size_t)n * s.W));
  ok(dalloc(&s.pair_wpre, (size_t)n * s.W));
  {
    // Work chunks of the narrow passes: kChunk items of one body each, the body's points in
    // Morton order of their rest positions, then its edges in the edge tree's leaf order
    // (also Morton order), so that a chunk covers a compact patch of the surface.  Each
    // chunk's rest-frame box bounds its items; a chunk whose box, moved by the body's DOFs,
    // overlaps no neighbouring body skips its queries.
    std::vector<int> eleaf(E > 0 ? E : 1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);  // the trees are built
    if (e == cudaSuccess && E > 0)
      e = cudaMemcpy(eleaf.data(), s.edge_tree.leaf_prim, sizeof(int) * E, cudaMemcpyDeviceToHost);
    std::vector<int> vperm(V);
    for (int b = 0; b < n; ++b) {
      const int v0 = d->vert_off[b], v1 = d->vert_off[b + 1];
      double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int v = v0; v < v1; ++v)
        for (int k = 0; k < 3; ++k) {
          lo[k] = std::min(lo[k], d->x0[3 * v + k]);
          hi[k] = std::max(hi[k], d->x0[3 * v + k]);
        }
      std::vector<std::pair<unsigned, int>> key;
      for (int v = v0; v < v1; ++v) {
        unsigned c[3];
        for (int k = 0; k < 3; ++k) {
          const double ext = hi[k] - lo[k];
          const double u = ext > 0 ? (d->x0[3 * v + k] - lo[k]) / ext : 0.0;
          c[k] = (unsigned)std::min(1023.0, std::max(0.0, u * 1024.0));
        }
        unsigned m = 0;
        for (int bit = 9; bit >= 0; --bit)
          for (int k = 0; k < 3; ++k) m = (m << 1) | ((c[k] >> bit) & 1u);
        key.push_back({m, v});
      }
      std::sort(key.begin(), key.end());
      for (int i = 0; i < v1 - v0; ++i) vperm[v0 + i] = key[i].second;
    }
    std::vector<int2> ch;
    std::vector<abd::Box> cbox;
    for (int b = 0; b < n; ++b) {
      const int nv = d->vert_off[b + 1] - d->vert_off[b], ne = d->edge_off[b + 1] - d->edge_off[b];
      const int items = nv + ne;
      // every body has at least one chunk: its first chunk also adds the body's own terms
      for (int i0 = 0; i0 < std::max(items, 1); i0 += abd::kChunk) {
        ch.push_back(make_int2(b, i0));
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        auto add = [&](int v) {
          for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], d->x0[3 * v + k]);
            hi[k] = std::max(hi[k], d->x0[3 * v + k]);
          }
        };
        for (int i = i0; i < std::min(items, i0 + abd::kChunk); ++i) {
          if (i < nv) {
            add(vperm[d->vert_off[b] + i]);
          } else {
            const int eg = eleaf[d->edge_off[b] + (i - nv)];
            add(d->edges[2 * eg]);
            add(d->edges[2 * eg + 1]);
          }
        }
        abd::Box B{};
        for (int k = 0; k < 3; ++k) {  // rounded outward to FP32
          B.lo[k] = items ? std::nextafter((float)lo[k], -INFINITY) : 0.f;
          B.hi[k] = items ? std::nextafter((float)hi[k], INFINITY) : 0.f;
        }
        cbox.push_back(B);
      }
    }
    s.nch = (int)ch.size();
    // each body's rest box: the union of its chunks' boxes
    std::vector<abd::Box> brest(n);
    for (int b = 0; b < n; ++b)
      for (int k = 0; k < 3; ++k) {
        brest[b].lo[k] = INFINITY;
        brest[b].hi[k] = -INFINITY;
      }
    for (size_t c = 0; c < ch.size(); ++c) {
      abd::Box& B = brest[ch[c].x];
      for (int k = 0; k < 3; ++k) {
        B.lo[k] = std::min(B.lo[k], cbox[c].lo[k]);
        B.hi[k] = std::max(B.hi[k], cbox[c].hi[k]);
      }
    }
    ok(upload(&s.body_rest, brest.data(), brest.size(), s.stream));
    std::vector<int4> slices;
    for (int b = 0; b < n; ++b)
      for (int v = d->vert_off[b]; v < d->vert_off[b + 1]; v += abd::kSlice)
        slices.push_back(make_int4(b, v, std::min(abd::kSlice, d->vert_off[b + 1] - v), 0));
    s.nslice = (int)slices.size();
    ok(upload(&s.slice, slices.data(), slices.size(), s.stream));
    ok(upload(&s.chunk, ch.data(), ch.size(), s.stream));
    ok(dalloc(&s.chunk_act, ch.size() + 1));
    ok(dalloc(&s.fric_mask, (size_t)n * s.W));
    ok(cudaMemsetAsync(s.fric_mask, 0, sizeof(uint32_t) * (size_t)n * s.W, s.stream));
    ok(upload(&s.chunk_box, cbox.data(), cbox.size(), s.stream));
    ok(upload(&s.vperm, vperm.data(), vperm.size(), s.stream));
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);  // host temporaries
  }
  ok(dalloc(&s.row_ptr, n + 1));
  ok(dalloc(&s.upper_ptr, n + 1));
  for (double** v : {&s.g, &s.dq, &s.r, &s.rh, &s.pv, &s.v, &s.y, &s.s, &s.z, &s.t})
    ok(dalloc(v, 12 * (size_t)n));
  if (ok(cudaMalloc(&s.cl_tab, abd::cluster_tables_bytes(n)))) {
    const abd::ClusterTables t = abd::cluster_tables_at(s.cl_tab, n);
    s.cl_ptr = t.cl_ptr;
    s.cl_body = t.cl_body;
    s.body_cl = t.body_cl;
    s.ncl_dev = t.ncl;
    s.cl_off = t.cl_off;
  }
  ok(dalloc(&s.diag, 144 * (size_t)n));
  // the clustering kernel's scratch, and room for the inverses of any clustering: a cluster of
  // s bodies takes (12 s)^2 doubles, and the sum of s^2 over clusters is at most kMaxCluster n
  if (ok(cudaMalloc(&s.cl_work_buf, abd::cluster_work_bytes(n)))) s.cl_work = abd::cluster_work_at(s.cl_work_buf, n);
  ok(dalloc(&s.cl_inv, 144 * (size_t)abd::kMaxCluster * n));
  ok(dalloc(&s.partials, abd::kRedSlots * (size_t)abd::kRedBlocks));
  s.red_grid = std::max(1, std::min(abd::kRedBlocks, (n + 7) / 8));
  s.cl_grid = std::max(1, std::min(abd::kRedBlocks, (n + 3) / 4));
  ok(dalloc(&s.red_count, abd::kRedSlots));
  ok(dalloc(&s.scal, 32));

  ok(dalloc(&s.box, 1));
  if (e == cudaSuccess) {
    s.dstat = s.box->dstat;
    s.energy_acc = &s.box->energy;
    s.dmin = &s.box->toi_key;
  }
  ok(dalloc(&s.dpar, abd::kNPar));
  ok(dalloc(&s.body_sup, n));
  ok(dalloc(&s.dint, 4));
  ok(dalloc(&s.q_last, 12 * (size_t)n));
  ok(dalloc(&s.dq_save, 12 * (size_t)n));
  ok(dalloc(&s.adj_x, 12 * (size_t)n));
  ok(dalloc(&s.highlight, n));
  if (e == cudaSuccess) e = cudaMemsetAsync(s.highlight, 0, sizeof(int) * n, s.stream);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.cap_stream2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.cap_stream3, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.cap_stream4, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.fork_a, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.fork_b, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.cap_stream5, cudaStreamNonBlocking);
  for (cudaEvent_t* ev : {&s.fork_ev[0], &s.fork_ev[1]})
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
  ok(dalloc(&s.row_cnt, n));
  ok(dalloc(&s.nbr, (size_t)n * abd::kNbList));
  ok(dalloc(&s.fdof, 24 * (size_t)n));
  ok(dalloc(&s.upper_cnt, n));
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.hstat, 32 * sizeof(int), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.hbox, sizeof(abd::Mailbox), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.hpar, abd::kNPar * sizeof(double), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&s.hval, 32 * sizeof(double), cudaHostAllocDefault);
  if (e == cudaSuccess) e = abd::rest_boxes(s);
  if (e == cudaSuccess && abd::prepare_solver(s) != ABD_OK) e = cudaErrorUnknown;
  if (e == cudaSuccess) e = abd::prepare_narrow(s);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.dq, 0, sizeof(double) * 12 * n, s.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.box, 0, sizeof(abd::Mailbox), s.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.dint, 0, 4 * sizeof(int), s.stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.cl_tab, 0, sizeof(int), s.stream);
  if (e == cudaSuccess) {  // dpar = {trial step, 1 (the full step of the CCD bound), 0, ...}
    for (int k = 0; k < abd::kNPar; ++k) s.hpar[k] = 0.0;
    s.hpar[1] = 1.0;
    e = cudaMemcpyAsync(s.dpar, s.hpar, abd::kNPar * sizeof(double), cudaMemcpyHostToDevice, s.stream);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(s.red_count, 0, sizeof(int) * abd::kRedSlots, s.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
  if (tcd) cudaFree(tcd);
  if (ecd) cudaFree(ecd);
  if (e != cudaSuccess) {
    abd_sim_destroy(h);
    return ABD_ERR_CUDA;
  }
  // initial capacities; min_capacity > 0 replaces them all (host-injected shortfalls)
  const int mc = prm->min_capacity;
  auto cap0 = [mc](int dflt) { return mc > 0 ? mc : dflt; };
  s.cap_pairs = 0;
  int r = grow_pairs(s, cap0(std::max(256, 8 * n)));
  if (!r) r = grow_act(s, cap0(std::max(1024, n)));
  if (!r) r = grow_contacts(s, cap0(std::max(4096, 8 * n)));
  if (!r) r = grow_fric(s, cap0(std::max(1024, 2 * n)));
  if (!r) r = grow_ccd(s, cap0(std::max(1 << 15, 32 * n)));
  if (!r) r = grow_ecand(s, cap0(std::max(1 << 15, 32 * n)));
  s.cap_pt = 0;
  s.cap_ee = 0;
  if (!r) r = grow_lists(s, cap0(std::max(1 << 14, V / 4)), cap0(std::max(1 << 14, E / 4)));
  s.cap_vg = cap0(std::max(1024, V));
  if (!r && dalloc(&s.vg_list, 2 * (size_t)s.cap_vg)) r = ABD_ERR_OVERFLOW;
  if (r) {
    abd_sim_destroy(h);
    return r;
  }
  *out = h;
  return ABD_OK;
}

int abd_sim_destroy(abd_sim* h) {
  if (!h) return ABD_ERR_INVALID;
  Sim& s = h->s;
  cudaStreamSynchronize(s.stream);
  free_tree(s.tri_tree);
  free_tree(s.edge_tree);
  void* bufs[] = {s.voff, s.toff, s.eoff, s.vbody, s.tbody, s.ebody, s.tris, s.edges, s.x0, s.mass, s.I0,
                  s.fixed, s.x, s.xk, s.body_box, s.pair_mask, s.row_ptr, s.upper_ptr, s.ij, s.adj_col,
                  s.adj_pair, s.pt_list, s.ee_list, s.vg_list, s.pair_cand, s.offdiag, s.pdiag, s.pgrad,
                  s.pair_active, s.pair_val, s.g, s.dq, s.diag,
                  s.r, s.rh, s.pv, s.v, s.y, s.s, s.z, s.t, s.partials, s.scal, s.box, s.dpar, s.dint,
                  s.row_cnt, s.upper_cnt, s.nbr, s.fdof, s.chunk_box, s.vperm,
                  s.cl_tab, s.cl_inv, s.pair_wpre, s.act_pairs, s.chunk,
                  s.red_count, s.body_bnd, s.contacts, s.contacts_by_pair, s.ccd_cand, s.ecand, s.body_rest,
                  s.body_sup, s.slice, s.q_last, s.highlight, s.cl_work_buf, s.dq_save, s.adj_x,
                  s.chunk_act, s.fric, s.fric_mask};
  for (void* q : bufs)
    if (q) cudaFree(q);
  for (abd::GraphSlot* g : {&s.g_ccd, &s.g_ccd_ev, &s.g_gh, &s.g_gh0, &s.g_kinit, &s.g_ls, &s.g_ls_dev, &s.g_step, &s.g_kadj})
    if (g->exec) cudaGraphExecDestroy(g->exec);
  for (cudaStream_t q : {s.cap_stream, s.cap_stream2, s.cap_stream3, s.cap_stream4, s.cap_stream5, s.fork_a, s.fork_b})
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t ev : {s.prof_ev[0], s.prof_ev[1], s.fork_ev[0], s.fork_ev[1]})
    if (ev) cudaEventDestroy(ev);
  for (void* q : {(void*)s.hstat, (void*)s.hval, (void*)s.hbox, (void*)s.hpar})
    if (q) cudaFreeHost(q);
  delete h;
  return ABD_OK;
}

// The kept line-search candidates no longer hold the next step's first GH candidates (a pass
// replaced them, or the parameters or states changed under them).
static int drop_superset(abd_sim* h) {
  CK(cudaMemsetAsync(h->s.dint + abd::kSupHave, 0, sizeof(int), h->s.stream));
  return ABD_OK;
}

int abd_sim_set_params(abd_sim* h, const abd_params* prm) {
  if (!h || !prm || bad_params(prm)) return ABD_ERR_INVALID;
  if (int r = drop_superset(h)) return r;
  h->s.prm = *prm;
  ++h->s.prm_version;  // parameters are kernel arguments of the captured passes
  return ABD_OK;
}

int abd_sim_set_stream(abd_sim* h, void* stream) {
  if (!h) return ABD_ERR_INVALID;
  h->s.stream = (cudaStream_t)stream;
  return ABD_OK;
}

int abd_sim_reset(abd_sim* h) {
  if (!h) return ABD_ERR_INVALID;
  CK(cudaMemsetAsync(h->s.dq, 0, sizeof(double) * 12 * h->s.n, h->s.stream));
  return drop_superset(h);
}

static int copy_vec(abd_sim* h, double* dst, const double* src) {
  if (!h || !dst || !src) return ABD_ERR_INVALID;
  CK(cudaMemcpyAsync(dst, src, sizeof(double) * 12 * h->s.n, cudaMemcpyDeviceToDevice, h->s.stream));
  CK(cudaStreamSynchronize(h->s.stream));
  return ABD_OK;
}
int abd_sim_get_dq(abd_sim* h, double* dst) { return h ? copy_vec(h, dst, h->s.dq) : ABD_ERR_INVALID; }
int abd_sim_set_dq(abd_sim* h, const double* src) {
  return h ? copy_vec(h, h->s.dq, src) : ABD_ERR_INVALID;
}
int abd_sim_get_g(abd_sim* h, double* dst) { return h ? copy_vec(h, dst, h->s.g) : ABD_ERR_INVALID; }

int abd_sim_sizes(const abd_sim* h, int* n, int* V, int* T, int* E) {
  if (!h) return ABD_ERR_INVALID;
  if (n) *n = h->s.n;
  if (V) *V = h->s.V;
  if (T) *T = h->s.T;
  if (E) *E = h->s.E;
  return ABD_OK;
}

long long abd_launch_count(const abd_sim* h) { return h ? h->s.launches : 0; }

int abd_profile(abd_sim* h, int enable) {
  if (!h) return ABD_ERR_INVALID;
  Sim& s = h->s;
  if (enable && !s.prof_ev[0]) {
    CK(cudaEventCreate(&s.prof_ev[0]));
    CK(cudaEventCreate(&s.prof_ev[1]));
  }
  s.prof_on = enable == 2 ? 2 : (enable ? 1 : 0);
  s.prof_tick = 0;
  s.prof_ms = s.prof_bytes = 0.0;
  s.prof_launches = 0;
  return ABD_OK;
}

int abd_profile_read(const abd_sim* h, double* ms, long long* launches, double* bytes) {
  if (!h) return ABD_ERR_INVALID;
  if (ms) *ms = h->s.prof_ms;
  if (launches) *launches = h->s.prof_launches;
  if (bytes) *bytes = h->s.prof_bytes;
  return ABD_OK;
}

int abd_get_highlight(abd_sim* h, int* out) {
  if (!h || !out) return ABD_ERR_INVALID;
  Sim& s = h->s;
  CK(cudaMemcpyAsync(out, s.highlight, sizeof(int) * s.n, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  return ABD_OK;
}

int abd_take_status(abd_sim* h, int* status) {
  if (!h || !status) return ABD_ERR_INVALID;
  *status = take_status(h);
  return ABD_OK;
}

int abd_update_mesh_vertex(abd_sim* h, const double* A, const double* p, double* x) {
  if (!h || !A || !p || !x) return ABD_ERR_INVALID;
  CK(abd::transform(h->s, A, p, x));
  return ABD_OK;
}

}  // extern "C"

namespace {

// lists (culling in LISTS mode) plus the VG list; counts = {pairs, PT, EE, VG}
int cull_lists(abd_sim* h, const double* A, const double* p, const double* A1, const double* p1, double* y0,
               double* y1, int counts[4]) {
  Sim& s = h->s;
  const abd::Dofs d0 = direct(A, p), d1 = direct(A1, p1);
  for (int tries = 0;; ++tries) {
    int r = culling(h, A ? &d0 : nullptr, A && A1 ? &d1 : nullptr, y0, y1, abd::NARROW_LISTS);
    if (r) return r;
    CK(y1 ? abd::vg_list_swept(s, y0, y1) : abd::vg_list(s, y0));
    if ((r = sync_read(s))) return r;
    if ((r = overflow(s)) > 0) return r;
    if (r == 0) break;
    if (tries >= kMaxReruns) return ABD_ERR_OVERFLOW;
  }
  counts[0] = s.n_pairs;
  counts[1] = s.hstat[abd::DS_PT_COUNT];
  counts[2] = s.hstat[abd::DS_EE_COUNT];
  counts[3] = s.hstat[abd::DS_VG_COUNT];
  for (int k = 0; k < 4; ++k) s.list_counts[k] = counts[k];
  return ABD_OK;
}

}  // namespace

extern "C" {

int abd_collision_set(abd_sim* h, const double* y0, const double* y1, int counts[4]) {
  if (!h || !y0 || !counts) return ABD_ERR_INVALID;
  if (int r = drop_superset(h)) return r;
  return cull_lists(h, nullptr, nullptr, nullptr, nullptr, const_cast<double*>(y0), const_cast<double*>(y1), counts);
}

int abd_collision_set_dofs(abd_sim* h, const double* A, const double* p, const double* A1, const double* p1,
                           int counts[4]) {
  if (!h || !A || !p || !counts || (!A1) != (!p1)) return ABD_ERR_INVALID;
  if (int r = drop_superset(h)) return r;
  Sim& s = h->s;
  return cull_lists(h, A, p, A1, p1, s.x, A1 ? s.xk : nullptr, counts);
}

int abd_export_lists(abd_sim* h, int* ij, int* pt, int* ee, int* vg, int cap) {
  if (!h || cap < 0) return ABD_ERR_INVALID;
  Sim& s = h->s;
  const int npairs = s.list_counts[0], npt = s.list_counts[1], nee = s.list_counts[2], nvg = s.list_counts[3];
  if (ij) CK(cudaMemcpyAsync(ij, s.ij, sizeof(int2) * std::min(cap, npairs), cudaMemcpyDeviceToDevice, s.stream));
  if (pt) CK(cudaMemcpyAsync(pt, s.pt_list, sizeof(int) * 5 * std::min(cap, npt), cudaMemcpyDeviceToDevice, s.stream));
  if (ee) CK(cudaMemcpyAsync(ee, s.ee_list, sizeof(int) * 5 * std::min(cap, nee), cudaMemcpyDeviceToDevice, s.stream));
  if (vg) CK(cudaMemcpyAsync(vg, s.vg_list, sizeof(int) * 2 * std::min(cap, nvg), cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaStreamSynchronize(s.stream));
  return ABD_OK;
}

int abd_ipc_gh(abd_sim* h, const abd_states* st, const double* A, const double* p, int* n_active) {
  if (!h || !st || !A || !p) return ABD_ERR_INVALID;
  return gh_at(h, *st, A, p, n_active ? n_active : nullptr);
}

int abd_export_system(abd_sim* h, double* g, double* diag, double* off, int* ij, int cap, int* n_pairs) {
  if (!h) return ABD_ERR_INVALID;
  Sim& s = h->s;
  if (g) CK(cudaMemcpyAsync(g, s.g, sizeof(double) * 12 * s.n, cudaMemcpyDeviceToDevice, s.stream));
  if (diag) CK(cudaMemcpyAsync(diag, s.diag, sizeof(double) * 144 * s.n, cudaMemcpyDeviceToDevice, s.stream));
  if (off) CK(abd::export_system(s, off, ij, cap));
  CK(cudaStreamSynchronize(s.stream));
  if (n_pairs) *n_pairs = s.n_pairs;
  return ABD_OK;
}

int abd_solve(abd_sim* h, double* dq, int* iters) {
  if (!h || !dq) return ABD_ERR_INVALID;
  int r = abd::build_preconditioner(h->s);
  if (r) return r;
  int it = 0;
  r = abd::krylov_solve(h->s, dq, &it);  // waits for the solve
  if (iters) *iters = it;
  return r;
}

int abd_compute_energy(abd_sim* h, const abd_states* st, const double* Ak, const double* pk, double* E) {
  if (!h || !st || !Ak || !pk || !E) return ABD_ERR_INVALID;
  return energy_at(h, *st, Ak, pk, E);
}

int abd_ccd(abd_sim* h, const double* A, const double* p, const double* A1, const double* p1, double* alpha,
            double* raw) {
  if (!h || !A || !p || !A1 || !p1 || !alpha) return ABD_ERR_INVALID;
  if (int r = drop_superset(h)) return r;  // the CCD pass clears the candidate count
  return ccd_at(h, A, p, A1, p1, alpha, raw);
}

int abd_energies_along(abd_sim* h, const abd_states* st, const double* A, const double* p, const double* alphas,
                       int K, double* E) {
  if (!h || !st || !A || !p || !alphas || !E || K < 0 || !st->Ak || !st->pk) return ABD_ERR_INVALID;
  for (int k = 0; k < K; ++k)
    if (!(alphas[k] >= 0.0 && alphas[k] <= 1.0)) return ABD_ERR_INVALID;
  if (K == 0) return ABD_OK;
  if (int r = drop_superset(h)) return r;  // the pass replaces the kept candidates
  Sim& s = h->s;
  double a1 = 0.0, raw = 0.0;
  int r = ccd_of(h, direct(A, p), updated(s, A, p, 1, st->Ak, st->pk), &a1, &raw, []() -> int { return ABD_OK; },
                 nullptr, 0, abd::NARROW_CCD_LS);
  for (int k0 = 0; !r && k0 < K; k0 += abd::kLsMax)
    r = ls_batch(h, *st, A, p, alphas + k0, std::min(abd::kLsMax, K - k0), E + k0, states_key(s, *st));
  return r;
}

}  // extern "C"

namespace {

// The step with the Newton iterations driven from the host (newton_loop = 1, and the fallback
// of the device loop when a line search needs a second batch of trials).
int step_host(abd_sim* h, const abd_states* stp, double* x_view, abd_step_info* info) {
  Sim& s = h->s;
  const abd_states& st = *stp;
  const abd_params& P = s.prm;
  const size_t nA = sizeof(double) * 9 * s.n, np = sizeof(double) * 3 * s.n;
  // q <- q0 (abd.py:124-128)
  CK(cudaMemcpyAsync(st.A, st.A0, nA, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaMemcpyAsync(st.p, st.p0, np, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaMemcpyAsync(st.Ak, st.A0, nA, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaMemcpyAsync(st.pk, st.p0, np, cudaMemcpyDeviceToDevice, s.stream));
  abd_step_info inf{};
  int r;
  double E0 = 0.0;
  int it = 0;
  for (;;) {
    int nact = 0;
    // the step's first GH pass also gives the energy at q0 (its own replay slot); the GH
    // passes take their candidates from the last CCD pass's line-search candidates (which the
    // step's CCD passes then replace: the first pass's kept list is consumed)
    // (the pass also forms the preconditioner's clusters)
    s.fric_lag = it == 0 && s.prm.friction_mu > 0.0 ? 1 : 0;
    r = gh_of(h, st, st.A, st.p, &nact, it == 0 ? &s.g_gh0 : &s.g_gh, it == 0, it == 0 ? 1 : 2);
    s.fric_lag = 0;
    if (r)
      return r;
    if (it == 0) CK(cudaMemsetAsync(s.dint + abd::kSupHave, 0, sizeof(int), s.stream));
    if (it == 0) {
      // the energy at q0 (abd.py:126-128): the GH pass at q0 sums the same terms as an
      // energy pass there
      E0 = xs_round_host(s.hbox->energy);
      inf.n_pt = s.hstat[abd::DS_PT_COUNT];
      inf.n_ee = s.hstat[abd::DS_EE_COUNT];
      inf.n_vg = s.hstat[abd::DS_VG_COUNT];
      inf.n_ij = s.n_pairs;
    }
    inf.n_active = nact;
    if ((r = abd::cluster_inverse(s))) return r;
    if ((r = abd::krylov_solve(s, s.dq, nullptr))) return r;  // outcome read with the CCD pass
    // dq.g, g.g (abd.py:148, 265) and the CCD bound between q and q - dq (abd.py:278-303),
    // one pass; Ak, pk = q - dq
    double alpha;
    // (on a branch of their own beside the pass's culling, which neither reads g nor writes
    // what they write)
    auto dots = [&]() -> int {
      CK(cudaEventRecord(s.fork_ev[0], s.stream));
      CK(cudaStreamWaitEvent(s.cap_stream2, s.fork_ev[0], 0));
      CK(abd::dots(s, s.dq, s.g, s.g, s.g, s.box->dots, s.cap_stream2));
      CK(cudaEventRecord(s.fork_ev[1], s.cap_stream2));
      s.fork_open = true;
      return ABD_OK;
    };
    // the CCD pass and the line search's first batch (its step lengths from the pass's time of
    // impact, on the device) before one wait
    const uint64_t skey = states_key(s, st);
    auto first_batch = [&]() -> int { return ls_launch(h, st, st.A, st.p, nullptr, 0, skey); };
    if ((r = ccd_of(h, direct(st.A, st.p), updated(s, st.A, st.p, 1, st.Ak, st.pk), &alpha, &inf.toi, dots,
                    &s.g_ccd, skey, abd::NARROW_CCD_LS, first_batch)))
      return r;
    inf.linear_iters += abd::krylov_outcome(s);
    const double qTg = s.hbox->dots[0], gTg = s.hbox->dots[1];
    // backtracking line search (abd.py:146-160): the trials alpha, alpha / 2, ... up to the
    // first below alpha_min, kLsMax per batch; the first trial that passes is taken, as in
    // the sequential search
    double E1 = E0;
    for (bool done = false, first = true; !done; first = false) {
      double al[abd::kLsMax], Eb[abd::kLsMax];
      const int K = trial_steps(alpha, P.alpha_min, al);
      if (first) {
        for (int k = 0; k < K; ++k) Eb[k] = xs_round_host(s.hbox->ls_energy[k]);
      } else if ((r = ls_batch(h, st, st.A, st.p, al, K, Eb, skey))) {
        return r;
      }
      for (int k = 0; k < K && !done; ++k) {
        alpha = al[k];
        E1 = Eb[k];
        ++inf.ls_trials;
        const bool wolfe = E1 < E0 + P.armijo_sign * P.c1 * alpha * qTg ||
                           std::fabs(E1 - E0) <= P.ls_noise_floor * std::fabs(E0);
        done = wolfe || alpha < P.alpha_min;
      }
      if (!done) alpha *= 0.5;
    }
    E0 = E1;
    CK(abd::update_dofs(s, st.A, st.p, s.dq, alpha, st.A, st.p));
    // Ak, pk: the DOFs of the accepted trial, as the sequential search leaves them
    CK(cudaMemcpyAsync(st.Ak, st.A, nA, cudaMemcpyDeviceToDevice, s.stream));
    CK(cudaMemcpyAsync(st.pk, st.p, np, cudaMemcpyDeviceToDevice, s.stream));
    ++it;
    inf.alpha = alpha;
    if (gTg < P.tol || it >= P.max_iter) break;
  }
  CK(abd::finish_step(s, st, x_view));
  // the last CCD pass's line-search candidates hold the next step's first GH candidates when
  // that step starts from these DOFs
  CK(cudaMemcpyAsync(s.q_last, st.A, nA, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaMemcpyAsync(s.q_last + 9 * (size_t)s.n, st.p, np, cudaMemcpyDeviceToDevice, s.stream));
  CK(cudaMemsetAsync(s.dint + abd::kSupHave, 1, 1, s.stream));
  inf.newton_iters = it;
  inf.energy = E0;
  inf.status = take_status(h);
  if (info) *info = inf;
  return (inf.status & (abd::ST_STACK_OVERFLOW | abd::ST_NAN)) ? ABD_ERR_DEVICE : ABD_OK;
}

// Enqueues a step with the Newton iterations as a device loop on s.stream, which must be
// capturing (newton.cu describes the loop); ends with the copy of the mailbox to the host
int step_issue(abd_sim* h, const abd_states& st, double* x_view) {
  Sim& s = h->s;
  auto dots = [&]() -> int {  // dq.g, g.g on a branch beside the CCD pass's culling
    CK(cudaEventRecord(s.fork_ev[0], s.stream));
    CK(cudaStreamWaitEvent(s.fork_b, s.fork_ev[0], 0));
    CK(abd::dots(s, s.dq, s.g, s.g, s.g, s.box->dots, s.fork_b));
    CK(cudaEventRecord(s.fork_ev[1], s.fork_b));
    s.fork_open = true;
    return ABD_OK;
  };
  auto iteration_tail = [&]() -> int {  // after a GH pass without overflow (the IF body)
    if (int r = abd::cluster_inverse(s)) return r;
    if (int r = abd::krylov_issue(s, s.dq)) return r;
    // the CCD bound between q and q - dq with the line-search candidates (abd.py:278-303),
    // Ak, pk = q - dq; the trials of the line search and the acceptance (the loop's last kernel
    // takes the accepted step)
    const abd::Dofs d0 = direct(st.A, st.p), d1 = updated(s, st.A, st.p, 1, st.Ak, st.pk);
    if (int r = ccd_issue(h, d0, d1, abd::NARROW_CCD_LS, dots)) return r;
    CK(abd::ls_energies(s, st, st.A, st.p, true));
    CK(abd::ls_accept(s));
    return ABD_OK;
  };
  const cudaStream_t top = s.stream;
  if (int r = clear_friction(s)) return r;  // the first Newton iteration's GH pass fixes them
  cudaGraphConditionalHandle hn;
  if (int r = abd::make_handle(top, &hn)) return r;
  // q <- q0 (abd.py:124-128); the warm start kept for a rerun
  CK(abd::step_begin(s, st, hn));
  cudaGraph_t nbody = nullptr;
  if (int r = abd::add_conditional(top, hn, cudaGraphCondTypeWhile, &nbody)) return r;
  const long long l0 = s.launches;
  int r = abd::capture_body(s, nbody, s.cap_stream3, [&]() -> int {
    s.side = s.fork_a;
    const int q0 = gh_issue(h, st, st.A, st.p, 3);
    s.side = nullptr;
    if (q0) return q0;
    cudaGraphConditionalHandle hi;
    if (int q = abd::make_handle(s.stream, &hi)) return q;
    CK(abd::gate_no_overflow(s, hi));
    cudaGraph_t ibody = nullptr;
    if (int q = abd::add_conditional(s.stream, hi, cudaGraphCondTypeIf, &ibody)) return q;
    if (int q = abd::capture_body(s, ibody, s.cap_stream4, iteration_tail)) return q;
    CK(abd::newton_end(s, st, hn));  // (with the accepted step's DOF update)
    return ABD_OK;
  });
  if (r) return r;
  s.step_launch[1] = s.launches - l0;
  CK(abd::finish_step_dev(s, st, x_view));
  CK(cudaMemcpyAsync(s.hbox, s.box, sizeof(abd::Mailbox), cudaMemcpyDeviceToHost, top));
  return ABD_OK;
}

// The key of a device-loop step's graph: everything its captured kernels read by value
uint64_t step_key(const Sim& s, const abd_states& st, const double* x_view) {
  abd::KeyHash k;
  k.add(states_key(s, st)).add(x_view).add(s.cap_pairs).add(s.cap_adj).add(s.cap_contacts).add(s.cap_act);
  k.add(s.ij).add(s.adj_col).add(s.adj_pair).add(s.contacts).add(s.contacts_by_pair).add(s.act_pairs);
  k.add(s.pair_cand).add(s.offdiag).add(s.pdiag).add(s.pgrad).add(s.pair_active).add(s.q_last).add(s.dint);
  k.add(s.cap_ccd).add(s.ccd_cand).add(s.cap_ecand).add(s.ecand).add(s.prof_on).add(s.cl_inv).add(s.dq_save);
  return k.h;
}

// The simulator's set-up around a device-loop step's capture and replay
void step_modes(Sim& s, bool on) {
  s.prof_events = on && s.prof_on ? -1 : 0;  // kernel timing by the global timer (no events)
  s.gh_energy = on ? 1 : 0;                  // the GH pass sums the energy at the first iteration
  s.energy_gate = on ? &s.box->step.it : nullptr;
  s.in_device_loop = on;                     // passes that usually skip in IF nodes
}

constexpr int kHostFinish = -2;

// After a device-loop step's graph ran (the mailbox on the host, the stream synchronised):
// 0 when the step is complete; kRerun when a list overflowed (the warm start restored, the
// kept candidates dropped, the list grown: run the step again); kHostFinish when a line search
// needed more trials (likewise restored: the host loop finishes the step); or an ABD error.
int step_outcome(abd_sim* h) {
  Sim& s = h->s;
  std::memcpy(s.hstat, s.hbox->dstat, sizeof(int) * abd::DS_NSLOTS);
  const abd::StepDev& S = s.hbox->step;
  s.launches += (long long)S.it * s.step_launch[1] + (long long)(S.lin + S.it) * s.step_launch[2];
  s.n_pairs = s.hstat[abd::DS_NPAIRS];
  s.n_adj = s.hstat[abd::DS_NADJ];
  const int bits = s.hstat[abd::DS_STATUS];
  if (!(bits & abd::kRerunMask)) return 0;
  CK(cudaMemcpyAsync(s.dq, s.dq_save, sizeof(double) * 12 * s.n, cudaMemcpyDeviceToDevice, s.stream));
  if (int r = drop_superset(h)) return r;
  const int g = overflow(s);  // grows what was short; clears the overflow bits on the device
  if (g > 0) return g;
  if (bits & abd::ST_LS_MORE) {
    s.hstat[abd::DS_STATUS] &= ~abd::ST_LS_MORE;
    CK(cudaMemcpyAsync(s.dstat + abd::DS_STATUS, &s.hstat[abd::DS_STATUS], sizeof(int), cudaMemcpyHostToDevice,
                       s.stream));
    CK(cudaStreamSynchronize(s.stream));
    return kHostFinish;
  }
  return kRerun;
}

// The step info of a completed device-loop step, from the mailbox; the step's status taken
int step_info(abd_sim* h, abd_step_info* info) {
  Sim& s = h->s;
  const abd::StepDev& S = s.hbox->step;
  if (s.prof_on) {
    s.prof_ms += 1e-6 * (double)S.prof_ns;
    s.prof_launches += (long long)S.prof_n;
    s.prof_bytes += S.prof_bytes;
  }
  abd_step_info inf{};
  inf.newton_iters = S.it;
  inf.linear_iters = S.lin;
  inf.ls_trials = S.ls;
  inf.n_pt = S.n_pt;
  inf.n_ee = S.n_ee;
  inf.n_vg = S.n_vg;
  inf.n_ij = S.n_ij;
  inf.n_active = S.n_active;
  inf.alpha = S.alpha;
  inf.toi = S.toi;
  inf.energy = S.E0;
  inf.status = take_status(h);
  if (info) *info = inf;
  return (inf.status & (abd::ST_STACK_OVERFLOW | abd::ST_NAN)) ? ABD_ERR_DEVICE : ABD_OK;
}

// The step with the Newton iterations as a device loop: one graph launch and one copy to the
// host per step, a rerun from the step's start when a list overflowed
int step_device(abd_sim* h, const abd_states* stp, double* x_view, abd_step_info* info) {
  Sim& s = h->s;
  const abd_states& st = *stp;
  int r = ABD_OK;
  // a rerun restarts the whole step and meets the next short list, so a step gets the reruns of
  // all its passes; each recaptures (the buffers and capacities are in the key)
  for (int tries = 0;; ++tries) {
    step_modes(s, true);
    const long long launches0 = s.launches;
    r = abd::run_graph(s, s.g_step, step_key(s, st, x_view), [&]() { return step_issue(h, st, x_view); });
    step_modes(s, false);
    if (r) return r;
    s.launches = launches0 + s.g_step.nlaunch - s.step_launch[1];  // the loops: step_outcome
    CK(cudaStreamSynchronize(s.stream));
    r = step_outcome(h);
    if (r == 0) break;
    if (r == kHostFinish) return step_host(h, stp, x_view, info);
    if (r > 0) return r;
    if (tries >= kMaxStepReruns) return ABD_ERR_OVERFLOW;
  }
  return step_info(h, info);
}

}  // namespace

extern "C" {

int abd_adjoint_step(abd_sim* h, const abd_states* st, const double* A, const double* p, const double* qb,
                     const double* qdb, double* qb_out, double* qdb_out, int* iters) {
  if (!h || !st || !A || !p || !qb || !qdb || !qb_out || !qdb_out) return ABD_ERR_INVALID;
  Sim& s = h->s;
  // the exact Hessian at (A, p): the GH pass with the exact contact and vertex-ground terms
  // (its candidates from the traversal: the kept line-search candidates are for the step)
  if (int r = drop_superset(h)) return r;
  s.exact_hessian = 1;
  int r = gh_of(h, *st, A, p, nullptr, nullptr, false, 0);
  s.exact_hessian = 0;
  if (r) return r;
  // H lambda = a by preconditioned BiCGSTAB from lambda = 0 (the exact Hessian need not be
  // positive definite), to the step's Krylov tolerance
  CK(abd::adjoint_rhs(s, qb, qdb));
  CK(cudaMemsetAsync(s.adj_x, 0, sizeof(double) * 12 * s.n, s.stream));
  if ((r = abd::cluster_inverse(s))) return r;
  const int solver = s.prm.solver;
  s.prm.solver = 0;
  int it = 0;
  r = abd::krylov_solve(s, s.adj_x, &it, &s.g_kadj);
  s.prm.solver = solver;
  if (r) return r;
  if (iters) *iters = it;
  CK(abd::adjoint_out(s, s.adj_x, qdb, qb_out, qdb_out));
  CK(cudaStreamSynchronize(s.stream));
  const int bits = take_status(h);
  return (bits & (abd::ST_STACK_OVERFLOW | abd::ST_NAN)) ? ABD_ERR_DEVICE : ABD_OK;
}

int abd_batch_create(int n, abd_sim* const* sims, void* stream, abd_batch** out) {
  if (n <= 0 || !sims || !out) return ABD_ERR_INVALID;
  for (int i = 0; i < n; ++i)
    if (!sims[i]) return ABD_ERR_INVALID;
  abd_batch* b = new (std::nothrow) abd_batch();
  if (!b) return ABD_ERR_OVERFLOW;
  b->sims.assign(sims, sims + n);
  b->stream = (cudaStream_t)stream;
  b->branch.assign(n, nullptr);
  b->join.assign(n, nullptr);
  b->top.assign(n, 0);
  cudaError_t e = ABD_NOTE(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  if (e == cudaSuccess) e = ABD_NOTE(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = ABD_NOTE(cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking));
    if (e == cudaSuccess) e = ABD_NOTE(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming));
  }
  if (e != cudaSuccess) {
    abd_batch_destroy(b);
    return ABD_ERR_CUDA;
  }
  *out = b;
  return ABD_OK;
}

int abd_batch_destroy(abd_batch* b) {
  if (!b) return ABD_ERR_INVALID;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaStream_t q : b->branch)
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t ev : b->join)
    if (ev) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
  return ABD_OK;
}

int abd_batch_step(abd_batch* b, const abd_states* st, double* const* x_view, abd_step_info* info) {
  if (!b || !st) return ABD_ERR_INVALID;
  const int n = (int)b->sims.size();
  for (abd_sim* h : b->sims)  // the device loop takes every step (one batch of trials)
    if (!(h->s.prm.alpha_min > 0x1p-15)) return ABD_ERR_INVALID;
  abd::KeyHash k;
  k.add(n);
  for (int i = 0; i < n; ++i) k.add(step_key(b->sims[i]->s, st[i], x_view ? x_view[i] : nullptr)).add(b->sims[i]);
  if (!b->exec || b->key != k.h) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    CK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    int r = ABD_NOTE(cudaEventRecord(b->fork, b->cap)) == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
    for (int i = 0; i < n && r == ABD_OK; ++i) {
      Sim& s = b->sims[i]->s;
      if (ABD_NOTE(cudaStreamWaitEvent(b->branch[i], b->fork, 0)) != cudaSuccess) {
        r = ABD_ERR_CUDA;
        break;
      }
      const cudaStream_t saved = s.stream;
      const long long l0 = s.launches;
      s.stream = b->branch[i];
      step_modes(s, true);
      r = step_issue(b->sims[i], st[i], x_view ? x_view[i] : nullptr);
      step_modes(s, false);
      s.stream = saved;
      b->top[i] = s.launches - l0 - s.step_launch[1];
      s.launches = l0;
      if (r == ABD_OK && (ABD_NOTE(cudaEventRecord(b->join[i], b->branch[i])) != cudaSuccess ||
                          ABD_NOTE(cudaStreamWaitEvent(b->cap, b->join[i], 0)) != cudaSuccess))
        r = ABD_ERR_CUDA;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = ABD_NOTE(cudaStreamEndCapture(b->cap, &graph));
    if (r == ABD_OK && e2 != cudaSuccess) r = ABD_ERR_CUDA;
    if (r == ABD_OK && ABD_NOTE(cudaGraphInstantiate(&b->exec, graph, 0)) != cudaSuccess) r = ABD_ERR_CUDA;
    if (graph) cudaGraphDestroy(graph);
    if (r != ABD_OK) {
      if (b->exec) cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
      return r;
    }
    b->key = k.h;
  }
  CK(cudaGraphLaunch(b->exec, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  int first_error = ABD_OK;
  for (int i = 0; i < n; ++i) {
    abd_sim* h = b->sims[i];
    h->s.launches += b->top[i];
    int r = step_outcome(h);
    abd_step_info* inf = info ? info + i : nullptr;
    if (r == 0) r = step_info(h, inf);
    else if (r == kRerun) r = step_device(h, &st[i], x_view ? x_view[i] : nullptr, inf);  // alone, grown
    else if (r == kHostFinish) r = step_host(h, &st[i], x_view ? x_view[i] : nullptr, inf);
    if (r != ABD_OK && first_error == ABD_OK) first_error = r;
  }
  return first_error;
}

int abd_step(abd_sim* h, const abd_states* stp, double* x_view, abd_step_info* info) {
  if (!h || !stp) return ABD_ERR_INVALID;
  // the device loop takes every step whose line search ends within one batch of trials
  // (alpha_min above 2^-15, the 16th halving of the largest step 1); else the host drives
  const bool device = h->s.prm.newton_loop == 0 && h->s.prm.alpha_min > 0x1p-15;
  return device ? step_device(h, stp, x_view, info) : step_host(h, stp, x_view, info);
}

}  // extern "C"
