/*
 * abd_b200.h - C ABI of the B200 (sm_100a) affine-body-dynamics implicit contact step.
 *
 * This is the drop-in boundary below the Python mirror of the reference's simulator API
 * (abd_warp_b200/simulator.py).  The reference (Luke-Skycrawler/abd-warp) is Python on
 * NVIDIA Warp and has no FFI of its own; each entry point below replaces the reference
 * function or Warp library call named beside it (paths are within the reference project).
 *
 * Conventions
 *  - All arrays named *_dev are device pointers on the simulator's device; everything else
 *    is host memory.  No entry point takes framework (torch) types.
 *  - Body state layout follows AffineBodyStates (abd/affine_body.py:7-21): A is [n][3][3]
 *    row-major with row k the DOF vector a_k, p is [n][3]; a rest vertex r maps to
 *    x = p + r0 a0 + r1 a1 + r2 a2 (abd/abd.py:313-316).  Gradients and Newton steps are
 *    [n][4][3] = per body (p, a0, a1, a2), as the reference's g / dq (abd/abd.py:49-50).
 *  - Calls are asynchronous on the simulator's stream unless they return a host value
 *    (counts, energies, step info), in which case they synchronise that stream.
 *  - Return value: ABD_OK or an ABD_ERR_* code; abd_status_string() describes it.
 *    A simulator whose call returned ABD_ERR_CUDA should be destroyed.
 */
#ifndef ABD_B200_H
#define ABD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ABD_OK = 0,
  ABD_ERR_CUDA = 1,      /* a CUDA runtime call failed */
  ABD_ERR_INVALID = 2,   /* bad argument (NULL pointer, size out of range, bad mesh index) */
  ABD_ERR_OVERFLOW = 3,  /* a capacity could not be grown (out of device memory) */
  ABD_ERR_DEVICE = 4     /* a kernel reported an internal error (traversal stack, NaN) */
};

/* Physics and solver parameters; the reference's module constants
 * (abd/const_params.py:24-44) and simulator_args (abd/abd.py:107-121) as one struct. */
typedef struct abd_params {
  double dt, dhat, d2hat, kappa, stiffness, gravity, tol, c1, alpha_min, ground, cg_tol, refine_tol;
  double ls_noise_floor; /* line search also accepts |E1 - E0| <= ls_noise_floor |E0| (0: off) */
  int max_iter;       /* Newton iteration cap (abd.py:114) */
  int armijo_sign;    /* -1: E1 < E0 - c1 a dq.g (default); +1: the reference's form (abd.py:156) */
  int ground_enabled; /* vertex-ground plane contact at y = ground (culling.py:54-82, vg_ipc.py) */
  int psd_ee;         /* contact_psd == 0 only: clamp EE eigenvalues as PT does */
  int enable_pt, enable_ee, enable_vg; /* const_params.py:41-43 */
  int solver;         /* 0: preconditioned BiCGSTAB (abd.py:244 uses bicgstab), 1: PCG (default) */
  int cg_max_iter;
  int precision;      /* 0: FP64 throughout (the only accepted value).  1, an FP32 Krylov solve
                         inside FP64 refinement, is rejected with ABD_ERR_INVALID: on contact
                         systems (cond(H) ~ 1e10 > 1 / eps_FP32) the refinement diverges */
  int contact_psd;    /* 1: PSD projection of the barrier Hessian; 0: the reference's form */
  int precond;        /* 1: contact-cluster block Jacobi (clusters of <= cluster_max bodies); 0: per body */
  int cluster_max;    /* 1..12 */
  int min_capacity;   /* 0: default capacities.  n > 0: every list of the simulator (body
                         pairs, candidates, contacts, active pairs, vertex-ground pairs) starts
                         with n entries (read by abd_sim_create) and the breadth-first
                         traversal frontier holds at most min(n, 512) nodes (read per pass),
                         so that small scenes run every grow-and-rerun path and the traversal's
                         depth-first fallback: a host-side way to inject capacity shortfalls */
  int newton_loop;    /* 0 (default): abd_step runs its Newton iterations as a device loop, one
                         CUDA graph launch and one copy to the host per step; 1: the host drives
                         them, waiting for the device twice per iteration.  Both give the same
                         results; the device loop hands a step over to the host loop when its
                         line search needs more than 16 trials (alpha_min <= 2^-15) */
  int ipc_full;       /* 0 (default): the reference's contact model -- interior point-triangle
                         and edge-edge pairs only (ipcsk/energy.py:20-22, 46-48; ccd.py:44-54).
                         1: the full IPC model -- the closest feature pair of every candidate
                         (point-triangle / -edge / -point; edge-edge / point-edge / point-point),
                         the barrier on its squared distance with the edge-edge mollifier, a
                         per-contact PSD projection of the exact local Hessian, and CCD roots on
                         the closed triangle / segments */
  double friction_mu;   /* lagged IPC friction (not in the reference; needs ipc_full = 1): the
                           Coulomb coefficient, 0 (default) = off.  At a step's start every
                           contact within dhat fixes its closest-point weights, a tangent basis
                           and its normal force; the step then adds mu lambda f0(|u|) per contact
                           (u: the tangential displacement over the step) to the energy, the
                           gradient and the Hessian, and keeps the contact's body pair in the
                           pair lists for the whole step */
  double friction_epsv; /* the slip velocity below which friction is static (eps = friction_epsv dt) */
} abd_params;

/* Scene description (host arrays, copied at creation).  Bodies are concatenated:
 * vertices of body b are [vert_off[b], vert_off[b+1]) etc.  Replaces the per-body WarpMesh
 * arrays (abd/affine_body.py:42-51, 84-97). */
typedef struct abd_scene_desc {
  int n_bodies;
  const int* vert_off;  /* [n+1] */
  const int* tri_off;   /* [n+1] */
  const int* edge_off;  /* [n+1] */
  const double* x0;     /* [V][3] rest positions (body frame) */
  const int* tris;      /* [T][3] global vertex indices */
  const int* edges;     /* [E][2] global vertex indices */
  const double* mass;   /* [n] */
  const double* I0;     /* [n] */
  const int* fixed;     /* [n] 1 = Dirichlet body (its DOFs never move) */
} abd_scene_desc;

/* Device pointers to the caller-owned body states (AffineBodyStates, affine_body.py:7-21). */
typedef struct abd_states {
  double *A, *p, *Ak, *pk, *Adot, *pdot, *A0, *p0;
} abd_states;

/* Counters of one time step. */
typedef struct abd_step_info {
  int newton_iters, linear_iters, ls_trials, n_pt, n_ee, n_vg, n_ij, n_active;
  double alpha, toi, energy;
  int status;          /* device status bits seen during the step (0 = clean) */
  int refine_iters;    /* FP64 refinement sweeps (0: precision 1 is not accepted) */
} abd_step_info;

typedef struct abd_sim abd_sim;
typedef struct abd_batch abd_batch;

/* Create a simulator for one scene on the current CUDA device; stream may be NULL (legacy
 * default stream).  Builds the per-body LBVHs (Morton codes, radix sort, Karras build).
 * Replaces AffineBodySimulator.__init__'s device setup (abd/abd.py:21-95).
 * Returns ABD_ERR_INVALID, before any device work, for a malformed scene: no bodies, a body
 * without vertices, offsets that do not start at 0 or decrease, a triangle or edge index
 * outside its body's vertices, a non-finite rest position, a free body without a positive
 * finite mass and I0, precision != 0 or min_capacity < 0; and, after the tree build, for a
 * body whose primitive tree is deeper than the traversal stack holds (3 ceil(H / 2) + 1 > 64
 * entries for H internal levels, which takes many primitives with one Morton code). */
int abd_sim_create(const abd_scene_desc* scene, const abd_params* prm, void* stream, abd_sim** out);
int abd_sim_destroy(abd_sim* sim);
int abd_sim_set_params(abd_sim* sim, const abd_params* prm);
int abd_sim_set_stream(abd_sim* sim, void* stream);
/* Zero the warm-started Newton step dq (AffineBodySimulator.reset, abd/abd.py:97-104). */
int abd_sim_reset(abd_sim* sim);
/* Copy the simulator's warm-started Newton step dq [n][12] / last gradient g [n][12]
 * (the reference's sim.dq / sim.g, abd/abd.py:49-50) to or from device buffers. */
int abd_sim_get_dq(abd_sim* sim, double* dst_dev);
int abd_sim_set_dq(abd_sim* sim, const double* src_dev);
int abd_sim_get_g(abd_sim* sim, double* dst_dev);
int abd_sim_sizes(const abd_sim* sim, int* n_bodies, int* n_verts, int* n_tris, int* n_edges);

/* One implicit time step (AffineBodySimulator.step, abd/abd.py:212-276): Newton on
 * inertia + orthogonality + IPC barrier energy with CCD-bounded backtracking line search,
 * then q0 <- q, qdot <- (q - q0)/dt and x_view_dev <- transform(q0).  x_view_dev may be NULL. */
int abd_step(abd_sim* sim, const abd_states* st, double* x_view_dev, abd_step_info* info);

/* Batched scenes (the reference steps one scene per simulator).  abd_batch_create groups n
 * simulators (one scene each, created by abd_sim_create and still owned by the caller, who
 * destroys them after the batch); stream is where the batch's steps run (NULL: legacy default
 * stream).  abd_batch_step steps every scene once: st[i] are scene i's states, x_view[i] its
 * vertex positions out (x_view or any x_view[i] may be NULL), info[i] its step info (info may
 * be NULL).  All scenes' device-loop steps are one CUDA graph, each scene a branch of its own
 * that holds its Newton loop, so one launch runs every scene's iterations concurrently with
 * each scene's own iteration counts, line search and convergence: each scene's result is the
 * one abd_step gives it.  A scene whose list overflowed is stepped again alone after the
 * list grew.  Needs alpha_min > 2^-15 in every scene (else ABD_ERR_INVALID).  Returns the
 * first error of a scene, or ABD_OK. */
int abd_batch_create(int n, abd_sim* const* sims, void* stream, abd_batch** out);
int abd_batch_destroy(abd_batch* batch);
int abd_batch_step(abd_batch* batch, const abd_states* st, double* const* x_view, abd_step_info* info);

/* One step of the adjoint of abd_step (the reference has none: hl_entry.py:4 sets
 * enable_backward = False).  A converged step solves grad E(q; q~) = 0 for q_{t+1}, with the
 * prediction q~ = q_t + dt qdot_t (+ dt^2 g on p), and qdot_{t+1} = (q_{t+1} - q_t) / dt.  Given
 * the adjoints qb_dev, qdb_dev [n][12] of q_{t+1} and qdot_{t+1} (per body [p, A rows], the
 * layout of g / dq), this returns those of q_t and qdot_t:
 *   a = qb + qdb / dt,  H lambda = a,  qb_out = M lambda - qdb / dt,  qdb_out = dt M lambda,
 * where H is the exact Hessian of the step's energy at q_{t+1} = (A_dev, p_dev) -- inertia,
 * orthogonality, and each active contact's unprojected barrier Hessian with every
 * second-derivative term (the Newton Hessian projects the barrier and, like the reference,
 * leaves out the derivatives of the closest-point coefficients: psd/vf.py:150-176,
 * psd/ee.py:94-116, and the vertex-ground 2 B' term: vg_ipc.py:28-33) -- and M the mass matrix
 * (mass on p, I0 on A).  H is solved by preconditioned BiCGSTAB to cg_tol; iters (host, may be
 * NULL) receives its iterations.  st supplies the inertia prediction (its A0 / p0 / Adot / pdot:
 * any values; H does not depend on them).  Fixed bodies get zero adjoints.  Valid where the
 * step converged (g.g below tol): the implicit-function derivative it computes is the
 * derivative of the step only there. */
int abd_adjoint_step(abd_sim* sim, const abd_states* st, const double* A_dev, const double* p_dev,
                     const double* qb_dev, const double* qdb_dev, double* qb_out_dev, double* qdb_out_dev,
                     int* iters);

/* x = p + sum_k r_k a_k for every vertex (update_mesh_vertex, abd/abd.py:305-324). */
int abd_update_mesh_vertex(abd_sim* sim, const double* A_dev, const double* p_dev, double* x_dev);

/* Broad + narrow culling on positions y0_dev (collision_set, abd/abd.py:187-207) or, when
 * y1_dev is not NULL, on the swept boxes y0 -> y1 (trajectory_intersection_set,
 * abd/abd.py:170-185).  counts[4] = {body pairs, PT, EE, VG} (host); the lists stay in the
 * simulator for abd_export_lists. */
int abd_collision_set(abd_sim* sim, const double* y0_dev, const double* y1_dev, int counts[4]);
/* The same culling at DOFs, the form the time step uses: positions x = transform(A, p) (and
 * xk = transform(A1, p1) for the swept boxes when A1_dev / p1_dev are not NULL) are computed
 * into the simulator's x / xk, and the tree's internal boxes are bounded by the affine
 * images of their rest-frame boxes instead of a refit.  Lists and counts as
 * abd_collision_set (update_mesh_vertex + collision_set / trajectory_intersection_set,
 * abd/abd.py:170-207, as step and ccd call them at abd.py:226-227, 278-280). */
int abd_collision_set_dofs(abd_sim* sim, const double* A_dev, const double* p_dev, const double* A1_dev,
                           const double* p1_dev, int counts[4]);
/* Copy the lists of the last abd_collision_set / abd_collision_set_dofs call (valid until the
 * next call that culls: abd_step, abd_ipc_gh, abd_compute_energy, abd_ccd,
 * abd_energies_along or another collision set) into device buffers of capacity cap rows:
 * ij [cap][2] (I < J), pt [cap][5] and ee [cap][5] as (I, J, pair, local prim of I, local
 * prim of J) like the reference's vec5i lists (culling.py:85-99), vg [cap][2] (body,
 * global vertex).  Any pointer may be NULL. */
int abd_export_lists(abd_sim* sim, int* ij_dev, int* pt_dev, int* ee_dev, int* vg_dev, int cap);

/* Gradient and Hessian at body DOFs (A_dev, p_dev) with prediction from st->A0/p0/Adot/pdot
 * (inertia: orthogonal_energy.py:17-22, contacts: ipc.py:54-62 -> pt_ipc / ee_ipc / vg_ipc,
 * assembly: put.py + bsr_set_from_triplets, abd/abd.py:240-243).  n_active (host, may be
 * NULL) receives the number of active PT + EE contacts. */
int abd_ipc_gh(abd_sim* sim, const abd_states* st, const double* A_dev, const double* p_dev, int* n_active);
/* Copy the last assembled system: g [n][12], diagonal blocks [n][12][12], off-diagonal blocks
 * [cap][12][12] (block (I,J), I < J, of body pair q in ij order) and ij [cap][2].
 * n_pairs (host) receives the number of body pairs. */
int abd_export_system(abd_sim* sim, double* g_dev, double* diag_dev, double* off_dev, int* ij_dev, int cap,
                      int* n_pairs);

/* Solve H dq = g of the last assembled system, dq_dev the warm start, overwritten
 * (warp.optim.linear.bicgstab call, abd/abd.py:244).  iters (host) may be NULL. */
int abd_solve(abd_sim* sim, double* dq_dev, int* iters);

/* Total energy at trial DOFs (Ak_dev, pk_dev) with prediction from st (compute_energy,
 * abd/abd.py:133-141: IPC barrier ipcsk/energy.py:9-48 + inertia orthogonal_energy.py:24-32). */
int abd_compute_energy(abd_sim* sim, const abd_states* st, const double* Ak_dev, const double* pk_dev, double* E);

/* CCD step bound between DOFs (A, p) and (A1, p1) (ccd, abd/abd.py:278-303; toi_vg ccd.py:9-18,
 * cubic CCD ccd.py:56-186 / cubic_roots.py:95-193 in place of abdtk).  alpha (host) gets
 * clamp(toi, 0, 1) * (0.9 if < 1), raw_toi (host, may be NULL) the unclamped minimum. */
int abd_ccd(abd_sim* sim, const double* A_dev, const double* p_dev, const double* A1_dev, const double* p1_dev,
            double* alpha, double* raw_toi);

/* Energies along the search direction: E[k] = the energy at (A, p) - alphas[k] dq (dq: the
 * simulator's, set by abd_sim_set_dq or left by abd_step) for K step lengths 0 <= alphas[k] <= 1
 * (host array), each bitwise equal to abd_compute_energy at those DOFs.  This is how abd_step
 * evaluates its line-search trials (abd.py:146-160 evaluates compute_energy once per trial):
 * one culling pass between (A, p) and (A, p) - dq collects every contact candidate that any
 * step length in [0, 1] can produce, then each batch of up to 16 trials re-evaluates only
 * those, with the reference's culling predicate applied at each trial's DOFs.  st->Ak, st->pk
 * receive (A, p) - dq. */
int abd_energies_along(abd_sim* sim, const abd_states* st, const double* A_dev, const double* p_dev,
                       const double* alphas, int K, double* E);

/* Inertia + orthogonality energy of n_bodies bodies at trial DOFs (Ak, pk), with the
 * prediction from st->A0 / p0 / Adot / pdot, written to E_dev (one double).  No counterpart in
 * the reference: it is the body part of abd_compute_energy, made for callers that may not
 * allocate device memory while running (fixed-budget real-time loops, plug-ins whose host
 * application owns all device memory).  It allocates nothing; its only scratch is a
 * fixed array inside the library (4096 doubles, so n_bodies <= 1,048,576, else
 * ABD_ERR_INVALID).  All calls share that array: calls that overlap on the GPU race.  The
 * first call on a device looks up the array's address (make it before any stream capture);
 * the address is kept for the process, so after cudaDeviceReset of a device this entry point
 * must not be called on it again.  The sum is a fixed-order tree (per CTA of 256 bodies, then
 * over the CTAs): deterministic, but it can differ in the last bits from abd_compute_energy,
 * whose sum is exact.  Fixed bodies contribute nothing.  Runs on `stream` (NULL: legacy
 * default stream). */
int abd_inertia_energy_noalloc(const abd_params* prm, int n_bodies, const abd_states* st, const double* Ak_dev,
                               const double* pk_dev, const double* mass_dev, const double* I0_dev,
                               const int* fixed_dev, double* E_dev, void* stream);

/* Per-body contact flags of the last gradient / Hessian pass (the step's last Newton
 * iteration, or abd_ipc_gh) into highlight_dev [n] (int, device): 1 when the body takes part
 * in an active PT or EE contact (d^2 < dhat^2 and a valid closest-point configuration) or has
 * an active vertex-ground contact, else 0.  The reference's step sets sim.highlight from its
 * contact pass every Newton iteration (abd/abd.py:238) and the viewer colours bodies by it
 * (abd/abd.py:412-413); ipc.py:59-60 keeps only the EE result and marks one body per contact
 * (pt_ipc.py:118, ee_ipc.py:98).  Here PT, EE and vertex-ground contacts all count, for both
 * bodies of a contact. */
int abd_get_highlight(abd_sim* sim, int* highlight_dev);

/* Where the last CUDA runtime call that failed in this thread failed, for an ABD_ERR_CUDA:
 * "file:line: error name: description" (empty if none has). */
const char* abd_error_detail(void);

/* Device status bits accumulated since the last call (and cleared). */
int abd_take_status(abd_sim* sim, int* status);
const char* abd_status_string(int code);

/* Number of kernel launches the simulator has issued since creation. */
long long abd_launch_count(const abd_sim* sim);

/* Kernel profiling (no counterpart in the reference; used by the benchmark's roofline).
 * abd_profile(sim, mode) resets the counters; from then on the step's CCD passes (which also
 * collect the line-search candidates) time their narrow-phase kernel: with the device Newton
 * loop (newton_loop 0) every launch, by the GPU's global timer (the kernel records its first
 * CTA's start and its last CTA's end); with the host loop by CUDA events on the simulator's
 * stream, every 4th pass in mode 1 and every pass in mode 2.  Mode 2 also counts the data the
 * kernel moves (and slows it down).
 * abd_profile_read returns the accumulated kernel time (ms), the number of launches and, for
 * mode 2, the algorithmic bytes (point queries 24 B, edge queries 36 B, (chunk, neighbour)
 * records 140 B, tree entries tested 36 B, candidates written 16 B).
 * abd_profile(sim, 0) stops. */
int abd_profile(abd_sim* sim, int enable);
/* The current device's FP64 throughput (TFLOP/s) measured by chains of fused multiply-adds
 * (no counterpart in the reference; the benchmark's FP64 roofline).  The library's kernels
 * are built without multiply-add contraction, so their own FP64 rate tops out at half of it. */
int abd_fp64_peak(double* tflops);
int abd_profile_read(const abd_sim* sim, double* ms, long long* launches, double* bytes);

#ifdef __cplusplus
}
#endif
#endif /* ABD_B200_H */
