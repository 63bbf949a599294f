/*
 * rodgpu.h - C ABI of the B200 rigid-rod contact hot path (librodgpu.so).
 *
 * One rg_system holds the device state of one periodic (or open) system of
 * capsules and advances it with the contact model of rod-dynamics-3d's
 * App::physicsStep (src/app/main.cpp:4333-4858):
 *   - "nsc":            free flight, detection, PSOR friction-cone sweeps,
 *                       semi-implicit position update, normal-only position
 *                       projection        (main.cpp:4383-4528)
 *   - "harmonic":       soft penalty contact with smooth / Cundall-Strack /
 *                       Karnopp friction, velocity Verlet (main.cpp:4610-4810)
 *   - "hertz-mindlin":  Hertz normal + Mindlin tangential spring with history
 *                       and rolling friction, applied to capsule contacts,
 *                       velocity Verlet    (main.cpp:4529-4609)
 *
 * Plain pointers and sizes only; no exceptions cross this boundary.  Every
 * entry point returns an rg_status (0 = ok).  Arrays are structure-of-arrays
 * FP64 in HOST memory unless the name says _dev.  A handle is not thread
 * safe; use one handle per host thread.
 *
 * The reference has no C ABI for this path.  The entry points below replace
 * the solver-class seam that App::physicsStep calls:
 *   ContactDetector::detectContacts   (include/physics/contact_detector.hpp:70)
 *   SoftContactSolver::computeForces  (include/physics/soft_contact.hpp:47)
 *   HertzMindlinSolver::computeForces (include/physics/hertz_mindlin.hpp:90)
 *   NscContactSolver::detectAndBuildManifolds / solveVelocities /
 *     projectPositions                (include/physics/nsc_contact.hpp:88-103)
 *   integrateHalfPos / integrateSecondHalf (include/physics/integrator.hpp:33-34)
 * and the free-function CUDA precedent cudaDetectCapsulePairsTwoPass
 *   (include/physics/cuda_broadphase.hpp:95-101).
 */
#ifndef RODGPU_H
#define RODGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RG_ABI_VERSION 2

typedef enum rg_status {
  RG_OK = 0,
  RG_ERR_ARG = 1,          /* bad argument (null pointer, n <= 0, ...)        */
  RG_ERR_CUDA = 2,         /* a CUDA runtime call failed                      */
  RG_ERR_CAPACITY = 3,     /* a device buffer overflowed and could not grow   */
  RG_ERR_NONFINITE = 4,    /* non-finite body state after a step              */
  RG_ERR_NOT_CONVERGED = 5,/* PSOR hit max sweeps above tolerance (strict)    */
  RG_ERR_NO_DEVICE = 6,    /* no CUDA device visible                          */
  RG_ERR_TIMEOUT = 7,      /* a bounded device-side wait gave up              */
  RG_ERR_STATE = 8         /* call out of order (e.g. step before bodies set) */
} rg_status;

typedef enum rg_model {
  RG_MODEL_NONE = 0,          /* physicsStep with no model enabled: no-op   */
  RG_MODEL_NSC = 1,           /* contact_model "nsc"                        */
  RG_MODEL_HARMONIC = 2,      /* contact_model "harmonic" (soft penalty)    */
  RG_MODEL_HERTZ_MINDLIN = 3  /* contact_model "hertz-mindlin" (capsules)   */
} rg_model;

typedef enum rg_friction_mode {  /* SoftContactSolver::computeFriction      */
  RG_FRICTION_SMOOTH = 0,        /* default (soft_contact.cpp:458-485)      */
  RG_FRICTION_CUNDALL = 1,       /* friction_cundall (soft_contact.cpp:317) */
  RG_FRICTION_KARNOPP = 2        /* friction_karnopp (soft_contact.cpp:369) */
} rg_friction_mode;

typedef enum rg_psor_order {
  RG_ORDER_COLORED = 0,  /* graph-coloured Gauss-Seidel (the device order)   */
  RG_ORDER_SORTED = 1    /* sequential sorted (a,b) order of the reference
                            (nsc_contact.cpp:91-102); oracle only           */
} rg_psor_order;

typedef enum rg_warm_start {
  RG_WARM_CACHE = 0,     /* previous-step impulses by pair (nsc_contact.cpp:305-317) */
  RG_WARM_NONE = 1,      /* cold start                                       */
  RG_WARM_MLP = 2        /* learned warm start from rg_mlp weights (for the
                            contacts nsc_mlp_scope selects; the others start
                            from the cache)                                  */
} rg_warm_start;

/* Configuration.  Field meanings and defaults follow AppCfg
 * (include/config/config.hpp:6-110); rg_config_default() fills them. */
typedef struct rg_config {
  int32_t n_bodies;
  int32_t model;                 /* rg_model */
  double dt;
  double gravity[3];
  double lin_damp, ang_damp, w_max;
  int32_t pbc_enabled;
  double pbc_min[3], pbc_max[3];

  /* SoftContactCfg (config.hpp:6-27) */
  double soft_delta, soft_k_scaler, soft_damping, soft_mu, soft_mu_static;
  double soft_nu, soft_kt, soft_vel_deadband;
  int32_t soft_enable_friction;
  int32_t soft_friction_mode;    /* rg_friction_mode */

  /* HertzMindlinCfg (config.hpp:29-64) */
  double hm_youngs_modulus, hm_poisson_ratio, hm_restitution;
  double hm_friction, hm_friction_static, hm_friction_transition_vel;
  double hm_rolling_friction;
  int32_t hm_enable_tangential, hm_enable_rolling;

  /* NscContactCfg (config.hpp:66-88) */
  double nsc_mu, nsc_beta, nsc_cfm, nsc_omega, nsc_slop, nsc_tol;
  int32_t nsc_velocity_iters, nsc_position_stabilization;
  int32_t nsc_position_iters, nsc_position_psor_iters;
  int32_t nsc_warm_start;        /* rg_warm_start */
  int32_t psor_order;            /* rg_psor_order; device supports COLORED */

  /* Neighbour-list broad phase (project-specific, no reference field). */
  double skin;                   /* Verlet skin; <= 0: max(d/2, L/10), means */
  int32_t max_neighbors;         /* initial per-rod list capacity; <= 0 auto */
  int32_t team_blocks;           /* blocks of the persistent NSC team; 0 auto */
  int32_t nsc_mlp_scope;         /* learned start for: 0 contacts new since
                                    the last step (not in the warm cache),
                                    1 every contact                          */
  int32_t nsc_mlp_min_sweeps;    /* ... in a step only when the previous one
                                    needed more PSOR sweeps than this, or the
                                    warm cache is empty (default 3; -1: in
                                    every step)                              */
  int32_t near_skin_pct;         /* near-list skin, % of the Verlet skin (0:
                                    automatic: 5 %, 50 % in all-pairs boxes;
                                    negative: the soft / HM detection tests
                                    the full lists every step)              */
  /* Bounded device waits.  Every team barrier of the persistent step polls
   * at most spin_limit times (0: the default 2e7 polls, about 1-2 s) and
   * then records RG_ERR_TIMEOUT; every block of the launch then returns and
   * the call restores the state it started from. */
  int32_t spin_limit;
  /* Test hook for failure detection, 0 in normal use: the team barriers of
   * the persistent step expect this many more blocks than the team has, so
   * their waits run out after spin_limit polls and the call returns
   * RG_ERR_TIMEOUT (no fault, no hang: the wait is the bounded one above). */
  int32_t test_absent_blocks;
  /* Cylindrical tube boundary (SceneCfg::cylinder, config.hpp:150-154):
   * an infinite tube of radius cylinder_radius about cylinder_axis through
   * the origin.  NSC: wall manifolds for the sample points of each capsule
   * (collideCapsuleInsideCylinder, collision.cpp:197-241; main.cpp:
   * 4431-4447) and spin about the rod axis projected out after the position
   * update (:4486-4494).  Soft model: a penalty spring with smooth Coulomb
   * friction at both force evaluations (:4661-4690, :4756-4787).  The
   * Hertz-Mindlin model has no wall term, as in the reference. */
  int32_t cylinder_enabled;
  double cylinder_radius;
  double cylinder_axis[3];
} rg_config;

/* Per-call statistics (the profile-CSV columns of main.cpp:3276-3355). */
typedef struct rg_step_stats {
  int64_t steps;            /* steps taken in this call                       */
  int64_t contacts;         /* contacts at the last detection                 */
  int64_t collisions;       /* NSC: manifolds with v_n_pre < -1e-6 (last step)*/
  int64_t psor_sweeps;      /* NSC: velocity sweeps summed over the call      */
  int64_t psor_sweeps_last; /* NSC: velocity sweeps of the last step          */
  int64_t list_rebuilds;    /* neighbour-list rebuilds in this call           */
  int64_t colors;           /* NSC: colours of the last velocity solve        */
  int64_t history_size;     /* HM / Cundall: live history entries             */
  double residual;          /* NSC: last PSOR residual (max |dλ| sum)         */
  double jn_sum, jt_sum;    /* NSC: Σ|λn| and Σ(|λt1|+|λt2|) of the last step
                               (the profile CSV's sums, main.cpp:3339-3343)   */
  double potential_energy;  /* soft / HM: last contact potential energy       */
  double kinetic_energy;    /* ½Σ m|v|² + ½Σ ω·Iω after the call              */
  double max_residual;      /* NSC: worst final residual over the call        */
  int64_t not_converged;    /* NSC: steps that stopped at max sweeps          */
  double device_ms;         /* device time of the call (CUDA events, stream)  */
  int64_t psor_row_sweeps;  /* NSC: Σ over steps of contacts x sweeps         */
  int64_t kernel_launches;  /* kernels this library launched during the call  */
  int64_t contact_steps;    /* NSC: Σ over steps of velocity-solve contacts;
                               soft / HM: Σ over force evaluations of contacts */
  int64_t near_rebuilds;    /* NSC: near-list rebuilds in this call           */
  int64_t reserved[1];
} rg_step_stats;

/* Stage timers (CUDA events on the system's stream), enabled per system.
 * Stages: 0 integrate, 1 detect (incl. list rebuild), 2 colour, 3 manifolds,
 * 4 PSOR sweeps, 5 position projection, 6 contact forces + history, 7 other. */
#define RG_NSTAGES 8

typedef struct rg_system rg_system;

/* ---- lifecycle ---------------------------------------------------------- */
int rg_abi_version(void);
void rg_config_default(rg_config* cfg);
const char* rg_status_string(int status);
/* Last error text of this handle (empty when none). */
const char* rg_last_error(const rg_system* sys);

/* Creates a system on the current CUDA device.  Replaces the solver objects
 * softContactSolver / hertzMindlinSolver / nscSolver owned by App
 * (src/app/main.cpp:439-442) as configured in App::resetScene (:1541-1590). */
int rg_create(const rg_config* cfg, rg_system** out);
int rg_destroy(rg_system* sys);
int rg_get_config(const rg_system* sys, rg_config* cfg);

/* Body properties, one value per body (RigidBody fields,
 * include/physics/rigid_body.hpp:30-41; makeCapsule rigid_body.cpp:11-47).
 * inertia = body-frame principal moments (Ixx, Iyy, Izz) per body, 3 per body.
 * mass <= 0 marks a static body (invMass = 0, App::createRod main.cpp:1523). */
int rg_set_bodies(rg_system* sys, const double* radius, const double* half_height,
                  const double* mass, const double* inertia,
                  const double* restitution);

/* State, structure of arrays: x[3N], q[4N] (w,x,y,z), v[3N], w[3N].
 * Forces f[3N], tau[3N] may be NULL on set (zeroed) or on get (skipped).
 * Soft / Hertz-Mindlin models: both force evaluations of a step start from
 * zero forces (the reference clears them in integrateSecondHalf,
 * src/physics/integrator.cpp:156-158); after a step f and tau hold the
 * forces at t + dt that its second half kick used, after rg_compute_forces
 * the forces it returned. */
int rg_set_state(rg_system* sys, const double* x, const double* q,
                 const double* v, const double* w,
                 const double* f, const double* tau);
int rg_get_state(const rg_system* sys, double* x, double* q, double* v,
                 double* w, double* f, double* tau);

/* Advances nsteps of App::physicsStep for the configured model.
 * stats may be NULL. */
int rg_step(rg_system* sys, int nsteps, rg_step_stats* stats);

/* Runs one detection at the current state (ContactDetector::detectContacts,
 * contact_detector.cpp:71-211, activation margin = the model's delta) and
 * copies the contacts, sorted by (a,b), to host buffers of capacity cap.
 * pairs[2*i] = a, pairs[2*i+1] = b (a < b);
 * geom[12*i..] = point_a(3), point_b(3), normal(3), distance, surface_limit,
 *                type (0 P2P, 1 E2P, 2 E2E as double);
 * shift[3*i..] = minimum-image shift applied to body b.
 * Any of geom / shift may be NULL.  *n receives the contact count even when
 * it exceeds cap (then only cap are written and RG_ERR_CAPACITY returned). */
int rg_detect(rg_system* sys, double delta, int32_t* pairs, double* geom,
              double* shift, size_t cap, size_t* n);

/* Contacts / impulses of the last NSC velocity solve, sorted by (a,b):
 * lambda[3*i..] = (λn, λt1, λt2); color[i] = PSOR colour (may be NULL). */
int rg_get_impulses(const rg_system* sys, int32_t* pairs, double* lambda,
                    int32_t* color, size_t cap, size_t* n);

/* Contact network of the last NSC velocity solve, the rows
 * App::logNetworkFrame writes for NSC scenes (src/app/main.cpp:3620-3700,
 * header "frame,rod_i,rod_j,contact_x..z,normal_x..z,phi,lambda_n,
 * lambda_t1,lambda_t2,vn_pre,vn_post").  Export must be enabled (it keeps
 * each manifold's normal, r_a, r_b, phi and v_n_pre on the device, 88 B
 * per contact) before the steps whose network is wanted.  Sorted by (a,b):
 * pairs[2*i..] = (rod_i, rod_j); rows[12*i..] = contact point x_a + r_a at
 * the current state (3), normal (3), phi, lambda_n, lambda_t1, lambda_t2,
 * v_n before the solve, v_n at the current velocities.  Returns
 * RG_ERR_CAPACITY (with *n set) when cap is too small. */
int rg_set_network_export(rg_system* sys, int enable);
int rg_get_contact_network(const rg_system* sys, int32_t* pairs, double* rows, size_t cap, size_t* n);

/* Per-body force and torque of one force evaluation at the current state
 * (soft or HM model), without integrating: f[3N], tau[3N].  Advances the
 * tangential history exactly like one computeForces call of the reference. */
int rg_compute_forces(rg_system* sys, double* f, double* tau, double* pe);

/* Tangential-history table (HM: ξ per pair; Cundall: F_t per pair), sorted
 * by pair: pairs[2*i..], value[3*i..], last_frame[i] (may be NULL). */
int rg_get_history(const rg_system* sys, int32_t* pairs, double* value,
                   int64_t* last_frame, size_t cap, size_t* n);

/* Enables (1) or disables (0) the stage timers; resets the accumulators. */
int rg_set_profiling(rg_system* sys, int enable);
/* Accumulated milliseconds and launch counts per stage since enabling. */
int rg_get_profile(const rg_system* sys, double* ms, int64_t* launches);
/* Phase times of the persistent NSC step since enabling (ms, n <= 12):
 * 0 free flight, 1 detection, 2 colouring, 3 manifold rows, 4 PSOR,
 * 5 position update, 6 projection detection, 7 projection colouring,
 * 8 projection sweeps. */
int rg_get_phase_times(const rg_system* sys, double* ms, int n);

/* ---- seeded packings generated on the device ------------------------------ */
/* Replaces the host populate of the reference's scenes ("nonoverlap",
 * src/app/main.cpp:1857-2140): up to n rods of length L and diameter d in
 * the periodic cube [lo, lo+side)^3, centres uniform, axes uniform on S^2,
 * no two closer than d (nearest periodic image).  Parallel random
 * sequential addition: every unplaced rod draws candidates at once, each
 * round; overlapping survivors keep the lower index.  Stops when every rod
 * is placed or the first rod has used max_attempts draws (the host loop
 * stops at its first unplaceable rod too).  x[3n], q[4n] (w,x,y,z): HOST
 * outputs, placed rods first, in index order; *placed = their number.  The
 * packing depends only on the arguments (not on thread timing).  Needs
 * side >= 3 (L + d) (RG_ERR_ARG otherwise).  Allocates device scratch. */
int rg_scene_rsa_device(int n, double L, double d, double lo, double side, uint64_t seed, int max_attempts,
                        double* x, double* q, int* placed);

/* ---- detection without device allocation --------------------------------- */
/* No counterpart in the reference: this entry point exists for callers that
 * cannot call cudaMalloc themselves or let a library do it (code running
 * under another framework's device allocator or inside a fixed memory
 * budget).  It finds the contacts rg_detect finds - same pairs (a < b,
 * sorted), same geometry, bit for bit - from DEVICE buffers the caller
 * owns, and allocates nothing: all intermediate data lives in one fixed
 * file-scope __device__ array sized for RG_NOALLOC_MAX_BODIES bodies
 * (about 0.6 MB), which every GPU that loads the library keeps until the
 * process exits.
 *
 *   x[3n], q[4n] (w,x,y,z), radius[n], half_height[n]: device, AoS.
 *   inv_mass[n]: device or NULL (NULL: every body dynamic); pairs of two
 *     static bodies are skipped as in rg_detect.
 *   pbc_min / pbc_max: HOST arrays of 3 (ignored when pbc_enabled == 0).
 *   pairs[2*cap], geom[12*cap] (may be NULL): device outputs, layout of
 *     rg_detect; count[1]: device, receives the contact count even when it
 *     exceeds cap (then only the first cap contacts are written).  Unlike
 *     rg_detect, an overflow is NOT reported by the return code: the count
 *     is known only on the device, after the call has returned.  Read
 *     *count once the stream has synchronised and compare it with cap; a
 *     larger count means the list is truncated and the call must be
 *     repeated with more room.
 *   stream: a cudaStream_t (NULL: the default stream).  The call only
 *     enqueues work; synchronise the stream before reading the outputs.
 * Returns RG_ERR_CAPACITY when n > RG_NOALLOC_MAX_BODIES and RG_ERR_ARG for
 * bad arguments, before any device work.  The first call on a device looks
 * the scratch address up with cudaGetSymbolAddress (once per device, with
 * that device current); make that first call before any stream capture.
 * Every call on a device shares the one scratch array: calls that overlap
 * on the GPU (other streams, other host threads) race and must be
 * serialised by the caller. */
#define RG_NOALLOC_MAX_BODIES 8192
int rg_detect_noalloc(const double* x, const double* q, const double* radius,
                      const double* half_height, const double* inv_mass, int n,
                      int pbc_enabled, const double* pbc_min, const double* pbc_max,
                      double delta, int32_t* pairs, double* geom, int cap,
                      int32_t* count, void* stream);

/* ---- learned PSOR warm start ------------------------------------------- */
/* MLP 8 -> 128 -> 128 -> 128 -> 3 (SiLU), BF16 weights and activations,
 * FP32 accumulation.  Features per contact (in this order): gap φ, v_n,
 * v_t1, v_t2, previous λn, λt1, λt2 (0 when new), contact-graph degree.
 * Targets: converged (λn, λt1, λt2).  Weights are held by the system. */
#define RG_MLP_IN 8
#define RG_MLP_HIDDEN 128
#define RG_MLP_OUT 3
/* Number of float parameters: W1 128x8, b1, W2 128x128, b2, W3 128x128, b3,
 * W4 3x128, b4, then input mean/scale (8+8) and output scale (3). */
size_t rg_mlp_param_count(void);
int rg_mlp_set_params(rg_system* sys, const float* params, size_t n);
int rg_mlp_get_params(const rg_system* sys, float* params, size_t n);
/* Records (features, converged impulses) of every NSC step taken while
 * recording is on are appended to a device buffer of capacity cap records. */
int rg_mlp_record(rg_system* sys, int enable, size_t cap);
int rg_mlp_records(const rg_system* sys, float* features, float* targets,
                   size_t cap, size_t* n);
/* Trains on host records with the device forward/backward kernels (Adam,
 * FP32 master weights, BF16 copies for the GEMMs): initialises the
 * normalisation from the records and the weights from seed, then runs
 * `epochs` passes of shuffled minibatches of `batch` records.  final_loss is
 * the mean squared error of the last epoch in normalised units. */
int rg_mlp_train(rg_system* sys, const float* features, const float* targets,
                 size_t n, int epochs, int batch, float lr, uint64_t seed,
                 float* final_loss);
/* Loss and gradient (rg_mlp_param_count floats, parameter layout; the
 * normalisation entries get 0) of the current weights on n records, by the
 * same device kernels as one training step.  For gradient checks. */
int rg_mlp_grad(rg_system* sys, const float* features, const float* targets,
                size_t n, float* grad, float* loss);
/* Inference with the in-step tensor-core routine: out[3*n] = predicted
 * impulses (previous impulse + predicted change) for features[8*n]. */
int rg_mlp_infer(rg_system* sys, const float* features, float* out, size_t n);

/* ---- batched independent systems ---------------------------------------- */
/* A batch runs many independent periodic systems of uneven size in one
 * device step (one launch sequence, CUDA-graph captured).  Each member has
 * its own rg_config (box, model, dt, μ, ...).  Bodies of member k occupy
 * global indices [offset_k, offset_k + n_k). */
typedef struct rg_batch rg_batch;
int rg_batch_create(const rg_config* cfgs, int n_systems, rg_batch** out);
int rg_batch_destroy(rg_batch* b);
int rg_batch_set_bodies(rg_batch* b, int k, const double* radius,
                        const double* half_height, const double* mass,
                        const double* inertia, const double* restitution);
int rg_batch_set_state(rg_batch* b, int k, const double* x, const double* q,
                       const double* v, const double* w);
int rg_batch_get_state(const rg_batch* b, int k, double* x, double* q,
                       double* v, double* w);
/* nsteps steps of every member; per_system (optional) gets n_systems stats,
 * each with device_ms = the whole batch call. */
int rg_batch_step(rg_batch* b, int nsteps, rg_step_stats* per_system);
/* States of all members at once: x[3T], q[4T], v[3T], w[3T] (host arrays,
 * member k's rods after those of members 0..k-1, T = total rods); forces
 * and torques are cleared as rg_set_state does.  One transfer per array:
 * page-locked arrays move at full host-link speed. */
int rg_batch_set_state_all(rg_batch* b, const double* x, const double* q,
                           const double* v, const double* w);
int rg_batch_get_state_all(rg_batch* b, double* x, double* q, double* v,
                           double* w);
/* Loads the same network into every NSC member. */
int rg_batch_set_mlp(rg_batch* b, const float* params, size_t n);
int rg_batch_size(const rg_batch* b);
/* Member k as a system handle (all single-system calls apply; it shares
 * the batch's stream and is destroyed with the batch). */
rg_system* rg_batch_member(rg_batch* b, int k);
const char* rg_batch_last_error(const rg_batch* b);
/* Schedule of the persistent launch: NSC members of at least 1.5 R work
 * units get a team of round(work/R) blocks, the rest share single-block
 * teams (R = rods_per_block; 0 = all single-block).  A member's work is its
 * rod count until a call has timed its steps on the device, then that
 * measured cost converted to rods at the batch's mean cost per rod.
 * R = -1: balanced plan - each member's step on nb blocks is modelled as
 * s + p / nb (+ a measured team overhead for nb > 1) from its timed
 * single-block solves (s) and the rest of its single-block step (p), and
 * the smallest makespan that fits the blocks is chosen (all single-block
 * until every member has been timed on one block).
 * use_graph: replay the launch from a CUDA graph. */
int rg_batch_set_schedule(rg_batch* b, int rods_per_block, int use_graph);
int rg_batch_get_schedule(const rg_batch* b, int* rods_per_block, int* grid,
                          int* nteams);
/* The cost model: each member's measured device cost (block-milliseconds
 * per step, 0 before its first timed call) and its team's block count in
 * the current plan. */
int rg_batch_get_costs(const rg_batch* b, double* cost_ms, int* team_blocks);
/* Device time of each team of the last full plan's launch (ms), its block
 * count and member count; at most cap teams, *nteams gets the number. */
int rg_batch_get_team_times(const rg_batch* b, double* ms, int* blocks, int* members, int cap,
                            int* nteams);
/* Autotuner: measures every member's step cost (all single-block), then
 * times trial_steps steps per candidate R (-1: balanced) after two untimed
 * steps, from the current state (state put back after each trial), and
 * selects the fastest; ms_out (optional) gets n_cand times. */
int rg_batch_autotune(rg_batch* b, const int* candidates, int n_cand,
                      int trial_steps, int* best, double* ms_out);

#ifdef __cplusplus
}
#endif
#endif /* RODGPU_H */
