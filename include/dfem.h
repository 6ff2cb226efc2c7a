/*
 * dfem.h — C ABI of the B200 projective-dynamics (PD) engine.
 *
 * This is the drop-in boundary for the hot path of diff_fem: one time step of
 * local–global projective dynamics (corotated FEM tets, muscle segments,
 * attachments, cloth strain/bending springs, obstacle and soft-soft contact
 * with friction, underwater drag)
 * and the vector–Jacobian product (VJP) of that step.
 *
 * Conventions
 *  - Every entry point returns an int status (DFEM_OK == 0).  On failure the
 *    message is available from dfem_last_error() (thread-local).
 *  - All buffers are caller-owned.  Positions/velocities are interleaved FP64
 *    [x0 y0 z0 x1 y1 z1 ...] of length 3N, ordered as the scene descriptor
 *    lists its vertices (diff_fem: Meshes, then Clothes; obstacles excluded).
 *  - `mem` arguments say where a buffer lives: DFEM_MEM_HOST or DFEM_MEM_DEVICE
 *    (a pointer on the scene's CUDA device).
 *  - One CUDA stream per scene; no process-wide mutable state apart from the
 *    thread-local error string.
 *
 * The reference interface each entry point replaces is cited beside it
 * (paths relative to the diff_fem repository).
 */
#ifndef DFEM_H_
#define DFEM_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DFEM_ABI_VERSION 6

enum dfem_status {
  DFEM_OK = 0,
  DFEM_ERR_INVALID = 1,       /* bad argument / descriptor                       */
  DFEM_ERR_CUDA = 2,          /* CUDA runtime error                              */
  DFEM_ERR_FACTOR = 3,        /* Cholesky failed even after regularisation      */
  DFEM_ERR_NONFINITE = 4,     /* NaN/Inf met in a step (status word set on GPU)  */
  DFEM_ERR_STATE = 5,         /* call out of order (e.g. backward before forward)*/
  DFEM_ERR_CAP = 6,           /* a bounded loop or wait hit its cap              */
  DFEM_ERR_NOMEM = 7,         /* allocation failed                               */
  DFEM_ERR_UNSUPPORTED = 8    /* feature combination the engine does not serve   */
};

enum dfem_mem { DFEM_MEM_HOST = 0, DFEM_MEM_DEVICE = 1 };

enum dfem_precision {
  DFEM_PREC_FP64 = 0,   /* plain form: everything FP64                          */
  DFEM_PREC_MIXED = 1   /* FP32 tet SVD and per-constraint force slots; FP64
                           projection tail, slot sums, factor, solves, state,
                           contact phase and adjoint                            */
};

/*
 * Scene descriptor: plain arrays, read once by dfem_scene_create.
 * Replaces the scene assembly of Environment::Environment / Dfobj::Initialize /
 * Dfcloth::Initialize / World::AddBody / World::Initialize
 * (sim/Environment.h:86-225, sim/Dfobj.h:442-611, sim/Dfcloth.h:198-300,
 *  sim/fem/World.h:248-591).  Optional arrays may be NULL when their count is 0.
 */
typedef struct dfem_scene_desc {
  /* vertices */
  int32_t n_vertices;
  const double *x0;            /* 3N rest positions                                  */
  const double *mass;          /* N lumped masses (World::mUnitMass)                 */
  const uint8_t *gravity_mask; /* N flags: 1 = vertex receives gravity (NULL = all)  */

  /* corotated FEM tets (CorotateFEMConstraint) */
  int32_t n_tets;
  const int32_t *tets;         /* 4T vertex indices (re-oriented like Dfobj.h:474-487)*/
  const double *youngs;        /* T Young's moduli E                                  */
  const double *poisson;       /* T Poisson ratios nu                                 */

  /* attachments (AttachmentConstraint) */
  int32_t n_attach;
  const int32_t *attach_vertex;   /* n_attach                                       */
  const double *attach_target;    /* 3*n_attach target points                        */
  const double *attach_stiffness; /* n_attach                                        */

  /* muscle constraints (LinearMuscleConstraint), grouped into segments */
  int32_t n_muscle;
  const int32_t *muscle_tets;     /* 4*n_muscle                                      */
  const double *muscle_fiber;     /* 3*n_muscle unit fibre directions                */
  const double *muscle_stiffness; /* n_muscle: muscle stiffness x distance weight    */
  const int32_t *muscle_segment;  /* n_muscle segment ids in [0, n_segments)         */
  int32_t n_segments;             /* activation channels: muscle segments and the
                                     channels of pneumatic springs (spring_channel) */

  /* cloth strain springs (SpringConstraint) */
  int32_t n_springs;
  const int32_t *spring_vertices; /* 2*n_springs                                     */
  const double *spring_rest;      /* n_springs rest lengths (NULL = from x0)         */
  const double *spring_weight;    /* n_springs weights w (J and L use sqrt(w))       */
  const int32_t *spring_channel;  /* n_springs activation channels, or NULL: -1 = plain
                                     spring; c in [0, n_segments) = pneumatic spring
                                     (PneumaticConstraint, sim/fem/Constraint/
                                     pneumaticEasy.h:133-147) whose projection uses
                                     rest * activation[c] as its length             */

  /* cloth bending stencils (BendingConstraint): centre vertex then 1-ring in order */
  int32_t n_bending;
  const int32_t *bend_offsets;    /* n_bending+1 offsets into bend_vertices          */
  const int32_t *bend_vertices;   /* centre first, then the ring (>= 3 vertices)     */
  const double *bend_weight;      /* n_bending weights                               */

  /* contact: soft surface (vertices + faces, global vertex ids) and obstacles */
  int32_t n_contact_vertices;
  const int32_t *contact_vertices;
  int32_t n_contact_faces;
  const int32_t *contact_faces;   /* 3 per face, global vertex ids                   */
  int32_t n_obstacle_vertices;
  const double *obstacle_x;       /* 3 per obstacle vertex (static)                  */
  int32_t n_obstacle_faces;
  const int32_t *obstacle_faces;  /* 3 per face, obstacle vertex ids                 */

  /* parameters (Environment.h:108-155, World.h:216-235) */
  double time_step;               /* h = 1 / "Simulation HZ"                         */
  int32_t max_iterations;         /* "Max Iteration" K                               */
  double damping;                 /* "Damping coefficient"                           */
  double gravity[3];
  int32_t handle_collision;       /* "Handle collision"                              */
  int32_t self_collision;         /* "Self-collision": soft-soft contact between the
                                     contact vertices and the contact faces (every
                                     face vertex must be a contact vertex; single
                                     scenes, not batches)                          */
  double alpha;                   /* "World Alpha" relaxation of the contact rhs     */
  double friction;                /* "World Friction" (soft-soft contact mu)         */
  double obstacle_friction;       /* obstacle mu (diff_fem hardcodes 1)              */
  int32_t precision;              /* enum dfem_precision                             */
  int32_t checkpoint_every;       /* adjoint checkpoint interval in steps (>= 1)     */

  /* underwater drag and lift (Environment::Step underwater branch,
   * Dfobj::ComputeDragForces, sim/Environment.h:236-247, sim/Dfobj.h:904-998):
   * with underwater != 0 no vertex receives gravity and every drag face adds
   * its drag + lift force (computed from the step's start state) to its three
   * vertices as the external force of World::TimeStepping */
  int32_t underwater;             /* "Is underwater"                                 */
  int32_t n_drag_faces;
  const int32_t *drag_faces;      /* 3 per face, global vertex ids, outward winding  */

  /* articulated skeleton ("Bones", read by Dfobj.h:254-288 into Link objects,
   * sim/constants.h:28-247, registered by World::AddBody, World.h:499-545):
   * link 0 is the one root (DFEM_JOINT_ALL: 6 dofs, a linearised rotation w
   * and a translation l); every other link has a parent of lower index and
   * one dof (DFEM_JOINT_ROTATIONAL: an angle about its axis;
   * DFEM_JOINT_PRISMATIC: a distance along it).  The vertices of a link move
   * rigidly with it; the other vertices are solved with the links through
   * the Schur complement of World::ComputeSolution (World.h:1600-1670).
   * Single FP64 scenes without contact.  dfem_step_backward differentiates
   * through the links too: dfem_set_joint_state_grad /
   * dfem_get_joint_state_grad carry the joint state's cotangents. */
  int32_t n_links;
  const int32_t *link_parent;     /* parent link, -1 for link 0                       */
  const int32_t *link_type;       /* enum dfem_joint                                  */
  const double *link_joint;       /* 3 per link: "Joint Pos"                          */
  const double *link_axis;        /* 3 per link: unit "Joint Axis" (root: unused)    */
  const int32_t *link_offsets;    /* n_links+1 offsets into link_vertices             */
  const int32_t *link_vertices;   /* the links' vertices (each in at most one link)   */
  const int32_t *link_channel;    /* n_links activation channels of the joint torques
                                     (World::mJointTorque, World.h:1638-1640) of the
                                     non-root links, -1 = none (NULL = none)       */
} dfem_scene_desc;

/* Joint types of the skeleton links (Link::JointType). */
enum dfem_joint { DFEM_JOINT_PRISMATIC = 0, DFEM_JOINT_ROTATIONAL = 1, DFEM_JOINT_ALL = 2 };

typedef struct dfem_scene dfem_scene;  /* opaque */

typedef struct dfem_scene_info {
  int32_t n_vertices, n_tets, n_attach, n_muscle, n_springs, n_bending;
  int32_t n_supernodes, n_levels;      /* supernodal Cholesky of the N x N matrix Hs */
  int64_t nnz_factor;                  /* stored entries of the Cholesky factor      */
  int32_t n_slots;                     /* per-constraint vertex slots of J*d         */
  int32_t device;
  double factor_regularisation;        /* 0 unless the retry loop added reg * I      */
} dfem_scene_info;

/* Build a scene on `device`: precomputation of J, L, H = M/h^2 + L and its
 * prefactorisation.  Replaces World::Initialize + World::PreComputation +
 * World::FactorizeLDLT (sim/fem/World.h:248-384, 1089-1139, 1212-1232). */
int dfem_scene_create(const dfem_scene_desc *desc, int device, dfem_scene **out);

/* A batch: n_scenes independent scenes stepped together as one handle.  The
 * parts are the disjoint union of the scenes: every per-vertex, per-tet and
 * per-segment array of the other calls (x, v, traj_x, youngs, poisson,
 * activations rows, gradients) is the concatenation of the scenes' arrays in
 * the given order.  Every part keeps its own convergence test and iteration
 * count (one World each, as a loop over scenes in the reference would run
 * them), its own factor and its own regularisation retry; the triangular
 * solves of all parts share one level schedule.  The scenes must share
 * time_step, damping, gravity, max_iterations, precision and
 * checkpoint_every; obstacle contact is not supported in a batch.  Parts
 * may mix underwater and dry scenes: drag faces stay with their part's
 * vertices, and gravity follows each part's own underwater flag. */
int dfem_scene_create_batch(const dfem_scene_desc *descs, int32_t n_scenes, int device, dfem_scene **out);

/* Part layout of a scene handle (a single scene is one part).  The offset
 * arrays (n_parts + 1 entries each; may be NULL) receive the first vertex,
 * tet and muscle segment of every part. */
int dfem_batch_layout(const dfem_scene *scene, int32_t *n_parts, int32_t *vertex_offsets,
                      int32_t *tet_offsets, int32_t *segment_offsets);

int dfem_scene_destroy(dfem_scene *scene);
int dfem_scene_get_info(const dfem_scene *scene, dfem_scene_info *info);

/* Per-tet materials; refactors H.  Replaces the COROTATE parameter update +
 * PreComputation of forward_all (python/pydifem.cc:207-221). */
int dfem_set_materials(dfem_scene *scene, const double *youngs, const double *poisson, int mem);

/* Muscle activation per segment for the next forward call(s).  Replaces
 * MuscleSegment::SetActivationLevel (sim/MuscleSegment.h:72-78). */
int dfem_set_activations(dfem_scene *scene, const double *activations, int mem);

/* Skeleton joint state (World::mJointQ / mJointQd as Link::WriteT lays them
 * out, sim/constants.h:206-221): the root's T (R row-major, 9 values; d, 3)
 * then the magnitude of every other link; jqd holds the previous step's
 * values (prevTr, prevmag).  12 + n_links - 1 doubles each (host memory).
 * dfem_step_forward starts from this state and leaves its end state here
 * (Link::ReadT / WriteT around every step, World.h:681-682,712-713).  A new
 * scene starts from the identity and zero magnitudes. */
int dfem_set_joint_state(dfem_scene *scene, const double *jq, const double *jqd);
int dfem_get_joint_state(const dfem_scene *scene, double *jq, double *jqd);

/* Cotangents dL/djq, dL/djqd of the joint state after the last forward's
 * final step, for the next dfem_step_backward only (without this call they
 * are zero); after it, dfem_get_joint_state_grad reads dL/djq, dL/djqd of the
 * joint state the forward started from.  The dldjq / dldjqd inputs and the
 * ansjq / ansjqd outputs of backward_act (python/pydifem.cc:91-180).  The
 * joint torques' gradient is the one of their activation channels. */
int dfem_set_joint_state_grad(dfem_scene *scene, const double *gjq, const double *gjqd);
int dfem_get_joint_state_grad(const dfem_scene *scene, double *gjq, double *gjqd);

/* Run n_steps time steps from (x, v); writes the final state, and optionally
 * every step's positions to traj_x ((n_steps) * 3N, may be NULL).
 * `activations`, if non-NULL, holds n_steps * n_segments values (one row per
 * step) and overrides dfem_set_activations for this call.
 * Records checkpoints so that dfem_step_backward can follow.
 * Replaces Environment::Step + World::TimeStepping + ProjectiveDynamicsMethod
 * (sim/Environment.h:228-293, sim/fem/World.h:673-1029) as driven by
 * forward_act / forward_all (python/pydifem.cc:39-86, 183-259). */
int dfem_step_forward(dfem_scene *scene, const double *x, const double *v,
                      const double *activations, int32_t n_steps,
                      double *x_out, double *v_out, double *traj_x, int mem);

/* VJP of the last dfem_step_forward call: given dL/dx_out and dL/dv_out,
 * writes dL/dx, dL/dv (3N each), dL/dE and dL/dnu per tet (may be NULL) and
 * dL/dactivation (n_steps * n_segments, may be NULL).
 * Replaces the CppAD tape + ADFun::Jacobian of backward_act / backward_all
 * (python/pydifem.cc:91-180, 262-301). */
int dfem_step_backward(dfem_scene *scene, const double *gx_out, const double *gv_out,
                       double *gx, double *gv, double *g_youngs, double *g_poisson,
                       double *g_activations, int mem);

/* The local step alone at positions x (3N, user order): every constraint's
 * projection d(x) and jd_out = J d(x) (3N, user order), i.e. the ori_c - b
 * of one PD iteration.  Uses the segment activations of dfem_set_activations.
 * Replaces World::EvaluateDVector + mJ * d (sim/fem/World.h:898-901,1194-1210). */
int dfem_eval_local(dfem_scene *scene, const double *x, double *jd_out, int mem);

/* Corotated-tet local step (J d of FEM tets) for callers that cannot allocate
 * device memory — e.g. code that must hand the library only pre-allocated
 * buffers from a pool owning the device heap, or a path where a cudaMalloc
 * would stall other work.  No counterpart in the reference.
 *
 * Allocates nothing: x (3N), tets (4T, already re-oriented), inv_dm (9T,
 * row-major Dm^-1 per tet), w_rot = mu*vol and w_vol = nu*mu*vol (T each),
 * the vertex -> (4*tet + corner) incidence CSR vtx_ptr (N+1) / vtx_slot (4T)
 * and jd_out (3N) are caller-owned device buffers; the work is enqueued on
 * `stream` (a cudaStream_t, NULL = default stream) and not waited for.
 * The per-(tet, corner) scratch is a static device array of
 * DFEM_NOALLOC_MAX_TETS * 12 doubles (6 MiB) that every GPU loading the
 * library holds until exit; n_tets above the limit is rejected with
 * DFEM_ERR_INVALID.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make it before any stream capture; the
 * address is kept for the life of the process, so a cudaDeviceReset between
 * calls is not supported.  All calls share the array: calls that overlap on
 * the GPU race.
 * Index ranges: tets entries in [0, n_vertices); vtx_ptr non-decreasing from
 * 0 to at most 4*n_tets; vtx_slot entries in [0, 4*n_tets).  The device skips
 * an index out of range (the affected outputs become NaN) and records it; the
 * next call on the device then first waits for `stream`, and returns
 * DFEM_ERR_INVALID (clearing the record).  Each call therefore also waits
 * for the work queued on `stream` before it, not for its own. */
#define DFEM_NOALLOC_MAX_TETS 65536
int dfem_eval_corotated_noalloc(int32_t n_vertices, int32_t n_tets, const double *x, const int32_t *tets,
                                const double *inv_dm, const double *w_rot, const double *w_vol,
                                const int32_t *vtx_ptr, const int32_t *vtx_slot, double *jd_out, void *stream);

/* Contact passes (detection rounds that found impacts) of each step of the
 * last forward call, host buffer of n values (0 without obstacle contact).
 * The loop of World::ProjectiveDynamicsMethod (sim/fem/World.h:928-1022). */
int dfem_get_contact_passes(const dfem_scene *scene, int32_t *passes, int32_t n);

/* Iteration counts of the last forward call: n steps x n_parts values
 * (row per step), host buffer. */
int dfem_get_iterations(const dfem_scene *scene, int32_t *iters, int32_t n);

/* Host-only diagnostic, needs no GPU: builds the scene's fill-reducing
 * ordering and supernodal Cholesky factor of Hs = M/h^2 + L_s on the host and
 * solves Hs X = B for 3 interleaved right-hand sides (3N, user vertex order).
 * `info` (may be NULL) receives the factor statistics.  Same role as
 * World::PreComputation + mDynamicSolver.solve (sim/fem/World.h:1089-1139,1660). */
int dfem_host_factor_solve(const dfem_scene_desc *desc, const double *b, double *x, dfem_scene_info *info);

/* The global solve's form.  request: -1 query, 0 autotune (time every form
 * on this scene's factor and keep the fastest; done once at creation),
 * 1 level kernels (one launch per elimination-tree level, launch class and
 * direction), 2 persistent (both triangular sweeps in one launch, supernodes
 * claimed in dependency order), 3 split (the levels below the autotuned cut
 * level as level kernels, the rest in one persistent launch), 4 cluster
 * (one thread-block cluster walks the levels, a cluster barrier between
 * levels; tried for factors of up to 4096 supernodes), 5 resident (single
 * scenes whose factor fits the shared memory of one thread-block cluster of
 * up to 16 CTAs: every block stays in shared memory for the launch,
 * contributions and solution values move between the CTAs over distributed
 * shared memory, a cluster barrier between levels), 6 dense (single scenes
 * of at most 4,096 vertices: X = Hs^-1 is formed from the factor after every
 * refactorisation, N_p^2 doubles twice with N_p = N rounded up to 64, and a
 * solve is one product with X; the autotune keeps it when its saving over
 * 100 solves exceeds the rebuild); a form requested with
 * 1-6 is used in every iteration (no per-iteration selection, see
 * dfem_solve_select).  *chosen (may
 * be NULL) receives the form in use (1-6), ms (may be NULL, 2 values)
 * the last autotune's time per solve of forms 1 and 2.  Forms 1-5 run the
 * same arithmetic per supernode: their results are identical; form 6 agrees
 * with them to rounding (and is deterministic).  No counterpart in
 * the reference (its solve is Eigen's SimplicialLDLT, sim/fem/World.h:1660). */
int dfem_solve_mode(dfem_scene *scene, int32_t request, int32_t *chosen, double *ms);

/* The last autotune's time per solve (ms) of the level-kernel, persistent,
 * best split, cluster, resident and dense forms (0: not timed), then the
 * time to build the dense form's inverse; writes the first min(n, 7). */
int dfem_solve_times(const dfem_scene *scene, double *ms, int32_t n);

/* The split form found by the last autotune: *cut_level (0: none), the
 * factor's number of levels, and its time per solve (ms). */
int dfem_solve_split(const dfem_scene *scene, int32_t *cut_level, int32_t *n_levels, double *ms_split);

/* Batches, after an autotune: the solve of an iteration takes the persistent
 * form when the parts still iterating hold less than *weight_threshold of the
 * factor's entries (*on = 1; 0: the tuned form in every iteration, as after an
 * explicit form request).  ms_one_part (may be NULL, 2 values): time per solve
 * with only the largest part active, tuned form and persistent form. */
int dfem_solve_select(const dfem_scene *scene, int32_t *on, double *weight_threshold, double *ms_one_part);

/* CUDA-event timing of every launch of the level-kernel solve form (a level
 * of the elimination tree, split into its small and its large supernodes;
 * forward and backward, `reps` launches each on the scene's stream, ms per
 * launch).  *n_segments receives the launch count per direction; the arrays
 * (cap entries each, may be NULL to query the count) receive the times, the
 * supernodes, the level of each launch and its CTA sizes (2 per launch:
 * forward, backward).  Instrumentation; no counterpart in the reference. */
int dfem_profile_levels(dfem_scene *scene, int32_t reps, int32_t cap, int32_t *n_segments, double *ms_fwd,
                        double *ms_bwd, int32_t *n_supernodes, int32_t *level, int32_t *threads);

/* Device memory (bytes) the adjoint may spend on storing the PD iterates of
 * every step of a forward call (default: 45 % of the device's memory, at most 60 % of the
 * memory free when the scene is made).  Within it the adjoint
 * replays no step (except steps with contact, whose contact iterations it
 * records on a replay); beyond it every step is recomputed from its
 * checkpoint.  Results are identical either way.  Invalidates the recorded
 * forward call.  No counterpart in the reference (its CppAD tape stores
 * everything). */
int dfem_set_adjoint_budget(dfem_scene *scene, int64_t bytes);

/* Number of kernels this scene has launched so far (CUDA-graph nodes counted
 * individually).  Instrumentation; no counterpart in the reference. */
int dfem_get_launch_count(const dfem_scene *scene, int64_t *count);

/* CUDA-event timing of the step's phases on the scene's stream, each phase
 * launched `reps` times after one warm-up on the state of the last forward
 * call: ms[0] local step (projection + J*d slots), ms[1] rhs gather,
 * ms[2] one full triangular solve (all levels, both sweeps), ms[3] adjoint
 * local step.  Instrumentation (diff_fem's TIMER_* macros, sim/utils/timer.h). */
int dfem_profile_phases(dfem_scene *scene, int32_t reps, double *ms);

/* Bounds of the engine's capped loops and waits, lowered for a scene (tests
 * of the failure paths, or a caller that wants a tighter bound); value < 0
 * restores the built-in cap, values above it are rejected.  When a bound is
 * reached the call that met it returns DFEM_ERR_CAP (the kernels finish
 * normally; the handle stays usable) and its results are not valid.
 *   DFEM_LIMIT_CONTACT_PASSES           detection passes of a step's contact
 *                                       phase that may still find new impacts
 *                                       (0..64; the reference's loop is uncapped,
 *                                       sim/fem/World.h:928-1022)
 *   DFEM_LIMIT_IMPACTS_PER_VERTEX       obstacle faces a contact vertex may hit (0..8)
 *   DFEM_LIMIT_SOFT_IMPACTS_PER_VERTEX  soft faces a contact vertex may hit in a step (0..16)
 *   DFEM_LIMIT_GROUP_MEMBERS            members of one soft-contact face group (0..32)
 *   DFEM_LIMIT_SOLVE_WAIT_POLLS         polls of a dependency wait of the persistent
 *                                       solve form (1..2^22)
 *   DFEM_LIMIT_BROAD_PHASE_CELLS        grid cells a contact vertex's swept box may
 *                                       cover in the obstacle detection's broad phase
 *                                       before the vertex tests every obstacle face
 *                                       (0..4096, default 64; 0: no broad phase).
 *                                       Never an error: results are identical either way.
 * No counterpart in the reference. */
enum dfem_limit {
  DFEM_LIMIT_CONTACT_PASSES = 0,
  DFEM_LIMIT_IMPACTS_PER_VERTEX = 1,
  DFEM_LIMIT_SOFT_IMPACTS_PER_VERTEX = 2,
  DFEM_LIMIT_GROUP_MEMBERS = 3,
  DFEM_LIMIT_SOLVE_WAIT_POLLS = 4,
  DFEM_LIMIT_BROAD_PHASE_CELLS = 5
};
int dfem_set_limit(dfem_scene *scene, int32_t which, int64_t value);

/* Execution options of a scene; results are identical under every setting.
 *   DFEM_OPTION_FUSED_CONTACT  1 (default for single scenes): a step's obstacle
 *                              contact phase (scenes without soft-soft contact)
 *                              runs as one cooperative launch with grid-wide
 *                              barriers between its detection and Jacobi phases;
 *                              0 (default for batches): as a conditional graph
 *                              loop of kernels (batches: gated per scene).
 *   DFEM_OPTION_SPLIT_FACTOR   1 (default): the refactorisation runs the levels
 *                              of few supernodes split over launches (several
 *                              CTAs per supernode); 0: one CTA per supernode
 *                              everywhere.  Applies from the next
 *                              refactorisation (dfem_set_materials).
 *   DFEM_OPTION_GATHER         0 (default): the per-vertex sums of the local
 *                              step's slots one warp per vertex below 65,536
 *                              vertices, one thread per vertex from there; 1:
 *                              one warp per vertex; 2: one thread per vertex.
 * No counterpart in the reference. */
enum dfem_option { DFEM_OPTION_FUSED_CONTACT = 0, DFEM_OPTION_SPLIT_FACTOR = 1, DFEM_OPTION_GATHER = 2 };
int dfem_set_option(dfem_scene *scene, int32_t which, int64_t value);

/* Failure injection for tests: the calling thread's device allocations by the
 * engine fail (DFEM_ERR_NOMEM) once `after` more have succeeded; after < 0
 * turns it off.  Thread-local; no counterpart in the reference. */
int dfem_debug_fail_allocations(int64_t after);

/* Synchronise the scene's stream. */
int dfem_synchronize(dfem_scene *scene);

/*
 * Asynchronous per-step OBJ output.  Replaces Environment::SaveObj / Save
 * (sim/Environment.h:295-327): for every body, `prefix + suffix[b]` receives
 * "v %06f %06f %06f" lines for the body's vertices and "f %d %d %d" lines
 * (1-based) for its surface faces.  dfem_obj_writer_enqueue copies the state
 * into one of `depth` staging slots (pinned host memory when a device is
 * present) and returns; a host thread formats and writes the files.  A
 * device state is copied on the scene's stream after the work already queued
 * there (the step that produced it), so the writes overlap the next steps.
 * Enqueue blocks only while every slot is in flight.
 */
typedef struct dfem_obj_writer dfem_obj_writer;  /* opaque */

/* Bodies: vertex_offsets (n_bodies+1) into the 3N state (user order),
 * face_offsets (n_bodies+1) into faces (3 body-local vertex ids each),
 * suffixes (n_bodies file-name suffixes, e.g. "_DfObj0.obj"). */
int dfem_obj_writer_create(int32_t n_bodies, const int32_t *vertex_offsets, const int32_t *face_offsets,
                           const int32_t *faces, const char *const *suffixes, int32_t depth,
                           dfem_obj_writer **out);
/* Queue one state x (3 * vertex_offsets[n_bodies] doubles; mem: enum
 * dfem_mem; a device state needs `scene`, whose stream orders the copy). */
int dfem_obj_writer_enqueue(dfem_obj_writer *writer, dfem_scene *scene, const char *prefix, const double *x, int mem);
/* Wait until every queued state is written; returns the first write error. */
int dfem_obj_writer_flush(dfem_obj_writer *writer);
int dfem_obj_writer_destroy(dfem_obj_writer *writer);

/* Last error message of the calling thread ("" if none). */
const char *dfem_last_error(void);

/* ABI version (DFEM_ABI_VERSION). */
int dfem_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DFEM_H_ */
