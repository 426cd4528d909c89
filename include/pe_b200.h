/*
 * pe_b200.h -- C ABI of the B200 rigid-body time step (libpe_b200.so).
 *
 * The library owns device memory and one CUDA stream per context.  Host arrays passed in are
 * copied; the caller keeps ownership.  Device memory comes from a stream-ordered pool per device
 * that keeps what destroyed contexts free, so a new context reuses it instead of mapping fresh
 * pages; pe_b200_release_memory hands the kept memory back to the device.  Every entry point returns a pe_b200_status; no C++
 * exception crosses this boundary.  A context is used by one host thread at a time.
 *
 * Each entry point replaces a piece of pe's compile-time plugin boundary (the
 * CollisionSystem<Config> specialisation selected by pe_CONSTRAINT_SOLVER,
 * pe/config/Collisions.h:90, pe/core/Configuration.h:84) and of the body/world API that feeds
 * it; the reference interface is cited beside each declaration (paths relative to pe's root).
 *
 * Body order: spheres are identified by their index in the arrays given to
 * pe_b200_upload_bodies (pe's creation order, hence pe's system-id order).  Walls (planes, then
 * boxes) follow the spheres in the id space used for contacts: id n + k for wall k.
 */
#ifndef PE_B200_H
#define PE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PE_B200_OK = 0,
    PE_B200_ERR_ARG = 1,       /* invalid argument (pe: std::invalid_argument) */
    PE_B200_ERR_CAPACITY = 2,  /* a buffer capacity was exceeded */
    PE_B200_ERR_NAN = 3,       /* non-finite state detected */
    PE_B200_ERR_TIMEOUT = 4,   /* a bounded device wait gave up */
    PE_B200_ERR_CUDA = 5,      /* CUDA runtime error */
    PE_B200_ERR_STATE = 6,     /* call out of order (e.g. step before upload) */
    PE_B200_ERR_NOMEM = 7,     /* device or host allocation failed */
    PE_B200_ERR_UNSUPPORTED = 8 /* model not supported (pe: std::runtime_error,
                                   HardContactSemiImplicitTimesteppingSolvers.h:1926) */
} pe_b200_status;

typedef enum {
    PE_B200_DEM = 0,    /* pe::response::DEMSolver (pe/core/collisionsystem/DEMSolver.h) */
    PE_B200_HCSITS = 1  /* pe::response::HardContactSemiImplicitTimesteppingSolvers */
} pe_b200_solver;

typedef enum {
    PE_B200_FP64 = 0,   /* everything in FP64, as pe's default real (pe/config/Precision.h) */
    PE_B200_MIXED = 1   /* FP64 positions; FP32 velocities, detection, forces and NBGS updates */
} pe_b200_precision;

typedef enum {
    /* pe's RelaxationModel, HardContactSemiImplicitTimesteppingSolvers.h:172-179 */
    PE_B200_INELASTIC_FRICTIONLESS = 0,
    PE_B200_APPROX_INELASTIC_COULOMB_DECOUPLING = 1,
    PE_B200_APPROX_INELASTIC_COULOMB_ORTHOGONAL_PROJECTIONS = 2,
    PE_B200_INELASTIC_COULOMB_DECOUPLING = 3,
    PE_B200_INELASTIC_COULOMB_ORTHOGONAL_PROJECTIONS = 4,
    PE_B200_INELASTIC_GENERALIZED_MAX_DISSIPATION = 5
} pe_b200_relaxation_model;

typedef struct {
    int32_t solver;            /* pe_b200_solver */
    int32_t precision;         /* pe_b200_precision */
    int32_t relaxation_model;  /* pe_b200_relaxation_model (HCSITS only) */
    int32_t max_iterations;    /* HCSITS sweeps per step; pe default 100 (HCSITS.h:421) */
    double erp;                /* HCSITS error reduction; pe default 0.7 (HCSITS.h:420) */
    double gravity[3];         /* World::setGravity (pe/core/World.h:754); default 0 */
    double damping;            /* World::setDamping, 1 = no drag (src/core/Settings.cpp:47) */
    int32_t device;            /* CUDA device ordinal */
    int32_t track_orientation; /* 1: integrate sphere quaternions (Default.h:190-193) */
    int64_t max_contacts;      /* HCSITS contact capacity; 0 = automatic (8 per sphere).
                                  DEM lists: initial capacity in entries (grown on demand);
                                  0 = automatic (16 per sphere); at most INT32_MAX */
    double skin;               /* DEM neighbour-list skin; <= 0: 0.1 x the smallest radius */
    int32_t neighbor_lists;    /* DEM: 1 = Verlet lists rebuilt on demand (default),
                                  0 = grid search every step */
    int32_t force_model;       /* DEM normal force law, pe's DEMConfig forceModel
                                  (pe/config/DEMConfig.h, pe/core/response/ForceModel.h):
                                  0 = linear spring-dashpot ('basic'), 1 = extended Hertz for
                                  sphere-sphere contacts ('hertz'; walls stay linear) */
} pe_b200_params;

/* createMaterial argument list, src/core/Materials.cpp:175 */
typedef struct {
    double density, cor, csf, cdf, poisson, young, stiffness, dampingN, dampingT;
} pe_b200_material;

typedef struct pe_b200_ctx pe_b200_ctx;

/* Fills *p with pe's defaults (zero gravity, no drag, DEM, FP64, 100 sweeps, erp 0.7).
 * Replaces: the compile-time defaults of the collision system constructors
 * (pe/core/collisionsystem/DEMSolver.h:340ff, HCSITS.h:408-426) and Settings (Settings.cpp:46-48). */
void pe_b200_default_params(pe_b200_params *p);

/* Creates a context (device buffers are allocated on upload).
 * Replaces: CollisionSystem<Config>::CollisionSystem() / theCollisionSystem()
 * (pe/core/CollisionSystem.h, DEMSolver.h:340, HCSITS.h:408). */
int pe_b200_create(const pe_b200_params *p, pe_b200_ctx **out);

/* Releases the context and all its device memory.
 * Replaces: CollisionSystem<Config>::~CollisionSystem (DEMSolver.h:441). */
int pe_b200_destroy(pe_b200_ctx *ctx);

/* Returns the device memory the library keeps for reuse on `device` (the buffers of destroyed
 * contexts) to the device; live contexts keep theirs.  No pe counterpart (pe allocates on the
 * host with new/delete). */
int pe_b200_release_memory(int32_t device);

/* Human-readable text of the last error on this context ("" if none). */
const char *pe_b200_last_error(const pe_b200_ctx *ctx);

/* Updates gravity and drag.  Replaces: World::setGravity / World::setDamping
 * (pe/core/World.h:736-767). */
int pe_b200_set_gravity(pe_b200_ctx *ctx, const double g[3]);
int pe_b200_set_damping(pe_b200_ctx *ctx, double damping);

/* HCSITS runtime setters.  Replace: setMaxIterations / setRelaxationModel /
 * setErrorReductionParameter (HardContactSemiImplicitTimesteppingSolvers.h:793, 814, 835). */
int pe_b200_set_max_iterations(pe_b200_ctx *ctx, int32_t n);
int pe_b200_set_relaxation_model(pe_b200_ctx *ctx, int32_t model);
int pe_b200_set_error_reduction(pe_b200_ctx *ctx, double erp);

/* Material table (validated like createMaterial, src/core/Materials.cpp:180-207).
 * Replaces: createMaterial / Material::get*(m1, m2) composition (pe/core/Materials.h:468-715). */
int pe_b200_set_materials(pe_b200_ctx *ctx, int32_t n, const pe_b200_material *m);

/* Fixed walls of scene `scene`: planes (4 doubles each: unit normal, displacement d with
 * n.x = d on the plane) and boxes (15 doubles each: centre, side lengths, row-major rotation).
 * Replaces: createPlane (src/core/rigidbody/Plane.cpp:1202) and createBox + setFixed
 * (src/core/rigidbody/Box.cpp:1312). */
int pe_b200_set_walls(pe_b200_ctx *ctx, int32_t scene, int32_t nplanes, const double *planes,
                      const int32_t *plane_mat, int32_t nboxes, const double *boxes,
                      const int32_t *box_mat);

/* Uploads the spheres of every scene at once: n spheres, interleaved xyz vectors, radii,
 * material ids and scene ids (scene may be NULL: all in scene 0).  nscenes scenes.
 * Replaces: createSphere (src/core/rigidbody/Sphere.cpp:1187) + setLinearVel/setAngularVel,
 * World::add -> CollisionSystem::add (src/core/World.cpp:262-277, DEMSolver.h:988-1008). */
int pe_b200_upload_bodies(pe_b200_ctx *ctx, int64_t n, const double *x, const double *v,
                          const double *w, const double *r, const int32_t *mat,
                          const int32_t *scene, int32_t nscenes);

/* Moving (non-fixed) boxes, after pe_b200_upload_bodies (which removes them again): m boxes,
 * centres x (3 each), orientations q (4 each, unit quaternion w x y z), linear and angular
 * velocities v, w (3 each), side lengths (3 each, > 0), material ids, scene ids (NULL: scene 0;
 * otherwise grouped by scene, non-decreasing).  FP64 contexts only (PE_B200_ERR_UNSUPPORTED
 * otherwise).  In contact ids box k is n + (all planes) + (all fixed boxes) + k, as if created
 * in pe after the fixed boxes.
 * Replaces: createBox + setOrientation / setLinearVel / setAngularVel for a box that is not fixed
 * (src/core/rigidbody/Box.cpp:1312-1330, 289-336).  The step then adds pe's box contacts
 * (MaxContacts.h:589-668 sphere/box, 867-2250 box/box, 2380-2528 box/plane), BoxTrait::move
 * (boxtrait/Default.h:149-220) for DEM and the box bodies of the hard-contact solver; the DEM
 * step runs on the cell grid (no neighbour lists) while boxes are present. */
int pe_b200_upload_boxes(pe_b200_ctx *ctx, int32_t m, const double *x, const double *q,
                         const double *v, const double *w, const double *lengths,
                         const int32_t *mat, const int32_t *scene);
/* Current state of the moving boxes (any pointer may be NULL).  Replaces: Box::getPosition /
 * getQuaternion / getLinearVel / getAngularVel. */
int pe_b200_download_boxes(pe_b200_ctx *ctx, double *x, double *q, double *v, double *w);
/* Number of moving boxes (-1 for a NULL context). */
int32_t pe_b200_box_count(const pe_b200_ctx *ctx);

/* Overwrites positions/velocities of the uploaded spheres (same order; any pointer may be NULL
 * to keep that field).  Replaces: RigidBody::setPosition / setLinearVel / setAngularVel. */
int pe_b200_set_state(pe_b200_ctx *ctx, const double *x, const double *v, const double *w);

/* Overwrites the orientations of the uploaded spheres (4 doubles each, unit quaternion w x y z,
 * upload order; they start as the identity).  Contexts created with track_orientation = 1 only
 * (PE_B200_ERR_STATE otherwise).  Replaces: RigidBody::setOrientation
 * (src/core/rigidbody/Sphere.cpp:319-332). */
int pe_b200_set_orientations(pe_b200_ctx *ctx, const double *q);

/* Advances every scene by nsteps steps of size dt.
 * Replaces: World::simulationStep (src/core/World.cpp:330-357) ->
 * CollisionSystem::simulationStep (DEMSolver.h:1155-1262, HCSITS.h:1472-1520).
 * dt <= 0 is rejected with PE_B200_ERR_ARG as World.cpp:333-334 throws. */
int pe_b200_step(pe_b200_ctx *ctx, int32_t nsteps, double dt);

/* Downloads sphere state in upload order (any pointer may be NULL).
 * Replaces: RigidBody::getPosition / getLinearVel / getAngularVel / getQuaternion. */
int pe_b200_download_bodies(pe_b200_ctx *ctx, double *x, double *v, double *w, double *q);

/* Contacts of the current state (detection only, no response), sorted by (b1, b2):
 * ids (2 per contact, wall k has id n + k of its scene's wall list), and 7 doubles per contact
 * (contact point xyz, normal xyz from body 2 to body 1, signed distance).  *n_out receives the
 * total count; at most cap records are written (ids/geom may be NULL when cap is 0).
 * Replaces: HashGrids::findContacts + MaxContacts::collide
 * (pe/core/detection/coarse/HashGrids.h:1121, pe/core/detection/fine/MaxContacts.h:242). */
int pe_b200_find_contacts(pe_b200_ctx *ctx, int64_t cap, int64_t *ids, double *geom,
                          int64_t *n_out);

/* Statistics of the last step: number of contacts, number of colours (HCSITS), the L-inf
 * impulse change of the last sweep (pe's delta_max, HCSITS.h:1893-1946) and the complementarity
 * residual of the final impulses in velocity units (computed in FP64 when requested by
 * pe_b200_set_residual(ctx, 1); otherwise -1; a tangential impulse within 1e-9 of the friction
 * cone, 1e-5 for FP32 impulses, counts as on the cone). */
int pe_b200_last_step_stats(pe_b200_ctx *ctx, int64_t *ncontacts, int32_t *ncolors,
                            double *delta_max, double *residual);
int pe_b200_set_residual(pe_b200_ctx *ctx, int32_t enabled);

/* Reverse-mode gradients of the FP64 DEM step (no counterpart in pe, which has no gradients).
 * pe_b200_adjoint_forward runs nsteps steps of size dt from the current state (the grid-search
 * DEM step, FP64, orientation tracking off), keeping a checkpoint every `checkpoint_every`
 * steps; the context is left at the final state.  pe_b200_adjoint_backward takes the gradient
 * of a loss with respect to the final state (gx, gv, gw: 3n doubles each, upload order),
 * recomputes each segment from its checkpoint and returns the gradient with respect to the
 * initial positions, velocities and angular velocities, and in gparams (4 doubles, may be NULL)
 * the derivative with respect to the contact coefficients k_n, c_n, c_t and mu, each summed over
 * all contacts (for one material: the derivative with respect to that composed coefficient). */
int pe_b200_adjoint_forward(pe_b200_ctx *ctx, int32_t nsteps, double dt, int32_t checkpoint_every);
int pe_b200_adjoint_backward(pe_b200_ctx *ctx, const double *gx, const double *gv,
                             const double *gw, double *gx0, double *gv0, double *gw0,
                             double *gparams);

/* DEM neighbour-list state: rebuilds so far, entries at the last rebuild, capacity, skin
 * (waits for the context's stream).  pe has no neighbour lists: its hash grids re-bin every
 * body every step (HashGrids.h:1121-1258); this reports the device-side replacement. */
int pe_b200_neighbor_list_stats(pe_b200_ctx *ctx, int64_t *rebuilds, int64_t *entries,
                                int64_t *capacity, double *skin);

/* Stage timers (CUDA events on the context's stream around each stage; off by default).
 * Replaces: pe's profiling sections and logProfilingSummary (pe/config/ProfilingMode.h:40,
 * pe/core/collisionsystem/DEMSolver.h:698-960).  Enabling resets the totals. */
int pe_b200_set_profiling(pe_b200_ctx *ctx, int32_t enabled);
/* Per stage: name, total milliseconds and number of timed launches since profiling was
 * enabled; *n_out receives the number of stages (at most cap are written). */
int pe_b200_profile(pe_b200_ctx *ctx, int32_t cap, const char **names, double *total_ms,
                    int64_t *count, int32_t *n_out);

/* CUDA graphs of the DEM neighbour-list step and of the hard-contact step of sphere scenes (no
 * pe counterpart; pe's step is a serial loop).  pe_b200_step(ctx, nsteps, dt) with
 * nsteps >= steps captures `steps` consecutive steps once and then replays the graph, so a
 * replay costs one launch; the remainder runs step by step.  Default 16; 0 (or 1) launches every
 * step; odd values are rounded down.  Graphs are not used while profiling is on.  The results
 * are the same as without graphs. */
int pe_b200_set_graph_steps(pe_b200_ctx *ctx, int32_t steps);
/* 1 when the context holds a captured graph it can replay. */
int pe_b200_graph_active(const pe_b200_ctx *ctx);
/* Graphs captured and graph launches since the context was created. */
int pe_b200_graph_stats(const pe_b200_ctx *ctx, int64_t *captures, int64_t *replays);

/* Launch shapes of the DEM neighbour-list step (no pe counterpart). */
typedef struct {
    int32_t dem_variant;     /* launch shape of the force/integration kernel, 0..variants-1 */
    int32_t rebuild_per_sm;  /* CTAs per SM of the persistent list rebuild; 0 = as many as fit;
                                -1 = one launch per rebuild stage (the same lists) */
    double skin;             /* neighbour-list skin (cells are re-planned to 2 r_max + skin) */
    double ms_per_step;      /* pe_b200_autotune: measured time of the winner; else -1 */
    int32_t variants;        /* output: number of launch shapes */
    int32_t nbgs_sweeps;     /* HCSITS sweeps: 0 automatic (4 when every colour fits one
                                block, else 5 when the bodies fit, else 2), 1 one thread-block
                                cluster with hardware barriers, 2 one cooperative grid with
                                barriers through global memory, 3 one launch per colour, 4 one
                                thread block with __syncthreads between colours (when every
                                colour fits it), 5 one cluster with the bodies' records in its
                                distributed shared memory (sphere scenes whose bodies fit) */
    int32_t dem_grid;        /* DEM grid step (cell search every step): 0 candidates read from an
                                FP32 position copy in cell order, with an exact FP64 test for the
                                close ones; 1 every candidate through its FP64 record (the same
                                results) */
    int32_t dem_split;       /* DEM list step: 0 the marked spheres' forces, then the integration
                                of every sphere; 1 the marked spheres (forces and integration) on a
                                second stream beside the integration of the others; 2 the same
                                overlap on one stream: the kernel that checks for (and runs) the
                                rebuild lets the integration of the unmarked spheres start, then
                                computes and integrates the marked ones (orientation tracking
                                runs form 0).  All forms give the same results */
} pe_b200_tuning;
int pe_b200_get_tuning(pe_b200_ctx *ctx, pe_b200_tuning *out);
int pe_b200_set_tuning(pe_b200_ctx *ctx, const pe_b200_tuning *t);
/* Times the DEM list step under candidate tunings from the current state (each trial restores
 * that state, forces one list rebuild and times trial_steps steps with CUDA events), applies the
 * fastest and restores the state.  Shapes do not change results; the skin changes them only in
 * the last bits (the summation order follows the re-sorted body order). */
int pe_b200_autotune(pe_b200_ctx *ctx, double dt, int32_t trial_steps, pe_b200_tuning *out);

/* Allocation-free DEM step.  This entry point has no counterpart in the reference.
 *
 * For callers that cannot allocate device memory -- an application that owns all device memory
 * through its own arena or pool, or a real-time loop that must not pay for an allocation's
 * implicit synchronisation -- it advances one scene by one FP64 DEM step (the same kernel as
 * pe_b200_step with PE_B200_DEM/PE_B200_FP64) without calling cudaMalloc, cudaFree or any
 * allocating routine.  Its scratch lives in one fixed __device__ array inside the library
 * (about 7.3 MB, held on every GPU that loads the library until the process exits).
 *
 *   x, v, w (3n doubles each, interleaved xyz), r (n), mat (n): device inputs;
 *   x_out, v_out, w_out: device outputs (may alias nothing of the inputs);
 *   mats/planes/boxes: host tables (as pe_b200_set_materials / pe_b200_set_walls);
 *   domain_lo/hi: finite box the grid covers (bodies outside are clamped into border cells,
 *   still exact); max_radius: finite, and no sphere may be larger (checked on the device: the
 *   call then returns PE_B200_ERR_ARG and leaves x_out, v_out and w_out unwritten, as it does
 *   for a material index outside [0, nmat)); stream: cudaStream_t to run on (NULL: the legacy
 *   default stream).
 * The call is synchronous: it returns after the step has finished on the device, copies its
 * tables from host memory and reads its status back.
 * Limits: n <= PE_B200_STATIC_MAX_SPHERES, <= 64 materials, <= 64 planes, <= 64 boxes (larger
 * requests return PE_B200_ERR_ARG before any work); the grid is coarsened to at most
 * PE_B200_STATIC_MAX_CELLS cells, whatever the domain's width.  All calls on a device share the
 * array: calls whose work overlaps on the GPU race and corrupt each other.  The first call on
 * each device (and the first after a cudaDeviceReset) looks up the array's device address,
 * which allocates nothing. */
#define PE_B200_STATIC_MAX_SPHERES 32768
#define PE_B200_STATIC_MAX_CELLS 131072
int pe_b200_dem_step_static(int64_t n, const double *x, const double *v, const double *w,
                            const double *r, const int32_t *mat, int32_t nmat,
                            const pe_b200_material *mats, int32_t nplanes, const double *planes,
                            const int32_t *plane_mat, int32_t nboxes, const double *boxes,
                            const int32_t *box_mat, const double gravity[3], double damping,
                            double dt, const double domain_lo[3], const double domain_hi[3],
                            double max_radius, double *x_out, double *v_out, double *w_out,
                            void *stream);

/* Consistency checks of the device state, run on the host (no pe counterpart beyond its debug
 * assertions, pe_INTERNAL_ASSERT, compiled out in release builds):
 *   - HCSITS: in the contact order of the last step no body appears twice in one colour (the
 *     condition under which the parallel Gauss-Seidel sweep of a colour is race-free);
 *   - DEM neighbour lists: entries in range, no self entries, every pair listed from both sides,
 *     orientation bit = (user id of the sphere < user id of the neighbour).
 * *problems receives the number of violations (0 = consistent).  Synchronises the stream. */
int pe_b200_validate(pe_b200_ctx *ctx, int64_t *problems);
/* Self-test of the bounded device waits: launches one kernel that waits on a flag nothing sets,
 * which gives up after `polls` polls (1 <= polls <= 2^24) and records a timeout.  Returns
 * PE_B200_ERR_TIMEOUT, as a real barrier or peer wait that ran out would, and leaves the context
 * usable. */
int pe_b200_selftest_timeout(pe_b200_ctx *ctx, int64_t polls);

/* Number of kernels this context launched since creation (device-side work accounting). */
int64_t pe_b200_kernel_launches(const pe_b200_ctx *ctx);

/* The CUDA stream (cudaStream_t) this context launches on, for event timing by the caller. */
void *pe_b200_stream(pe_b200_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* PE_B200_H */
