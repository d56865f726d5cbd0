/*
 * beatbox.h -- C ABI of the B200 rigid-body step library (libbeatbox.so).
 *
 * This is the drop-in boundary for beat-box's per-step rigid-body pipeline.  The
 * reference exposes that pipeline as the C++ class beatbox::RigidBodyManager
 * (src/rigid_body_manager.hpp:12-264), fed by SceneManager::load_scene
 * (src/scene_manager.hpp:825-929) and configured by StatusManager
 * (src/status_manager.hpp:204-373).  Each entry point below names the reference
 * interface it replaces.  Plain pointers and sizes only; no exceptions cross this
 * boundary; every function returns a bb_status (0 = OK) unless stated otherwise.
 *
 * Threading: a bb_world is used by one host thread at a time.  bb_step() enqueues
 * work on the world's CUDA stream and returns; bb_sync() waits for it.  Readback
 * functions synchronise the world's stream before copying.
 */
#ifndef BEATBOX_H
#define BEATBOX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
typedef int32_t bb_status;
#define BB_OK 0
#define BB_E_INVALID 1      /* bad argument or call order */
#define BB_E_CAPACITY 2     /* a per-step buffer (pairs, manifolds) overflowed; reserve more */
#define BB_E_CUDA 3         /* a CUDA runtime call failed; see bb_last_error_string() */
#define BB_E_DEVICE_LIMIT 4 /* a bounded device loop (spin, traversal stack) gave up */
#define BB_E_BUDGET 5       /* serving admission refused: HBM budget exhausted */
#define BB_E_UNSUPPORTED 6  /* feature of the reference not provided by this build */

/* ---- body flags: the reference RigidBodyFlag bits (include/shared.inl:94-100) ----- */
#define BB_BODY_DYNAMIC (1u << 1)
#define BB_BODY_GRAVITY (1u << 2)
#define BB_BODY_SLEEPING (1u << 3)
/* Set by bb_world_pause on every dynamic body of a paused (sub-)world: the body counts as
 * asleep, and the step leaves it and its contacts exactly as they are (no sleep-timer update,
 * contacts carried over unchanged) until the world is resumed.  No reference counterpart. */
#define BB_BODY_PAUSED (1u << 5)

/* ---- shapes ---------------------------------------------------------------------- */
#define BB_SHAPE_BOX 0u    /* reference OBB body: RigidBody::minimum/maximum (shared.inl:349-352) */
#define BB_SHAPE_SPHERE 1u /* no reference counterpart: written from first principles */
#define BB_SHAPE_VOXEL 2u  /* concave body: occupancy bitmask + surface cells (VoxelShape,
                              include/shared.inl:938-951; RigidBody::shape_index != 0) */
#define BB_VOXEL_MAX_DIM 256u /* cells per axis: surface cells pack x | y<<8 | z<<16 */

/* ---- inertia construction modes for bb_add_bodies -------------------------------- */
#define BB_INERTIA_PHYSICAL 0u  /* solid box / sphere inverse inertia from mass */
#define BB_INERTIA_REFERENCE 1u /* cuboid_get_inverse_intertia(inv_mass, min, max): the reference
                                   scene builder passes inverse mass as mass
                                   (src/scene_manager.hpp:861, include/math.hpp:106-130) */
#define BB_INERTIA_EXPLICIT 2u  /* use bb_body_desc.inv_inertia (+ inv_inertia_off) as given */
/* Voxel bodies always take their inertia from the shape (BB_INERTIA_PHYSICAL and
 * BB_INERTIA_REFERENCE both mean "from the shape") unless BB_INERTIA_EXPLICIT. */

/* ---- solver types: SimSolverType (include/shared.inl:210-216) ---------------------- */
#define BB_SOLVER_PGS 0u      /* Baumgarte PGS: only on the reference's per-island path */
#define BB_SOLVER_PGS_SOFT 1u /* soft-step PGS on graph colours (reference default PGS family) */
#define BB_SOLVER_AVBD 2u     /* augmented vertex block descent (reference default solver) */

/* ---- sim flags: SimFlag (include/shared.inl:150-161) -------------------------------- */
#define BB_SIM_ACCUM_IMPULSE (1u << 0)
#define BB_SIM_FRICTION (1u << 1)
#define BB_SIM_WARM_STARTING (1u << 2)
#define BB_SIM_ADVECTION (1u << 3)
#define BB_SIM_DEBUG_INFO (1u << 4)
#define BB_SIM_USE_GRAPH_COLORING (1u << 5)
#define BB_SIM_SLEEPING_ENABLED (1u << 7)
/* reference defaults (src/rigid_body_manager.hpp:140-147) */
#define BB_SIM_DEFAULT_FLAGS                                                                        \
  (BB_SIM_ACCUM_IMPULSE | BB_SIM_FRICTION | BB_SIM_WARM_STARTING | BB_SIM_ADVECTION |               \
   BB_SIM_DEBUG_INFO | BB_SIM_USE_GRAPH_COLORING | BB_SIM_SLEEPING_ENABLED)

/* ---- reference arithmetic kept as switchable behaviours ----------------------------
 * Each bit reproduces one piece of the reference step's arithmetic exactly.  Clearing a
 * bit selects the physically consistent formula instead.                             */
#define BB_QUIRK_GRAVITY_IMPULSE (1u << 0)   /* PGS advect: v += g*dt*inv_mass (apply_impulse,
                                                src/shaders/extensions.slang:127-134,169-178) */
#define BB_QUIRK_SAT_FRAME (1u << 1)         /* box-box SAT relative rotation C = R_A*R_B^T
                                                (collision_detection.slang:572) */
#define BB_QUIRK_INERTIA_TRANSPOSE (1u << 2) /* world inverse inertia R^T*I^-1*R
                                                (extensions.slang:184-188) */
#define BB_QUIRKS_REFERENCE (BB_QUIRK_GRAVITY_IMPULSE | BB_QUIRK_SAT_FRAME | BB_QUIRK_INERTIA_TRANSPOSE)
#define BB_QUIRKS_PHYSICAL 0u

/* ---- Morton normalisation box ---------------------------------------------------- */
#define BB_BOUNDS_FIXED 0u /* use bb_solver_params.world_min / world_extent (reference: -64, 128,
                              src/shaders/simulation/RB_sim.slang:96-101) */
#define BB_BOUNDS_AUTO 1u  /* per substep: min/max of body positions */

/* ---- colour-sweep schedules ------------------------------------------------------------
 * DATAFLOW: every (sweep, manifold) item waits on per-body sequence counters for exactly the
 * items that precede it on its two bodies in (sweep, colour, manifold) order -- the order the
 * reference's per-colour dispatches impose -- so no grid-wide barrier is needed.
 * COLOUR_BARRIER: one grid barrier between colours, as the reference's dispatch sequence. */
#define BB_SCHEDULE_DATAFLOW 0u
#define BB_SCHEDULE_COLOUR_BARRIER 1u

/* Solver and material parameters.  Every reference constant is a field whose default (from
 * bb_default_solver_params) is the reference value; replaces StatusManager::set_solver /
 * flag toggles (src/status_manager.hpp:204-373) and the compile-time constants of
 * include/shared.inl:77-83,760-839 and include/defines.hpp:352-364. */
typedef struct bb_solver_params {
  uint32_t solver;             /* BB_SOLVER_* (default AVBD) */
  uint32_t flags;              /* BB_SIM_* (default BB_SIM_DEFAULT_FLAGS) */
  uint32_t quirks;             /* BB_QUIRK_* (default BB_QUIRKS_REFERENCE) */
  uint32_t iterations;         /* PGS solve sweeps per substep (reference create() arg, default 5) */
  uint32_t relax_iterations;   /* PGS relax sweeps per substep (reference: = iterations) */
  uint32_t gc_rounds;          /* edge-colouring rounds (RBM GRAPH_COLOR_MAX_ROUNDS = 32) */
  float gravity;               /* y acceleration, default -9.81 */
  float linear_damping;        /* 0.1 /s */
  float angular_damping;       /* 0.1 /s */
  float contact_hertz;         /* MIN_CONTACT_HERTZ = 30 */
  float penetration_cap;       /* narrow-phase depth floor, -0.25 */
  /* sleeping (shared.inl:793-797, RB_sim.slang:556-737) */
  float sleep_lin_vel2;        /* 0.0144 */
  float sleep_ang_vel2;        /* 0.0225 */
  uint32_t sleep_steps;        /* 30 */
  /* AVBD (shared.inl:798-838) */
  uint32_t avbd_iterations;    /* 10 */
  float avbd_beta;             /* 1e5 */
  float avbd_gamma;            /* 0.99 */
  float avbd_k_min;            /* 1 */
  float avbd_k_max;            /* 1e9 */
  float avbd_margin;           /* 0.0005 */
  float avbd_stick_thresh;     /* 0.01 */
  float avbd_stick_slop;       /* 0.001 */
  uint32_t avbd_color_rounds;  /* 16 */
  uint32_t avbd_shock_layers;  /* 12 */
  uint32_t avbd_post_stab_sweeps; /* 4 */
  /* execution schedule of the colour sweeps (results are identical either way) */
  uint32_t schedule;           /* BB_SCHEDULE_* (default BB_SCHEDULE_COLOUR_BARRIER) */
  /* launch geometry (results are identical for every value; 0 = default; bb_autotune picks) */
  uint32_t broad_threads;        /* broad-phase block size: 32, 64 or 128 (default 128) */
  uint32_t narrow_blocks_per_sm; /* narrow-phase grid, 128-thread blocks per SM: 1..64 (default 16) */
  uint32_t pgs_stage_next;       /* colour-barrier PGS_SOFT: 1 stages each thread's next item of a colour in shared
                                    memory while the current one computes (large worlds); 0 loads it after (default) */
  /* Morton normalisation */
  uint32_t bounds_mode;        /* BB_BOUNDS_* */
  float world_min[3];          /* default -64 */
  float world_extent[3];       /* default 128 */
} bb_solver_params;

/* World creation.  max_bodies sizes the body arrays; pair_capacity and contact capacity
 * are derived from pairs_per_body (pairs <= pairs_per_body * max_bodies). */
typedef struct bb_world_desc {
  uint32_t max_bodies;
  uint32_t pairs_per_body; /* 0 = default (16) */
  int32_t device;          /* CUDA device ordinal; -1 = current */
  void* stream;            /* cudaStream_t to run on; NULL = the world creates its own */
} bb_world_desc;

/* One body.  Replaces the RigidBody initialiser used by SceneManager scenes
 * (src/scene_manager.hpp:114-823) plus the id / mass / inertia assignment of
 * load_scene (src/scene_manager.hpp:850-887). */
typedef struct bb_body_desc {
  float position[3];
  float rotation[4];     /* quaternion x, y, z, w (reference Quaternion{v, w}) */
  float velocity[3];
  float omega[3];
  uint32_t shape;        /* handle from bb_add_box_shape / bb_add_sphere_shape */
  uint32_t flags;        /* BB_BODY_* */
  float mass;            /* > 0: used as given; 0: density * volume (0 density = static) */
  float density;
  float friction;
  float restitution;     /* stored; unused by the reference solvers (solvers.slang:49-56) */
  uint32_t inertia_mode; /* BB_INERTIA_* */
  float inv_inertia[3];  /* body-frame diagonal, BB_INERTIA_EXPLICIT only */
  float inv_inertia_off[3]; /* body-frame off-diagonal (xy, xz, yz), BB_INERTIA_EXPLICIT only;
                               the reference RigidBody::inv_inertia is a full 3x3
                               (include/shared.inl:366) */
} bb_body_desc;

/* Per-step counters: the reference SimConfig readback (src/rigid_body_manager.cpp:1681-1693,
 * include/shared.inl:571-665) plus this build's capacity and error reporting. */
typedef struct bb_step_stats {
  uint32_t body_count;
  uint32_t active_body_count;
  uint32_t pair_count;            /* broad_phase_collision_count */
  uint32_t manifold_count;        /* g_c_info.collision_count */
  uint32_t contact_count;
  uint32_t island_count;
  uint32_t graph_color_count;     /* colours used by the edge colouring */
  uint32_t graph_color_overflow;  /* manifolds solved by the serial overflow bucket */
  uint32_t graph_color_violations;
  uint32_t avbd_color_count;
  uint32_t avbd_violations;
  uint32_t sleeping_count;
  uint32_t fresh_contacts;        /* dbg_fresh: contacts that failed warm-start matching */
  uint32_t stick_count;           /* avbd_stick_count */
  float max_penetration;          /* deepest contact penetration (positive metres) */
  uint32_t error_flags;           /* BB_ERRF_* bits raised on the device */
  uint32_t pair_capacity;
  uint32_t substeps_run;          /* substeps run since the world was created */
  uint32_t solved_manifolds;      /* last substep's colour sweeps: manifolds with an awake body */
  uint32_t solved_contacts;       /* and their contacts (0 under AVBD and the per-island path) */
  uint32_t graph_color_rounds;    /* bid/commit rounds the last edge colouring ran (at most gc_rounds) */
  uint32_t error_site;            /* where the first bounded wait gave up (BB_ERRF_SPIN_LIMIT): 0 none,
                                     1 sort look-back, 2 dataflow PGS wait, 3 generation barrier, 4 scan
                                     look-back, 16 + k grid barrier k (0 edge colouring, 1 PGS_SOFT, 2 AVBD
                                     colouring, 3..5 AVBD solve phases, 7 connected components) */
} bb_step_stats;

/* device error bits (bb_step_stats.error_flags) */
#define BB_ERRF_PAIR_OVERFLOW (1u << 0)
#define BB_ERRF_STACK_OVERFLOW (1u << 1)
#define BB_ERRF_SPIN_LIMIT (1u << 2)
#define BB_ERRF_CAS_LIMIT (1u << 3)
#define BB_ERRF_CONTACT_OVERFLOW (1u << 4)

/* intermediate buffers readable with bb_debug_read (for parity tests and tools) */
#define BB_DBG_MORTON 1u       /* u32 x N: Morton code of each body, by body id */
#define BB_DBG_SORTED_KEYS 2u  /* u32 x N */
#define BB_DBG_SORTED_IDS 3u   /* u32 x N: body id at each sorted position */
#define BB_DBG_LBVH_CHILD 4u   /* i32 x 2(N-1): left, right of internal nodes; >= N-1 = leaf */
#define BB_DBG_LEAF_AABB 5u    /* f32 x 6N: min xyz, max xyz per sorted leaf */
#define BB_DBG_NODE_AABB 6u    /* f32 x 6(N-1) */
#define BB_DBG_PAIRS 7u        /* u32 x 2P: (sorted a, sorted b), a < b */
#define BB_DBG_MANIFOLDS 8u    /* bb_manifold_info x M */
#define BB_DBG_CONTACTS 9u     /* bb_contact_info x 8M (slot j of manifold m at 8m+j) */
#define BB_DBG_EDGE_COLORS 10u /* u32 x M (0xFFFFFFFF = overflow, 0xFFFFFFFE = resting: the manifold's
                                  island has no awake body, so it is neither coloured nor solved) */
#define BB_EDGE_COLOR_OVERFLOW 0xFFFFFFFFu
#define BB_EDGE_COLOR_RESTING 0xFFFFFFFEu
#define BB_DBG_BODY_COLORS 11u /* u32 x N by body id (AVBD colouring) */
#define BB_DBG_ISLANDS 12u     /* u32 x N by body id (0xFFFFFFFF = static / no island) */
#define BB_DBG_SUPPORT_DEPTH 13u /* u32 x N by body id (AVBD shock-propagation depth) */
#define BB_DBG_BODY_INERTIA 14u  /* f32 x 6N by body id: body-frame inverse inertia xx yy zz xy xz yz */

typedef struct bb_manifold_info {
  uint32_t body_a;       /* body ids; a has the lower sorted position this substep */
  uint32_t body_b;
  int32_t key;           /* SAT axis (0-14), 20 sphere-sphere, 21/22 box-sphere */
  int32_t contact_count;
  float normal[3];       /* from a towards b */
  uint32_t color;        /* edge colour */
  float tangent[2][3];
} bb_manifold_info;

typedef struct bb_contact_info {
  float position[3];
  float penetration;     /* <= 0 when overlapping */
  float normal_impulse;  /* PGS impulse, or AVBD lambda */
  float tangent_impulse[2];
  uint32_t feature;      /* packed feature pair: in_ref | out_ref<<8 | in_inc<<16 | out_inc<<24 */
  uint32_t warm_start;   /* persistence counter (0 = fresh) */
  float penalty;         /* AVBD normal penalty k (mass_coefficient) */
} bb_contact_info;

/* ---- entry points ------------------------------------------------------------------ */

/* Fill p with the reference defaults listed in bb_solver_params.  No reference
 * counterpart: the reference compiles these in. */
void bb_default_solver_params(bb_solver_params* p);

/* Replaces RigidBodyManager::RigidBodyManager + create()
 * (src/rigid_body_manager.hpp:14-18, src/rigid_body_manager.cpp:6-283). */
bb_status bb_world_create(const bb_world_desc* desc, void** out_world);
/* Replaces RigidBodyManager::~RigidBodyManager (src/rigid_body_manager.hpp:16). */
bb_status bb_world_destroy(void* world);

/* Shape table.  The reference stores the box extents in each RigidBody (min/max,
 * shared.inl:351-352); here bodies reference a shape handle. */
bb_status bb_add_box_shape(void* world, float hx, float hy, float hz, uint32_t* out_shape);
bb_status bb_add_sphere_shape(void* world, float radius, uint32_t* out_shape);

/* Voxel shape from an occupancy grid: solid[x + y*nx + z*nx*ny] != 0 marks a solid cell
 * (nx, ny, nz <= BB_VOXEL_MAX_DIM, at least one solid cell).  The body origin is the
 * centre of mass of the solid cells.  Replaces SceneManager::build_voxel_shape
 * (src/scene_manager.hpp:488-560) and the voxel pools it fills (shared.inl:771-774). */
bb_status bb_add_voxel_shape(void* world, uint32_t nx, uint32_t ny, uint32_t nz, float voxel_size,
                             const uint8_t* solid, uint32_t* out_shape);

/* What bb_add_voxel_shape derives from a grid, on the host (no world, no GPU). */
typedef struct bb_voxel_info {
  float grid_origin[3];       /* body-frame corner of cell (0,0,0) = minus the centre of mass */
  float box_min[3];           /* RigidBody::minimum (= grid_origin) */
  float box_max[3];           /* RigidBody::maximum (= grid_origin + dims * voxel_size) */
  uint32_t solid_count;
  uint32_t surface_count;     /* solid cells with an empty face neighbour */
  float unit_mass;            /* mass at density 1: solid_count * voxel_size^3 */
  float unit_inv_inertia[6];  /* inverse inertia about the centre of mass at density 1,
                                 body frame: xx, yy, zz, xy, xz, yz */
} bb_voxel_info;
/* surface: NULL, or room for surface_count entries packed x | y<<8 | z<<16 | dir<<24 with dir
 * the first empty neighbour in the order -x, +x, -y, +y, -z, +z (scene_manager.hpp:536-546).
 * A body of mass M has inverse inertia unit_inv_inertia * (unit_mass / M) (float). */
bb_status bb_voxel_shape_info(uint32_t nx, uint32_t ny, uint32_t nz, float voxel_size, const uint8_t* solid,
                              bb_voxel_info* out, uint32_t* surface, uint32_t surface_capacity);

/* Append n bodies; their ids are consecutive from *out_first_id.  Replaces the body
 * push + id/mass/inertia assignment of SceneManager::load_scene
 * (src/scene_manager.hpp:850-887) and RBM::update_active_rigid_body_list
 * (src/rigid_body_manager.cpp:90-119,1695-1712). */
bb_status bb_add_bodies(void* world, const bb_body_desc* bodies, uint32_t n, uint32_t* out_first_id);

/* Batched worlds: append an independent world of n bodies (its own ground included) to a
 * world object; bodies of different worlds never interact.  Ids stay consecutive per world
 * (*out_first_id); keys sort by (world, Morton code), the LBVH keeps each world in one subtree,
 * and colouring priorities use world-local ids, so every world evolves exactly as it would
 * alone.  world_min/world_extent: the world's Morton normalisation box.  Not mixable with
 * bb_add_bodies on the same object.  No reference counterpart (the reference is one world). */
typedef struct bb_batch_world_desc {
  float world_min[3];
  float world_extent[3];
} bb_batch_world_desc;
bb_status bb_add_world(void* world, const bb_batch_world_desc* desc, const bb_body_desc* bodies, uint32_t n,
                       uint32_t* out_world_index, uint32_t* out_first_id);
uint32_t bb_world_count(void* world);

/* Batch slots for continuous batching.  A batch is one object stepped as a whole; these two
 * calls let a serving loop keep worlds resident in it while they have no work, and reuse the
 * slot of a finished world for a new one, without touching the other worlds.
 *
 * bb_world_pause: paused = 1 pauses world `world_index` of the batch (0 for a plain world):
 * its dynamic bodies count as asleep (BB_BODY_PAUSED), and every later step leaves the world
 * exactly as it is -- poses, velocities, sleep timers, and its contacts, which are carried from
 * substep to substep unchanged.  paused = 0 resumes it: it then steps bit for bit as if the
 * steps taken while it was paused had not happened.  Asynchronous on the world's stream.
 *
 * bb_world_refill: puts `count` new bodies into world `world_index`'s slot (ids
 * [first, first + slot size), slot size = the body count the world was added with), with new
 * Morton bounds; the slot's unused bodies are parked as static specks far outside the box.  The
 * slot's old bodies, their contacts and their sorted order are discarded: the new world starts
 * as a world just added does (and steps as it would alone).  count above the slot size returns
 * BB_E_CAPACITY.  Waits for the world's stream.  No reference counterpart (the reference steps
 * one scene, src/rigid_body_manager.cpp:1606-1622). */
bb_status bb_world_pause(void* world, uint32_t world_index, uint32_t paused);
bb_status bb_world_refill(void* world, uint32_t world_index, const bb_batch_world_desc* desc,
                          const bb_body_desc* bodies, uint32_t count);

/* Change the friction/restitution of bodies [first, first+n).  No separate reference
 * entry point (materials are per body, shared.inl:360-361). */
bb_status bb_set_material(void* world, uint32_t first, uint32_t n, float friction, float restitution);

/* Replaces StatusManager::set_solver + flag toggles (src/status_manager.hpp:204-373),
 * RBM::set_sim_flags/clear_sim_flags/set_sim_type (src/rigid_body_manager.hpp:22-40). */
bb_status bb_set_solver_params(void* world, const bb_solver_params* params);
bb_status bb_get_solver_params(void* world, bb_solver_params* params);

/* Advance every body by dt in `substeps` full pipeline passes of h = dt/substeps.
 * Replaces RigidBodyManager::simulate (src/rigid_body_manager.cpp:1606-1622), which runs
 * one pass at the fixed TIME_STEP.  Asynchronous on the world's stream. */
bb_status bb_step(void* world, float dt, uint32_t substeps);
/* Wait for queued steps; returns BB_E_CAPACITY / BB_E_DEVICE_LIMIT if a step raised an
 * error flag (see bb_step_stats.error_flags). */
bb_status bb_sync(void* world);

/* Read / overwrite body state by id (any pointer may be NULL).  position 3N, rotation 4N
 * (x y z w), velocity 3N, omega 3N.  The reference never reads bodies back to the host
 * (transforms go to the TLAS, src/shaders/AS_mngr.slang:5-36). */
bb_status bb_read_state(void* world, float* position, float* rotation, float* velocity, float* omega);
bb_status bb_write_state(void* world, const float* position, const float* rotation,
                         const float* velocity, const float* omega);
/* Per-body flags (BB_BODY_*, including SLEEPING) by id. */
bb_status bb_read_flags(void* world, uint32_t* flags);
uint32_t bb_body_count(void* world);

/* Replaces RBM::read_back_sim_config (src/rigid_body_manager.cpp:1681-1693). */
bb_status bb_read_stats(void* world, bb_step_stats* stats);

/* Replaces RBM::skip_warm_starting_once (src/rigid_body_manager.hpp:29-31). */
bb_status bb_skip_warm_starting_once(void* world);

/* Run the collision front end of one substep on the current state without moving bodies:
 * Morton codes, radix sort, LBVH build + refit, broad phase (stage = 1), and the narrow
 * phase with warm-start matching (stage = 2).  Results are readable with bb_debug_read.
 * No reference counterpart (the reference only runs the whole task graph). */
bb_status bb_debug_collide(void* world, uint32_t stage);
/* Copy an intermediate buffer (BB_DBG_*) of the last substep to host memory.  *count
 * receives the element count; at most max_bytes are written. */
bb_status bb_debug_read(void* world, uint32_t which, void* dst, uint64_t max_bytes, uint64_t* count);

/* Bounded device waits, for tests of the failure path.  polls: how many polls a grid-barrier
 * wait of this world's persistent kernels makes before it gives up (0 = the default, 2^22),
 * raising BB_ERRF_SPIN_LIMIT so that bb_sync returns BB_E_DEVICE_LIMIT.  abandon_block = 1
 * makes the last block of the PGS_SOFT colour-sweep kernel leave before its first grid barrier
 * (when the kernel runs on more than one block), so the other blocks wait for a block that
 * never arrives until their bounded waits give up; the step's results are then undefined, and
 * bb_world_clear (which also clears the error bits) makes the world usable again.  No
 * counterpart in the reference: its bounded loops (avbd.slang:559, collision_detection.slang:921,
 * LBVH.slang:226,278) stop without reporting. */
bb_status bb_debug_wait_limit(void* world, uint32_t polls, uint32_t abandon_block);

/* CUDA stream the world runs on (cudaStream_t). */
void* bb_world_stream(void* world);
/* Per-stage device timing (ms, summed over substeps since the last reset) for profiling.
 * names: a NUL-separated list of stage names, written to names (may be NULL). */
bb_status bb_set_profiling(void* world, int32_t enabled);
bb_status bb_read_stage_times(void* world, float* ms, uint32_t max_stages, uint32_t* n_stages,
                              char* names, uint32_t names_bytes);
/* Device memory held by the world (all its buffers), in bytes; bb_world_bytes_for gives the
 * same figure for a world not yet created.  No reference counterpart. */
uint64_t bb_world_device_bytes(void* world);
uint64_t bb_world_bytes_for(uint32_t max_bodies, uint32_t pairs_per_body);
/* Remove all bodies and shapes, keeping the world's buffers, stream and parameters, so the
 * object can hold a different scene (bodies added next restart the persistent state).  No
 * reference counterpart (the reference reloads a scene into fixed buffers, RBM:224-254). */
bb_status bb_world_clear(void* world);

/* Saved world state, for checkpoints and for resuming evicted worlds bit for bit.
 * bb_world_save_state writes an image of the world (its device arrays and the host fields that
 * steer the next step: manifold parity, solver parameters, pending warm-start skip) into dst;
 * with dst = NULL it only returns the size in *bytes.  The image holds the persistent contacts
 * (both manifold buffers with impulses, anchors and warm-start counters), per-body lists, sort
 * order, sleep timers and island roots, so a world loaded from it steps exactly as the saved
 * world would have.  Its size is the world's device footprint (bb_world_device_bytes).
 * bb_world_load_state restores an image into a world created with the same bb_world_desc
 * capacity that holds the same bodies (the same shapes and bodies added in the same order);
 * anything else returns BB_E_INVALID.  Both wait for the world's stream.  The reference's
 * counterpart is a pause of the whole step (src/status_manager.hpp:133-152); it saves nothing. */
/* Automatic regrow of the pair capacity.  With max_pairs_per_body > 0, bb_step first copies
 * the world's device state (once, before the first step since the last bb_sync; the copy needs as
 * much device memory again as the world holds), and when bb_sync finds that a step overflowed the
 * pair or manifold capacity it reallocates the world with twice the pairs per body (up to the
 * limit), restores the copy and runs the steps issued since again: the world then steps exactly
 * as a world created with the larger capacity would.  bb_sync returns BB_E_CAPACITY only when the
 * limit is reached.  Calls that change bodies, poses or parameters between a step and its
 * bb_sync drop the copy (an overflow before them is then reported, not repaired).  0 turns it
 * off (the default).  The reference instead clamps silently at its N^2 buffer sizes
 * (include/shared.inl:770-776, RB_sim.slang:454,466). */
bb_status bb_world_set_auto_regrow(void* world, uint32_t max_pairs_per_body);

bb_status bb_world_save_state(void* world, void* dst, uint64_t max_bytes, uint64_t* bytes);
bb_status bb_world_load_state(void* world, const void* src, uint64_t bytes);

/* Number of kernels this library launched on the world's stream since creation. */
uint64_t bb_kernel_launch_count(void* world);

/* Stable LSD radix sort of n (key, value) pairs held in DEVICE memory: keys_out/vals_out
 * receive the pairs ordered by the low key_bits (1..32) of the key, ties kept in input order.
 * The step's Morton-code sort (onesweep with decoupled look-back), exposed on caller arrays;
 * the reference sorts inside its task graph (src/shaders/simulation/RB_sim.slang:113-203,
 * LBVH.slang:34-152).  Asynchronous on `stream` (cudaStream_t, NULL = legacy default).
 * Its scratch is allocated with cudaMalloc on first use per device and reused afterwards. */
bb_status bb_radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                              uint32_t* vals_out, uint32_t n, uint32_t key_bits, void* stream);

/* bb_radix_sort_pairs with the same results that allocates nothing: its scratch (about 2.3 MB)
 * is a fixed device array in the library, so n is limited to BB_SORT_STATIC_MAX_KEYS (larger n
 * returns BB_E_INVALID).  The first call on a device (with that device current) looks the
 * array's address up; make it before any stream capture.  Every call clears the part of the
 * scratch that must start at zero on `stream` itself.  Calls on one device share the scratch:
 * calls that overlap in time (different streams without ordering, several host threads) race
 * and give wrong results.  The looked-up address is kept with the id of the CUDA context; after
 * cudaDeviceReset (a new context) the next call looks it up again.  No counterpart in the
 * reference. */
#define BB_SORT_STATIC_MAX_KEYS 262144u
bb_status bb_radix_sort_pairs_static(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, uint32_t n, uint32_t key_bits, void* stream);

/* BB_OK from either sort means its work was launched, not that it finished: a look-back wait
 * that reached its bound (BB_ERRF_SPIN_LIMIT) leaves the output undefined.  This waits for
 * `stream` and returns in *error_flags the device error bits (BB_ERRF_*) of the last sort on the
 * current device: static_scratch = 1 for bb_radix_sort_pairs_static, 0 for bb_radix_sort_pairs.
 * 0 means that sort ran to the end.  Allocates nothing.  No counterpart in the reference (its
 * sort passes clamp silently, LBVH.slang:34-152). */
bb_status bb_radix_sort_error_flags(uint32_t static_scratch, void* stream, uint32_t* error_flags);

/* Pick the launch geometry and colour-sweep schedule of this world by timing candidates
 * (coordinate descent over bb_solver_params.schedule, broad_threads, narrow_blocks_per_sm,
 * pgs_stage_next; each candidate timed between two runs of the incumbent).  All candidates
 * give bit-identical results, so the trial steps are ordinary steps (about 21 x
 * (trial_steps + 1) of them): use it in place of warm-up.  The
 * winner is set on the world and copied to *chosen (may be NULL).  The reference has no
 * autotuner (its dispatch sizes are fixed in the task graph, src/rigid_body_manager.cpp:1284-1427). */
bb_status bb_autotune(void* world, float dt, uint32_t substeps, uint32_t trial_steps, bb_solver_params* chosen);

/* ---- serving loop ---------------------------------------------------------------------
 * Step requests for many worlds, kept resident on the device between requests, admitted by an
 * HBM budget (continuous batching).  Worlds of one step class (solver parameters, dt,
 * substeps) sit as slots of one batched world, and each step of that batch advances every
 * running request in it; requests that arrive while others run join at the next step.  A
 * request either creates a world (its key not seen before; shapes and bodies given) or
 * continues one.  A world runs its requests one after another in submission order; its result
 * does not depend on the other requests in flight.  A world that changes step class moves to
 * that class's batch (warm-start contacts restart); idle worlds may be evicted to make room
 * (their body state is kept on the host).  No reference counterpart: the reference steps one
 * scene per frame from its render loop (src/renderer_manager.cpp:254). */
typedef struct bb_shape_desc {
  uint32_t type;   /* BB_SHAPE_BOX or BB_SHAPE_SPHERE */
  float half[3];   /* half extents; sphere radius in half[0] */
} bb_shape_desc;

typedef struct bb_server_desc {
  uint64_t hbm_budget_bytes; /* device memory the server may hold in worlds */
  uint32_t max_active;       /* requests in flight at once (0 = 64) */
  uint32_t pairs_per_body;   /* pair capacity of the worlds it creates (0 = 8) */
  int32_t device;            /* -1 = current device */
} bb_server_desc;

typedef struct bb_request {
  uint64_t world;               /* caller's world key */
  const bb_shape_desc* shapes;  /* new world: shape table (body.shape indexes it); else NULL */
  uint32_t n_shapes;
  const bb_body_desc* bodies;   /* new world: its bodies (copied by submit); else NULL */
  uint32_t n_bodies;
  float world_min[3];           /* new world: Morton normalisation box */
  float world_extent[3];
  bb_solver_params params;      /* this request's solver settings (Morton box fields ignored) */
  float dt;
  uint32_t substeps;
  uint32_t steps;               /* bb_step(dt, substeps) calls */
} bb_request;

typedef struct bb_request_status {
  uint32_t done;     /* 1 once finished */
  bb_status result;  /* BB_OK, BB_E_BUDGET (the world can never fit the budget), ... */
  double submit_s;   /* server clock, seconds since bb_server_create */
  double start_s;
  double finish_s;
  uint32_t error_flags; /* BB_ERRF_* seen in the world's batch by the end of the request's last step */
  uint32_t error_site;  /* bb_step_stats.error_site of the batch at that point */
} bb_request_status;

typedef struct bb_server_stats {
  uint64_t submitted, completed, failed;
  uint64_t body_steps;       /* bodies x steps of the completed requests */
  uint64_t evictions, worlds_created;
  uint64_t resident_bytes;   /* device bytes held in resident and pooled worlds */
  uint32_t active, queued, resident_worlds, known_worlds;
  double materialise_s;      /* worker time spent creating / loading worlds */
  double issue_s;            /* worker time spent enqueueing steps (includes graph captures) */
  uint64_t batch_steps;      /* steps of batched worlds enqueued */
  uint64_t slot_steps;       /* world-steps they advanced (running requests per batch step, summed) */
} bb_server_stats;

bb_status bb_server_create(const bb_server_desc* desc, void** out_server);
bb_status bb_server_destroy(void* server); /* finishes queued requests first */
bb_status bb_server_submit(void* server, const bb_request* req, uint64_t* out_ticket);
bb_status bb_server_poll(void* server, uint64_t ticket, bb_request_status* out);
bb_status bb_server_wait(void* server, uint64_t ticket, bb_request_status* out);
/* Body state of a world after its last finished request (waits for a running one). */
bb_status bb_server_read_state(void* server, uint64_t world, float* position, float* rotation, float* velocity,
                               float* omega, uint32_t* n_bodies);
bb_status bb_server_get_stats(void* server, bb_server_stats* out);

/* ---- render feed (no graphics API: device and host buffers) ----------------------------
 * Per body the 3 x 4 row-major affine transform [R | t] (world = R * local + t), the layout of a
 * ray-tracing instance transform.  Replaces the TLAS instance update of the reference
 * (src/shaders/AS_mngr.slang:5-36, include/shared.inl:377-419), which feeds its path tracer.
 * bb_update_transforms refreshes the device buffer on the world's stream (asynchronous);
 * bb_transforms_device returns that buffer (12 floats per body id, valid for the world's life);
 * bb_read_transforms refreshes it and copies it to host memory. */
bb_status bb_update_transforms(void* world);
const float* bb_transforms_device(void* world);
bb_status bb_read_transforms(void* world, float* transforms);
/* Contact points of the last substep (x, y, z, depth; depth <= 0 on penetration), in manifold
 * order; up to max_points are copied and *count receives the total.  Replaces the reference's
 * debug contact-point buffer for its renderer (src/shaders/simulation/RB_sim.slang:1583-1653). */
bb_status bb_read_contact_points(void* world, float* points, uint32_t max_points, uint32_t* count);

/* Last error message of the calling thread (static storage, never NULL). */
const char* bb_last_error_string(void);
/* Library version string. */
const char* bb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* BEATBOX_H */
