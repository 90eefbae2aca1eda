/*
 * avbd.h: C ABI of the B200 (sm_100a) backend for three-avbd's 3D Augmented Vertex Block Descent step.
 *
 * This is the drop-in boundary for the reference's `GpuSolver3D` (src/avbd3d/gpu/solver.ts:598),
 * the object `World` (src/lib/world.ts:729-731) delegates every physics call to. A host binding
 * (N-API/FFI from TypeScript, ctypes from Python) implements the GpuSolver3D member list on top of
 * these functions; each declaration below names the reference member it replaces.
 *
 * Conventions:
 *   - Every function returns an int status: AVBD_OK (0) or a negative AVBD_ERR_* code, and leaves
 *     the world unchanged on invalid input (the reference throws before any state change,
 *     gpu/solver.ts appendJoints). avbd_last_error() gives the message.
 *   - Host buffers are caller-owned; device buffers are world-owned. One CUDA stream per world:
 *     a world is not thread-safe, distinct worlds are.
 *   - Records are the reference's GPU records, bit-compatible: a body is 40 floats
 *     (src/avbd3d/gpu/layout.ts:8-59), a joint 40 floats plus a 4-int info
 *     (layout.ts:77-110, 232-243), a manifold 8 words and a contact 16 words (layout.ts:118-127).
 *   - Overflow of pair/contact storage is a counter bit, not an error (layout.ts C_OVERFLOW);
 *     storage grows at the next step, as the reference's adapt() does (gpu/solver.ts:2362-2377).
 */
#ifndef AVBD_H
#define AVBD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AVBD_ABI_VERSION 3

enum {
  AVBD_OK = 0,
  AVBD_ERR_INVALID = -1,   /* bad argument (index, count, NaN, size) */
  AVBD_ERR_CAPACITY = -2,  /* past a fixed capacity (bodies, joints) */
  AVBD_ERR_CUDA = -3,      /* a CUDA call failed; the message says which */
  AVBD_ERR_TIMEOUT = -4,   /* a bounded device wait gave up (the step's results are not valid) */
  AVBD_ERR_NO_DEVICE = -5, /* no CUDA device, or not sm_100 */
};

/* Shape codes in avbd_body.shape (layout.ts:143-151). */
#define AVBD_SHAPE_BOX 0
#define AVBD_SHAPE_SPHERE 1
#define AVBD_SHAPE_SAIL 2
/* A hull body's shape is AVBD_SHAPE_HULL + its hull's header offset (vec4s) in the world's hull
 * buffer (layout.ts:150-151): the offset avbd_add_hull returns. */
#define AVBD_SHAPE_HULL 3
/* Most vertices a hull keeps (hull.ts:51); faces and edges at most 255 each. */
#define AVBD_MAX_HULL_VERTICES 32
/* Joint slot types (avbd_joint_info.type, layout.ts:153-154, avbd2d/gpu/layout.ts:74). */
#define AVBD_T_NONE 0
#define AVBD_T_JOINT 1
#define AVBD_T_SPRING 2
/* GPU-only rules (gpu/solver.ts:174-231; the reference's parity tests turn every one off). */
#define AVBD_FLAG_MATCH_NEAREST 1u
#define AVBD_FLAG_FACE_BIAS 2u
/* reuseContacts (gpu/solver.ts:181, wgsl-collision.ts:20-44, 706-753): a pair keeps last step's contact
 * points (C(x-) evaluated again, warm starts as usual) when neither body moved more than 2 mm or turned
 * more than 0.002 rad since the step that generated them; its narrowphase is skipped. */
#define AVBD_FLAG_REUSE_CONTACTS 4u
#define AVBD_FLAG_START_AT_REST 8u
#define AVBD_FLAG_MASS_PENALTY 16u
/* Contact key bit: static friction held last step (layout.ts:130). */
#define AVBD_STICK_BIT 0x80000000u
/* Colour state (avbd2d/gpu/layout.ts:42-43, wgsl-topology.ts:81). */
#define AVBD_NO_COLOR 255u
#define AVBD_PENDING 256u
#define AVBD_MAX_COLORS 64u
/* Unbounded stiffness / thresholds are stored as BIG; a row is hard at >= 1e30 (avbd2d/gpu/layout.ts:99-100). */
#define AVBD_BIG 3.0e38f

/* One body: the reference's 10-vec4 record (layout.ts:8-59, struct Body at :219-230). */
typedef struct avbd_body {
  float pos[3], friction;
  float rot[4];            /* quaternion x, y, z, w */
  float initial_pos[3];    /* x- (pose at the start of the step) */
  float flags;             /* 1: rewritten slot (no contact history), 2: disabled, 4: cold */
  float initial_rot[4];
  float size[3], mass;     /* full widths; mass 0 = static */
  float moment[3], radius; /* principal moments; bounding radius */
  float inertial_pos[3];   /* inertial target y */
  float moved_step;        /* u32 bits: the step the body last moved past the contact-reuse tolerances */
  float inertial_rot[4];
  float vel[3], prev_up_vel; /* velocity; last step's velocity along up */
  float ang_vel[3], shape;   /* angular velocity; AVBD_SHAPE_* */
} avbd_body;

/* One joint or spring slot: the reference's 10-vec4 record (layout.ts:77-110, :232-243). */
typedef struct avbd_joint {
  float pen_lin[3], stiffness_lin; /* spring: w = its stiffness */
  float pen_ang[3], stiffness_ang;
  float lam_lin[3], fracture;      /* fracture on |lam_ang| (negative: on |lam_lin| too); BIG: never */
  float lam_ang[3], torque_arm;
  float c0_lin[4];
  float c0_ang[3], yield_force;    /* BIG: never yields */
  float r_a[3], spring_rest;       /* r_a: world point when a = -1 */
  float r_b[3], break_bend;        /* BIG: never */
  float rest[4];                   /* rotB = rotA * rest */
  float rest_start[4];
} avbd_joint;

typedef struct avbd_joint_info {
  int32_t type; /* AVBD_T_* */
  int32_t a;    /* body index, -1: the world */
  int32_t b;
  int32_t meta; /* 0 */
} avbd_joint_info;

/* A contact pair (layout.ts:118-120, struct Manifold :245-248): a > b, contacts [first, first+count). */
typedef struct avbd_manifold {
  uint32_t a, b, first, count;
  float normal[3], friction; /* normal from B to A */
} avbd_manifold;

/* A contact point (layout.ts:122-127, struct Contact :254-263). */
typedef struct avbd_contact {
  float r_a[3];
  uint32_t key; /* feature | AVBD_STICK_BIT */
  float r_b[3], c0_n;
  float pen[3], c0_t1;
  float lam[3], c0_t2;
} avbd_contact;

/* SolverParams (ref/solver.ts:139-165) and the GPU flags (gpu/solver.ts:174-231). */
typedef struct avbd_params {
  float dt, gravity, alpha, beta_lin, beta_ang, gamma;
  float contact_margin;
  int32_t iterations;
  uint32_t flags; /* AVBD_FLAG_* */
  float up[3];    /* unit vector; gravity pulls along -up */
  /* The wind on sails (GpuParams3D windSpeed, windAngle, windGust, windPressure, gpu/solver.ts:200-206,
   * applied in warmStartBodies, wgsl-solve.ts:262-335): speed (m/s) towards wind_angle (rad from +x
   * about z), gusts of wind_gust of the speed, wind_pressure = 1/2 rho C_d (kg/m^3); 0: no air. */
  float wind_speed, wind_angle, wind_gust, wind_pressure;
} avbd_params;

typedef struct avbd_config {
  uint32_t body_capacity;  /* 0: 1024 */
  uint32_t joint_capacity; /* 0: 256 */
  uint32_t pair_capacity;  /* 0: max(65536, 8 x body_capacity); grows on overflow */
  int32_t device;          /* CUDA device ordinal */
} avbd_config;

/* readCounters (gpu/solver.ts:2305-2309). */
typedef struct avbd_counters {
  uint32_t pairs, contacts, manifolds, overflow; /* overflow: 1 pairs, 2 contacts, 4 manifolds */
  uint32_t clashes, colors, rounds, error;       /* error: nonzero after a bounded wait gave up */
  uint32_t steps, pair_capacity, graphs, launches; /* graphs: steps replay a CUDA graph; launches: kernels per step */
} avbd_counters;

typedef struct avbd_world avbd_world;

/* Library. */
int avbd_abi_version(void);
/* Device name and SM count, for reports. */
int avbd_device_info(int device, char* name, size_t name_cap, int* sm_count);

/* Construction: `new GpuSolver3D(device, ref, options)` (gpu/solver.ts:722) / World.create (world.ts:880-927). */
int avbd_world_create(const avbd_config* config, avbd_world** out);
/* destroy() (gpu/solver.ts:2439-2459): idempotent on NULL. */
int avbd_world_destroy(avbd_world* world);
const char* avbd_last_error(const avbd_world* world);

/* params (GpuParams3D, gpu/solver.ts:163-231). */
int avbd_set_params(avbd_world* world, const avbd_params* params);
int avbd_get_params(const avbd_world* world, avbd_params* params);
/* Defaults of the reference's SolverParams with every GPU-only rule off, up = +z and no air (sails
 * fall as the reference's CPU solver lets them: the reference's parity setting,
 * avbd3d-gpu.gpu.test.ts:47-52). */
int avbd_default_params(avbd_params* params);
/* gpuParams3D() (gpu/solver.ts:216-230), what a World runs with: the reference's SolverParams, every
 * GPU-only rule on (matchNearest, faceBias, reuseContacts, startAtRest, massPenalty), contact margin
 * 0.01, up = +y, calm air (speed 0, gusts 0.4, pressure 0.72). */
int avbd_world_params(avbd_params* params);

/* addBodies (gpu/solver.ts:1469-1481): appends; *first = index of the first. */
int avbd_add_bodies(avbd_world* world, const avbd_body* bodies, uint32_t n, uint32_t* first);
/* rewriteBodies / patchBody (gpu/solver.ts:1113-1139): overwrite bodies [first, first+n);
 * keep_contacts != 0 keeps their contact history (seedFrom), else the slots start fresh. */
int avbd_write_bodies(avbd_world* world, uint32_t first, const avbd_body* bodies, uint32_t n, int keep_contacts);
/* rewriteBodies(indices, bodies) (gpu/solver.ts:1774-1784) for any list of existing slots: every
 * record is checked before any is written; each slot starts afresh. */
int avbd_write_bodies_at(avbd_world* world, const uint32_t* indices, const avbd_body* bodies, uint32_t n);
/* appendJoints / appendSprings (gpu/solver.ts:1484-1533): appends slots; *first = first slot. */
int avbd_add_joints(avbd_world* world, const avbd_joint* joints, const avbd_joint_info* info, uint32_t n, uint32_t* first);
/* seedFrom's joint rewrite (gpu/solver.ts:1330-1331). */
int avbd_write_joints(avbd_world* world, uint32_t first, const avbd_joint* joints, const avbd_joint_info* info, uint32_t n);
/* appendJoints / appendSprings through appendConstraints (gpu/solver.ts:1709-1738): released slots
 * are taken first (lowest first), then new slots at the end; slots[k] receives joint k's slot. */
int avbd_append_joints(avbd_world* world, const avbd_joint* joints, const avbd_joint_info* info, uint32_t n, uint32_t* slots);
/* releaseJoints (gpu/solver.ts:1745-1771): each slot in range and not yet released stops acting (record
 * zeroed, info AVBD_T_NONE with bodies -1), its two bodies collide again, and the slot goes to the
 * free list that avbd_append_joints takes from. Slots out of range or already released are ignored. */
int avbd_release_joints(avbd_world* world, const uint32_t* slots, uint32_t n);
/* disableConstraint (gpu/solver.ts:1941-1947): penalties, stiffnesses and multipliers zeroed
 * (fracture and torque arm kept); the slot stays taken. */
int avbd_disable_joints(avbd_world* world, const uint32_t* slots, uint32_t n);
/* appendWorldJoint(b, anchorWorld, anchorBody) with the 'legacy' policy (gpu/solver.ts:1592-1623):
 * appends a joint holding body b's point anchor_body (body frame) at the world point anchor_world:
 * hard linear rows, no angular rows (the body turns freely about the point), never breaking, torque
 * arm |size|^2 of the body. *slot receives its slot. ('inertial-hard' needs the reference's native
 * sensor shaders and has no counterpart.) */
int avbd_add_world_joint(avbd_world* world, uint32_t body, const float anchor_world[3], const float anchor_body[3], uint32_t* slot);
/* setWorldAnchor(slot, p) (gpu/solver.ts:1937-1939): the slot's r_a (a world joint's world point)
 * becomes p from the next step on. */
int avbd_set_world_anchor(avbd_world* world, uint32_t slot, const float p[3]);
/* IgnoreCollision pairs (ref/forces.ts:384-390; no-collide table gpu/no-collide.ts). */
int avbd_add_ignore_pairs(avbd_world* world, const uint32_t* pairs_ab, uint32_t n);
/* setFilters (gpu/solver.ts): groups_mask[2i] = groups, [2i+1] = collides-with mask. */
int avbd_set_filters(avbd_world* world, uint32_t first, const uint32_t* groups_mask, uint32_t n);
/* setFilters(indices, groups, collidesWith) (gpu/solver.ts:1791-1801) for any list of slots. */
int avbd_set_filters_at(avbd_world* world, const uint32_t* indices, const uint32_t* groups, const uint32_t* collides_with, uint32_t n);
/* setBodyAux(indices, scales, linear?, angular?) (gpu/solver.ts:1814-1845; record layout.ts:33-46):
 * per-slot gravity scale (default 1) and linear / angular damping rates in 1/s (default 0; a
 * dynamic body's incoming velocities decay by exp(-rate dt) once per step, before its inertial
 * target). linear and angular: both given, or both NULL, when a lone slot (no consecutive
 * neighbour in `indices`) keeps its rates and a run of consecutive slots gets the default rates, as
 * setBodyAux writes whole records for runs (:1826-1845). */
int avbd_set_body_aux(avbd_world* world, const uint32_t* indices, uint32_t n, const float* scales, const float* linear, const float* angular);
/* The aux records of slots first .. first + n - 1: 4 floats each (scale, linear, angular, 0). */
int avbd_read_body_aux(avbd_world* world, uint32_t first, float* aux4, uint32_t n);
/* setLifecycle(index, bits) (gpu/solver.ts:2069-2076): bits 2 disabled (the body takes no part),
 * 4 cold (its joints start the next step without warm start); the slot loses its contact history. */
int avbd_set_lifecycle(avbd_world* world, uint32_t index, uint32_t bits);

/* Convex hulls (src/avbd3d/hull.ts, gpu/wgsl-hull.ts). A hull record is the reference's packed
 * layout (gpu/solver.ts:313-338 packHull with its header at vec4 0), 4 words per vec4:
 *   header: vertex start, vertex count, face start, face count | edge start, edge count, index start, 0
 *   vertices (x, y, z as f32 bits), faces (normal + plane offset as f32 bits, then first index and
 *   vertex count), vertex indices (4 a vec4), edges (vertex a, vertex b, face on each side),
 * all in the body's principal frame. */
typedef struct avbd_hull_props {
  double volume;                   /* per unit density */
  double moments[3];               /* principal moments per unit density */
  double size[3];                  /* full widths of the vertex bounds (principal frame) */
  double radius;                   /* farthest vertex from the centre of mass */
  double center[3];                /* where the principal frame sits in the points' frame */
  double rotation[4];              /* its rotation, x y z w */
  uint32_t vertices, faces, edges; /* counts */
} avbd_hull_props;
/* convexHull(points) (hull.ts:60-75): the hull of n xyz points, simplified to
 * AVBD_MAX_HULL_VERTICES by farthest-point sampling; AVBD_ERR_INVALID when the points span no
 * volume. Host code (no device needed). *vec4s receives the record's size; with packed NULL only
 * the size and props are returned. */
int avbd_hull_build(const float* points, uint32_t n, uint32_t* packed, uint32_t cap_vec4s, uint32_t* vec4s, avbd_hull_props* props);
/* The hull buffer's append (gpu/solver.ts:1390-1410, pinHull): copies one packed record (header at
 * vec4 0) into the world's hull buffer; *offset receives its header offset (shape code - 3).
 * Records are validated (counts, index ranges); a body naming an offset that is not a hull header
 * is rejected by avbd_add_bodies / avbd_write_bodies. */
int avbd_add_hull(avbd_world* world, const uint32_t* packed, uint32_t vec4s, uint32_t* offset);
/* releaseHull (gpu/solver.ts:1408-1414, unpinHull :1448-1454): the record's run goes to the free list
 * (merged with free neighbours) and the next avbd_add_hull that fits reuses it. Refused while a
 * body's shape names the record. Reference counting per shape stays with the caller. */
int avbd_release_hull(avbd_world* world, uint32_t offset);
/* The hull buffer: top (vec4s in use or freed), device capacity and the largest free run; an
 * adaptive world grows, so a hull always fits (canPinHull, :1421-1432). */
int avbd_hull_storage(const avbd_world* world, uint32_t* top, uint32_t* capacity, uint32_t* largest_free);
/* seedFrom's contact import (gpu/solver.ts:1320-1359): last step's manifolds and contacts, the
 * next step's warm-start source. manifold.first indexes `contacts`. */
int avbd_seed_contacts(avbd_world* world, const avbd_manifold* manifolds, uint32_t n_manifolds, const avbd_contact* contacts,
                       uint32_t n_contacts);
/* fixedColors (gpu/solver.ts:560, 2130-2134): one colour per body (AVBD_NO_COLOR for none), or
 * NULL to return to the Jones-Plassmann colouring. */
int avbd_set_fixed_colors(avbd_world* world, const uint32_t* colors, uint32_t n);

/* step() (gpu/solver.ts:2112-2295): n steps, enqueued on the world's stream (asynchronous). */
int avbd_step(avbd_world* world, int n);
/* step(options) (GpuStepOptions, gpu/solver.ts:42-50). reuse_manifolds != 0: the step detects no pair
 * and keeps every manifold of the step before (normals, anchors, keys), evaluating C(x-) again and
 * warm-starting as usual, for substeps after a detecting step; it applies only while last step's
 * manifolds are valid (a step ran and no body, joint, filter, lifecycle or contact write came since),
 * else the step detects as usual. NULL options: avbd_step. */
typedef struct avbd_step_options {
  uint32_t reuse_manifolds;
} avbd_step_options;
int avbd_step_with(avbd_world* world, int n, const avbd_step_options* options);
/* Contact-reuse state: per body its reference pose (8 floats: x y z 0 and rotation x y z w; a zero
 * rotation: none yet; the step it last moved is the body record's moved_step word, as u32 bits), and
 * per manifold (avbd_read_contacts' order) the step whose narrowphase generated its points. */
int avbd_read_reuse_state(avbd_world* world, float* ref_poses, uint32_t body_cap, uint32_t* n_bodies, uint32_t* generations, uint32_t manifold_cap,
                          uint32_t* n_manifolds);
/* Waits for the world's stream; reports a device error or a bounded wait that gave up. */
int avbd_synchronize(avbd_world* world);

/* Readbacks (synchronous): readBodies / readJoints / readContactList / readPairs / readCounters
 * (gpu/solver.ts:2297-2360). *n receives the number available; at most `cap` are written. */
int avbd_read_bodies(avbd_world* world, avbd_body* dst, uint32_t cap, uint32_t* n);
int avbd_read_joints(avbd_world* world, avbd_joint* dst, avbd_joint_info* info, uint32_t cap, uint32_t* n);
int avbd_read_contacts(avbd_world* world, avbd_manifold* manifolds, uint32_t manifold_cap, uint32_t* n_manifolds, avbd_contact* contacts,
                       uint32_t contact_cap, uint32_t* n_contacts);
int avbd_read_pairs(avbd_world* world, uint32_t* dst_ab, uint32_t cap, uint32_t* n);
int avbd_read_colors(avbd_world* world, uint32_t* dst, uint32_t cap, uint32_t* n);
int avbd_read_counters(avbd_world* world, avbd_counters* counters);

/* Asynchronous pose readback into caller memory (pinned for overlap): World.read (world.ts:2102-2224). */
int avbd_read_bodies_async(avbd_world* world, avbd_body* dst, uint32_t cap);

/* Per-step statistics (profileNextStep / readCounters, gpu/solver.ts:1951-1953, 2305-2309): with
 * avbd_enable_step_stats(world, capacity) each step writes the device-clock times of its two phases
 * (collision: from the step's first kernel to the solve kernel's start; solve: the topology+solve
 * kernel) and a snapshot of its counters into a device ring of `capacity` entries, inside the step
 * (so it works under graph replay, without host synchronisation); avbd_read_step_stats returns the
 * entries oldest first. capacity 0 turns it off. */
typedef struct avbd_step_stats {
  float collision_ms, solve_ms;  /* broadphase + narrowphase; topology + warm start + iterations + velocities */
  uint32_t pairs, contacts, manifolds, adjacency, incidences, dynamic_bodies, colors, rounds, launches, error;
} avbd_step_stats;
int avbd_enable_step_stats(avbd_world* world, uint32_t capacity);
int avbd_read_step_stats(avbd_world* world, avbd_step_stats* dst, uint32_t cap, uint32_t* n);

/* Device time (ms from the start of the topology+solve launch) at each of its grid barriers in the
 * last step: the per-phase profile of the persistent kernel (profileNextStep's phases, gpu/solver.ts:2159-2172). */
int avbd_read_phase_clocks(avbd_world* world, double* dst, uint32_t cap, uint32_t* n);

/* Steps replay a captured CUDA graph (default on; per-step statistics launch directly). */
int avbd_use_graphs(avbd_world* world, int enable);

/* Blocks of the cooperative topology + solve launch (0: every co-resident block, the default). The
 * lane groups a body's rows are summed in depend on the launch's thread count, so results differ in
 * the last bits between launch shapes; one block reproduces a batched world's step bit for bit. */
int avbd_set_solve_blocks(avbd_world* world, int blocks);

/* The broadphase's classification of bodies by bounding radius (gpu/radii.ts largestSmall, and
 * uploadStatics, gpu/solver.ts:1263-1318): the largest radius still small (at most 2 x the median,
 * or, past 64 larger bodies, the largest left), which sizes the grid cells (2 x it), and the radius
 * above which a body is "large" and tested against every body (halfway to the smallest large one).
 * Host code (no device needed). */
int avbd_broadphase_radii(const double* radii, uint32_t n, double* largest_small, double* large_threshold);

/* The world's CUDA stream (cudaStream_t) for callers that order their own device work with its steps. */
int avbd_world_stream(avbd_world* world, void** stream);

/* Device views of the world's storage for CUDA consumers on its device, as the reference hands its
 * buffers to ContactWatch, Pusher and BodyMover (bodyBuffer, contactStorage / contactStorages(),
 * gpu/solver.ts:638-650; world.ts:854-862). Read or write them in stream order with the world's
 * steps (avbd_world_stream). Body arrays stay where they are for the world's lifetime (the body
 * capacity is fixed at creation); contact arrays move when pair storage grows (at a step, after 80 %
 * use or an overflow bit), so query them again after each step. */
typedef struct avbd_body_view {
  void* fields[10];   /* one float4 array per row of the avbd_body record, in record order:
                         pos + friction, rot, initial pos + flags, initial rot, size + mass,
                         moment + radius, inertial pos, inertial rot, vel + prev up vel, ang vel + shape */
  uint32_t count;     /* bodies in use */
  uint32_t capacity;  /* length of each array */
} avbd_body_view;
int avbd_body_storage(avbd_world* world, avbd_body_view* out);

typedef struct avbd_contact_view {
  const void* pairs;         /* uint4 per pair slot: a, b, first point slot (8 x slot), count | step << 4; count 0: no manifold */
  const void* normals;       /* float4 per pair slot: normal (B to A), friction */
  const void* points;        /* avbd_contact per point slot: pair slot p's points at 8p .. 8p + count - 1 */
  const uint32_t* counters;  /* the world's device counter words */
  uint32_t count_word;       /* counters[count_word]: pair slots this storage holds */
  uint32_t pair_capacity;    /* pair slots (points: 8 x) */
} avbd_contact_view;
/* which 0: the storage the last step wrote (contactStorage); 1: the one the step before wrote, which
 * the next step overwrites (the other entry of contactStorages()). */
int avbd_contact_storage(avbd_world* world, uint32_t which, avbd_contact_view* out);

/* Pose/velocity update from caller memory (pinned for overlap), enqueued on the world's stream
 * without validation or synchronisation: shapes, masses and radii must be unchanged (use
 * avbd_write_bodies for those). Keeps the bodies' contact history. */
int avbd_write_bodies_async(avbd_world* world, uint32_t first, const avbd_body* bodies, uint32_t n);

/* Broadphase without allocation. No counterpart in the reference. The step's candidate pairs
 * (the rule of the step's broadphase: groups/mask, bounding spheres, AABBs + 1e-4, face separation)
 * of n <= AVBD_NOALLOC_MAX_BODIES host body records, found in one block with every intermediate array
 * in one fixed device array of AVBD_NOALLOC_SCRATCH_BYTES; it allocates no device or pinned memory.
 * For callers that cannot allocate (a thread querying pairs while steps run on other streams, since
 * cudaMalloc/cudaFree synchronise the device; hosts whose allocator owns all device memory).
 * groups_mask: NULL (all collide) or 2 x n words, (groups, mask) per body; the buffer must hold all
 * 2 x n words. Shapes: boxes, spheres and sails (a hull's shape code is refused with
 * AVBD_ERR_INVALID: this call has no hull buffer). Writes up to cap (a, b) pairs, a > b, in no
 * particular order, to pairs_ab and the number found to *count; returns AVBD_ERR_CAPACITY when n is
 * past the maximum (*count 0) or more pairs were found than cap or AVBD_NOALLOC_MAX_PAIRS (*count:
 * all that were found). Runs on `stream` (a cudaStream_t, NULL: the default stream) of the current
 * device and waits for it. Every call looks up the fixed array's device address on the current
 * device; the first call on a device also loads the library's device code there, so make it before
 * any stream capture on that device. All calls share the fixed array and each clears what it counts
 * in: calls whose GPU work overlaps (two host threads, two streams) race on it. */
#define AVBD_NOALLOC_MAX_BODIES 4096u
#define AVBD_NOALLOC_MAX_PAIRS 32768u
#define AVBD_NOALLOC_SCRATCH_BYTES 1065472u
int avbd_find_pairs_noalloc(const avbd_body* bodies, uint32_t n, const uint32_t* groups_mask, uint32_t* pairs_ab, uint32_t cap, uint32_t* count,
                            void* stream);

/* ---- Around the step: impulses, contact events, raycasts -------------------------------------------
 * The passes a World runs beside the solver (world.ts:1736-1738 and its queries), on the world's
 * device state and stream. */

/* Pusher.apply (src/lib/push.ts:103-131): impulses on bodies before the next step. Per pushed body (each
 * slot at most once: sum a body's pushes first, as addImpulse does): lin the whole linear impulse (N s),
 * off_lin the part of it applied at points, moment those parts' moment about the world origin plus any
 * angular impulse. A dynamic, enabled body's velocity gains lin / mass and its angular velocity
 * I^-1 (moment - x cross off_lin) taken in its principal frame, at the pose the device holds; static and
 * disabled bodies are left alone. Waits for the world's stream. */
typedef struct avbd_push {
  uint32_t body;
  float lin[3];
  float off_lin[3];
  float moment[3];
} avbd_push;
int avbd_apply_pushes(avbd_world* world, const avbd_push* pushes, uint32_t n);

/* ContactWatch (src/lib/contacts.ts:129-267): after each step (avbd_contact_watch_run), the touching
 * pairs with a reporting body go into this step's set; a pair missing from last step's set began
 * touching (where: its points' mean on body a; how hard: |sum of its normal multipliers| dt; the normal
 * from b to a), and one of last step's set missing from this step's ended. Bodies are reported by
 * lifetime IDs (1 .. 2^31 - 1) set per slot, so events survive slot reuse. Events accumulate on the
 * device until avbd_contact_watch_read; past `capacity` they are counted as dropped; a step with more
 * touching pairs than a set holds (2 x `pairs`, a power of two) sets `full`, and that step's events
 * are unreliable. The watch reads the world's storage: destroy it before the world. */
#define AVBD_CONTACT_BEGIN 1u
#define AVBD_CONTACT_END 2u
typedef struct avbd_contact_event {
  uint32_t kind, a, b, step; /* AVBD_CONTACT_*, lifetime IDs of the pair's bodies (a's slot > b's), the step */
  float point[3], impulse;   /* a begin's point and normal impulse */
  float normal[3], pad;      /* a begin's normal (b to a) */
} avbd_contact_event;
typedef struct avbd_contact_watch avbd_contact_watch;
int avbd_contact_watch_create(avbd_world* world, uint32_t pairs, uint32_t capacity, avbd_contact_watch** out);
int avbd_contact_watch_destroy(avbd_contact_watch* watch);
const char* avbd_contact_watch_last_error(const avbd_contact_watch* watch);
/* setWatched(indices, ids, on): slot indices[k] reports (on[k] != 0) under lifetime ID ids[k] */
int avbd_contact_watch_set(avbd_contact_watch* watch, const uint32_t* indices, const uint32_t* ids, const uint32_t* on, uint32_t n);
/* run(storage, pairs, step, dt): after a step, enqueued on the world's stream */
int avbd_contact_watch_run(avbd_contact_watch* watch, uint32_t step, float dt);
/* read(): the events since the last read, in step order (within a step as the device wrote them), and
 * clears them; *n the events held, *dropped those past the capacity, *full whether a set overflowed */
int avbd_contact_watch_read(avbd_contact_watch* watch, avbd_contact_event* dst, uint32_t cap, uint32_t* n, uint32_t* dropped, uint32_t* full);

/* Raycaster.cast (src/lib/raycast.ts:170-251): the nearest hit of each ray among the world's bodies
 * (boxes and sails by their faces, spheres, hulls by their face planes) at the poses the device holds,
 * skipping disabled bodies, bodies whose groups miss `mask`, and the `ignore` slots. A hit at the same
 * distance as another goes to the lower slot. direction is normalised here (a zero direction stays
 * zero); max_distance caps the hit distance (values past 3e38: no cap). A ray starting inside a body
 * hits it at distance 0 with the normal against the ray. hit.body -1 (distance -1): no hit. */
#define AVBD_RAY_MAX 65535u
#define AVBD_RAY_MAX_IGNORED 16u
typedef struct avbd_ray {
  float origin[3], max_distance;
  float direction[3], pad;
} avbd_ray;
typedef struct avbd_ray_hit {
  int32_t body;
  float distance;
  float point[3];  /* origin + direction * distance */
  float normal[3]; /* world axes */
} avbd_ray_hit;
int avbd_raycast(avbd_world* world, const avbd_ray* rays, uint32_t n, const uint32_t* ignore, uint32_t n_ignore, uint32_t mask, avbd_ray_hit* hits);

/* ---- Pose capture: the frames of the pose cache (src/bake/pose-cache.ts) -------------------------
 * A recorder on the device: up to max_frames frames of the listed body slots, a frame being the
 * world's step word (steps since the world was made) and 7 f32 per slot, position then rotation
 * x y z w (the cache's slot layout, POSE_FLOATS), or +0 for a disabled slot. A frame is gathered by
 * one kernel on the world's stream when the stream reaches it, so capturing every k-th step costs no
 * host synchronisation; the host side writes the cache format (avbd_b200.pose_cache). */
typedef struct avbd_pose_capture avbd_pose_capture;
int avbd_pose_capture_create(avbd_world* world, const uint32_t* slots, uint32_t n, uint32_t max_frames, avbd_pose_capture** out);
/* One frame of the poses the world holds when its stream gets here; past max_frames it is dropped
 * and counted. */
int avbd_pose_capture_frame(avbd_pose_capture* capture);
/* Waits for the world's stream; *frames = frames held, *dropped = frames refused for room; copies
 * min(frames, cap) frames: steps[cap], poses[cap x n x 7]. */
int avbd_pose_capture_read(avbd_pose_capture* capture, uint32_t* steps, float* poses, uint32_t cap, uint32_t* frames, uint32_t* dropped);
int avbd_pose_capture_reset(avbd_pose_capture* capture);
int avbd_pose_capture_destroy(avbd_pose_capture* capture);

/* ---- Adjoint --------------------------------------------------------------------------------------
 * No counterpart in the reference (it has no differentiation). Gradients of a pose loss
 * L = sum over dynamic bodies of |x_T - x*|^2 + |q_T - q*|^2 after a recorded rollout, with respect
 * to every body's initial linear and angular velocity, mass (moments in proportion) and friction
 * coefficient, in double precision, for batched worlds of boxes on static bodies (no joints). The
 * step is differentiated with its contact structure frozen from the recording: per step the pairs
 * and their normal bases, each point's body-frame anchors and the last-step point it warm-starts
 * from, and the colouring; everything else (C(x-), warm starts, inertial targets, the coloured
 * primal solves, duals with penalty ramps and friction cone, velocities) is differentiated. The
 * replay keeps a checkpoint every `checkpoint` steps and recomputes between them. A world holds at
 * most 128 bodies and 1024 points a step. */
typedef struct avbd_adjoint avbd_adjoint;
typedef struct avbd_adjoint_desc {
  uint32_t worlds, steps, iterations, checkpoint; /* checkpoint 0: every 10 steps */
  double dt, gravity, alpha, gamma, beta_lin, contact_margin;
  const uint32_t* world_first_body;    /* worlds + 1 */
  const double* bodies;                /* 13 per body: pos3 rot4 prev_up_vel unit_moment3 dynamic friction */
  const uint32_t* step_first_manifold; /* steps x (worlds + 1), global indices */
  const uint32_t* step_first_point;    /* steps x (worlds + 1) */
  const int32_t* manifold_bodies;      /* 2 per manifold, world-local (a > b) */
  const double* manifold_basis;        /* 9 per manifold: rows n (B to A), t1, t2 */
  const double* point_anchors;         /* 6 per point: rA, rB in body frames */
  const int32_t* point_manifold;       /* global manifold index */
  const int32_t* point_prev;           /* global index of the last step's point it warm-starts from, or -1 */
  const int32_t* colors;               /* steps x bodies (-1: static) */
  const int32_t* color_counts;         /* steps x worlds */
  int32_t device;
} avbd_adjoint_desc;
int avbd_adjoint_create(const avbd_adjoint_desc* desc, avbd_adjoint** out);
int avbd_adjoint_destroy(avbd_adjoint* adjoint);
const char* avbd_adjoint_last_error(const avbd_adjoint* adjoint);
/* target: 7 per body (pos, rot x y z w) */
int avbd_adjoint_set_target(avbd_adjoint* adjoint, const double* target);
/* params: 8 per body (v0 xyz, omega0 xyz, mass, friction); loss per world; final poses 7 per body (or NULL) */
int avbd_adjoint_forward(avbd_adjoint* adjoint, const double* params, double* loss, double* final_pose);
/* the reverse sweep, after a replay unless the last call was a forward with the same params: grad 8
 * per body (as params), loss per world (or NULL) */
int avbd_adjoint_backward(avbd_adjoint* adjoint, const double* params, double* grad, double* loss);

/* ---- Batched worlds ------------------------------------------------------------------------------
 * No counterpart in the reference, which steps one world per GpuSolver3D (gpu/solver.ts:598). A batch
 * holds many small independent worlds (1 to AVBD_BATCH_MAX_WORLD_BODIES bodies each) and steps them
 * all with two launches per step, one block per world, captured in a CUDA graph. Each world runs
 * exactly the single-world step (pair rule, narrowphase, warm start, Jones-Plassmann colouring,
 * Gauss-Seidel solve, dual, velocities) on its own bodies; indices inside a world are local to it.
 * The worlds share one avbd_params. Not thread-safe; one stream per batch. */
typedef struct avbd_batch avbd_batch;

#define AVBD_BATCH_MAX_WORLD_BODIES 4096u
#define AVBD_BATCH_TUNE_CANDIDATES 16

typedef struct avbd_batch_config {
  uint32_t world_capacity; /* worlds */
  uint32_t body_capacity;  /* bodies over all worlds */
  uint32_t joint_capacity; /* joints over all worlds */
  uint32_t pairs_per_body; /* a new world's pair slots per body (0: 6); grows per world as needed */
  int32_t device;
} avbd_batch_config;

typedef struct avbd_batch_world {
  uint32_t first_body, bodies, first_joint, joints, pair_capacity, fixed_colors;
} avbd_batch_world;

typedef struct avbd_batch_status {
  uint32_t worlds, bodies, joints, steps;
  uint64_t pair_slots;
  uint32_t relayouts; /* times pair storage was laid out again for a world that outgrew it */
  uint32_t collide_threads, collide_blocks, solve_blocks, graphs;
  uint32_t rows_per_lane; /* the solve's least rows a lane of a body's group */
  uint32_t world_threads; /* the solve's threads a world: 256 (a block a world), 128, 64 or 32 */
} avbd_batch_status;

/* The autotuner's measurements: per candidate launch shape (collision block size, solve blocks,
 * bodies per warp as the least rows a lane of a body's group takes: 1, or 4, and the threads a world:
 * a block, four, two or one warp) its mean step time */
typedef struct avbd_batch_tuning {
  uint32_t candidates;
  uint32_t candidate_threads[AVBD_BATCH_TUNE_CANDIDATES];
  uint32_t candidate_solve_blocks[AVBD_BATCH_TUNE_CANDIDATES];
  uint32_t candidate_rows_per_lane[AVBD_BATCH_TUNE_CANDIDATES];
  float candidate_ms[AVBD_BATCH_TUNE_CANDIDATES];
  uint32_t collide_threads, solve_blocks, rows_per_lane; /* the choice */
  float ms_per_step;
  uint32_t steps_taken; /* tuning steps are real steps: the worlds advance by this many */
  uint32_t candidate_world_threads[AVBD_BATCH_TUNE_CANDIDATES]; /* 256: a block a world; 128, 64, 32: part of one */
  uint32_t world_threads;                                        /* the choice */
} avbd_batch_tuning;

int avbd_batch_create(const avbd_batch_config* config, avbd_batch** out);
int avbd_batch_destroy(avbd_batch* batch);
const char* avbd_batch_last_error(const avbd_batch* batch);
int avbd_batch_set_params(avbd_batch* batch, const avbd_params* params);
/* A new world from host records (as avbd_add_bodies + avbd_add_joints + avbd_add_ignore_pairs on a
 * fresh world); joint and ignore-pair indices are local to the world. */
int avbd_batch_add_world(avbd_batch* batch, const avbd_body* bodies, uint32_t n, const avbd_joint* joints, const avbd_joint_info* info,
                         uint32_t n_joints, const uint32_t* ignore_pairs_ab, uint32_t n_ignore, uint32_t* index);
/* A new world that continues a single world exactly: bodies, joints, filters, no-collide pairs, last
 * step's contacts (warm starts), colour state and fixed colours are copied from it. */
int avbd_batch_add_world_from(avbd_batch* batch, avbd_world* world, uint32_t* index);
int avbd_batch_world_info(avbd_batch* batch, uint32_t world, avbd_batch_world* out);
int avbd_batch_step(avbd_batch* batch, int n);
int avbd_batch_synchronize(avbd_batch* batch);
int avbd_batch_read_bodies(avbd_batch* batch, uint32_t world, avbd_body* dst, uint32_t cap, uint32_t* n);
int avbd_batch_read_joints(avbd_batch* batch, uint32_t world, avbd_joint* dst, avbd_joint_info* info, uint32_t cap, uint32_t* n);
int avbd_batch_read_colors(avbd_batch* batch, uint32_t world, uint32_t* dst, uint32_t cap, uint32_t* n);
int avbd_batch_read_counters(avbd_batch* batch, uint32_t world, avbd_counters* counters);
/* Every world's bodies in batch order (world w at its first_body), on the batch's stream */
int avbd_batch_read_all_bodies_async(avbd_batch* batch, avbd_body* dst, uint32_t cap);
int avbd_batch_write_all_bodies_async(avbd_batch* batch, const avbd_body* src, uint32_t n);
int avbd_batch_use_graphs(avbd_batch* batch, int enable);
int avbd_batch_stream(avbd_batch* batch, void** stream);
/* Times each candidate launch shape over `steps` real steps and keeps the fastest: the collision
 * block size first, then the solve's threads a world x solve blocks, then four rows a lane. */
int avbd_batch_tune(avbd_batch* batch, int steps, avbd_batch_tuning* out);
/* Sets the launch shape the tuner would choose: collision block size (64, 128 or 256), solve blocks
 * (0: as many as fit), the least rows a lane (1 to 8) and the solve's threads a world (256: a block a
 * world; 128, 64 or 32: two, four or eight worlds a block). Every shape gives the same results bit for
 * bit. No counterpart in the reference (it has no batched worlds). */
int avbd_batch_set_launch(avbd_batch* batch, uint32_t collide_threads, uint32_t solve_blocks, uint32_t rows_per_lane, uint32_t world_threads);
int avbd_batch_info(avbd_batch* batch, avbd_batch_status* out);

/* ---- Recording a batched rollout for the adjoint -------------------------------------------------
 * No counterpart in the reference. The next `steps` avbd_batch_step calls append their contact
 * structure (per step the manifolds with their normal bases, each point's body-frame anchors and
 * the last-step point it warm-started from, the colouring) to a device recording, three extra
 * launches per step. The batch must hold boxes only, no joints, default contact rules and up = +z;
 * the first recorded step must not warm-start from an earlier step (a fresh batch, or bodies
 * written again with avbd_batch_write_all_bodies_async and flag 1). points_per_body (0: 8) sizes the
 * recording: steps x bodies x points_per_body points. */
int avbd_batch_record_start(avbd_batch* batch, uint32_t steps, uint32_t points_per_body);
/* steps recorded so far, manifolds and points, problems (bits: 1 out of room, 2 warm start from before
 * the recording, 4 sphere contacts, 8 more than 64 colours) */
int avbd_batch_record_status(avbd_batch* batch, uint32_t* steps, uint64_t* manifolds, uint64_t* points, uint32_t* problems);
/* An adjoint of the recorded rollout: it adopts the batch's finished recording (the batch then
 * holds none) and starts from the bodies as they were when recording began; worlds, steps and the
 * step parameters are the batch's. */
int avbd_adjoint_create_from_batch(avbd_batch* batch, uint32_t checkpoint, avbd_adjoint** out);
/* The parameters the recording ran with: 8 per body (v0 xyz, omega0 xyz, mass, friction); zero for
 * an adjoint built from a host description */
int avbd_adjoint_nominal(const avbd_adjoint* adjoint, double* params);
/* The adjoint's recording in the avbd_adjoint_desc layout (all worlds, global indices; sizes from
 * avbd_adjoint_info): what avbd_adjoint_create would take to build the same adjoint */
int avbd_adjoint_read_recording(const avbd_adjoint* adjoint, double* bodies, int32_t* step_first_manifold, int32_t* step_first_point,
                                int32_t* manifold_bodies, double* manifold_basis, double* point_anchors, int32_t* point_manifold, int32_t* point_prev,
                                int32_t* colors, int32_t* color_counts);
/* worlds, steps, bodies, the most points of one world in one step, manifolds and points recorded */
int avbd_adjoint_info(const avbd_adjoint* adjoint, uint32_t* worlds, uint32_t* steps, uint32_t* bodies, uint32_t* max_points, uint64_t* manifolds,
                      uint64_t* points);

#ifdef __cplusplus
}
#endif

#endif /* AVBD_H */
