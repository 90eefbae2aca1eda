// Device-side layout and maths of the B200 AVBD step.
//
// Body state is structure-of-arrays of float4 (one 128-bit load per field); the field meanings
// are the reference's body record (src/avbd3d/gpu/layout.ts:8-59). Contacts live in fixed slots,
// eight per broadphase pair (pair p's points at 8p .. 8p+7), in four float4 arrays with the
// reference's contact words (layout.ts:122-127): no atomics are needed to place them and the
// points of one manifold are contiguous.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace avbd {

constexpr float PENALTY_MIN = 1.0f;        // ref/body.ts:8
constexpr float PENALTY_MAX = 1e10f;       // ref/body.ts:9
constexpr float STICK_THRESH = 0.00001f;   // ref/body.ts:11
constexpr float PIVOT_FLOOR = 1e-5f;       // gpu/layout.ts:192
constexpr float BIG = 3.0e38f;             // avbd2d/gpu/layout.ts:99
constexpr float HARD = 1e30f;              // avbd2d/gpu/layout.ts:100
constexpr uint32_t STICK_BIT = 0x80000000u;
constexpr uint32_t SPHERE_FEATURE = 3u << 24;
constexpr uint32_t NO_COLOR = 255u, PENDING = 256u;
constexpr int MAX_COLORS = 64;
constexpr int MAX_CONTACTS = 8;
constexpr float SHAPE_SPHERE_F = 1.0f;
constexpr float SHAPE_SAIL_F = 2.0f;  // a box that catches the wind on its local z faces (layout.ts:145)
constexpr uint32_t T_NONE = 0, T_JOINT = 1, T_SPRING = 2;
constexpr uint32_t FLAG_MATCH_NEAREST = 1, FLAG_FACE_BIAS = 2, FLAG_REUSE_CONTACTS = 4, FLAG_START_AT_REST = 8, FLAG_MASS_PENALTY = 16;
constexpr float REUSE_LIN_TOL = 0.002f, REUSE_ANG_TOL = 0.002f;  // gpu/layout.ts:174-175
constexpr float REST_SPEED = 0.1f;
constexpr float NEAREST_FRACTION = 0.05f;
constexpr uint32_t OWNER_BIT = 0x80000000u;  // incidence entry: this body updates the constraint's dual
// incidence partner word: index | PARTNER_DYNAMIC | PARTNER_EARLIER (its colour comes first in the sweep)
constexpr uint32_t PARTNER_DYNAMIC = 0x80000000u, PARTNER_EARLIER = 0x40000000u, PARTNER_MASK = 0x3fffffffu;
constexpr int LANE_CLASSES = 6;                // 1, 2, 4, 8, 16, 32 lanes per body
constexpr int BUCKETS = MAX_COLORS * LANE_CLASSES;
constexpr int BUCKET_WORDS = 5 * BUCKETS;  // counts | starts + total | fill cursors | lane bases | lane totals (64)
enum : int { K_RA = 0, K_RB = 1, K_PEN = 2, K_LAM = 3 };

// Counter words (device memory)
enum : int {
  C_PAIRS = 0, C_CONTACTS = 1, C_MANIFOLDS = 2, C_OVERFLOW = 3, C_CLASHES = 4, C_COLORS = 5, C_ROUNDS = 6, C_ERROR = 7,
  C_PREV_PAIRS = 8, C_ADJ = 9, C_INC = 10, C_DYN = 11, C_STEP = 12, C_PENDING = 16,  // 16..16+2*MAX_ROUND_PAIRS: pending counts per round pair
  COUNTER_WORDS = 128,
};
constexpr int MAX_ROUND_PAIRS = 32;
constexpr int MAX_CLOCKS = 1023;  // barrier timestamps kept per step
constexpr int CLOCK_T0 = MAX_CLOCKS + 1, CLOCK_WORDS = MAX_CLOCKS + 2;
constexpr int STAT_WORDS = 16;    // collision ns, solve ns, then counters (pairs, contacts, manifolds, adjacency, incidences, dynamic, colours, rounds, launches, error)
constexpr int C_STATS_NEXT = 13;  // counter word: next ring entry
constexpr int C_HULL_PAIRS = 14;  // counter word: pairs deferred to the warp-per-pair hull narrowphase
// Error bits
constexpr uint32_t ERR_BARRIER_TIMEOUT = 1, ERR_ADJ_OVERFLOW = 2, ERR_INC_OVERFLOW = 4, ERR_DEPENDENCY_TIMEOUT = 8;

// Joint record words (layout.ts:84-110), as float4 slots
enum : int { J_PEN_LIN = 0, J_PEN_ANG = 1, J_LAM_LIN = 2, J_LAM_ANG = 3, J_C0_LIN = 4, J_C0_ANG = 5, J_RA = 6, J_RB = 7, J_REST = 8, J_REST_START = 9, JOINT_VEC4 = 10 };

struct StepParams {
  float dt, gravity, alpha, betaLin, betaAng, gamma, margin;
  uint32_t flags;
  int iterations;
  float upx, upy, upz;
  // the wind on sails: velocity (x, y; m/s), gust fraction, pressure coefficient 1/2 rho C_d
  float windX, windY, windGust, windPressure;
  // broadphase
  float cellSize, largeThreshold;
  uint32_t tableMask, nLarge, nNoCollide, anyDynamicLarge;
  // sizes
  uint32_t n, nj, pairCap, hashMask, incCap, adjCap;
  uint32_t step;
  uint32_t fixedColors;  // colours come from the host (validation), no Jones-Plassmann
  uint32_t colorCap;
  uint32_t rowsPerLane;  // the least rows a lane of a body's group takes (0, 1: as the colour's size asks)
  int cur;               // which manifold/contact buffers this step writes
};

struct DWorld {
  // bodies (SoA, capacity bodyCap)
  float4 *pos, *rot, *ipos, *irot, *size, *moment, *ypos, *yrot, *vel, *avel;
  float4* aux;  // per body: gravity scale, linear and angular damping rates (1/s), 0; null: 1, 0, 0, 0
  uint2* filters;
  uint4* hulls;  // hull records (wgsl-hull.ts layout), or null when the world has none
  uint32_t* hullPairs;  // pair slots whose narrowphase runs one warp per pair (hull against hull or box)
  // joints: JOINT_VEC4 float4 per slot, AoS (a joint row reads the whole record)
  float4* joint;
  int4* jinfo;
  // broadphase statics: large body indices, then (hi, lo, slot) no-collide triples sorted by (hi, lo)
  uint32_t *large, *nocollide;
  // broadphase scratch
  uint32_t *keyA, *keyB, *valA, *valB, *radixHist;
  int4* cell;
  uint32_t *cellStart, *cellEnd;
  float4* sortedPR;  // per sorted slot: position, bounding radius
  int4* sortedCell;  // per sorted slot: cell x, y, z, body index | dynamic << 31
  float4* aabb;      // per body: world AABB half extents (this step), then per sorted slot (sortedAabb)
  float4* sortedAabb;
  uint2* pairs;
  // contact pairs and points, double-buffered (cur: this step, 1 - cur: last step)
  uint4* mIds[2];   // a, b, first (= 8 * slot), count | step << 4
  float4* mGeo[2];  // normal (B to A), friction
  float4* cPt[2];   // 4 float4 per point (layout.ts:124-127): rA + key, rB + C0.n, pen + C0.t1, lam + C0.t2
  uint32_t* hash;   // last step's pairs: slot + 1, open addressing
  // topology
  uint32_t *adjStart, *adjFill;
  uint4* adjList;  // per (body, constraint): sort key hi, key lo, constraint | rows << 28, other | dynamic << 31
  uint32_t *colorA, *colorB, *colorHist, *colorStart, *colorBodies, *fixedColor;
  uint32_t *incCount, *incStart;
  uint2* incList;         // per incidence: constraint row (joint slot, or nj + point slot) | OWNER_BIT, partner word
  uint32_t* done;         // per body: iterations finished in this step's dataflow sweep (pose and owned rows)
  uint32_t* poseDone;     // per body: iterations whose pose is written (published before its owned rows)
  uint4* laneTable;       // per lane of the dataflow sweep: body, first row, row end, L | sub << 8
  uint32_t* bucket;       // BUCKET_WORDS: counts, starts (+ total), fill cursors, lane bases, lane totals per colour
  // Per body, the step's unknowns relative to x- (kept by the solve, precise at any distance from the
  // origin, where an absolute f32 position rounds to its magnitude's ulp): dlin = x - x- and
  // dang = (2 vec(r), r.w) with r the rotation since x- (q = r q-, so qsub(q, q-) = dang.xyz); and
  // the inertial target y the same way: ylin = y - x-, yang = the rotation from q- to y's rotation.
  float4 *dlin, *dang, *ylin, *yang;
  // contact reuse (wgsl-collision.ts:20-44): per body its reference pose (zero rotation: none yet);
  // the step it last moved past the tolerances is kept in ypos.w (the record's moved_step word)
  float4 *refPos, *refRot;
  uint32_t* scanScratch;
  // bookkeeping
  uint32_t* counters;
  uint32_t* barrier;  // [0] arrive count, [1] generation
  unsigned long long* clocks;  // [0] count, [1..] device time (ns) at each grid barrier of the last step's solve, [CLOCK_T0] collision start
  uint32_t* statsRing;          // per-step statistics ring (STAT_WORDS a step), or null
  uint32_t statsCap;
};

// One world of a batch: where its slices start in the batch's concatenated arrays, and its sizes
struct WorldDesc {
  uint32_t body, n, joint, nj;          // bodies (the world's local indices start at `body`), joints
  uint32_t pair, pairCap, hash, hashMask;
  uint32_t adj, adjCap, inc, incCap;
  float largeThreshold;                 // the world's broadphase classification (radii.ts)
  uint32_t nNoCollide, noCollide;       // nNoCollide (hi, lo, slot) triples from word noCollide, world-local indices
  uint32_t flags;                       // WORLD_FIXED_COLORS
};
constexpr uint32_t WORLD_FIXED_COLORS = 1u;

// The view of world `wi` of a batch: every pointer moved to the world's slice
__host__ __device__ inline DWorld worldView(const DWorld& b, const WorldDesc& d, uint32_t wi) {
  DWorld v = b;
  float4** bodyArrays[] = {&v.pos, &v.rot, &v.ipos, &v.irot, &v.size, &v.moment, &v.ypos, &v.yrot, &v.vel, &v.avel, &v.dlin, &v.dang, &v.ylin, &v.yang, &v.refPos, &v.refRot, &v.aabb};
  for (float4** a : bodyArrays) *a += d.body;
  v.filters += d.body;
  if (v.aux) v.aux += d.body;
  v.cell += d.body;
  v.joint += size_t(d.joint) * JOINT_VEC4;
  v.jinfo += d.joint;
  v.nocollide = b.nocollide + d.noCollide;
  v.pairs += d.pair;
  for (int k = 0; k < 2; k++) {
    v.mIds[k] += d.pair;
    v.mGeo[k] += d.pair;
    v.cPt[k] += size_t(d.pair) * MAX_CONTACTS * 4;
  }
  v.hash += d.hash;
  v.adjStart += d.body + wi;
  v.adjFill += d.body + wi;
  v.adjList += d.adj;
  v.colorA += d.body;
  v.colorB += d.body;
  v.colorBodies += d.body;
  v.fixedColor += d.body;
  v.done = nullptr;
  v.laneTable = nullptr;
  v.incCount += d.body;
  v.incStart += d.body + wi;
  v.incList += d.inc;
  v.bucket += size_t(wi) * BUCKET_WORDS;
  v.colorStart += size_t(wi) * (MAX_COLORS + 1);
  v.scanScratch += size_t(wi) * 2;
  v.counters += size_t(wi) * COUNTER_WORDS;
  v.clocks = nullptr;
  v.statsRing = nullptr;
  v.statsCap = 0;
  return v;
}

// The step parameters of one world of a batch: the batch's shared ones with the world's sizes
__host__ __device__ inline StepParams worldParams(const StepParams& shared, const WorldDesc& d) {
  StepParams p = shared;
  p.n = d.n;
  p.nj = d.nj;
  p.pairCap = d.pairCap;
  p.hashMask = d.hashMask;
  p.incCap = d.incCap;
  p.adjCap = d.adjCap;
  p.largeThreshold = d.largeThreshold;
  p.nLarge = 0;
  p.nNoCollide = d.nNoCollide;
  p.fixedColors = (d.flags & WORLD_FIXED_COLORS) ? 1u : 0u;
  return p;
}

// --- vector / quaternion helpers (operation order of the reference's WGSL, wgsl layout.ts:307-340) ---
__host__ __device__ inline float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__host__ __device__ inline float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__host__ __device__ inline float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ inline float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__host__ __device__ inline float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline float3 cross3(float3 a, float3 b) { return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
__host__ __device__ inline float3 abs3(float3 a) { return make_float3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__host__ __device__ inline float len3(float3 a) { return sqrtf(dot3(a, a)); }
__host__ __device__ inline float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__host__ __device__ inline float4 qmul(float4 a, float4 b) {
  return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                     a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
__host__ __device__ inline float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
// The reference's rotate (ref/math.ts:115-126): t = 2 u x v; v + t w + u x t
__host__ __device__ inline float3 qrotate(float4 q, float3 v) {
  float tx = (q.y * v.z - q.z * v.y) * 2.0f;
  float ty = (q.z * v.x - q.x * v.z) * 2.0f;
  float tz = (q.x * v.y - q.y * v.x) * 2.0f;
  return make_float3(v.x + tx * q.w + (q.y * tz - q.z * ty), v.y + ty * q.w + (q.z * tx - q.x * tz), v.z + tz * q.w + (q.x * ty - q.y * tx));
}
// qsub (ref/math.ts:86-89): 2 vec(a b^-1), b^-1 = conj(b) / |b|^2
__host__ __device__ inline float3 qsub(float4 a, float4 b) {
  float l = (b.x * b.x + b.y * b.y + b.z * b.z) + b.w * b.w;
  float4 inv = make_float4(-b.x / l, -b.y / l, -b.z / l, b.w / l);
  float4 s = qmul(a, inv);
  return make_float3(s.x * 2.0f, s.y * 2.0f, s.z * 2.0f);
}
// qaddv (ref/math.ts:109-113): normalize(a + (v, 0) a / 2)
__host__ __device__ inline float4 qadd(float4 a, float3 v) {
  float4 s = qmul(make_float4(v.x, v.y, v.z, 0.0f), a);
  float4 q = make_float4(a.x + s.x * 0.5f, a.y + s.y * 0.5f, a.z + s.z * 0.5f, a.w + s.w * 0.5f);
  float l = sqrtf((q.x * q.x + q.y * q.y + q.z * q.z) + q.w * q.w);
  return make_float4(q.x / l, q.y / l, q.z / l, q.w / l);
}
// orthonormal (ref/math.ts:228-238): rows n, t1, t2
__host__ __device__ inline void orthonormal(float3 n, float3& t1, float3& t2) {
  float3 t = fabsf(n.x) > fabsf(n.z) ? make_float3(-n.y, n.x, 0.0f) : make_float3(0.0f, -n.z, n.y);
  float l = sqrtf(dot3(t, t));
  t1 = make_float3(t.x / l, t.y / l, t.z / l);
  t2 = cross3(n, t1);
}
__host__ __device__ inline uint32_t hash32(uint32_t x) {  // avbd2d/gpu/layout.ts:107-115 (lowbias32)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__host__ __device__ inline uint32_t pairHash(uint32_t a, uint32_t b) { return hash32((a * 0x9e3779b1u) ^ hash32(b)); }  // wgsl-collision.ts:344

inline uint32_t grid_for(uint32_t n, uint32_t block) { return (n + block - 1) / block; }

// Host launchers (avbd_collide.cu)
uint32_t launch_collision(const DWorld& w, const StepParams& p, uint32_t tableSize, bool reuseManifolds, cudaStream_t s);
void launch_step_stats(const DWorld& w, uint32_t launches, cudaStream_t s);
// Batched worlds: one block per world over a queue of world indices (largest first)
struct BatchLaunch {
  DWorld base;
  const WorldDesc* worlds;
  const uint32_t* order;  // world indices, largest first
  uint32_t nWorlds;
  uint32_t* queue;        // [0] collision queue, [1] solve queue (zeroed before the launches)
  uint32_t* status;       // [0] storage bits (BATCH_*), [1] error bits of any world
  StepParams p;           // shared parameters; per-world sizes come from the WorldDesc
};
constexpr uint32_t BATCH_OVERFLOW = 1u, BATCH_NEAR_FULL = 2u;
cudaError_t launch_batch_collision(const BatchLaunch& b, int blocks, int threads, cudaStream_t s);
// worldThreads: 256, a block a world; 32, a warp a world (eight worlds a block)
cudaError_t launch_batch_solve(const BatchLaunch& b, int blocks, int worldThreads, cudaStream_t s);
int batch_collide_blocks_per_sm(int threads);
int batch_solve_blocks_per_sm(int worldThreads);
constexpr int BATCH_SOLVE_THREADS = 256;  // the solve's block size (its shared tables assume it)
constexpr uint32_t BATCH_MAX_WORLD_BODIES = 4096;

// The contact structure of a batched rollout, recorded step by step for the adjoint (avbd_record.cu).
// Step s of the recording holds every world's manifolds, then every world's points, world after
// world; manFirst/ptFirst (K x (W + 1) global indices) give each world's range. Indices of bodies
// are world-local, of manifolds and points global.
struct RecordDev {
  uint32_t K, W, nb;  // steps, worlds, bodies over all worlds
  uint64_t manCap, ptCap;
  int* manFirst;      // K x (W + 1)
  int* ptFirst;       // K x (W + 1)
  int* manCount;      // W: the step's manifolds and points per world (scratch)
  int* ptCount;
  int2* manAB;        // per manifold: bodies a > b
  double* basis;      // 9 per manifold: n (B to A), t1, t2 as the solve builds them
  int* manSlot;       // the world-local pair slot it was found in (ascending within a world's step)
  int* manPt0;        // global index of its first point
  double* anchors;    // 6 per point: rA, rB in the bodies' frames
  int* ptMan;         // global manifold index
  int* ptPrev;        // global index of the last step's point it warm-started from, or -1
  int* color;         // K x nb: the body's colour, -1 for a static body
  int* ncol;          // K x W: colours of the world's step
  unsigned long long* totals;  // [0] manifolds, [1] points recorded so far
  uint32_t* status;            // [0] REC_* bits, [1] most points of one world in one step
};
constexpr uint32_t REC_CAPACITY = 1u, REC_HISTORY = 2u, REC_SPHERE = 4u, REC_COLORS = 8u, REC_ORDER = 16u;
// Appends step s (the step L just ran) to the recording
cudaError_t launch_record_step(const BatchLaunch& L, const RecordDev& R, uint32_t s, int blocks, cudaStream_t st);

// Host launchers (avbd_solve.cu)
int solve_grid_blocks(int device);
cudaError_t launch_topology_solve(const DWorld& w, const StepParams& p, int blocks, cudaStream_t s);

}  // namespace avbd
