// Collision phase of the B200 AVBD step: last step's pairs into the warm-start hash, cell keys,
// a counting sort of the bodies on their cell hash (a one-digit radix sort, stable by body index),
// cell ranges, pair emission, and the narrowphase.
//
// This file is compiled with --fmad=false: every product and sum is rounded on its own, in the
// operation order of the reference's WGSL (src/avbd3d/gpu/wgsl-collision.ts), so the pair tests
// and the SAT axis choice (hence the feature keys) agree bit for bit with an f32 CPU
// restatement compiled with -ffp-contract=off.
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <vector>

#include "avbd_device.cuh"
#include "avbd_host.hpp"

namespace cg = cooperative_groups;

namespace avbd {


constexpr int GS_BLOCKS = 148 * 8;  // grid-stride kernels over device-side counts

__device__ inline bool enabled(const DWorld& w, uint32_t i) {
  uint32_t f = (uint32_t)w.ipos[i].w;
  return (f & 2u) == 0u;
}

__device__ inline float3 aabbOf(const DWorld& w, uint32_t i);

// --- begin: rotate counters (wgsl-collision.ts:96-107) -------------------------------------------
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void k_begin(DWorld w, StepParams p) {
  w.clocks[CLOCK_T0] = gtimer();
  uint32_t* c = w.counters;
  uint32_t pairs = c[C_PAIRS];
  c[C_PREV_PAIRS] = pairs < p.pairCap ? pairs : p.pairCap;
  c[C_STEP] += 1;  // steps since the world was made (the manifold's generation word)
  c[C_PAIRS] = 0;
  c[C_CONTACTS] = 0;
  c[C_MANIFOLDS] = 0;
  c[C_OVERFLOW] = 0;
  c[C_CLASHES] = 0;
  c[C_COLORS] = 0;
  c[C_ROUNDS] = 0;
  c[C_ERROR] = 0;
  c[C_HULL_PAIRS] = 0;
  for (int k = 0; k < 2 * MAX_ROUND_PAIRS + 2; k++) c[C_PENDING + k] = 0;
}

// --- last step's pairs into the hash table (wgsl-collision.ts:354-368), compare-and-swap probing ---
__global__ void k_hash_insert(DWorld w, StepParams p) {
  const int prev = 1 - p.cur;
  const uint32_t count = w.counters[C_PREV_PAIRS];
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < count; m += gridDim.x * blockDim.x) {
    uint4 ids = w.mIds[prev][m];
    if ((ids.w & 15u) == 0u) continue;
    // Rewritten slots have no contact history
    if (w.ipos[ids.x].w != 0.0f || w.ipos[ids.y].w != 0.0f) continue;
    uint32_t h = pairHash(ids.x, ids.y) & p.hashMask;
    for (uint32_t probe = 0; probe <= p.hashMask; probe++) {
      if (atomicCAS(&w.hash[h], 0u, m + 1u) == 0u) break;
      h = (h + 1u) & p.hashMask;
    }
  }
}

__device__ inline int hashFind(const DWorld& w, const StepParams& p, uint32_t a, uint32_t b) {
  const int prev = 1 - p.cur;
  uint32_t h = pairHash(a, b) & p.hashMask;
  for (uint32_t probe = 0; probe <= p.hashMask; probe++) {
    uint32_t v = w.hash[h];
    if (v == 0u) return -1;
    uint4 ids = w.mIds[prev][v - 1u];
    if (ids.x == a && ids.y == b) return int(v - 1u);
    h = (h + 1u) & p.hashMask;
  }
  return -1;
}

// --- contact reuse (wgsl-collision.ts:20-44, 706-762) -------------------------------------------------
// updateRefs: a body without a reference pose, or moved or turned past the tolerance since it, takes
// its pose (x-) as the new reference and stamps this step into its moved_step word (ypos.w)
__device__ inline void updateRef(const DWorld& w, uint32_t i, uint32_t step) {
  const float3 pos = f3(w.pos[i]);
  const float4 rot = w.rot[i];
  const float4 ref = w.refRot[i];
  bool moved = ((ref.x * ref.x + ref.y * ref.y) + ref.z * ref.z) + ref.w * ref.w == 0.0f || len3(pos - f3(w.refPos[i])) > REUSE_LIN_TOL ||
               len3(qsub(rot, ref)) > REUSE_ANG_TOL;
  if (moved) {
    w.refPos[i] = make_float4(pos.x, pos.y, pos.z, 0.0f);
    w.refRot[i] = rot;
    w.ypos[i].w = __uint_as_float(step);
  }
}
__global__ void k_update_refs(DWorld w, StepParams p) {
  const uint32_t step = w.counters[C_STEP];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x)
    if (((uint32_t)w.ipos[i].w & 2u) == 0u) updateRef(w, i, step);
}

// A contact's least normal penalty (wgsl-collision.ts contactPenaltyMin): with FLAG_MASS_PENALTY the
// lighter dynamic body's m/dt^2
__device__ inline float contactPenaltyMin(const DWorld& w, const StepParams& p, uint32_t a, uint32_t b) {
  if (!(p.flags & FLAG_MASS_PENALTY)) return PENALTY_MIN;
  float mA = w.size[a].w <= 0.0f ? 3.4e38f : w.size[a].w;
  float mB = w.size[b].w <= 0.0f ? 3.4e38f : w.size[b].w;
  return fminf(fmaxf(fminf(mA, mB) / (p.dt * p.dt), PENALTY_MIN), PENALTY_MAX);
}

// Counts a manifold of `count` points into the step's counters, one atomic per coalesced group
__device__ __forceinline__ void countManifold(const DWorld& w, uint32_t count) {
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t pts = cg::reduce(g, count, cg::plus<uint32_t>());
  uint32_t nonEmpty = cg::reduce(g, count > 0u ? 1u : 0u, cg::plus<uint32_t>());
  if (g.thread_rank() == 0) {
    atomicAdd(&w.counters[C_CONTACTS], pts);
    atomicAdd(&w.counters[C_MANIFOLDS], nonEmpty);
  }
}

// copyContacts (wgsl-collision.ts:721-753): last step's manifold in slot pm kept as this step's
// manifold in slot pi (ids with its generation step, normal, friction, points with their keys and
// anchors), each point's C(x-) evaluated at the current poses and its multipliers and penalties
// warm-started as a fresh point's are
__device__ void copyContacts(const DWorld& w, const StepParams& p, uint32_t pi, uint32_t pm) {
  const int cur = p.cur, prev = 1 - cur;
  const uint4 ids = w.mIds[prev][pm];
  const uint32_t a = ids.x, b = ids.y, count = min(ids.w & 15u, (uint32_t)MAX_CONTACTS);
  const float4 geo = w.mGeo[prev][pm];
  w.mIds[cur][pi] = make_uint4(a, b, pi * MAX_CONTACTS, ids.w);
  w.mGeo[cur][pi] = geo;
  countManifold(w, count);
  const float3 n = f3(geo);
  float3 t1, t2;
  orthonormal(n, t1, t2);
  const float3 cA = f3(w.pos[a]), cB = f3(w.pos[b]);
  const float4 qA = w.rot[a], qB = w.rot[b];
  const float penaltyMin = contactPenaltyMin(w, p, a, b);
  for (uint32_t i = 0; i < count; i++) {
    const float4* q = w.cPt[prev] + 4 * (size_t(ids.z) + i);
    const float4 ra = q[K_RA], rb = q[K_RB];
    float3 pen = f3(q[K_PEN]), lam = f3(q[K_LAM]);
    const float3 d = (cA - cB) + (qrotate(qA, f3(ra)) - qrotate(qB, f3(rb)));
    const float c0x = dot3(n, d) + p.margin, c0y = dot3(t1, d), c0z = dot3(t2, d);
    lam = lam * p.alpha * p.gamma;
    pen = make_float3(fminf(fmaxf(pen.x * p.gamma, PENALTY_MIN), PENALTY_MAX), fminf(fmaxf(pen.y * p.gamma, PENALTY_MIN), PENALTY_MAX),
                      fminf(fmaxf(pen.z * p.gamma, PENALTY_MIN), PENALTY_MAX));
    pen.x = fmaxf(pen.x, penaltyMin);
    float4* o = w.cPt[cur] + 4 * (size_t(pi) * MAX_CONTACTS + i);
    o[K_RA] = ra;
    o[K_RB] = make_float4(rb.x, rb.y, rb.z, c0x);
    o[K_PEN] = make_float4(pen.x, pen.y, pen.z, c0y);
    o[K_LAM] = make_float4(lam.x, lam.y, lam.z, c0z);
  }
}

// reuseContacts (wgsl-collision.ts:706-717): the pair keeps last step's points when they were
// generated no earlier than either body's last move
__device__ inline bool reusePair(const DWorld& w, const StepParams& p, uint32_t pi, uint32_t a, uint32_t b) {
  const int pm = hashFind(w, p, a, b);
  if (pm < 0) return false;
  const uint32_t idw = w.mIds[1 - p.cur][pm].w;
  const uint32_t moved = max(__float_as_uint(w.ypos[a].w), __float_as_uint(w.ypos[b].w));
  if ((idw & 15u) == 0u || (idw >> 4) < moved) return false;
  copyContacts(w, p, pi, (uint32_t)pm);
  return true;
}

// reuseManifolds (wgsl-collision.ts:755-762): every pair slot of last step kept in the same slot,
// its manifold copied; the step detects no pair
__global__ void k_reuse_manifolds(DWorld w, StepParams p) {
  const uint32_t total = w.counters[C_PREV_PAIRS];
  const int prev = 1 - p.cur;
  if (blockIdx.x == 0 && threadIdx.x == 0) w.counters[C_PAIRS] = total;
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < total; m += gridDim.x * blockDim.x) {
    const uint4 ids = w.mIds[prev][m];
    w.pairs[m] = make_uint2(ids.x, ids.y);
    if ((ids.w & 15u) == 0u) {
      w.mIds[p.cur][m] = make_uint4(ids.x, ids.y, m * MAX_CONTACTS, ids.w & ~15u);
      continue;
    }
    copyContacts(w, p, m, m);
  }
}

// --- grid keys: cellHash (wgsl-collision.ts:121-128), one level -----------------------------------
__device__ inline int4 cellOf(float3 x, float size) {
  return make_int4((int)floorf(x.x / size), (int)floorf(x.y / size), (int)floorf(x.z / size), 0);
}
__device__ inline uint32_t cellHash(int4 c, uint32_t mask) {
  return (((uint32_t)c.x * 73856093u) ^ ((uint32_t)c.y * 19349663u) ^ ((uint32_t)c.z * 83492791u)) & mask;
}

__global__ void k_cell_keys(DWorld w, StepParams p) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  bool small = enabled(w, i) && w.moment[i].w <= p.largeThreshold;
  int4 c = cellOf(f3(w.pos[i]), p.cellSize);
  w.cell[i] = c;
  w.keyA[i] = small ? cellHash(c, p.tableMask) : p.tableMask + 1u;  // large and disabled bodies sort last
  w.valA[i] = i;
}

// --- counting sort of bodies by cell hash (a single radix pass on the whole key) -------------------
// Count (each body keeps its rank in its bucket), exclusive scan of the bucket counts, scatter. The
// order of bodies within a bucket follows the atomics and changes nothing downstream: pairs are a
// set, and every body sums its rows in a sorted order of its own.
__global__ void k_bucket_count(const uint32_t* keys, uint32_t n, uint32_t* count, uint32_t* rank, uint32_t sentinel) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = keys[i];
  rank[i] = k == sentinel ? 0u : atomicAdd(&count[k], 1u);
}

// Exclusive scan, three kernels: block tiles of 4096 (totals out), the totals, the tiles' offsets.
constexpr int SCAN_THREADS = 1024, SCAN_ITEMS = 4, SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
__device__ uint32_t block_exclusive_scan_1024(uint32_t v, uint32_t* warpSums) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpSums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = warpSums[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warpSums[lane] = t;
  }
  __syncthreads();
  uint32_t r = x - v + (warp > 0 ? warpSums[warp - 1] : 0u);
  __syncthreads();
  return r;
}
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(uint32_t* data, uint32_t len, uint32_t* totals) {
  __shared__ uint32_t warpSums[32];
  uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
  uint32_t v[SCAN_ITEMS], sum = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    v[k] = base + k < len ? data[base + k] : 0u;
    sum += v[k];
  }
  uint32_t run = block_exclusive_scan_1024(sum, warpSums);
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++) {
    if (base + k < len) data[base + k] = run;
    run += v[k];
  }
  if (threadIdx.x == SCAN_THREADS - 1) totals[blockIdx.x] = run;
}
__global__ void __launch_bounds__(1024) k_scan_single(uint32_t* data, uint32_t len) {
  __shared__ uint32_t warpSums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < len; base += 1024) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < len ? data[i] : 0u;
    uint32_t ex = block_exclusive_scan_1024(v, warpSums) + carry;
    if (i < len) data[i] = ex;
    __syncthreads();
    if (threadIdx.x == 1023) carry = ex + v;
    __syncthreads();
  }
}
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_add(uint32_t* data, uint32_t len, const uint32_t* totals) {
  uint32_t add = totals[blockIdx.x];
  uint32_t base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; k++)
    if (base + k < len) data[base + k] += add;
}

// cellEnd held the counts: make it start + count
__global__ void k_bucket_finish(const uint32_t* start, uint32_t* end, uint32_t len) {
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h < len) end[h] += start[h];
}

// Bodies into bucket order, with each sorted slot's candidate record (position and radius, exact cell
// and body with its dynamic bit) so a cell walk reads contiguous memory.
__global__ void k_bucket_scatter(DWorld w, uint32_t n, uint32_t sentinel) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = w.keyA[i];
  if (k == sentinel) return;
  uint32_t slot = w.cellStart[k] + w.valB[i];
  float4 pi = w.pos[i];
  w.sortedPR[slot] = make_float4(pi.x, pi.y, pi.z, w.moment[i].w);
  int4 c = w.cell[i];
  w.sortedCell[slot] = make_int4(c.x, c.y, c.z, (int)(i | (w.size[i].w > 0.0f ? 0x80000000u : 0u)));
  float3 a = aabbOf(w, i);
  w.sortedAabb[slot] = make_float4(a.x, a.y, a.z, 0.0f);
}

// --- pair tests (wgsl-collision.ts:150-234) ------------------------------------------------------------
struct Shape {
  float3 ax0, ax1, ax2, h;
  bool sphere;
};
__device__ inline Shape shapeOf(const DWorld& w, uint32_t i) {
  float4 q = w.rot[i];
  Shape s;
  float4 sz = w.size[i];
  s.h = make_float3(sz.x * 0.5f, sz.y * 0.5f, sz.z * 0.5f);
  s.sphere = w.avel[i].w == SHAPE_SPHERE_F;
  s.ax0 = qrotate(q, make_float3(1.0f, 0.0f, 0.0f));
  s.ax1 = qrotate(q, make_float3(0.0f, 1.0f, 0.0f));
  s.ax2 = qrotate(q, make_float3(0.0f, 0.0f, 1.0f));
  return s;
}
__device__ inline float extentOf(const Shape& s, float3 n) {
  if (s.sphere) return s.h.x;
  return s.h.x * fabsf(dot3(n, s.ax0)) + s.h.y * fabsf(dot3(n, s.ax1)) + s.h.z * fabsf(dot3(n, s.ax2));
}
__device__ inline float3 aabbHalf(const Shape& s) {
  if (s.sphere) return make_float3(s.h.x, s.h.x, s.h.x);
  return abs3(s.ax0) * s.h.x + abs3(s.ax1) * s.h.y + abs3(s.ax2) * s.h.z;
}
__device__ inline bool faceSeparated(const Shape& A, const Shape& B, float3 d) {
  const float3 a[3] = {A.ax0, A.ax1, A.ax2};
  const float3 b[3] = {B.ax0, B.ax1, B.ax2};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (fabsf(dot3(d, a[k])) - extentOf(A, a[k]) - extentOf(B, a[k]) > 1e-3f) return true;
    if (fabsf(dot3(d, b[k])) - extentOf(A, b[k]) - extentOf(B, b[k]) > 1e-3f) return true;
  }
  return false;
}

__device__ inline float3 aabbOf(const DWorld& w, uint32_t i) { return aabbHalf(shapeOf(w, i)); }

struct Probe {
  uint32_t index;
  float3 pos, aabb;
  float radius;
  bool dynamic;
  uint2 filter;
  Shape shape;
};
__device__ inline Probe probeOf(const DWorld& w, uint32_t i) {
  Probe P;
  P.index = i;
  P.pos = f3(w.pos[i]);
  P.radius = w.moment[i].w;
  P.shape = shapeOf(w, i);
  P.aabb = aabbHalf(P.shape);
  P.dynamic = w.size[i].w > 0.0f;
  P.filter = w.filters[i];
  return P;
}

// No-collide list, binary search (wgsl-collision.ts:53-76)
__device__ inline bool ignored(const DWorld& w, const StepParams& p, uint32_t hi, uint32_t lo) {
  const uint32_t* t = w.nocollide;
  uint32_t first = 0, count = p.nNoCollide;
  while (count > 0u) {
    uint32_t step = count / 2u, mid = first + step;
    uint32_t mh = t[3u * mid], ml = t[3u * mid + 1u];
    if (mh < hi || (mh == hi && ml < lo)) {
      first = mid + 1u;
      count -= step + 1u;
    } else {
      count = step;
    }
  }
  for (uint32_t k = first; k < p.nNoCollide; k++) {
    if (t[3u * k] != hi || t[3u * k + 1u] != lo) break;
    uint32_t j = t[3u * k + 2u];
    if (j == 0xffffffffu) return true;
    float4 pl = w.joint[j * JOINT_VEC4 + J_PEN_LIN], pa = w.joint[j * JOINT_VEC4 + J_PEN_ANG];
    if (pl.w != 0.0f || pa.w != 0.0f) return true;
  }
  return false;
}

__device__ inline void emitPair(const DWorld& w, const StepParams& p, uint32_t a, uint32_t b) {
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(&w.counters[C_PAIRS], g.size());
  base = g.shfl(base, 0);
  uint32_t slot = base + g.thread_rank();
  if (slot >= p.pairCap) {
    atomicOr(&w.counters[C_OVERFLOW], 1u);
    return;
  }
  w.pairs[slot] = make_uint2(a, b);
}

__device__ inline void testPair(const DWorld& w, const StepParams& p, const Probe& P, uint32_t j) {
  if (!enabled(w, j)) return;
  if (!P.dynamic && w.size[j].w <= 0.0f) return;
  uint2 fj = w.filters[j];
  if ((P.filter.x & fj.y) == 0u || (fj.x & P.filter.y) == 0u) return;
  float3 d = P.pos - f3(w.pos[j]);
  float r = P.radius + w.moment[j].w;
  if (dot3(d, d) > r * r) return;
  Shape B = shapeOf(w, j);
  float3 bh = aabbHalf(B);
  if (fabsf(d.x) > P.aabb.x + bh.x + 1e-4f || fabsf(d.y) > P.aabb.y + bh.y + 1e-4f || fabsf(d.z) > P.aabb.z + bh.z + 1e-4f) return;
  if (faceSeparated(P.shape, B, d)) return;
  uint32_t a = max(P.index, j), b = min(P.index, j);
  if (ignored(w, p, a, b)) return;
  emitPair(w, p, a, b);
}

// Which body's view a pair is tested from (findPairs / findFixedLarge ownership, wgsl-collision.ts:
// 242-323): two small dynamic bodies from the higher index, small against large from the small one,
// two large dynamic ones from the lower index, a fixed body's pair from the mover, except a small
// fixed body against a large mover (findFixedLarge). The f32 tests round differently from either
// side, so the GPU's own choice is kept.
__device__ inline uint32_t proberOf(const DWorld& w, const StepParams& p, uint32_t i, uint32_t j) {
  bool di = w.size[i].w > 0.0f, dj = w.size[j].w > 0.0f;
  bool li = w.moment[i].w > p.largeThreshold, lj = w.moment[j].w > p.largeThreshold;
  if (di && dj) {
    if (!li && !lj) return max(i, j);
    if (li != lj) return li ? j : i;
    return min(i, j);
  }
  uint32_t dyn = di ? i : j, fix = di ? j : i;
  bool lfix = di ? lj : li, ldyn = di ? li : lj;
  if (!lfix && ldyn) return fix;
  return dyn;
}

__device__ inline void testFromProber(const DWorld& w, const StepParams& p, const Probe& P, uint32_t j) {
  uint32_t pr = proberOf(w, p, P.index, j);
  if (pr == P.index) testPair(w, p, P, j);
  else testPair(w, p, probeOf(w, pr), P.index);
}

// The grid walk: every small body (fixed ones too) visits its own cell (bodies of lower index) and
// the 13 cells of its forward half-shell, so each small-small pair is visited once; cells are at
// least twice the largest small radius, so this covers every overlap. Large bodies test against
// everything (the large list), as the reference's do.
//
// One cell of small body i's walk: offset o = 0 is its own cell, 1..13 the forward half-shell
// ((dx, dy, dz) > 0 in (z, y, x) order)
__device__ inline void walkCell(const DWorld& w, const StepParams& p, const Probe& P, bool dyn, int4 c, int o) {
  const uint32_t i = P.index;
  const int q = o == 0 ? 13 : 13 + o;
  const int4 cc = make_int4(c.x + q % 3 - 1, c.y + (q / 3) % 3 - 1, c.z + q / 9 - 1, 0);
  const uint32_t h = cellHash(cc, p.tableMask);
  const uint32_t end = w.cellEnd[h];
  for (uint32_t k = w.cellStart[h]; k < end; k++) {
    int4 cj = w.sortedCell[k];
    uint32_t j = (uint32_t)cj.w & 0x7fffffffu;
    bool dj = ((uint32_t)cj.w & 0x80000000u) != 0u;
    if (o == 0 && j >= i) continue;
    if (!dyn && !dj) continue;
    if (cj.x != cc.x || cj.y != cc.y || cj.z != cc.z) continue;
    float4 pr = w.sortedPR[k];
    float3 d = P.pos - make_float3(pr.x, pr.y, pr.z);
    float r = P.radius + pr.w;
    if (dot3(d, d) > r * r) continue;  // the sphere test, the same in both views
    float4 ab = w.sortedAabb[k];         // and the AABB test (its sums commute)
    if (fabsf(d.x) > P.aabb.x + ab.x + 1e-4f || fabsf(d.y) > P.aabb.y + ab.y + 1e-4f || fabsf(d.z) > P.aabb.z + ab.z + 1e-4f) continue;
    testFromProber(w, p, P, j);
  }
}
// A small body against the large list
__device__ inline void smallAgainstLarge(const DWorld& w, const StepParams& p, const Probe& P, bool dyn) {
  if (!dyn && !p.anyDynamicLarge) return;
  for (uint32_t k = 0; k < p.nLarge; k++) {
    uint32_t l = w.large[k];
    if (!dyn && (!enabled(w, l) || w.size[l].w <= 0.0f)) continue;
    testPair(w, p, P, l);
  }
}
// A large dynamic body against the large list (each pair of large bodies once)
__device__ inline void largeAgainstLarge(const DWorld& w, const StepParams& p, const Probe& P) {
  for (uint32_t k = 0; k < p.nLarge; k++) {
    uint32_t l = w.large[k];
    if (l == P.index || (l < P.index && w.size[l].w > 0.0f)) continue;
    testPair(w, p, P, l);
  }
}

// One thread per body walks its cells with the cheap tests (cell, sphere, AABB); the candidates
// that pass go to a per-warp queue in shared memory, and whenever it holds a warp's worth, the warp
// takes the full test (the prober's view, the face separation, the no-collide list) one candidate a
// lane, so that the long test runs on full warps instead of on the few lanes whose walk found one.
constexpr uint32_t PAIR_WALK_THREADS = 128, PAIR_QUEUE = 64;
__device__ __forceinline__ void testCandidate(const DWorld& w, const StepParams& p, uint2 e) {
  const uint32_t pr = proberOf(w, p, e.x, e.y);
  testPair(w, p, probeOf(w, pr), pr == e.x ? e.y : e.x);
}
// Lanes take the queue's first min(count, 32) candidates and test them; the rest move to the front.
__device__ __forceinline__ void drainQueue(const DWorld& w, const StepParams& p, uint2* Q, uint32_t& count, uint32_t lane) {
  const uint32_t take = min(count, 32u);
  const uint2 e = lane < take ? Q[lane] : make_uint2(0u, 0u);
  __syncwarp();
  if (lane + take < count) Q[lane] = Q[lane + take];
  __syncwarp();
  count -= take;
  if (lane < take) testCandidate(w, p, e);
}
__global__ void __launch_bounds__(PAIR_WALK_THREADS) k_find_pairs(DWorld w, StepParams p) {
  __shared__ uint2 s_queue[PAIR_WALK_THREADS / 32][PAIR_QUEUE];
  const uint32_t lane = threadIdx.x & 31u;
  uint2* Q = s_queue[threadIdx.x >> 5];
  uint32_t count = 0;  // the warp's queue length (the same in every lane)
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool on = i < p.n && enabled(w, i);
  const bool dyn = on && w.size[i].w > 0.0f;
  const bool small = on && w.moment[i].w <= p.largeThreshold;
  float3 pos = make_float3(0.0f, 0.0f, 0.0f), aabb = pos;
  float radius = 0.0f;
  int4 c = make_int4(0, 0, 0, 0);
  if (small) {
    pos = f3(w.pos[i]);
    radius = w.moment[i].w;
    aabb = aabbOf(w, i);
    c = w.cell[i];
  }
#pragma unroll 1
  for (int o = 0; o < 14; o++) {
    // offset o = 0: the own cell; 1..13: (dx, dy, dz) > 0 in (z, y, x) order
    const int q = o == 0 ? 13 : 13 + o;
    const int4 cc = make_int4(c.x + q % 3 - 1, c.y + (q / 3) % 3 - 1, c.z + q / 9 - 1, 0);
    uint32_t k = 0, end = 0;
    if (small) {
      const uint32_t h = cellHash(cc, p.tableMask);
      k = w.cellStart[h];
      end = w.cellEnd[h];
    }
    auto candidate = [&](uint32_t kk, uint32_t& jj) -> bool {
      const int4 cj = w.sortedCell[kk];
      jj = (uint32_t)cj.w & 0x7fffffffu;
      const bool dj = ((uint32_t)cj.w & 0x80000000u) != 0u;
      if ((o == 0 && jj >= i) || !(dyn || dj) || cj.x != cc.x || cj.y != cc.y || cj.z != cc.z) return false;
      const float4 pr = w.sortedPR[kk];
      const float3 d = pos - make_float3(pr.x, pr.y, pr.z);
      const float r = radius + pr.w;
      if (dot3(d, d) > r * r) return false;  // the sphere test, the same in both views
      const float4 ab = w.sortedAabb[kk];      // and the AABB test (its sums commute)
      return !(fabsf(d.x) > aabb.x + ab.x + 1e-4f || fabsf(d.y) > aabb.y + ab.y + 1e-4f || fabsf(d.z) > aabb.z + ab.z + 1e-4f);
    };
    auto enqueue = [&](bool push, uint32_t jj) {
      const uint32_t m = __ballot_sync(0xffffffffu, push);
      if (m) {
        if (push) Q[count + __popc(m & ((1u << lane) - 1u))] = make_uint2(i, jj);
        count += __popc(m);
        __syncwarp();
        if (count >= 32u) drainQueue(w, p, Q, count, lane);
      }
    };
    while (__any_sync(0xffffffffu, k < end)) {
      uint32_t j0 = 0, j1 = 0;
      const bool p0 = k < end && candidate(k, j0);
      const bool p1 = k + 1 < end && candidate(k + 1, j1);
      k += 2;
      enqueue(p0, j0);
      enqueue(p1, j1);
    }
  }
  while (count > 0u) drainQueue(w, p, Q, count, lane);
  if (small) {
    smallAgainstLarge(w, p, probeOf(w, i), dyn);
  } else if (dyn) {
    largeAgainstLarge(w, p, probeOf(w, i));
  }
}

// --- narrowphase: box SAT + clipping (wgsl-collision.ts:385-599, ref/collide.ts) ---------------------
constexpr float SAT_AXIS_EPSILON = 1.0e-6f, PLANE_EPSILON = 1.0e-5f, CONTACT_MERGE_DIST_SQ = 1.0e-6f;
constexpr uint32_t AXIS_FACE_A = 0, AXIS_FACE_B = 1, AXIS_EDGE = 2;

struct Box {
  float3 c, h;
  float3 ax[3];
};
struct Sat {
  uint32_t kind, ia, ib;
  float sep;
  float3 n;
  bool valid;
};
struct Found {
  uint32_t feature[MAX_CONTACTS];
  float3 xA[MAX_CONTACTS], xB[MAX_CONTACTS];
  uint32_t count;
};

__device__ inline Box makeBox(const DWorld& w, uint32_t i) {
  float4 q = w.rot[i];
  float4 sz = w.size[i];
  Box b;
  b.c = f3(w.pos[i]);
  b.h = make_float3(sz.x * 0.5f, sz.y * 0.5f, sz.z * 0.5f);
  b.ax[0] = qrotate(q, make_float3(1.0f, 0.0f, 0.0f));
  b.ax[1] = qrotate(q, make_float3(0.0f, 1.0f, 0.0f));
  b.ax[2] = qrotate(q, make_float3(0.0f, 0.0f, 1.0f));
  return b;
}
__device__ inline float projRadius(const Box& b, float3 n) {
  return b.h.x * fabsf(dot3(n, b.ax[0])) + b.h.y * fabsf(dot3(n, b.ax[1])) + b.h.z * fabsf(dot3(n, b.ax[2]));
}
__device__ inline bool testAxis(const Box& A, const Box& B, float3 delta, float3 axis, uint32_t kind, uint32_t ia, uint32_t ib, Sat& best) {
  float lenSq = dot3(axis, axis);
  if (lenSq < SAT_AXIS_EPSILON) return true;
  float invLen = 1.0f / sqrtf(lenSq);
  float3 n = axis * invLen;
  if (dot3(n, delta) < 0.0f) n = -n;
  float distance = fabsf(dot3(delta, n));
  float rA = projRadius(A, n);
  float rB = projRadius(B, n);
  float sep = distance - (rA + rB);
  if (sep > 0.0f) return false;
  if (!best.valid || sep > best.sep) {
    best.valid = true;
    best.kind = kind;
    best.ia = ia;
    best.ib = ib;
    best.sep = sep;
    best.n = n;
  }
  return true;
}
__device__ inline float3 support(const Box& b, float3 dir) {
  float sx = dot3(dir, b.ax[0]) >= 0.0f ? 1.0f : -1.0f;
  float sy = dot3(dir, b.ax[1]) >= 0.0f ? 1.0f : -1.0f;
  float sz = dot3(dir, b.ax[2]) >= 0.0f ? 1.0f : -1.0f;
  float3 p = b.c + b.ax[0] * (b.h.x * sx);
  p = p + b.ax[1] * (b.h.y * sy);
  return p + b.ax[2] * (b.h.z * sz);
}
__device__ inline void addFound(Found& f, float3 xA, float3 xB, uint32_t feature) {
  float3 mid = (xA + xB) * 0.5f;
  for (uint32_t i = 0; i < f.count; i++) {
    float3 m = (f.xA[i] + f.xB[i]) * 0.5f;
    float3 d = mid - m;
    if (dot3(d, d) < CONTACT_MERGE_DIST_SQ) return;
  }
  if (f.count >= MAX_CONTACTS) return;
  f.feature[f.count] = feature;
  f.xA[f.count] = xA;
  f.xB[f.count] = xB;
  f.count++;
}
// Sutherland-Hodgman against dot(pn, x) <= offset (a quad clipped by four planes keeps <= 8 vertices)
__device__ inline uint32_t clipPlane(const float3* src, uint32_t n, float3* dst, float3 pn, float offset) {
  if (n == 0u) return 0u;
  uint32_t count = 0;
  float3 a = src[n - 1u];
  float da = dot3(pn, a) - offset;
  for (uint32_t i = 0; i < n; i++) {
    float3 b = src[i];
    float db = dot3(pn, b) - offset;
    bool aIn = da <= PLANE_EPSILON, bIn = db <= PLANE_EPSILON;
    if (aIn != bIn) {
      float t = 0.0f;
      float denom = da - db;
      if (fabsf(denom) > SAT_AXIS_EPSILON) t = fminf(fmaxf(da / denom, 0.0f), 1.0f);
      if (count < 8u) dst[count++] = a + (b - a) * t;
    }
    if (bIn && count < 8u) dst[count++] = b;
    a = b;
    da = db;
  }
  return count;
}
__device__ inline uint32_t faceU(uint32_t k) { return k == 0u ? 1u : 0u; }
__device__ inline uint32_t faceV(uint32_t k) { return k != 2u ? 2u : 1u; }

__device__ void faceManifold(const Box& A, const Box& B, bool refIsA, uint32_t refAxis, float3 nAB, Found& found) {
  const Box& R = refIsA ? A : B;
  const Box& I = refIsA ? B : A;
  float3 outward = refIsA ? nAB : -nAB;
  float rs = dot3(outward, R.ax[refAxis]) >= 0.0f ? 1.0f : -1.0f;
  float3 rn = R.ax[refAxis] * rs;
  float3 rc = R.c + rn * comp(R.h, refAxis);
  float3 ru = R.ax[faceU(refAxis)], rv = R.ax[faceV(refAxis)];
  float eu = comp(R.h, faceU(refAxis)), ev = comp(R.h, faceV(refAxis));
  uint32_t incAxis = 0;
  float bestDot = -3.4028234663852886e38f;
  for (uint32_t k = 0; k < 3u; k++) {
    float d = fabsf(dot3(I.ax[k], rn));
    if (d > bestDot) {
      bestDot = d;
      incAxis = k;
    }
  }
  float is = dot3(I.ax[incAxis], rn) > 0.0f ? -1.0f : 1.0f;
  float3 fn = I.ax[incAxis] * is;
  float3 fc = I.c + fn * comp(I.h, incAxis);
  float3 u = I.ax[faceU(incAxis)], v = I.ax[faceV(incAxis)];
  float eU = comp(I.h, faceU(incAxis)), eV = comp(I.h, faceV(incAxis));
  float3 poly[8], tmp[8];
  // vert(su, sv) = fc + u (su eU) + v (sv eV)
  poly[0] = (fc + u * (1.0f * eU)) + v * (1.0f * eV);
  poly[1] = (fc + u * (-1.0f * eU)) + v * (1.0f * eV);
  poly[2] = (fc + u * (-1.0f * eU)) + v * (-1.0f * eV);
  poly[3] = (fc + u * (1.0f * eU)) + v * (-1.0f * eV);
  uint32_t n = 4;
  float3 nru = -ru, nrv = -rv;
  n = clipPlane(poly, n, tmp, ru, dot3(ru, rc) + eu);
  n = clipPlane(tmp, n, poly, nru, dot3(nru, rc) + eu);
  n = clipPlane(poly, n, tmp, rv, dot3(rv, rc) + ev);
  n = clipPlane(tmp, n, poly, nrv, dot3(nrv, rc) + ev);
  if (n == 0u) return;
  uint32_t prefix = ((refIsA ? AXIS_FACE_A : AXIS_FACE_B) << 24) | (refAxis << 16) | (incAxis << 8);
  for (uint32_t i = 0; i < n && found.count < MAX_CONTACTS; i++) {
    float3 q = poly[i];
    float dist = dot3(q - rc, rn);
    if (dist > PLANE_EPSILON) continue;
    float3 onRef = q + rn * (-dist);
    addFound(found, refIsA ? onRef : q, refIsA ? q : onRef, prefix | i);
  }
  if (found.count == 0u) addFound(found, support(A, nAB), support(B, -nAB), prefix);
}
__device__ inline void supportEdge(const Box& b, uint32_t k, float3 dir, float3& e0, float3& e1) {
  uint32_t k1 = (k + 1u) % 3u, k2 = (k + 2u) % 3u;
  float s1 = dot3(dir, b.ax[k1]) >= 0.0f ? 1.0f : -1.0f;
  float s2 = dot3(dir, b.ax[k2]) >= 0.0f ? 1.0f : -1.0f;
  float3 c = b.c + b.ax[k1] * (comp(b.h, k1) * s1);
  c = c + b.ax[k2] * (comp(b.h, k2) * s2);
  float3 e = b.ax[k] * comp(b.h, k);
  e0 = c - e;
  e1 = c + e;
}
__device__ void edgeContact(const Box& A, const Box& B, uint32_t ia, uint32_t ib, float3 nAB, Found& found) {
  float3 p0, p1, q0, q1;
  supportEdge(A, ia, nAB, p0, p1);
  supportEdge(B, ib, -nAB, q0, q1);
  float3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  float a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
  float s = 0.0f, t = 0.0f;
  if (a <= SAT_AXIS_EPSILON && e <= SAT_AXIS_EPSILON) {
  } else if (a <= SAT_AXIS_EPSILON) {
    t = fminf(fmaxf(f / e, 0.0f), 1.0f);
  } else {
    float c = dot3(d1, r);
    if (e <= SAT_AXIS_EPSILON) {
      s = fminf(fmaxf(-c / a, 0.0f), 1.0f);
    } else {
      float b = dot3(d1, d2);
      float denom = a * e - b * b;
      if (fabsf(denom) > SAT_AXIS_EPSILON) s = fminf(fmaxf((b * f - c * e) / denom, 0.0f), 1.0f);
      t = (b * s + f) / e;
      if (t < 0.0f) {
        t = 0.0f;
        s = fminf(fmaxf(-c / a, 0.0f), 1.0f);
      } else if (t > 1.0f) {
        t = 1.0f;
        s = fminf(fmaxf((b - c) / a, 0.0f), 1.0f);
      }
    }
  }
  uint32_t key = (AXIS_EDGE << 24) | (ia << 8) | ib;
  addFound(found, p0 + d1 * s, q0 + d2 * t, key);
  if (found.count == 0u) addFound(found, support(A, nAB), support(B, -nAB), key);
}
// collide (wgsl-collision.ts:656-683); sat.n points from A towards B
__device__ void collideBoxes(const Box& A, const Box& B, bool faceBias, Sat& sat, Found& found) {
  float3 delta = B.c - A.c;
  Sat face, edge;
  face.valid = false;
  edge.valid = false;
  face.sep = 0.0f;
  edge.sep = 0.0f;
  for (uint32_t i = 0; i < 3u; i++)
    if (!testAxis(A, B, delta, A.ax[i], AXIS_FACE_A, i, 0u, face)) return;
  for (uint32_t i = 0; i < 3u; i++)
    if (!testAxis(A, B, delta, B.ax[i], AXIS_FACE_B, 0u, i, face)) return;
  for (uint32_t i = 0; i < 3u; i++)
    for (uint32_t j = 0; j < 3u; j++)
      if (!testAxis(A, B, delta, cross3(A.ax[i], B.ax[j]), AXIS_EDGE, i, j, edge)) return;
  if (!face.valid) return;
  Sat best = face;
  if (edge.valid) {
    bool edgeWins = 0.95f * edge.sep > face.sep + 0.01f;
    if (faceBias) edgeWins = edge.sep > 0.95f * face.sep + 0.01f;
    if (edgeWins) best = edge;
  }
  sat = best;
  if (best.kind == AXIS_EDGE) edgeContact(A, B, best.ia, best.ib, best.n, found);
  else faceManifold(A, B, best.kind == AXIS_FACE_A, best.kind == AXIS_FACE_A ? best.ia : best.ib, best.n, found);
}
// Spheres (wgsl-collision.ts:604-653)
__device__ void sphereSphere(const Box& A, const Box& B, Sat& sat, Found& found) {
  float3 d = B.c - A.c;
  float dist = sqrtf(dot3(d, d));
  if (dist > A.h.x + B.h.x) return;
  float3 n = make_float3(0.0f, 0.0f, 1.0f);
  if (dist > 0.0f) n = d / dist;
  sat.n = n;
  addFound(found, A.c + n * A.h.x, B.c - n * B.h.x, SPHERE_FEATURE);
}
__device__ bool sphereBox(const Box& S, const Box& X, float4 qX, float3& onSphere, float3& onBox, float3& nOut) {
  float3 p = qrotate(qconj(qX), S.c - X.c);
  float3 q = make_float3(fminf(fmaxf(p.x, -X.h.x), X.h.x), fminf(fmaxf(p.y, -X.h.y), X.h.y), fminf(fmaxf(p.z, -X.h.z), X.h.z));
  float r = S.h.x;
  float3 nLocal;
  float3 ob = q;
  if (p.x != q.x || p.y != q.y || p.z != q.z) {
    float3 d = p - q;
    float dist = sqrtf(dot3(d, d));
    if (dist > r) return false;
    nLocal = d / dist;
  } else {
    float3 depth = X.h - abs3(p);
    int k = 0;
    if (depth.y < comp(depth, k)) k = 1;
    if (depth.z < comp(depth, k)) k = 2;
    float s = comp(p, k) >= 0.0f ? 1.0f : -1.0f;
    nLocal = make_float3(k == 0 ? s : 0.0f, k == 1 ? s : 0.0f, k == 2 ? s : 0.0f);
    if (k == 0) ob.x = s * X.h.x;
    else if (k == 1) ob.y = s * X.h.y;
    else ob.z = s * X.h.z;
  }
  float3 n = qrotate(qX, nLocal);
  nOut = -n;
  onBox = X.c + qrotate(qX, ob);
  onSphere = S.c - n * r;
  return true;
}

// Contact pair p: manifold slot p with its points at 8p .. 8p+count-1, warm-started from last step's
// pair (a, b) by feature key (wgsl-collision.ts:767-892).
// --- convex hulls (wgsl-hull.ts) -------------------------------------------------------------------------
// A pair with a hull on either side (the other a hull, a box or a sphere) collides here: SAT over
// both shapes' face normals by support points and the edge pairs whose Gauss-map arcs cross
// (queryFaces, queryEdges), then the incident face clipped by the reference face's side planes, or
// the closest points of two edges. A box takes part as a hull of its own topology. These run one
// thread per pair with their clip polygons in local memory, kept out of the box path (noinline).
constexpr uint32_t NO_HULL = 0xffffffffu, MAX_CLIP = 64;
constexpr float SHAPE_HULL_F = 3.0f;
__constant__ uint8_t BOX_FACE_VERTS[24] = {1, 3, 7, 5, 0, 2, 6, 4, 2, 3, 7, 6, 0, 1, 5, 4, 4, 5, 7, 6, 0, 1, 3, 2};
__constant__ uint8_t BOX_EDGES[12][4] = {{0, 1, 3, 5}, {2, 3, 2, 5}, {4, 5, 3, 4}, {6, 7, 2, 4}, {0, 2, 1, 5}, {1, 3, 0, 5},
                                         {4, 6, 1, 4}, {5, 7, 0, 4}, {0, 4, 1, 3}, {1, 5, 0, 3}, {2, 6, 1, 2}, {3, 7, 0, 2}};

struct Poly {
  float3 c, h;
  float4 q;
  uint32_t hull, vs, nv, fs, nf, es, ne, is;
};
__device__ inline bool isHull(const DWorld& w, uint32_t i) { return w.avel[i].w >= SHAPE_HULL_F; }
__device__ inline Poly polyOf(const DWorld& w, uint32_t i) {  // wgsl-hull.ts:47-63
  Poly P;
  P.c = f3(w.pos[i]);
  P.q = w.rot[i];
  P.h = f3(w.size[i]) * 0.5f;
  P.hull = NO_HULL;
  P.nv = 8u;
  P.nf = 6u;
  P.ne = 12u;
  P.vs = P.fs = P.es = P.is = 0u;
  if (isHull(w, i)) {
    uint32_t h = (uint32_t)(w.avel[i].w - SHAPE_HULL_F + 0.5f);
    uint4 h0 = w.hulls[h], h1 = w.hulls[h + 1u];
    P.hull = h;
    P.vs = h0.x;
    P.nv = h0.y;
    P.fs = h0.z;
    P.nf = h0.w;
    P.es = h1.x;
    P.ne = h1.y;
    P.is = h1.z;
  }
  return P;
}
__device__ inline float3 u4f3(uint4 u) { return make_float3(__uint_as_float(u.x), __uint_as_float(u.y), __uint_as_float(u.z)); }
__device__ inline float3 vertLocal(const DWorld& w, const Poly& P, uint32_t v) {
  if (P.hull == NO_HULL) return make_float3((v & 1u) ? P.h.x : -P.h.x, (v & 2u) ? P.h.y : -P.h.y, (v & 4u) ? P.h.z : -P.h.z);
  return u4f3(w.hulls[P.vs + v]);
}
__device__ inline float3 vert(const DWorld& w, const Poly& P, uint32_t v) { return P.c + qrotate(P.q, vertLocal(w, P, v)); }
__device__ inline float3 faceNormalLocal(const DWorld& w, const Poly& P, uint32_t f) {
  if (P.hull == NO_HULL) {
    float3 n = make_float3(0.0f, 0.0f, 0.0f);
    float s = (f & 1u) ? -1.0f : 1.0f;
    if (f / 2u == 0u) n.x = s;
    else if (f / 2u == 1u) n.y = s;
    else n.z = s;
    return n;
  }
  return u4f3(w.hulls[P.fs + 2u * f]);
}
__device__ inline float4 facePlane(const DWorld& w, const Poly& P, uint32_t f) {  // wgsl-hull.ts:75-92
  float3 nl;
  float d;
  if (P.hull == NO_HULL) {
    nl = faceNormalLocal(w, P, f);
    uint32_t k = f / 2u;
    d = k == 0u ? P.h.x : (k == 1u ? P.h.y : P.h.z);
  } else {
    uint4 u = w.hulls[P.fs + 2u * f];
    nl = u4f3(u);
    d = __uint_as_float(u.w);
  }
  float3 n = qrotate(P.q, nl);
  return make_float4(n.x, n.y, n.z, d + dot3(n, P.c));
}
__device__ inline uint32_t faceVertCount(const DWorld& w, const Poly& P, uint32_t f) { return P.hull == NO_HULL ? 4u : w.hulls[P.fs + 2u * f + 1u].y; }
__device__ inline uint32_t faceVert(const DWorld& w, const Poly& P, uint32_t f, uint32_t j) {
  if (P.hull == NO_HULL) return BOX_FACE_VERTS[f * 4u + j];
  uint32_t k = w.hulls[P.fs + 2u * f + 1u].x + j;
  uint4 q = w.hulls[P.is + k / 4u];
  uint32_t m = k % 4u;
  return m == 0u ? q.x : (m == 1u ? q.y : (m == 2u ? q.z : q.w));
}
__device__ inline uint4 edgeOf(const DWorld& w, const Poly& P, uint32_t e) {
  if (P.hull == NO_HULL) return make_uint4(BOX_EDGES[e][0], BOX_EDGES[e][1], BOX_EDGES[e][2], BOX_EDGES[e][3]);
  return w.hulls[P.es + e];
}
__device__ inline float3 polySupport(const DWorld& w, const Poly& P, float3 dir) {  // wgsl-hull.ts:104-115
  float3 l = qrotate(qconj(P.q), dir);
  if (P.hull == NO_HULL)
    return P.c + qrotate(P.q, make_float3(l.x >= 0.0f ? P.h.x : -P.h.x, l.y >= 0.0f ? P.h.y : -P.h.y, l.z >= 0.0f ? P.h.z : -P.h.z));
  float best = -3.4e38f;
  float3 at = make_float3(0.0f, 0.0f, 0.0f);
  for (uint32_t v = 0; v < P.nv; v++) {
    float3 q = u4f3(w.hulls[P.vs + v]);
    float s = dot3(q, l);
    if (s > best) {
      best = s;
      at = q;
    }
  }
  return P.c + qrotate(P.q, at);
}
// The face of A whose plane B sticks out of least (wgsl-hull.ts:120-128)
__device__ inline void queryFaces(const DWorld& w, const Poly& A, const Poly& B, float& sep, uint32_t& face) {
  sep = -3.4e38f;
  face = 0u;
  for (uint32_t f = 0; f < A.nf; f++) {
    float4 pl = facePlane(w, A, f);
    float3 n = make_float3(pl.x, pl.y, pl.z);
    float s = dot3(n, polySupport(w, B, -n)) - pl.w;
    if (s > sep) {
      sep = s;
      face = f;
    }
  }
}
__device__ inline bool minkowskiFace(float3 a, float3 b, float3 c, float3 d) {  // wgsl-hull.ts:131-142
  float3 bxa = cross3(b, a), dxc = cross3(d, c);
  float cba = dot3(c, bxa), dba = dot3(d, bxa), adc = dot3(a, dxc), bdc = dot3(b, dxc);
  return cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f;
}
struct EdgeQuery {
  float sep;
  uint32_t ea, eb;
  float3 n;
  bool valid;
};
__device__ __noinline__ EdgeQuery queryEdges(const DWorld& w, const Poly& A, const Poly& B) {  // wgsl-hull.ts:155-183
  EdgeQuery out;
  out.sep = -3.4e38f;
  out.ea = out.eb = 0u;
  out.n = make_float3(0.0f, 0.0f, 0.0f);
  out.valid = false;
  float4 toB = qmul(qconj(B.q), A.q);
  for (uint32_t i = 0; i < A.ne; i++) {
    uint4 ea = edgeOf(w, A, i);
    float3 a = qrotate(toB, faceNormalLocal(w, A, ea.z));
    float3 b = qrotate(toB, faceNormalLocal(w, A, ea.w));
    for (uint32_t j = 0; j < B.ne; j++) {
      uint4 eb = edgeOf(w, B, j);
      if (!minkowskiFace(a, b, -faceNormalLocal(w, B, eb.z), -faceNormalLocal(w, B, eb.w))) continue;
      float3 pa = vert(w, A, ea.x), qa = vert(w, A, ea.y), pb = vert(w, B, eb.x), qb = vert(w, B, eb.y);
      float3 n = cross3(qa - pa, qb - pb);
      float l = len3(n);
      if (l < 1e-5f * len3(qa - pa) * len3(qb - pb)) continue;
      n = n / l;
      if (dot3(n, pa - A.c) < 0.0f) n = -n;
      float s = dot3(n, pb - pa);
      if (s > out.sep) {
        out.sep = s;
        out.ea = i;
        out.eb = j;
        out.n = n;
        out.valid = true;
      }
    }
  }
  return out;
}
__device__ inline uint32_t clipHull(const float3* src, uint32_t n, float3* dst, float3 pn, float offset) {  // wgsl-hull.ts:186-204
  if (n == 0u) return 0u;
  uint32_t count = 0;
  float3 a = src[n - 1u];
  float da = dot3(pn, a) - offset;
  for (uint32_t i = 0; i < n; i++) {
    float3 b = src[i];
    float db = dot3(pn, b) - offset;
    if ((da <= PLANE_EPSILON) != (db <= PLANE_EPSILON)) {
      float t = 0.0f;
      if (fabsf(da - db) > SAT_AXIS_EPSILON) t = fminf(fmaxf(da / (da - db), 0.0f), 1.0f);
      if (count < MAX_CLIP) dst[count++] = a + (b - a) * t;
    }
    if (db <= PLANE_EPSILON && count < MAX_CLIP) dst[count++] = b;
    a = b;
    da = db;
  }
  return count;
}
// Face contact (wgsl-hull.ts:207-291): the other shape's face clipped to the reference face
__device__ __noinline__ void hullFaceContact(const DWorld& w, const Poly& A, const Poly& B, bool refIsA, uint32_t refFace, Found& found) {
  const Poly& R = refIsA ? A : B;
  const Poly& I = refIsA ? B : A;
  float4 plane = facePlane(w, R, refFace);
  float3 rn = make_float3(plane.x, plane.y, plane.z);
  uint32_t deepest = 0;
  float low = 3.4e38f;
  for (uint32_t v = 0; v < I.nv; v++) {
    float d = dot3(vert(w, I, v), rn);
    if (d < low) {
      low = d;
      deepest = v;
    }
  }
  uint32_t inc = 0;
  float least = 3.4e38f;
  for (uint32_t f = 0; f < I.nf; f++) {
    bool touches = false;
    uint32_t cnt = faceVertCount(w, I, f);
    for (uint32_t j = 0; j < cnt; j++)
      if (faceVert(w, I, f, j) == deepest) {
        touches = true;
        break;
      }
    if (!touches) continue;
    float4 pf = facePlane(w, I, f);
    float d = dot3(make_float3(pf.x, pf.y, pf.z), rn);
    if (d < least) {
      least = d;
      inc = f;
    }
  }
  float3 poly[MAX_CLIP], tmp[MAX_CLIP];
  uint32_t n = min(faceVertCount(w, I, inc), MAX_CLIP);
  for (uint32_t j = 0; j < n; j++) poly[j] = vert(w, I, faceVert(w, I, inc, j));
  const uint32_t k = faceVertCount(w, R, refFace);
  float3 centre = make_float3(0.0f, 0.0f, 0.0f);
  for (uint32_t j = 0; j < k; j++) centre = centre + vert(w, R, faceVert(w, R, refFace, j));
  centre = centre / (float)k;
  for (uint32_t j = 0; j < k && n > 0u; j++) {
    float3 v0 = vert(w, R, faceVert(w, R, refFace, j));
    float3 v1 = vert(w, R, faceVert(w, R, refFace, (j + 1u) % k));
    float3 sd = cross3(v1 - v0, rn);
    float l = len3(sd);
    if (l < SAT_AXIS_EPSILON) continue;
    sd = sd / l;
    if (dot3(sd, centre - v0) > 0.0f) sd = -sd;
    n = clipHull(poly, n, tmp, sd, dot3(sd, v0));
    for (uint32_t m = 0; m < n; m++) poly[m] = tmp[m];
  }
  float depth[MAX_CLIP];
  uint32_t index[MAX_CLIP];
  bool chosen[MAX_CLIP];
  uint32_t keep = 0;
  for (uint32_t m = 0; m < n; m++) {
    float dist = dot3(rn, poly[m]) - plane.w;
    if (dist <= PLANE_EPSILON) {
      tmp[keep] = poly[m];
      depth[keep] = dist;
      index[keep] = m;
      chosen[keep] = false;
      keep++;
    }
  }
  const uint32_t prefix = ((refIsA ? AXIS_FACE_A : AXIS_FACE_B) << 24) | (min(refFace, 255u) << 16) | (min(inc, 255u) << 8);
  for (uint32_t c = 0; c < min(keep, (uint32_t)MAX_CONTACTS); c++) {
    uint32_t pick = 0;
    float bestScore = -3.4e38f;
    for (uint32_t m = 0; m < keep; m++) {
      if (chosen[m]) continue;
      float score = -depth[m];
      if (c > 0u) {
        score = 3.4e38f;
        for (uint32_t o = 0; o < keep; o++)
          if (chosen[o]) score = fminf(score, dot3(tmp[m] - tmp[o], tmp[m] - tmp[o]));
      }
      if (score > bestScore) {
        bestScore = score;
        pick = m;
      }
    }
    chosen[pick] = true;
    float3 pp = tmp[pick];
    float3 onRef = pp - rn * depth[pick];
    addFound(found, refIsA ? onRef : pp, refIsA ? pp : onRef, prefix | min(index[pick], 255u));
  }
  if (found.count == 0u) {
    float3 nAB = refIsA ? rn : -rn;
    addFound(found, polySupport(w, A, nAB), polySupport(w, B, -nAB), prefix);
  }
}
// Edge contact (wgsl-hull.ts:293-315): closest points of the two edges
__device__ inline void hullEdgeContact(const DWorld& w, const Poly& A, const Poly& B, const EdgeQuery& q, Found& found) {
  uint4 ea = edgeOf(w, A, q.ea), eb = edgeOf(w, B, q.eb);
  float3 p0 = vert(w, A, ea.x), q0 = vert(w, B, eb.x);
  float3 d1 = vert(w, A, ea.y) - p0, d2 = vert(w, B, eb.y) - q0;
  float3 r = p0 - q0;
  float a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r), c = dot3(d1, r), b = dot3(d1, d2);
  float denom = a * e - b * b;
  float s = 0.0f;
  if (fabsf(denom) > SAT_AXIS_EPSILON * a * e) s = fminf(fmaxf((b * f - c * e) / denom, 0.0f), 1.0f);
  float t = (b * s + f) / fmaxf(e, SAT_AXIS_EPSILON);
  if (t < 0.0f) {
    t = 0.0f;
    s = fminf(fmaxf(-c / fmaxf(a, SAT_AXIS_EPSILON), 0.0f), 1.0f);
  } else if (t > 1.0f) {
    t = 1.0f;
    s = fminf(fmaxf((b - c) / fmaxf(a, SAT_AXIS_EPSILON), 0.0f), 1.0f);
  }
  addFound(found, p0 + d1 * s, q0 + d2 * t, (AXIS_EDGE << 24) | (min(q.ea, 255u) << 8) | min(q.eb, 255u));
}
// collidePoly (wgsl-hull.ts:318-341): sat.n from A towards B
__device__ __noinline__ void collidePoly(const DWorld& w, const Poly& A, const Poly& B, bool faceBias, Sat& sat, Found& found) {
  float faSep, fbSep;
  uint32_t faFace, fbFace;
  queryFaces(w, A, B, faSep, faFace);
  if (faSep > 0.0f) return;
  queryFaces(w, B, A, fbSep, fbFace);
  if (fbSep > 0.0f) return;
  EdgeQuery eq = queryEdges(w, A, B);
  if (eq.valid && eq.sep > 0.0f) return;
  float faceSep = fmaxf(faSep, fbSep);
  bool edgeWins = eq.valid && eq.sep > 0.95f * faceSep + 0.01f;
  if (!faceBias) edgeWins = eq.valid && 0.95f * eq.sep > faceSep + 0.01f;
  if (edgeWins) {
    sat.kind = AXIS_EDGE;
    sat.ia = eq.ea;
    sat.ib = eq.eb;
    sat.sep = eq.sep;
    sat.n = eq.n;
    sat.valid = true;
    hullEdgeContact(w, A, B, eq, found);
    return;
  }
  if (fbSep > faSep) {
    float4 pl = facePlane(w, B, fbFace);
    sat.kind = AXIS_FACE_B;
    sat.ia = 0u;
    sat.ib = fbFace;
    sat.sep = fbSep;
    sat.n = -make_float3(pl.x, pl.y, pl.z);
    sat.valid = true;
    hullFaceContact(w, A, B, false, fbFace, found);
    return;
  }
  float4 pl = facePlane(w, A, faFace);
  sat.kind = AXIS_FACE_A;
  sat.ia = faFace;
  sat.ib = 0u;
  sat.sep = faSep;
  sat.n = make_float3(pl.x, pl.y, pl.z);
  sat.valid = true;
  hullFaceContact(w, A, B, true, faFace, found);
}
__device__ inline float3 segmentPoint(float3 a, float3 b, float3 p) {  // wgsl-hull.ts:344-347
  float3 d = b - a;
  return a + d * fminf(fmaxf(dot3(p - a, d) / fmaxf(dot3(d, d), 1e-20f), 0.0f), 1.0f);
}
// Sphere (centre c, radius r) against hull X (wgsl-hull.ts:350-405): n from the sphere towards X
__device__ __noinline__ bool sphereHull(const DWorld& w, float3 c, float r, const Poly& X, float3& onSphere, float3& onHull, float3& nOut) {
  float deepest = -3.4e38f;
  uint32_t deepFace = 0;
  for (uint32_t f = 0; f < X.nf; f++) {
    float4 pl = facePlane(w, X, f);
    float s = dot3(make_float3(pl.x, pl.y, pl.z), c) - pl.w;
    if (s > deepest) {
      deepest = s;
      deepFace = f;
    }
  }
  if (deepest > r) return false;
  if (deepest <= 0.0f) {
    float4 pl = facePlane(w, X, deepFace);
    float3 n = make_float3(pl.x, pl.y, pl.z);
    nOut = -n;
    onHull = c - n * deepest;
    onSphere = c - n * r;
    return true;
  }
  float3 best = make_float3(0.0f, 0.0f, 0.0f);
  float bestDist = 3.4e38f;
  for (uint32_t f = 0; f < X.nf; f++) {
    float4 pl = facePlane(w, X, f);
    float3 pn = make_float3(pl.x, pl.y, pl.z);
    float s = dot3(pn, c) - pl.w;
    if (s <= 0.0f) continue;
    float3 pp = c - pn * s;
    uint32_t k = faceVertCount(w, X, f);
    float3 centre = make_float3(0.0f, 0.0f, 0.0f);
    for (uint32_t j = 0; j < k; j++) centre = centre + vert(w, X, faceVert(w, X, f, j));
    centre = centre / (float)k;
    bool inside = true;
    float3 edgeBest = make_float3(0.0f, 0.0f, 0.0f);
    float edgeDist = 3.4e38f;
    for (uint32_t j = 0; j < k; j++) {
      float3 v0 = vert(w, X, faceVert(w, X, f, j));
      float3 v1 = vert(w, X, faceVert(w, X, f, (j + 1u) % k));
      float3 side = cross3(v1 - v0, pn);
      if (dot3(side, centre - v0) > 0.0f) side = -side;
      if (dot3(side, pp - v0) > 0.0f) inside = false;
      float3 q = segmentPoint(v0, v1, c);
      float dq = dot3(q - c, q - c);
      if (dq < edgeDist) {
        edgeDist = dq;
        edgeBest = q;
      }
    }
    if (!inside) pp = edgeBest;
    float dist = len3(pp - c);
    if (dist < bestDist) {
      bestDist = dist;
      best = pp;
    }
  }
  if (bestDist > r) return false;
  float3 n = make_float3(0.0f, 0.0f, 1.0f);
  if (bestDist > 0.0f) n = (c - best) / bestDist;
  nOut = -n;
  onHull = best;
  onSphere = c - n * r;
  return true;
}


// --- hull pairs, one warp per pair ---------------------------------------------------------------------
// The SAT queries of collidePoly with the faces, and the edge pairs (i, j) in i-major order, dealt to
// the lanes; each lane evaluates its candidates exactly as the sequential loops do, and a warp
// reduction keeps the largest separation, the lowest index among equals: the candidate the
// sequential loop's strict "greater" keeps. The contact itself is built by lane 0.
__device__ inline void warpArgMax(float& v, uint32_t& i) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    float ov = __shfl_xor_sync(0xffffffffu, v, off);
    uint32_t oi = __shfl_xor_sync(0xffffffffu, i, off);
    if (ov > v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
}
__device__ inline void queryFacesWarp(const DWorld& w, const Poly& A, const Poly& B, uint32_t lane, float& sep, uint32_t& face) {
  float best = -3.4e38f;
  uint32_t at = 0xffffffffu;
  for (uint32_t f = lane; f < A.nf; f += 32u) {
    float4 pl = facePlane(w, A, f);
    float3 n = make_float3(pl.x, pl.y, pl.z);
    float s = dot3(n, polySupport(w, B, -n)) - pl.w;
    if (s > best) {  // lanes take ascending faces: the first of equals stays
      best = s;
      at = f;
    }
  }
  warpArgMax(best, at);
  sep = best;
  face = at == 0xffffffffu ? 0u : at;
}
__device__ inline EdgeQuery queryEdgesWarp(const DWorld& w, const Poly& A, const Poly& B, uint32_t lane) {
  const float4 toB = qmul(qconj(B.q), A.q);
  const uint32_t total = A.ne * B.ne;
  float best = -3.4e38f;
  uint32_t at = 0xffffffffu;
  float3 bestN = make_float3(0.0f, 0.0f, 0.0f);
  for (uint32_t k = lane; k < total; k += 32u) {
    const uint32_t i = k / B.ne, j = k - i * B.ne;
    uint4 ea = edgeOf(w, A, i);
    float3 a = qrotate(toB, faceNormalLocal(w, A, ea.z));
    float3 b = qrotate(toB, faceNormalLocal(w, A, ea.w));
    uint4 eb = edgeOf(w, B, j);
    if (!minkowskiFace(a, b, -faceNormalLocal(w, B, eb.z), -faceNormalLocal(w, B, eb.w))) continue;
    float3 pa = vert(w, A, ea.x), qa = vert(w, A, ea.y), pb = vert(w, B, eb.x), qb = vert(w, B, eb.y);
    float3 n = cross3(qa - pa, qb - pb);
    float l = len3(n);
    if (l < 1e-5f * len3(qa - pa) * len3(qb - pb)) continue;
    n = n / l;
    if (dot3(n, pa - A.c) < 0.0f) n = -n;
    float s = dot3(n, pb - pa);
    if (s > best) {
      best = s;
      at = k;
      bestN = n;
    }
  }
  const uint32_t mine = at;
  warpArgMax(best, at);
  const uint32_t src = __ffs(__ballot_sync(0xffffffffu, mine == at && at != 0xffffffffu)) - 1u;
  EdgeQuery out;
  out.valid = at != 0xffffffffu;
  out.sep = best;
  out.ea = out.valid ? at / B.ne : 0u;
  out.eb = out.valid ? at - out.ea * B.ne : 0u;
  out.n = out.valid ? make_float3(__shfl_sync(0xffffffffu, bestN.x, src), __shfl_sync(0xffffffffu, bestN.y, src), __shfl_sync(0xffffffffu, bestN.z, src))
                    : make_float3(0.0f, 0.0f, 0.0f);
  return out;
}
// collidePoly (wgsl-hull.ts:318-341) with the queries spread over the warp; the result is lane 0's
__device__ void collidePolyWarp(const DWorld& w, const Poly& A, const Poly& B, bool faceBias, uint32_t lane, Sat& sat, Found& found) {
  float faSep, fbSep;
  uint32_t faFace, fbFace;
  queryFacesWarp(w, A, B, lane, faSep, faFace);
  if (faSep > 0.0f) return;
  queryFacesWarp(w, B, A, lane, fbSep, fbFace);
  if (fbSep > 0.0f) return;
  EdgeQuery eq = queryEdgesWarp(w, A, B, lane);
  if (eq.valid && eq.sep > 0.0f) return;
  if (lane != 0u) return;
  float faceSep = fmaxf(faSep, fbSep);
  bool edgeWins = eq.valid && eq.sep > 0.95f * faceSep + 0.01f;
  if (!faceBias) edgeWins = eq.valid && 0.95f * eq.sep > faceSep + 0.01f;
  if (edgeWins) {
    sat.kind = AXIS_EDGE;
    sat.ia = eq.ea;
    sat.ib = eq.eb;
    sat.sep = eq.sep;
    sat.n = eq.n;
    sat.valid = true;
    hullEdgeContact(w, A, B, eq, found);
    return;
  }
  if (fbSep > faSep) {
    float4 pl = facePlane(w, B, fbFace);
    sat.kind = AXIS_FACE_B;
    sat.ia = 0u;
    sat.ib = fbFace;
    sat.sep = fbSep;
    sat.n = -make_float3(pl.x, pl.y, pl.z);
    sat.valid = true;
    hullFaceContact(w, A, B, false, fbFace, found);
    return;
  }
  float4 pl = facePlane(w, A, faFace);
  sat.kind = AXIS_FACE_A;
  sat.ia = faFace;
  sat.ib = 0u;
  sat.sep = faSep;
  sat.n = make_float3(pl.x, pl.y, pl.z);
  sat.valid = true;
  hullFaceContact(w, A, B, true, faFace, found);
}

__device__ __forceinline__ void writeManifold(const DWorld& w, const StepParams& p, uint32_t pi, uint32_t a, uint32_t b, const Box& A, const Box& B, const Sat& sat,
                              const Found& found, bool anySphere);

__device__ void narrowPair(const DWorld& w, const StepParams& p, uint32_t pi) {
  {
    uint2 pr = w.pairs[pi];
    uint32_t a = pr.x, b = pr.y;
    Box A = makeBox(w, a), B = makeBox(w, b);
    Sat sat;
    sat.n = make_float3(0.0f, 0.0f, 0.0f);
    sat.valid = false;
    Found found;
    found.count = 0;
    if ((p.flags & FLAG_REUSE_CONTACTS) && reusePair(w, p, pi, a, b)) return;
    bool sphereA = w.avel[a].w == SHAPE_SPHERE_F, sphereB = w.avel[b].w == SHAPE_SPHERE_F;
    float4 qA = w.rot[a], qB = w.rot[b];
    if (sphereA && sphereB) {
      sphereSphere(A, B, sat, found);
    } else if (w.hulls && (isHull(w, a) || isHull(w, b))) {
      if (sphereA || sphereB) {
        float3 onS, onX, nn;
        if (sphereA) {
          bool hit = sphereHull(w, A.c, A.h.x, polyOf(w, b), onS, onX, nn);
          sat.n = nn;
          if (hit) addFound(found, onS, onX, SPHERE_FEATURE);
        } else {
          bool hit = sphereHull(w, B.c, B.h.x, polyOf(w, a), onS, onX, nn);
          sat.n = -nn;
          if (hit) addFound(found, onX, onS, SPHERE_FEATURE);
        }
      } else {
        // hull against hull or box: one warp per pair (k_hull_narrowphase) writes this slot
        w.hullPairs[atomicAdd(&w.counters[C_HULL_PAIRS], 1u)] = pi;
        return;
      }
    } else if (sphereA || sphereB) {
      float3 onS, onX, nn;
      if (sphereA) {
        bool hit = sphereBox(A, B, qB, onS, onX, nn);
        sat.n = nn;
        if (hit) addFound(found, onS, onX, SPHERE_FEATURE);
      } else {
        bool hit = sphereBox(B, A, qA, onS, onX, nn);
        sat.n = -nn;
        if (hit) addFound(found, onX, onS, SPHERE_FEATURE);
      }
    } else {
      collideBoxes(A, B, (p.flags & FLAG_FACE_BIAS) != 0u, sat, found);
    }
    writeManifold(w, p, pi, a, b, A, B, sat, found, sphereA || sphereB);
  }
}

// Pair slot pi's manifold from its contacts: ids, normal and friction, and every point warm-started
// from last step's point of the same feature (wgsl-collision.ts:812-900)
__device__ __forceinline__ void writeManifold(const DWorld& w, const StepParams& p, uint32_t pi, uint32_t a, uint32_t b, const Box& A, const Box& B, const Sat& sat,
                              const Found& found, bool anySphere) {
  const int cur = p.cur, prev = 1 - cur;
  {
    float4 qA = w.rot[a], qB = w.rot[b];
    uint32_t count = found.count;
    float3 n = -sat.n;
    float fa = w.pos[a].w, fb = w.pos[b].w;
    w.mIds[cur][pi] = make_uint4(a, b, pi * MAX_CONTACTS, count | (w.counters[C_STEP] << 4));
    w.mGeo[cur][pi] = make_float4(n.x, n.y, n.z, sqrtf(fa * fb));
    countManifold(w, count);
    if (count == 0u) return;
    float3 t1, t2;
    orthonormal(n, t1, t2);
    uint32_t prevFirst = 0, prevCount = 0;
    int pm = hashFind(w, p, a, b);
    if (pm >= 0) {
      uint4 pid = w.mIds[prev][pm];
      prevFirst = pid.z;
      prevCount = min(pid.w & 15u, (uint32_t)MAX_CONTACTS);
    }
    bool matchNearest = (p.flags & FLAG_MATCH_NEAREST) != 0u;
    float minSide = fminf(fminf(fminf(A.h.x, A.h.y), A.h.z), fminf(fminf(B.h.x, B.h.y), B.h.z)) * 2.0f;
    const float penaltyMin = contactPenaltyMin(w, p, a, b);
    float3 cA = A.c, cB = B.c;
    for (uint32_t i = 0; i < count; i++) {
      float3 rA = qrotate(qconj(qA), found.xA[i] - cA);
      float3 rB = qrotate(qconj(qB), found.xB[i] - cB);
      float3 pen = make_float3(0.0f, 0.0f, 0.0f), lam = make_float3(0.0f, 0.0f, 0.0f);
      uint32_t stick = 0;
      int j = -1;
      for (uint32_t c = prevFirst; c < prevFirst + prevCount; c++) {
        if ((__float_as_uint(w.cPt[prev][4 * c + K_RA].w) & ~STICK_BIT) == found.feature[i]) {
          j = int(c);
          break;
        }
      }
      if (j < 0 && matchNearest) {
        float bestDist = NEAREST_FRACTION * minSide;
        for (uint32_t c = prevFirst; c < prevFirst + prevCount; c++) {
          float3 d = f3(w.cPt[prev][4 * c + K_RA]) - rA;
          float dist = sqrtf(dot3(d, d));
          if (dist <= bestDist) {
            bestDist = dist;
            j = int(c);
          }
        }
      }
      if (j >= 0) {
        const float4* q = w.cPt[prev] + 4 * j;
        float4 pra = q[K_RA];
        pen = f3(q[K_PEN]);
        lam = f3(q[K_LAM]);
        stick = __float_as_uint(pra.w) & STICK_BIT;
        if (stick != 0u && !anySphere) {
          rA = f3(pra);
          rB = f3(q[K_RB]);
        }
      }
      // the centres' difference first (exact for nearby bodies at any distance from the origin)
      float3 d = (cA - cB) + (qrotate(qA, rA) - qrotate(qB, rB));
      float c0x = dot3(n, d) + p.margin, c0y = dot3(t1, d), c0z = dot3(t2, d);
      lam = lam * p.alpha * p.gamma;
      pen = make_float3(fminf(fmaxf(pen.x * p.gamma, PENALTY_MIN), PENALTY_MAX), fminf(fmaxf(pen.y * p.gamma, PENALTY_MIN), PENALTY_MAX),
                        fminf(fmaxf(pen.z * p.gamma, PENALTY_MIN), PENALTY_MAX));
      pen.x = fmaxf(pen.x, penaltyMin);
      uint32_t slot = pi * MAX_CONTACTS + i;
      float4* o = w.cPt[cur] + 4 * slot;
      o[K_RA] = make_float4(rA.x, rA.y, rA.z, __uint_as_float(found.feature[i] | stick));
      o[K_RB] = make_float4(rB.x, rB.y, rB.z, c0x);
      o[K_PEN] = make_float4(pen.x, pen.y, pen.z, c0y);
      o[K_LAM] = make_float4(lam.x, lam.y, lam.z, c0z);
    }
  }
}

// The deferred hull pairs, one warp each
__global__ void __launch_bounds__(256) k_hull_narrowphase(DWorld w, StepParams p) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t total = w.counters[C_HULL_PAIRS];
  for (uint32_t k = warp; k < total; k += nwarps) {
    const uint32_t pi = w.hullPairs[k];
    const uint2 pr = w.pairs[pi];
    Sat sat;
    sat.n = make_float3(0.0f, 0.0f, 0.0f);
    sat.valid = false;
    Found found;
    found.count = 0;
    collidePolyWarp(w, polyOf(w, pr.x), polyOf(w, pr.y), (p.flags & FLAG_FACE_BIAS) != 0u, lane, sat, found);
    if (lane == 0u) writeManifold(w, p, pi, pr.x, pr.y, makeBox(w, pr.x), makeBox(w, pr.y), sat, found, false);
    __syncwarp();
  }
}

__global__ void __launch_bounds__(128) k_narrowphase(DWorld w, StepParams p) {
  uint32_t total = w.counters[C_PAIRS];
  if (total > p.pairCap) total = p.pairCap;
  for (uint32_t pi = blockIdx.x * blockDim.x + threadIdx.x; pi < total; pi += gridDim.x * blockDim.x) narrowPair(w, p, pi);
}

// --- batched worlds: one block per world ------------------------------------------------------------------
// A world of a batch holds at most a few hundred bodies: its pairs are found by testing every pair
// of bodies against the broadphase rule (the same set the grid walk finds), then collided.
__global__ void __launch_bounds__(256) k_batch_collide(BatchLaunch B) {
  __shared__ uint32_t s_world;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_world = atomicAdd(&B.queue[0], 1u);
    __syncthreads();
    const uint32_t qi = s_world;
    if (qi >= B.nWorlds) return;
    const uint32_t wi = B.order[qi];
    const WorldDesc d = B.worlds[wi];
    const DWorld w = worldView(B.base, d, wi);
    const StepParams p = worldParams(B.p, d);
    uint32_t* c = w.counters;
    const uint32_t prevPairs = min(c[C_PAIRS], d.pairCap);
    __syncthreads();
    if (threadIdx.x == 0) {
      c[C_PREV_PAIRS] = prevPairs;
      c[C_STEP] += 1;
      c[C_PAIRS] = 0;
      c[C_CONTACTS] = 0;
      c[C_MANIFOLDS] = 0;
      c[C_OVERFLOW] = 0;
      c[C_CLASHES] = 0;
      c[C_COLORS] = 0;
      c[C_ROUNDS] = 0;
      c[C_ERROR] = 0;
      for (int k = 0; k < 2 * MAX_ROUND_PAIRS + 2; k++) c[C_PENDING + k] = 0;
    }
    for (uint32_t h = threadIdx.x; h <= d.hashMask; h += blockDim.x) w.hash[h] = 0u;
    __syncthreads();
    if (p.flags & FLAG_REUSE_CONTACTS)  // updateRefs, per world
      for (uint32_t i = threadIdx.x; i < d.n; i += blockDim.x)
        if (((uint32_t)w.ipos[i].w & 2u) == 0u) updateRef(w, i, c[C_STEP]);
    const int prev = 1 - p.cur;
    for (uint32_t m = threadIdx.x; m < prevPairs; m += blockDim.x) {  // hashInsert, per world
      uint4 ids = w.mIds[prev][m];
      if ((ids.w & 15u) == 0u) continue;
      if (w.ipos[ids.x].w != 0.0f || w.ipos[ids.y].w != 0.0f) continue;
      uint32_t h = pairHash(ids.x, ids.y) & d.hashMask;
      for (uint32_t probe = 0; probe <= d.hashMask; probe++) {
        if (atomicCAS(&w.hash[h], 0u, m + 1u) == 0u) break;
        h = (h + 1u) & d.hashMask;
      }
    }
    __syncthreads();
    // every pair (i > j): triangular index k -> (i, j)
    const uint32_t n = d.n;
    const uint32_t total = n * (n - 1u) / 2u;
    for (uint32_t k = threadIdx.x; k < total; k += blockDim.x) {
      uint32_t i = (uint32_t)((1.0f + sqrtf(1.0f + 8.0f * (float)k)) * 0.5f);
      while (i * (i - 1u) / 2u > k) i--;
      while ((i + 1u) * i / 2u <= k) i++;
      uint32_t j = k - i * (i - 1u) / 2u;
      if (!enabled(w, i) || !enabled(w, j)) continue;
      bool di = w.size[i].w > 0.0f, dj = w.size[j].w > 0.0f;
      if (!di && !dj) continue;
      float4 pi4 = w.pos[i], pj4 = w.pos[j];
      float3 dd = make_float3(pi4.x - pj4.x, pi4.y - pj4.y, pi4.z - pj4.z);
      float r = w.moment[i].w + w.moment[j].w;
      if (dot3(dd, dd) > r * r) continue;  // the sphere test: the same from either body's view
      uint32_t pr = proberOf(w, p, i, j);
      testPair(w, p, probeOf(w, pr), pr == i ? j : i);
    }
    __syncthreads();
    const uint32_t found = c[C_PAIRS];
    const uint32_t pairs = min(found, d.pairCap);
    for (uint32_t pi = threadIdx.x; pi < pairs; pi += blockDim.x) narrowPair(w, p, pi);
    if (threadIdx.x == 0) {
      uint32_t bits = (c[C_OVERFLOW] & 1u) ? BATCH_OVERFLOW : 0u;
      if (uint64_t(found) * 10u > uint64_t(d.pairCap) * 8u) bits |= BATCH_NEAR_FULL;
      if (bits) atomicOr(&B.status[0], bits);
    }
  }
}

int batch_collide_blocks_per_sm(int threads) {
  int perSm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_batch_collide, threads, 0);
  return perSm;
}

cudaError_t launch_batch_collision(const BatchLaunch& b, int blocks, int threads, cudaStream_t s) {
  k_batch_collide<<<blocks, threads, 0, s>>>(b);
  return cudaGetLastError();
}

// The step's statistics into the ring: phase times from the device clocks, then the counters
__global__ void k_step_stats(DWorld w, uint32_t launches) {
  if (threadIdx.x != 0 || !w.statsRing || !w.statsCap) return;
  const uint32_t* c = w.counters;
  uint32_t slot = c[C_STATS_NEXT] % w.statsCap;
  uint32_t* o = w.statsRing + size_t(slot) * STAT_WORDS;
  unsigned long long n = w.clocks[0], t0 = w.clocks[CLOCK_T0], t1 = w.clocks[1], t2 = n ? w.clocks[n] : t1;
  o[0] = (uint32_t)(t1 - t0);
  o[1] = (uint32_t)(t2 - t1);
  o[2] = c[C_PAIRS];
  o[3] = c[C_CONTACTS];
  o[4] = c[C_MANIFOLDS];
  o[5] = c[C_ADJ];
  o[6] = c[C_INC];
  o[7] = c[C_DYN];
  o[8] = c[C_COLORS];
  o[9] = c[C_ROUNDS];
  o[10] = launches;
  o[11] = c[C_ERROR];
  w.counters[C_STATS_NEXT] = c[C_STATS_NEXT] + 1;
}
void launch_step_stats(const DWorld& w, uint32_t launches, cudaStream_t s) { k_step_stats<<<1, 32, 0, s>>>(w, launches); }

// Host: the collision phase, enqueued on `s`. Returns the number of kernels it launched.
uint32_t launch_collision(const DWorld& w, const StepParams& p, uint32_t tableSize, bool reuseManifolds, cudaStream_t s) {
  const uint32_t n = p.n;
  k_begin<<<1, 1, 0, s>>>(w, p);
  uint32_t launches = 1;
  if ((p.flags & FLAG_REUSE_CONTACTS) && n > 0) {
    k_update_refs<<<grid_for(n, 256), 256, 0, s>>>(w, p);
    launches++;
  }
  if (reuseManifolds) {
    k_reuse_manifolds<<<GS_BLOCKS, 128, 0, s>>>(w, p);
    return launches + 1;
  }
  launches += 2;  // hash insert, narrowphase
  cudaMemsetAsync(w.hash, 0, (size_t(p.hashMask) + 1) * 4, s);
  k_hash_insert<<<GS_BLOCKS, 256, 0, s>>>(w, p);
  if (n > 0) {
    const uint32_t sentinel = p.tableMask + 1u;
    cudaMemsetAsync(w.cellStart, 0, size_t(tableSize) * 4, s);
    k_cell_keys<<<grid_for(n, 256), 256, 0, s>>>(w, p);
    k_bucket_count<<<grid_for(n, 256), 256, 0, s>>>(w.keyA, n, w.cellStart, w.valB, sentinel);
    // cellEnd = counts before the scan turns them into starts
    cudaMemcpyAsync(w.cellEnd, w.cellStart, size_t(tableSize) * 4, cudaMemcpyDeviceToDevice, s);
    uint32_t tiles = grid_for(tableSize, SCAN_TILE);
    k_scan_tiles<<<tiles, SCAN_THREADS, 0, s>>>(w.cellStart, tableSize, w.radixHist);
    k_scan_single<<<1, 1024, 0, s>>>(w.radixHist, tiles);
    k_scan_add<<<tiles, SCAN_THREADS, 0, s>>>(w.cellStart, tableSize, w.radixHist);
    k_bucket_finish<<<grid_for(tableSize, 256), 256, 0, s>>>(w.cellStart, w.cellEnd, tableSize);
    k_bucket_scatter<<<grid_for(n, 256), 256, 0, s>>>(w, n, sentinel);
    k_find_pairs<<<grid_for(n, PAIR_WALK_THREADS), PAIR_WALK_THREADS, 0, s>>>(w, p);
    launches += 8;
  }
  k_narrowphase<<<GS_BLOCKS, 128, 0, s>>>(w, p);
  if (w.hulls) {
    k_hull_narrowphase<<<GS_BLOCKS, 256, 0, s>>>(w, p);
    launches++;
  }
  return launches;
}

}  // namespace avbd

// --- broadphase without allocation -------------------------------------------------------------------
// No counterpart in the reference. avbd_find_pairs_noalloc runs the step's broadphase (cell keys,
// counting sort, half-shell walk, large bodies against all; the pair rule of k_find_pairs) over up
// to NOALLOC_MAX_BODIES bodies given as host records, in ONE block, with every intermediate array in
// the file-scope device array below. Callers that cannot allocate device memory use it: a render or
// input thread that queries candidate pairs between steps (cudaMalloc and cudaFree synchronise the
// whole device, so they would stall the steps in flight on other streams), and hosts that hand all
// device memory to their own allocator. Every call shares the one array: calls whose GPU work
// overlaps (two streams, two host threads) race on it and their results are undefined.
namespace avbd {

constexpr uint32_t NOALLOC_MAX_BODIES = AVBD_NOALLOC_MAX_BODIES;
constexpr uint32_t NOALLOC_MAX_PAIRS = AVBD_NOALLOC_MAX_PAIRS;
constexpr uint32_t NOALLOC_TABLE = 2 * NOALLOC_MAX_BODIES;  // cell hash buckets (a power of two)
constexpr uint32_t NOALLOC_THREADS = 1024;
static_assert((NOALLOC_TABLE & (NOALLOC_TABLE - 1)) == 0 && NOALLOC_TABLE % NOALLOC_THREADS == 0, "table");

// Byte offsets of the scratch arrays (each a multiple of 256)
struct NoAllocLayout {
  static constexpr size_t B = NOALLOC_MAX_BODIES, T = NOALLOC_TABLE;
  static constexpr size_t POS = 0, ROT = POS + 16 * B, IPOS = ROT + 16 * B, SIZE = IPOS + 16 * B, MOMENT = SIZE + 16 * B, AVEL = MOMENT + 16 * B,
                          FILTERS = AVEL + 16 * B, CELL = FILTERS + 8 * B, KEY = CELL + 16 * B, RANK = KEY + 4 * B, START = RANK + 4 * B,
                          END = START + 4 * T, SPR = END + 4 * T, SCELL = SPR + 16 * B, SAABB = SCELL + 16 * B, LARGE = SAABB + 16 * B,
                          PAIRS = LARGE + 4 * B, COUNTERS = PAIRS + 8 * size_t(NOALLOC_MAX_PAIRS), BYTES = COUNTERS + 4 * COUNTER_WORDS;
};
static_assert(NoAllocLayout::BYTES == AVBD_NOALLOC_SCRATCH_BYTES, "the header states the scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NoAllocLayout::BYTES];

// One block: counts into buckets, scans them, scatters the candidate records, walks the cells.
// What must start at zero (the bucket counts and the pair counters) is cleared here, every call.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_find_pairs_noalloc(DWorld w, StepParams p, uint32_t* key, uint32_t* rank) {
  const uint32_t n = p.n, T = NOALLOC_TABLE, sentinel = T;
  __shared__ uint32_t s_warp[NOALLOC_THREADS / 32];
  for (uint32_t h = threadIdx.x; h < T; h += blockDim.x) w.cellStart[h] = 0u;
  if (threadIdx.x == 0) {
    w.counters[C_PAIRS] = 0u;
    w.counters[C_OVERFLOW] = 0u;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {  // k_cell_keys + k_bucket_count
    bool small = enabled(w, i) && w.moment[i].w <= p.largeThreshold;
    int4 c = cellOf(f3(w.pos[i]), p.cellSize);
    w.cell[i] = c;
    uint32_t k = small ? cellHash(c, p.tableMask) : sentinel;
    key[i] = k;
    if (k != sentinel) rank[i] = atomicAdd(&w.cellStart[k], 1u);
  }
  __syncthreads();
  {  // exclusive scan of the bucket counts: each thread owns T / threads consecutive buckets
    constexpr uint32_t PER = NOALLOC_TABLE / NOALLOC_THREADS;
    const uint32_t base = threadIdx.x * PER, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t v[PER], sum = 0;
    for (uint32_t k = 0; k < PER; k++) {
      v[k] = w.cellStart[base + k];
      sum += v[k];
    }
    uint32_t x = sum;
    for (uint32_t o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t k = 0; k < warp; k++) before += s_warp[k];
    uint32_t run = before + x - sum;
    for (uint32_t k = 0; k < PER; k++) {
      w.cellStart[base + k] = run;
      w.cellEnd[base + k] = run + v[k];
      run += v[k];
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {  // k_bucket_scatter
    uint32_t k = key[i];
    if (k == sentinel) continue;
    uint32_t slot = w.cellStart[k] + rank[i];
    float4 pi = w.pos[i];
    w.sortedPR[slot] = make_float4(pi.x, pi.y, pi.z, w.moment[i].w);
    int4 c = w.cell[i];
    w.sortedCell[slot] = make_int4(c.x, c.y, c.z, (int)(i | (w.size[i].w > 0.0f ? 0x80000000u : 0u)));
    float3 a = aabbOf(w, i);
    w.sortedAabb[slot] = make_float4(a.x, a.y, a.z, 0.0f);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {  // the walk of k_find_pairs, body i
    if (!enabled(w, i)) continue;
    const bool dyn = w.size[i].w > 0.0f;
    const Probe P = probeOf(w, i);
    if (w.moment[i].w <= p.largeThreshold) {
      const int4 c = w.cell[i];
      for (int o = 0; o < 14; o++) walkCell(w, p, P, dyn, c, o);
      smallAgainstLarge(w, p, P, dyn);
    } else if (dyn) {
      largeAgainstLarge(w, p, P);
    }
  }
}

}  // namespace avbd

extern "C" int avbd_find_pairs_noalloc(const avbd_body* bodies, uint32_t n, const uint32_t* groups_mask, uint32_t* pairs_ab, uint32_t cap,
                                       uint32_t* count, void* stream) {
  using namespace avbd;
  using L = NoAllocLayout;
  if (count) *count = 0;
  if ((n && !bodies) || (cap && !pairs_ab) || !count) return AVBD_ERR_INVALID;
  if (n > NOALLOC_MAX_BODIES) return AVBD_ERR_CAPACITY;  // at most AVBD_NOALLOC_MAX_BODIES bodies
  if (!bodyProblem(bodies, n).empty()) return AVBD_ERR_INVALID;
  // boxes, spheres and sails only: this call has no hull buffer to read a hull's shape code against
  for (uint32_t i = 0; i < n; i++)
    if (bodies[i].shape != 0.0f && bodies[i].shape != 1.0f && bodies[i].shape != 2.0f) return AVBD_ERR_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return AVBD_ERR_NO_DEVICE;
  // The scratch array's address on the current device, looked up on every call (no allocation): in
  // host code g_noalloc_scratch names a host-side stand-in, and a context torn down and made again
  // (cudaDeviceReset) may load the module at another address, so no address is kept between calls.
  // The first call on a device loads the module there; make it before any stream capture.
  void* scratch = nullptr;
  if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess || !scratch) return AVBD_ERR_CUDA;
  unsigned char* base = static_cast<unsigned char*>(scratch);
  if (n == 0) return AVBD_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the broadphase configuration of uploadStatics (solver.ts:1263-1318), from the radii
  std::vector<double> radii(n);
  for (uint32_t i = 0; i < n; i++) radii[i] = bodies[i].radius;
  const double maxSmall = largestSmall(radii);
  const float threshold = float(largeThreshold(radii));
  std::vector<uint32_t> large;
  uint32_t anyDynamicLarge = 0;
  for (uint32_t i = 0; i < n; i++)
    if (bodies[i].radius > threshold) {
      large.push_back(i);
      if (bodies[i].mass > 0.0f) anyDynamicLarge = 1;
    }
  DWorld w{};
  w.pos = reinterpret_cast<float4*>(base + L::POS);
  w.rot = reinterpret_cast<float4*>(base + L::ROT);
  w.ipos = reinterpret_cast<float4*>(base + L::IPOS);
  w.size = reinterpret_cast<float4*>(base + L::SIZE);
  w.moment = reinterpret_cast<float4*>(base + L::MOMENT);
  w.avel = reinterpret_cast<float4*>(base + L::AVEL);
  w.filters = reinterpret_cast<uint2*>(base + L::FILTERS);
  w.cell = reinterpret_cast<int4*>(base + L::CELL);
  w.cellStart = reinterpret_cast<uint32_t*>(base + L::START);
  w.cellEnd = reinterpret_cast<uint32_t*>(base + L::END);
  w.sortedPR = reinterpret_cast<float4*>(base + L::SPR);
  w.sortedCell = reinterpret_cast<int4*>(base + L::SCELL);
  w.sortedAabb = reinterpret_cast<float4*>(base + L::SAABB);
  w.large = reinterpret_cast<uint32_t*>(base + L::LARGE);
  w.pairs = reinterpret_cast<uint2*>(base + L::PAIRS);
  w.counters = reinterpret_cast<uint32_t*>(base + L::COUNTERS);
  StepParams p{};
  p.n = n;
  p.largeThreshold = threshold;
  p.cellSize = float(std::max(2.0 * maxSmall * (1 + 1e-4), 1e-3));
  p.tableMask = NOALLOC_TABLE - 1u;
  p.nLarge = uint32_t(large.size());
  p.anyDynamicLarge = anyDynamicLarge;
  p.pairCap = NOALLOC_MAX_PAIRS;
  p.nNoCollide = 0;
  // the record fields the pair rule reads, strided out of the host records
  const size_t fieldIndex[6] = {0, 1, 2, 4, 5, 9};
  float4* fields[6] = {w.pos, w.rot, w.ipos, w.size, w.moment, w.avel};
  for (int f = 0; f < 6; f++)
    if (cudaMemcpy2DAsync(fields[f], sizeof(float4), reinterpret_cast<const char*>(bodies) + fieldIndex[f] * sizeof(float4), sizeof(avbd_body), sizeof(float4),
                          n, cudaMemcpyHostToDevice, s) != cudaSuccess)
      return AVBD_ERR_CUDA;
  cudaError_t e = groups_mask ? cudaMemcpyAsync(w.filters, groups_mask, size_t(n) * sizeof(uint2), cudaMemcpyHostToDevice, s)
                              : cudaMemsetAsync(w.filters, 0xff, size_t(n) * sizeof(uint2), s);
  if (e != cudaSuccess) return AVBD_ERR_CUDA;
  if (!large.empty() && cudaMemcpyAsync(w.large, large.data(), large.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return AVBD_ERR_CUDA;
  k_find_pairs_noalloc<<<1, NOALLOC_THREADS, 0, s>>>(w, p, reinterpret_cast<uint32_t*>(base + L::KEY), reinterpret_cast<uint32_t*>(base + L::RANK));
  if (cudaGetLastError() != cudaSuccess) return AVBD_ERR_CUDA;
  uint32_t found = 0;
  if (cudaMemcpyAsync(&found, w.counters + C_PAIRS, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return AVBD_ERR_CUDA;
  // the host sources above must outlive their copies, and the count is needed below
  if (cudaStreamSynchronize(s) != cudaSuccess) return AVBD_ERR_CUDA;
  *count = found;
  const uint32_t k = std::min(std::min(found, cap), NOALLOC_MAX_PAIRS);
  if (k && (cudaMemcpyAsync(pairs_ab, w.pairs, size_t(k) * sizeof(uint2), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess))
    return AVBD_ERR_CUDA;
  return found > NOALLOC_MAX_PAIRS || found > cap ? AVBD_ERR_CAPACITY : AVBD_OK;
}
