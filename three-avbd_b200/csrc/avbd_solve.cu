// Topology and solve of the B200 AVBD step: one cooperative persistent kernel.
//
//   adjacency (degree, scan, fill, per-body sort)        avbd2d/gpu/wgsl-topology.ts:63-153
//   Jones-Plassmann colouring (compact, mark, rounds)    wgsl-topology.ts:155-262
//   colour buckets, stable by body index                 wgsl-topology.ts:264-328
//   incidence list: per colour, per body, per row         (new: constraints sorted by colour and body)
//   joint and body warm starts                           avbd3d/gpu/wgsl-solve.ts:235-335
//   iterations x colours: primal + fused dual            wgsl-solve.ts:337-670
//   velocities                                           wgsl-solve.ts:672-684
//
// Phases are separated by a grid barrier whose every wait is bounded (a clock budget, then an
// error bit in the counters and an orderly exit of every block); the launch is cooperative, so
// every block is resident and the barrier completes.
//
// The dual update of a constraint is fused into the primal pass of the colour that solves its
// last dynamic body (the "owner" bit of its incidence): once both its bodies have moved in this
// iteration nothing reads its multipliers until the next iteration, so updating it there equals
// the reference's separate dual pass after every colour (solver.ts:2246-2259), with one grid
// barrier per iteration fewer and the contact rows still in cache.
#include "avbd_device.cuh"

namespace avbd {

constexpr int SOLVE_THREADS = 256;
constexpr long long BARRIER_CYCLES = 4000000000LL;  // about two seconds of SM clock

__device__ __forceinline__ uint32_t ldv(const uint32_t* p) { return *(const volatile uint32_t*)p; }

// Grid barrier (arrive counter + generation), bounded wait. Returns false when the step must stop.
__device__ bool grid_sync(uint32_t* bar, uint32_t* counters) {
  __shared__ uint32_t s_abort;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t gen = ldv(bar + 1);
    uint32_t ab = 0;
    __threadfence();
    uint32_t arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long t0 = clock64();
      while (ldv(bar + 1) == gen) {
        if (ldv(&counters[C_ERROR]) & ERR_BARRIER_TIMEOUT) { ab = 1; break; }
        if (clock64() - t0 > BARRIER_CYCLES) {
          atomicOr(&counters[C_ERROR], ERR_BARRIER_TIMEOUT);
          ab = 1;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_abort = ab;
  }
  __syncthreads();
  return s_abort == 0;
}

// Exclusive scan of one block's range [lo, hi) in place; returns the range total (all threads).
__device__ uint32_t block_scan_range(uint32_t* data, uint32_t lo, uint32_t hi) {
  __shared__ uint32_t warpSums[SOLVE_THREADS / 32];
  __shared__ uint32_t s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t base = lo; base < hi; base += SOLVE_THREADS) {
    uint32_t i = base + threadIdx.x;
    uint32_t v = i < hi ? data[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[warp] = x;
    __syncthreads();
    uint32_t before = 0, total = 0;
#pragma unroll
    for (int k = 0; k < SOLVE_THREADS / 32; k++) {
      uint32_t s = warpSums[k];
      if (k < warp) before += s;
      total += s;
    }
    uint32_t carry = s_carry;
    if (i < hi) data[i] = carry + before + x - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + total;
    __syncthreads();
  }
  return s_carry;
}

// Exclusive scan of data[0, len) across the grid; scratch[gridDim.x] receives the total.
__device__ bool grid_scan(uint32_t* data, uint32_t len, uint32_t* scratch, uint32_t* bar, uint32_t* counters) {
  uint32_t chunk = (len + gridDim.x - 1) / gridDim.x;
  uint32_t lo = min(len, blockIdx.x * chunk), hi = min(len, lo + chunk);
  uint32_t total = block_scan_range(data, lo, hi);
  if (threadIdx.x == 0) scratch[blockIdx.x] = total;
  if (!grid_sync(bar, counters)) return false;
  if (blockIdx.x == 0) {
    uint32_t all = block_scan_range(scratch, 0, gridDim.x);
    if (threadIdx.x == 0) scratch[gridDim.x] = all;
  }
  if (!grid_sync(bar, counters)) return false;
  uint32_t add = scratch[blockIdx.x];
  for (uint32_t i = lo + threadIdx.x; i < hi; i += SOLVE_THREADS) data[i] += add;
  return grid_sync(bar, counters);
}

// --- constraint endpoints and activity (gpu/layout.ts:356-369) ----------------------------------------
__device__ inline bool enabledBody(const DWorld& w, uint32_t i) { return ((uint32_t)w.ipos[i].w & 2u) == 0u; }
__device__ inline bool dynBody(const DWorld& w, int i) { return i >= 0 && w.size[i].w > 0.0f && enabledBody(w, (uint32_t)i); }

// Endpoints of constraint c (joints first, then contact pair slots); false when it does not act.
__device__ inline bool endpoints(const DWorld& w, const StepParams& p, uint32_t c, int& ea, int& eb, uint32_t& count) {
  if (c < p.nj) {
    int4 in = w.jinfo[c];
    if (in.x == (int)T_NONE) return false;
    float4 pl = w.joint[c * JOINT_VEC4 + J_PEN_LIN], pa = w.joint[c * JOINT_VEC4 + J_PEN_ANG];
    if (pl.w == 0.0f && pa.w == 0.0f) return false;
    if (in.y >= 0 && !enabledBody(w, (uint32_t)in.y)) return false;
    if (!enabledBody(w, (uint32_t)in.z)) return false;
    ea = in.y;
    eb = in.z;
    count = 1;
    return true;
  }
  uint4 ids = w.mIds[p.cur][c - p.nj];
  count = ids.w & 15u;
  if (count == 0u) return false;
  ea = (int)ids.x;
  eb = (int)ids.y;
  return true;
}

// Summation order of a body's constraints (wgsl-topology.ts:116-125): joints by slot, then contact
// pairs by (other body + 2, first point's feature key).
__device__ inline unsigned long long adjKey(const DWorld& w, const StepParams& p, uint32_t b, uint32_t c) {
  if (c < p.nj) return (unsigned long long)c;
  uint4 ids = w.mIds[p.cur][c - p.nj];
  uint32_t other = ids.x == b ? ids.y : ids.x;
  uint32_t feature = __float_as_uint(w.cRA[p.cur][ids.z].w) & ~STICK_BIT;
  return ((unsigned long long)(other + 2u) << 32) | feature;
}

// --- Jones-Plassmann (wgsl-topology.ts:157-262) ---------------------------------------------------------
__device__ inline uint32_t priority(uint32_t i) { return hash32(i + 0x9e3779b9u); }
__device__ inline bool beats(uint32_t i, uint32_t j) {
  uint32_t pi = priority(i), pj = priority(j);
  return pi > pj || (pi == pj && i > j);
}
__device__ inline int neighbour(const DWorld& w, const StepParams& p, uint32_t b, uint32_t e) {
  uint32_t c = w.adjList[e];
  int ea, eb;
  uint32_t cnt;
  if (c < p.nj) {
    int4 in = w.jinfo[c];
    ea = in.y;
    eb = in.z;
  } else {
    uint4 ids = w.mIds[p.cur][c - p.nj];
    ea = (int)ids.x;
    eb = (int)ids.y;
  }
  (void)cnt;
  int other = ea == (int)b ? eb : ea;
  return dynBody(w, other) ? other : -1;
}
__device__ inline uint32_t smallestFree(const DWorld& w, const StepParams& p, uint32_t b, const uint32_t* src, bool skipPending) {
  uint32_t lo = 0, hi = 0;
  for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1]; e++) {
    int j = neighbour(w, p, b, e);
    if (j < 0) continue;
    uint32_t s = src[j];
    if (skipPending && (s & PENDING)) continue;
    uint32_t col = s & 0xffu;
    if (col == NO_COLOR) continue;
    if (col < 32u) lo |= 1u << col;
    else hi |= 1u << (col - 32u);
  }
  if (~lo != 0u) return __ffs(~lo) - 1;
  if (~hi != 0u) return 32u + __ffs(~hi) - 1;
  return MAX_COLORS;
}

// --- stable bucket scatter of one block's chunk (64 colours) ---------------------------------------------
// Bodies of [lo, hi) go to colorBodies in index order within each colour, at the block's scanned
// per-colour offsets colorHist[c * gridDim.x + blockIdx.x].
__device__ void color_scatter_chunk(const DWorld& w, uint32_t lo, uint32_t hi) {
  __shared__ uint32_t running[MAX_COLORS];
  __shared__ uint32_t warpCount[SOLVE_THREADS / 32][MAX_COLORS];
  __shared__ uint32_t tileCount[MAX_COLORS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < MAX_COLORS) running[threadIdx.x] = w.colorHist[threadIdx.x * gridDim.x + blockIdx.x];
  for (uint32_t base = lo; base < hi; base += SOLVE_THREADS) {
    for (int k = threadIdx.x; k < (SOLVE_THREADS / 32) * MAX_COLORS; k += SOLVE_THREADS) (&warpCount[0][0])[k] = 0;
    __syncthreads();
    uint32_t b = base + threadIdx.x;
    bool live = b < hi && (w.colorB[b] != 0xffffffffu);
    uint32_t col = live ? (w.colorA[b] & 0xffu) : 0xffffffffu;
    uint32_t peers = __match_any_sync(0xffffffffu, col);
    uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (live && rank == 0) warpCount[warp][col] = __popc(peers);
    __syncthreads();
    if (threadIdx.x < MAX_COLORS) {
      uint32_t s = 0;
      for (int k = 0; k < SOLVE_THREADS / 32; k++) {
        uint32_t c = warpCount[k][threadIdx.x];
        warpCount[k][threadIdx.x] = s;
        s += c;
      }
      tileCount[threadIdx.x] = s;
    }
    __syncthreads();
    if (live) w.colorBodies[running[col] + warpCount[warp][col] + rank] = b;
    __syncthreads();
    if (threadIdx.x < MAX_COLORS) running[threadIdx.x] += tileCount[threadIdx.x];
    __syncthreads();
  }
}

// --- body poses -----------------------------------------------------------------------------------------
struct Pose {
  float3 x, x0, dLin, dAng;
  float4 q, q0;
};
__device__ inline Pose loadPose(const DWorld& w, uint32_t i) {
  Pose P;
  float4 p = w.pos[i], q = w.rot[i], p0 = w.ipos[i], q0 = w.irot[i];
  P.x = f3(p);
  P.q = q;
  P.x0 = f3(p0);
  P.q0 = q0;
  P.dLin = P.x - P.x0;
  P.dAng = qsub(q, q0);
  return P;
}
__device__ inline void setPose(Pose& P, float3 x, float4 q) {
  P.x = x;
  P.q = q;
  P.dLin = x - P.x0;
  P.dAng = qsub(q, P.q0);
}

// The Newton system of one body (wgsl-solve.ts:56-75): lin and ang symmetric (upper triangles),
// cross with row = angular index and column = linear index, and the gradient.
struct Acc {
  float v[27];  // lin 00 01 02 11 12 22 | ang 00 01 02 11 12 22 | cross 9 | rLin 3 | rAng 3
};
__device__ inline void accZero(Acc& a) {
#pragma unroll
  for (int k = 0; k < 27; k++) a.v[k] = 0.0f;
}
__device__ inline void addRow(Acc& A, float3 l, float3 a, float k, float f) {
  float3 kl = l * k, ka = a * k;
  A.v[0] += kl.x * l.x; A.v[1] += kl.x * l.y; A.v[2] += kl.x * l.z; A.v[3] += kl.y * l.y; A.v[4] += kl.y * l.z; A.v[5] += kl.z * l.z;
  A.v[6] += ka.x * a.x; A.v[7] += ka.x * a.y; A.v[8] += ka.x * a.z; A.v[9] += ka.y * a.y; A.v[10] += ka.y * a.z; A.v[11] += ka.z * a.z;
  A.v[12] += ka.x * l.x; A.v[13] += ka.x * l.y; A.v[14] += ka.x * l.z;
  A.v[15] += ka.y * l.x; A.v[16] += ka.y * l.y; A.v[17] += ka.y * l.z;
  A.v[18] += ka.z * l.x; A.v[19] += ka.z * l.y; A.v[20] += ka.z * l.z;
  A.v[21] += l.x * f; A.v[22] += l.y * f; A.v[23] += l.z * f;
  A.v[24] += a.x * f; A.v[25] += a.y * f; A.v[26] += a.z * f;
}

// --- contacts (wgsl-solve.ts:169-231) ----------------------------------------------------------------------
struct ContactEval {
  float3 rAW, rBW, C, F;
  float frictionScale, bounds;
};
__device__ inline void evalContact(float4 ra, float4 rb, float4 pen, float4 lam, float3 n, float3 t1, float3 t2, float friction, const Pose& A,
                                   const Pose& B, float alpha, ContactEval& e) {
  uint32_t key = __float_as_uint(ra.w);
  bool rolling = (key & ~STICK_BIT) == SPHERE_FEATURE;
  e.rAW = qrotate(rolling ? A.q0 : A.q, f3(ra));
  e.rBW = qrotate(rolling ? B.q0 : B.q, f3(rb));
  float keep = 1.0f - alpha;
  e.C.x = rb.w * keep + dot3(n, A.dLin) - dot3(n, B.dLin) + dot3(cross3(e.rAW, n), A.dAng) + dot3(cross3(e.rBW, -n), B.dAng);
  e.C.y = pen.w * keep + dot3(t1, A.dLin) - dot3(t1, B.dLin) + dot3(cross3(e.rAW, t1), A.dAng) + dot3(cross3(e.rBW, -t1), B.dAng);
  e.C.z = lam.w * keep + dot3(t2, A.dLin) - dot3(t2, B.dLin) + dot3(cross3(e.rAW, t2), A.dAng) + dot3(cross3(e.rBW, -t2), B.dAng);
  float3 F = make_float3(pen.x * e.C.x + lam.x, pen.y * e.C.y + lam.y, pen.z * e.C.z + lam.z);
  F.x = fminf(F.x, 0.0f);
  e.bounds = fabsf(F.x) * friction;
  e.frictionScale = sqrtf(F.y * F.y + F.z * F.z);
  if (e.frictionScale > e.bounds && e.frictionScale > 0.0f) {
    float s = e.bounds / e.frictionScale;
    F.y = F.y * s;
    F.z = F.z * s;
  }
  e.F = F;
}

// --- joints and springs (wgsl-solve.ts:79-165, 562-635) --------------------------------------------------
struct Bodies2 {  // poses of a joint's bodies; `own` is the body being solved (its pose in registers)
  const DWorld* w;
  uint32_t own;
  const Pose* ownPose;
  __device__ inline float3 pos(int i) const { return (uint32_t)i == own ? ownPose->x : f3(w->pos[i]); }
  __device__ inline float4 rot(int i) const { return (uint32_t)i == own ? ownPose->q : w->rot[i]; }
};
__device__ inline float3 jointLinC(const float4* k, int a, int b, const Bodies2& B) {
  float3 anchorA = a < 0 ? f3(k[J_RA]) : qrotate(B.rot(a), f3(k[J_RA])) + B.pos(a);
  return anchorA - (qrotate(B.rot(b), f3(k[J_RB])) + B.pos(b));
}
__device__ inline float3 jointAngC(const float4* k, int a, int b, const Bodies2& B) {
  float4 qb = B.rot(b);
  float4 ra = a < 0 ? make_float4(0.0f, 0.0f, 0.0f, 1.0f) : B.rot(a);
  float l = ((qb.x * qb.x + qb.y * qb.y) + qb.z * qb.z) + qb.w * qb.w;
  float4 inv = make_float4(-qb.x / l, -qb.y / l, -qb.z / l, qb.w / l);
  float4 d = qmul(qmul(ra, k[J_REST]), inv);
  if (d.w < 0.0f) d = make_float4(-d.x, -d.y, -d.z, -d.w);
  float s = 2.0f * k[J_LAM_ANG].w;
  return make_float3(d.x * s, d.y * s, d.z * s);
}
__device__ inline void loadJoint(const DWorld& w, uint32_t j, float4* k) {
#pragma unroll
  for (int i = 0; i < JOINT_VEC4; i++) k[i] = w.joint[j * JOINT_VEC4 + i];
}

__device__ void addJoint(Acc& acc, const DWorld& w, uint32_t j, float alpha, uint32_t i, const Bodies2& B) {
  int4 info = w.jinfo[j];
  int a = info.y, b = info.z;
  float4 k[JOINT_VEC4];
  loadJoint(w, j, k);
  bool isA = (int)i == a;
  float sg = isA ? 1.0f : -1.0f;
  if ((uint32_t)info.x == T_SPRING) {
    float3 rAW = qrotate(B.rot(a), f3(k[J_RA]));
    float3 rBW = qrotate(B.rot(b), f3(k[J_RB]));
    float3 d = (rAW + B.pos(a)) - (rBW + B.pos(b));
    float len = len3(d);
    if (len <= 1.0e-6f) return;
    float3 n = d / len;
    float stiffness = k[J_PEN_LIN].w;
    float3 r = isA ? rAW : rBW;
    addRow(acc, n * sg, cross3(r, n) * sg, stiffness, stiffness * (len - k[J_RA].w));
    return;
  }
  float3 penLin = f3(k[J_PEN_LIN]), penAng = f3(k[J_PEN_ANG]);
  if (dot3(penLin, penLin) > 0.0f) {
    float3 C = jointLinC(k, a, b, B);
    if (k[J_PEN_LIN].w >= HARD) C = C - f3(k[J_C0_LIN]) * alpha;
    float3 F = penLin * C + f3(k[J_LAM_LIN]);
    float3 r = isA ? qrotate(B.rot(a), f3(k[J_RA])) : -qrotate(B.rot(b), f3(k[J_RB]));
    float3 v = -r;
    addRow(acc, make_float3(sg, 0.0f, 0.0f), make_float3(0.0f, -v.z, v.y), penLin.x, F.x);
    addRow(acc, make_float3(0.0f, sg, 0.0f), make_float3(v.z, 0.0f, -v.x), penLin.y, F.y);
    addRow(acc, make_float3(0.0f, 0.0f, sg), make_float3(-v.y, v.x, 0.0f), penLin.z, F.z);
    float rf = dot3(r, F);
    acc.v[6] += len3(r * F.x - make_float3(rf, 0.0f, 0.0f));
    acc.v[9] += len3(r * F.y - make_float3(0.0f, rf, 0.0f));
    acc.v[11] += len3(r * F.z - make_float3(0.0f, 0.0f, rf));
  }
  if (dot3(penAng, penAng) > 0.0f) {
    float3 C = jointAngC(k, a, b, B);
    if (k[J_PEN_ANG].w >= HARD) C = C - f3(k[J_C0_ANG]) * alpha;
    float3 F = penAng * C + f3(k[J_LAM_ANG]);
    float s = sg * k[J_LAM_ANG].w;
    float3 z = make_float3(0.0f, 0.0f, 0.0f);
    addRow(acc, z, make_float3(s, 0.0f, 0.0f), penAng.x, F.x);
    addRow(acc, z, make_float3(0.0f, s, 0.0f), penAng.y, F.y);
    addRow(acc, z, make_float3(0.0f, 0.0f, s), penAng.z, F.z);
  }
}

__device__ void dualJoint(const DWorld& w, const StepParams& p, uint32_t j, const Bodies2& B) {
  int4 info = w.jinfo[j];
  if ((uint32_t)info.x != T_JOINT) return;
  int a = info.y, b = info.z;
  float4 k[JOINT_VEC4];
  loadJoint(w, j, k);
  const float alpha = p.alpha;
  float4 penLin = k[J_PEN_LIN], penAng = k[J_PEN_ANG], lamLin = k[J_LAM_LIN], lamAng = k[J_LAM_ANG];
  if (dot3(f3(penLin), f3(penLin)) > 0.0f) {
    float3 C = jointLinC(k, a, b, B);
    if (penLin.w >= HARD) C = C - f3(k[J_C0_LIN]) * alpha;
    if (penLin.w >= HARD) {
      float3 l = f3(penLin) * C + f3(lamLin);
      lamLin = make_float4(l.x, l.y, l.z, lamLin.w);
    }
    float cap = fminf(penLin.w, PENALTY_MAX);
    float3 pl = f3(penLin) + abs3(C) * p.betaLin;
    penLin = make_float4(fminf(pl.x, cap), fminf(pl.y, cap), fminf(pl.z, cap), penLin.w);
  }
  float frac = lamLin.w;
  float limit = fabsf(frac);
  bool yielded = false;
  if (dot3(f3(penAng), f3(penAng)) > 0.0f) {
    float3 C = jointAngC(k, a, b, B);
    if (penAng.w >= HARD) C = C - f3(k[J_C0_ANG]) * alpha;
    if (penAng.w >= HARD) {
      float3 l = f3(penAng) * C + f3(lamAng);
      lamAng = make_float4(l.x, l.y, l.z, lamAng.w);
      float yieldForce = k[J_C0_ANG].w;
      if (yieldForce < BIG) {
        float force = len3(f3(lamAng));
        if (force > yieldForce && !(limit < BIG && force > limit)) {
          float3 l2 = f3(lamAng) * (yieldForce / force);
          lamAng = make_float4(l2.x, l2.y, l2.z, lamAng.w);
          yielded = true;
        }
      }
    }
    if (!yielded) {
      float cap = fminf(penAng.w, PENALTY_MAX);
      float3 pa = f3(penAng) + abs3(C) * p.betaAng;
      penAng = make_float4(fminf(pa.x, cap), fminf(pa.y, cap), fminf(pa.z, cap), penAng.w);
    }
  }
  float4 rest = k[J_REST];
  bool bentOff = false;
  if (yielded) {
    float4 ra = a < 0 ? make_float4(0.0f, 0.0f, 0.0f, 1.0f) : B.rot(a);
    float4 q = qmul(qconj(ra), B.rot(b));
    float l = sqrtf(((q.x * q.x + q.y * q.y) + q.z * q.z) + q.w * q.w);
    rest = make_float4(q.x / l, q.y / l, q.z / l, q.w / l);
    if (k[J_RB].w < BIG) {
      float4 d = qmul(qconj(k[J_REST_START]), rest);
      bentOff = 2.0f * atan2f(sqrtf(d.x * d.x + d.y * d.y + d.z * d.z), fabsf(d.w)) > k[J_RB].w;
    }
  }
  bool linear = frac < 0.0f && dot3(f3(lamLin), f3(lamLin)) > limit * limit;
  if ((limit < BIG && (dot3(f3(lamAng), f3(lamAng)) > limit * limit || linear)) || bentOff) {
    penLin = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    penAng = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    lamLin = make_float4(0.0f, 0.0f, 0.0f, frac);
    lamAng = make_float4(0.0f, 0.0f, 0.0f, lamAng.w);
  }
  float4* out = w.joint + j * JOINT_VEC4;
  out[J_PEN_LIN] = penLin;
  out[J_PEN_ANG] = penAng;
  out[J_LAM_LIN] = lamLin;
  out[J_LAM_ANG] = lamAng;
  if (yielded) {
    out[J_REST] = rest;
    out[J_C0_ANG] = make_float4(0.0f, 0.0f, 0.0f, k[J_C0_ANG].w);
  }
}

// --- the 6x6 LDLT with pivot floor and the pose update (wgsl-solve.ts:504-558) ------------------------------
__device__ inline void finishBody(const Acc& acc, float3& x, float4& q) {
  const float* v = acc.v;
  float A11 = v[0], A21 = v[1], A22 = v[3], A31 = v[2], A32 = v[4], A33 = v[5];
  float A41 = v[12], A42 = v[13], A43 = v[14], A44 = v[6];
  float A51 = v[15], A52 = v[16], A53 = v[17], A54 = v[7], A55 = v[9];
  float A61 = v[18], A62 = v[19], A63 = v[20], A64 = v[8], A65 = v[10], A66 = v[11];
  float D1 = A11;
  float L21 = A21 / D1, L31 = A31 / D1, L41 = A41 / D1, L51 = A51 / D1, L61 = A61 / D1;
  float D2 = fmaxf(A22 - L21 * L21 * D1, A22 * PIVOT_FLOOR);
  float L32 = (A32 - L21 * L31 * D1) / D2;
  float L42 = (A42 - L21 * L41 * D1) / D2;
  float L52 = (A52 - L21 * L51 * D1) / D2;
  float L62 = (A62 - L21 * L61 * D1) / D2;
  float D3 = fmaxf(A33 - (L31 * L31 * D1 + L32 * L32 * D2), A33 * PIVOT_FLOOR);
  float L43 = (A43 - L31 * L41 * D1 - L32 * L42 * D2) / D3;
  float L53 = (A53 - L31 * L51 * D1 - L32 * L52 * D2) / D3;
  float L63 = (A63 - L31 * L61 * D1 - L32 * L62 * D2) / D3;
  float D4 = fmaxf(A44 - (L41 * L41 * D1 + L42 * L42 * D2 + L43 * L43 * D3), A44 * PIVOT_FLOOR);
  float L54 = (A54 - L41 * L51 * D1 - L42 * L52 * D2 - L43 * L53 * D3) / D4;
  float L64 = (A64 - L41 * L61 * D1 - L42 * L62 * D2 - L43 * L63 * D3) / D4;
  float D5 = fmaxf(A55 - (L51 * L51 * D1 + L52 * L52 * D2 + L53 * L53 * D3 + L54 * L54 * D4), A55 * PIVOT_FLOOR);
  float L65 = (A65 - L51 * L61 * D1 - L52 * L62 * D2 - L53 * L63 * D3 - L54 * L64 * D4) / D5;
  float D6 = fmaxf(A66 - (L61 * L61 * D1 + L62 * L62 * D2 + L63 * L63 * D3 + L64 * L64 * D4 + L65 * L65 * D5), A66 * PIVOT_FLOOR);
  float y1 = v[21];
  float y2 = v[22] - L21 * y1;
  float y3 = v[23] - L31 * y1 - L32 * y2;
  float y4 = v[24] - L41 * y1 - L42 * y2 - L43 * y3;
  float y5 = v[25] - L51 * y1 - L52 * y2 - L53 * y3 - L54 * y4;
  float y6 = v[26] - L61 * y1 - L62 * y2 - L63 * y3 - L64 * y4 - L65 * y5;
  float w3 = y6 / D6;
  float w2 = y5 / D5 - L65 * w3;
  float w1 = y4 / D4 - L54 * w2 - L64 * w3;
  float v3 = y3 / D3 - L43 * w1 - L53 * w2 - L63 * w3;
  float v2 = y2 / D2 - L32 * v3 - L42 * w1 - L52 * w2 - L62 * w3;
  float v1 = y1 / D1 - L21 * v2 - L31 * v3 - L41 * w1 - L51 * w2 - L61 * w3;
  x = make_float3(x.x - v1, x.y - v2, x.z - v3);
  q = qadd(q, make_float3(-w1, -w2, -w3));
}

// One lane's share of one incidence: a joint, or a contact point of a pair.
__device__ inline void accumulateIncidence(Acc& acc, const DWorld& w, const StepParams& p, uint32_t id, uint32_t i, const Pose& own) {
  if (id < p.nj) {
    Bodies2 B{&w, i, &own};
    addJoint(acc, w, id, p.alpha, i, B);
    return;
  }
  uint32_t cs = id - p.nj;
  uint32_t m = cs / MAX_CONTACTS;
  uint4 ids = w.mIds[p.cur][m];
  float4 geo = w.mGeo[p.cur][m];
  bool isA = ids.x == i;
  Pose other = loadPose(w, isA ? ids.y : ids.x);
  const Pose& A = isA ? own : other;
  const Pose& B = isA ? other : own;
  float3 n = f3(geo), t1, t2;
  orthonormal(n, t1, t2);
  ContactEval e;
  evalContact(w.cRA[p.cur][cs], w.cRB[p.cur][cs], w.cPen[p.cur][cs], w.cLam[p.cur][cs], n, t1, t2, geo.w, A, B, p.alpha, e);
  float4 pen = w.cPen[p.cur][cs];
  float sg = isA ? 1.0f : -1.0f;
  float3 r = isA ? e.rAW : e.rBW;
  float3 l0 = n * sg, l1 = t1 * sg, l2 = t2 * sg;
  addRow(acc, l0, cross3(r, l0), pen.x, e.F.x);
  addRow(acc, l1, cross3(r, l1), pen.y, e.F.y);
  addRow(acc, l2, cross3(r, l2), pen.z, e.F.z);
}

// The dual update of one owned incidence (wgsl-solve.ts:562-662)
__device__ inline void dualIncidence(const DWorld& w, const StepParams& p, uint32_t id, uint32_t i, const Pose& own) {
  if (id < p.nj) {
    Bodies2 B{&w, i, &own};
    dualJoint(w, p, id, B);
    return;
  }
  uint32_t cs = id - p.nj;
  uint32_t m = cs / MAX_CONTACTS;
  uint4 ids = w.mIds[p.cur][m];
  float4 geo = w.mGeo[p.cur][m];
  bool isA = ids.x == i;
  Pose other = loadPose(w, isA ? ids.y : ids.x);
  const Pose& A = isA ? own : other;
  const Pose& B = isA ? other : own;
  float3 n = f3(geo), t1, t2;
  orthonormal(n, t1, t2);
  float4 ra = w.cRA[p.cur][cs], pen = w.cPen[p.cur][cs], lam = w.cLam[p.cur][cs];
  ContactEval e;
  evalContact(ra, w.cRB[p.cur][cs], pen, lam, n, t1, t2, geo.w, A, B, p.alpha, e);
  w.cLam[p.cur][cs] = make_float4(e.F.x, e.F.y, e.F.z, lam.w);
  if (e.F.x < 0.0f) pen.x = fminf(pen.x + p.betaLin * fabsf(e.C.x), PENALTY_MAX);
  if (e.frictionScale <= e.bounds) {
    pen.y = fminf(pen.y + p.betaLin * fabsf(e.C.y), PENALTY_MAX);
    pen.z = fminf(pen.z + p.betaLin * fabsf(e.C.z), PENALTY_MAX);
    bool stick = sqrtf(e.C.y * e.C.y + e.C.z * e.C.z) < STICK_THRESH;
    uint32_t key = __float_as_uint(ra.w);
    uint32_t nk = (key & ~STICK_BIT) | (stick ? STICK_BIT : 0u);
    if (nk != key) w.cRA[p.cur][cs].w = __uint_as_float(nk);
  }
  w.cPen[p.cur][cs] = pen;
}

// --- the kernel -----------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(SOLVE_THREADS, 2) k_topology_solve(DWorld w, StepParams p) {
  const uint32_t T = gridDim.x * blockDim.x;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = p.n, nj = p.nj;
  uint32_t* ctr = w.counters;
  uint32_t* bar = w.barrier;
#define GSYNC \
  if (!grid_sync(bar, ctr)) return;
  uint32_t npairs = ldv(&ctr[C_PAIRS]);
  if (npairs > p.pairCap) npairs = p.pairCap;
  const uint32_t ncons = nj + npairs;

  // A. degrees (adjStart[0, n] zeroed by the host)
  for (uint32_t c = tid; c < ncons; c += T) {
    int ea, eb;
    uint32_t cnt;
    if (!endpoints(w, p, c, ea, eb, cnt)) continue;
    if (dynBody(w, ea)) atomicAdd(&w.adjStart[ea], 1u);
    if (dynBody(w, eb)) atomicAdd(&w.adjStart[eb], 1u);
  }
  GSYNC
  if (!grid_scan(w.adjStart, n + 1, w.scanScratch, bar, ctr)) return;
  if (tid == 0) ctr[C_ADJ] = w.adjStart[n];
  // B. fill (adjFill zeroed by the host), then each body's list sorted into its summation order
  for (uint32_t c = tid; c < ncons; c += T) {
    int ea, eb;
    uint32_t cnt;
    if (!endpoints(w, p, c, ea, eb, cnt)) continue;
    if (dynBody(w, ea)) w.adjList[w.adjStart[ea] + atomicAdd(&w.adjFill[ea], 1u)] = c;
    if (dynBody(w, eb)) w.adjList[w.adjStart[eb] + atomicAdd(&w.adjFill[eb], 1u)] = c;
  }
  GSYNC
  for (uint32_t b = tid; b < n; b += T) {
    uint32_t lo = w.adjStart[b], hi = w.adjStart[b + 1];
    for (uint32_t i = lo + 1; i < hi; i++) {
      uint32_t id = w.adjList[i];
      unsigned long long key = adjKey(w, p, b, id);
      uint32_t j = i;
      while (j > lo) {
        uint32_t prevId = w.adjList[j - 1];
        if (!(key < adjKey(w, p, b, prevId))) break;
        w.adjList[j] = prevId;
        j--;
      }
      w.adjList[j] = id;
    }
  }
  GSYNC

  // C. colouring: state A persists between steps (colour | PENDING); B is scratch
  const uint32_t cap = p.colorCap;
  if (p.fixedColors) {
    for (uint32_t b = tid; b < n; b += T) w.colorA[b] = dynBody(w, (int)b) ? w.fixedColor[b] : NO_COLOR;
    if (tid == 0) ctr[C_ROUNDS] = 0;
    GSYNC
  } else {
    for (uint32_t b = tid; b < n; b += T) {  // compaction: A -> B
      if (!dynBody(w, (int)b)) {
        w.colorB[b] = NO_COLOR;
        continue;
      }
      uint32_t col = w.colorA[b] & 0xffu;
      if (col != NO_COLOR) {
        bool isMax = true;
        for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1] && isMax; e++) {
          int j = neighbour(w, p, b, e);
          if (j >= 0 && !beats(b, (uint32_t)j)) isMax = false;
        }
        if (isMax) col = min(col, smallestFree(w, p, b, w.colorA, false));
      }
      w.colorB[b] = col;
    }
    GSYNC
    {
      uint32_t pending = 0;
      for (uint32_t b = tid; b < n; b += T) {  // pending: B -> A
        if (!dynBody(w, (int)b)) {
          w.colorA[b] = NO_COLOR;
          continue;
        }
        uint32_t col = w.colorB[b] & 0xffu;
        bool pend = col == NO_COLOR;
        for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1] && !pend; e++) {
          int j = neighbour(w, p, b, e);
          if (j >= 0 && (w.colorB[j] & 0xffu) == col && beats((uint32_t)j, b)) pend = true;
        }
        w.colorA[b] = col | (pend ? PENDING : 0u);
        pending += pend ? 1u : 0u;
      }
      if (pending) atomicAdd(&ctr[C_PENDING], pending);
    }
    GSYNC
    uint32_t r = 0;
    while (r < MAX_ROUND_PAIRS / 2 && ldv(&ctr[C_PENDING + r]) > 0u) {
      for (int half = 0; half < 2; half++) {
        const uint32_t* src = half == 0 ? w.colorA : w.colorB;
        uint32_t* dst = half == 0 ? w.colorB : w.colorA;
        uint32_t pending = 0;
        for (uint32_t b = tid; b < n; b += T) {
          uint32_t s = src[b];
          if (!(s & PENDING)) {
            dst[b] = s;
            continue;
          }
          bool isMax = true;
          for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1] && isMax; e++) {
            int j = neighbour(w, p, b, e);
            if (j >= 0 && (src[j] & PENDING) && !beats(b, (uint32_t)j)) isMax = false;
          }
          uint32_t out = s;
          if (isMax) {
            uint32_t f = smallestFree(w, p, b, src, true);
            out = f >= cap ? ((cap - 1u) | PENDING) : f;
          }
          dst[b] = out;
          if (half == 1 && (out & PENDING) && dynBody(w, (int)b)) pending++;
        }
        if (half == 1 && pending) atomicAdd(&ctr[C_PENDING + r + 1], pending);
        GSYNC
      }
      r++;
    }
    if (tid == 0) ctr[C_ROUNDS] = 2u * r;
  }

  // D. final colours (NO_COLOR -> cap - 1, pending kept and counted) and per-block histograms over
  // contiguous chunks; colorB marks non-dynamic bodies (0xffffffff) for the scatter
  const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const uint32_t lo = min(n, blockIdx.x * chunk), hi = min(n, lo + chunk);
  {
    __shared__ uint32_t hist[MAX_COLORS];
    if (threadIdx.x < MAX_COLORS) hist[threadIdx.x] = 0;
    __syncthreads();
    uint32_t clashes = 0, maxc = 0;
    for (uint32_t b = lo + threadIdx.x; b < hi; b += SOLVE_THREADS) {
      if (!dynBody(w, (int)b)) {
        w.colorB[b] = 0xffffffffu;
        continue;
      }
      uint32_t s = w.colorA[b];
      uint32_t col = s & 0xffu;
      if (s & PENDING) clashes++;
      if (col == NO_COLOR || col >= (uint32_t)MAX_COLORS) col = cap - 1u;
      w.colorA[b] = col | (s & PENDING);
      w.colorB[b] = 0;
      atomicAdd(&hist[col], 1u);
      maxc = max(maxc, col + 1u);
    }
    if (clashes) atomicAdd(&ctr[C_CLASHES], clashes);
    if (maxc) atomicMax(&ctr[C_COLORS], maxc);
    __syncthreads();
    if (threadIdx.x < MAX_COLORS) w.colorHist[threadIdx.x * gridDim.x + blockIdx.x] = hist[threadIdx.x];
  }
  GSYNC
  if (blockIdx.x == 0) {
    uint32_t total = block_scan_range(w.colorHist, 0, MAX_COLORS * gridDim.x);
    __syncthreads();
    if (threadIdx.x < MAX_COLORS) w.colorStart[threadIdx.x] = w.colorHist[threadIdx.x * gridDim.x];
    if (threadIdx.x == 0) w.colorStart[MAX_COLORS] = total;
  }
  GSYNC
  color_scatter_chunk(w, lo, hi);
  GSYNC

  // E. incidence list: for each colour position s (body b = colorBodies[s]) its rows in order,
  // joints as one entry, contact pairs as one entry per point; OWNER_BIT where b is the last of the
  // constraint's dynamic bodies to move in an iteration
  const uint32_t numDyn = ldv(&w.colorStart[MAX_COLORS]);
  const uint32_t numColors = ldv(&ctr[C_COLORS]);
  for (uint32_t s = tid; s < numDyn; s += T) {
    uint32_t b = w.colorBodies[s];
    uint32_t count = 0;
    for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1]; e++) {
      uint32_t c = w.adjList[e];
      count += c < nj ? 1u : (w.mIds[p.cur][c - nj].w & 15u);
    }
    w.incStart[s] = count;
  }
  if (tid == 0) w.incStart[numDyn] = 0;
  GSYNC
  if (!grid_scan(w.incStart, numDyn + 1, w.scanScratch, bar, ctr)) return;
  const uint32_t totalInc = ldv(&w.scanScratch[gridDim.x]);
  if (tid == 0) {
    ctr[C_INC] = totalInc;
    ctr[C_DYN] = numDyn;
  }
  if (totalInc > p.incCap) {
    if (tid == 0) atomicOr(&ctr[C_ERROR], ERR_INC_OVERFLOW);
    return;  // uniform: every block read the same total after the barrier
  }
  for (uint32_t s = tid; s < numDyn; s += T) {
    uint32_t b = w.colorBodies[s];
    uint32_t colB = w.colorA[b] & 0xffu;
    uint32_t out = w.incStart[s];
    for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1]; e++) {
      uint32_t c = w.adjList[e];
      int ea, eb;
      uint32_t cnt;
      if (c < nj) {
        int4 in = w.jinfo[c];
        ea = in.y;
        eb = in.z;
        cnt = 1;
      } else {
        uint4 ids = w.mIds[p.cur][c - nj];
        ea = (int)ids.x;
        eb = (int)ids.y;
        cnt = ids.w & 15u;
      }
      int other = ea == (int)b ? eb : ea;
      bool owner = true;
      if (dynBody(w, other)) {
        uint32_t colO = w.colorA[other] & 0xffu;
        owner = colO < colB || (colO == colB && (uint32_t)other < b);
      }
      uint32_t flag = owner ? OWNER_BIT : 0u;
      if (c < nj) w.incList[out++] = c | flag;
      else
        for (uint32_t k = 0; k < cnt; k++) w.incList[out++] = (nj + (c - nj) * MAX_CONTACTS + k) | flag;
    }
  }

  // F. warm starts: joints (C(x-) at the poses the step starts from), then bodies
  for (uint32_t j = tid; j < nj; j += T) {
    int4 info = w.jinfo[j];
    if ((uint32_t)info.x != T_JOINT) continue;
    int a = info.y, b = info.z;
    if ((a >= 0 && !enabledBody(w, (uint32_t)a)) || !enabledBody(w, (uint32_t)b)) continue;
    float4 k[JOINT_VEC4];
    loadJoint(w, j, k);
    Pose dummy;
    Bodies2 B{&w, 0xffffffffu, &dummy};
    float3 cl = jointLinC(k, a, b, B), ca = jointAngC(k, a, b, B);
    float4* o = w.joint + j * JOINT_VEC4;
    o[J_C0_LIN] = make_float4(cl.x, cl.y, cl.z, 0.0f);
    o[J_C0_ANG] = make_float4(ca.x, ca.y, ca.z, k[J_C0_ANG].w);
    float decay = p.alpha * p.gamma;
    o[J_LAM_LIN] = make_float4(k[J_LAM_LIN].x * decay, k[J_LAM_LIN].y * decay, k[J_LAM_LIN].z * decay, k[J_LAM_LIN].w);
    o[J_LAM_ANG] = make_float4(k[J_LAM_ANG].x * decay, k[J_LAM_ANG].y * decay, k[J_LAM_ANG].z * decay, k[J_LAM_ANG].w);
    float4 pl = k[J_PEN_LIN], pa = k[J_PEN_ANG];
    auto wp = [&](float x, float stiff) { return fminf(fminf(fmaxf(x * p.gamma, PENALTY_MIN), PENALTY_MAX), stiff); };
    o[J_PEN_LIN] = make_float4(wp(pl.x, pl.w), wp(pl.y, pl.w), wp(pl.z, pl.w), pl.w);
    o[J_PEN_ANG] = make_float4(wp(pa.x, pa.w), wp(pa.y, pa.w), wp(pa.z, pa.w), pa.w);
  }
  GSYNC
  const float dt = p.dt, g = p.gravity;
  const float3 up = make_float3(p.upx, p.upy, p.upz);
  for (uint32_t i = tid; i < n; i += T) {
    if (!enabledBody(w, i)) continue;
    float4 pos = w.pos[i], rot = w.rot[i], vel = w.vel[i];
    float3 av = f3(w.avel[i]);
    bool dynamic = w.size[i].w > 0.0f;
    float3 y = f3(pos) + f3(vel) * dt;
    if (dynamic) y = y + up * (g * (dt * dt));
    w.ypos[i] = make_float4(y.x, y.y, y.z, w.ypos[i].w);
    w.yrot[i] = qadd(rot, av * dt);
    float wgt = 0.0f;
    if (fabsf(g) > 0.0f) wgt = fminf(fmaxf((dot3(f3(vel), up) - vel.w) / dt * (g < 0.0f ? -1.0f : 1.0f) / fabsf(g), 0.0f), 1.0f);
    bool slow = len3(f3(vel)) + len3(av) * w.moment[i].w < REST_SPEED;
    bool atRest = (p.flags & FLAG_START_AT_REST) != 0u && slow;
    w.ipos[i] = make_float4(pos.x, pos.y, pos.z, 0.0f);
    w.irot[i] = rot;
    if (dynamic && !atRest) {
      float3 x = f3(pos) + f3(vel) * dt + up * (g * (wgt * dt * dt));
      w.pos[i] = make_float4(x.x, x.y, x.z, pos.w);
      w.rot[i] = qadd(rot, av * dt);
    }
    if (!dynamic && (vel.x != 0.0f || vel.y != 0.0f || vel.z != 0.0f || av.x != 0.0f || av.y != 0.0f || av.z != 0.0f)) {
      float3 x = f3(pos) + f3(vel) * dt;
      w.pos[i] = make_float4(x.x, x.y, x.z, pos.w);
      w.rot[i] = qadd(rot, av * dt);
    }
  }
  GSYNC

  // G. iterations: each colour one sweep of its bodies, `lanes` threads per body
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warpGlobal = tid >> 5, nwarps = T >> 5;
  const float dt2 = dt * dt;
  for (int it = 0; it < p.iterations; it++) {
    for (uint32_t c = 0; c < numColors; c++) {
      const uint32_t s0 = w.colorStart[c], nb = w.colorStart[c + 1] - s0;
      uint32_t L = 1;
      while (L < 16u && nb * L * 2u <= T) L <<= 1;
      const uint32_t groupsPerWarp = 32u / L;
      const uint32_t sub = lane & (L - 1u), leader = lane & ~(L - 1u);
      for (uint32_t base = warpGlobal * groupsPerWarp; base < nb; base += nwarps * groupsPerWarp) {
        const uint32_t g = base + lane / L;
        const bool active = g < nb;
        uint32_t body = 0, e0 = 0, e1 = 0;
        Pose own;
        Acc acc;
        accZero(acc);
        if (active) {
          body = w.colorBodies[s0 + g];
          e0 = w.incStart[s0 + g];
          e1 = w.incStart[s0 + g + 1];
          own = loadPose(w, body);
          if (sub == 0) {
            float m = w.size[body].w / dt2;
            float3 I = f3(w.moment[body]) / dt2;
            acc.v[0] = m;
            acc.v[3] = m;
            acc.v[5] = m;
            acc.v[6] = I.x;
            acc.v[9] = I.y;
            acc.v[11] = I.z;
            float3 rl = (own.x - f3(w.ypos[body])) * m;
            float3 ra = I * qsub(own.q, w.yrot[body]);
            acc.v[21] = rl.x;
            acc.v[22] = rl.y;
            acc.v[23] = rl.z;
            acc.v[24] = ra.x;
            acc.v[25] = ra.y;
            acc.v[26] = ra.z;
          }
          for (uint32_t e = e0 + sub; e < e1; e += L) accumulateIncidence(acc, w, p, w.incList[e] & ~OWNER_BIT, body, own);
        }
        for (uint32_t off = L >> 1; off > 0; off >>= 1) {
#pragma unroll
          for (int k = 0; k < 27; k++) acc.v[k] += __shfl_xor_sync(0xffffffffu, acc.v[k], off);
        }
        float3 x = own.x;
        float4 q = own.q;
        if (active && sub == 0) {
          finishBody(acc, x, q);
          w.pos[body] = make_float4(x.x, x.y, x.z, w.pos[body].w);
          w.rot[body] = q;
        }
        x.x = __shfl_sync(0xffffffffu, x.x, leader);
        x.y = __shfl_sync(0xffffffffu, x.y, leader);
        x.z = __shfl_sync(0xffffffffu, x.z, leader);
        q.x = __shfl_sync(0xffffffffu, q.x, leader);
        q.y = __shfl_sync(0xffffffffu, q.y, leader);
        q.z = __shfl_sync(0xffffffffu, q.z, leader);
        q.w = __shfl_sync(0xffffffffu, q.w, leader);
        if (active) {
          setPose(own, x, q);
          for (uint32_t e = e0 + sub; e < e1; e += L) {
            uint32_t id = w.incList[e];
            if (id & OWNER_BIT) dualIncidence(w, p, id & ~OWNER_BIT, body, own);
          }
        }
      }
      GSYNC
    }
  }

  // H. velocities (BDF1)
  for (uint32_t i = tid; i < n; i += T) {
    if (!enabledBody(w, i)) continue;
    float4 vel = w.vel[i];
    float prevUp = dot3(f3(vel), up);
    if (w.size[i].w > 0.0f) {
      float3 v = (f3(w.pos[i]) - f3(w.ipos[i])) / dt;
      w.vel[i] = make_float4(v.x, v.y, v.z, prevUp);
      float3 av = qsub(w.rot[i], w.irot[i]) / dt;
      w.avel[i] = make_float4(av.x, av.y, av.z, w.avel[i].w);
    } else {
      w.vel[i] = make_float4(vel.x, vel.y, vel.z, prevUp);
    }
  }
#undef GSYNC
}

int solve_grid_blocks(int device) {
  int sms = 0, perSm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_topology_solve, SOLVE_THREADS, 0);
  if (perSm < 1) perSm = 1;
  return sms * perSm;
}

cudaError_t launch_topology_solve(const DWorld& w, const StepParams& p, int blocks, cudaStream_t s) {
  cudaMemsetAsync(w.barrier, 0, 2 * sizeof(uint32_t), s);
  cudaMemsetAsync(w.adjStart, 0, (size_t(p.n) + 1) * sizeof(uint32_t), s);
  cudaMemsetAsync(w.adjFill, 0, (size_t(p.n) + 1) * sizeof(uint32_t), s);
  DWorld wc = w;
  StepParams pc = p;
  void* args[] = {&wc, &pc};
  return cudaLaunchCooperativeKernel((const void*)k_topology_solve, dim3(blocks), dim3(SOLVE_THREADS), args, 0, s);
}

}  // namespace avbd
