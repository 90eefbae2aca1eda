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
constexpr uint32_t ADJ_SORT_LOCAL = 24;  // adjacency lists up to this long are sorted in local memory
constexpr long long BARRIER_CYCLES = 4000000000LL;  // about two seconds of SM clock

__device__ __forceinline__ uint32_t ldv(const uint32_t* p) { return *(const volatile uint32_t*)p; }

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t atom_add_release_gpu(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier: a monotonic arrival counter (zeroed before the launch); the k-th barrier completes
// when it reaches k x gridDim.x. Arrival is a release, the wait an acquire (PTX memory model), so
// every block's writes before the barrier are visible to every block after it. The wait is bounded:
// past the clock budget the block sets an error bit and returns false, and every other block
// leaves at its next wait. The last block to arrive stamps the device time for the phase profile.
__device__ unsigned long long* g_clocks;
__shared__ uint32_t s_epoch;
__device__ bool grid_sync(uint32_t* bar, uint32_t* counters) {
  __shared__ uint32_t s_abort;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t target = (++s_epoch) * gridDim.x;
    uint32_t ab = 0;
    uint32_t old = atom_add_release_gpu(bar, 1u);
    if (old + 1u == target) {
      unsigned long long* ck = g_clocks;
      if (ck) {
        unsigned long long k = ck[0];
        if (k < (unsigned long long)MAX_CLOCKS) {
          ck[1 + k] = globaltimer();
          ck[0] = k + 1;
        }
      }
    } else {
      long long t0 = clock64();
      while (ld_acquire_gpu(bar) < target) {
        if (ldv(&counters[C_ERROR]) & (ERR_BARRIER_TIMEOUT | ERR_DEPENDENCY_TIMEOUT)) { ab = 1; break; }
        if (clock64() - t0 > BARRIER_CYCLES) {
          atomicOr(&counters[C_ERROR], ERR_BARRIER_TIMEOUT);
          ab = 1;
          break;
        }
        __nanosleep(32);
      }
    }
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

// Exclusive scan of one warp's range [lo, hi) in place; returns the range total (all lanes).
__device__ uint32_t warp_scan_range(uint32_t* data, uint32_t lo, uint32_t hi) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t carry = 0;
  for (uint32_t base = lo; base < hi; base += 32u) {
    const uint32_t i = base + lane;
    const uint32_t v = i < hi ? data[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (i < hi) data[i] = carry + x - v;
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
  __syncwarp();
  return carry;
}

// The scopes the topology+solve code runs at: the whole grid (one large world, cooperative launch,
// bounded grid barriers), one block (one small world of a batch, __syncthreads) or part of a block
// (one small world of a batch on a warp, two or four warps, SubTeam). A team's "unit" is the part of
// it that shares one copy of the shared-memory tables: a block, or a sub-block team itself.
// laneBudget is the thread count the lane classes are sized by: a sub-block team sizes them as a
// block does, so that every body gets the same lanes and sums its rows in the same order.
struct GridTeam {
  static constexpr bool kDataflow = true;  // colour passes as a dataflow sweep (no grid barrier per colour)
  static constexpr uint32_t kUnits = 1;
  uint32_t* bar;
  uint32_t* ctr;
  __device__ uint32_t rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ uint32_t size() const { return gridDim.x * blockDim.x; }
  __device__ uint32_t block() const { return blockIdx.x; }
  __device__ uint32_t blocks() const { return gridDim.x; }
  __device__ bool sync() { return grid_sync(bar, ctr); }
  __device__ uint32_t unit() const { return 0; }
  __device__ uint32_t lrank() const { return threadIdx.x; }
  __device__ uint32_t lsize() const { return blockDim.x; }
  __device__ void lsync() const { __syncthreads(); }
  __device__ uint32_t scan(uint32_t* data, uint32_t lo, uint32_t hi) const { return block_scan_range(data, lo, hi); }
  __device__ uint32_t laneBudget() const { return size(); }
};
struct BlockTeam {
  static constexpr bool kDataflow = false;  // a block's __syncthreads per colour costs little
  static constexpr uint32_t kUnits = 1;
  __device__ uint32_t rank() const { return threadIdx.x; }
  __device__ uint32_t size() const { return blockDim.x; }
  __device__ uint32_t block() const { return 0; }
  __device__ uint32_t blocks() const { return 1; }
  __device__ bool sync() {
    __syncthreads();
    return true;
  }
  __device__ uint32_t unit() const { return 0; }
  __device__ uint32_t lrank() const { return threadIdx.x; }
  __device__ uint32_t lsize() const { return blockDim.x; }
  __device__ void lsync() const { __syncthreads(); }
  __device__ uint32_t scan(uint32_t* data, uint32_t lo, uint32_t hi) const { return block_scan_range(data, lo, hi); }
  __device__ uint32_t laneBudget() const { return size(); }
};
// Exclusive scan of a sub-block team's range [lo, hi) in place (kT threads, two or four warps, synced
// by named barrier 1 + unit); returns the range total (all threads).
template <uint32_t kT>
__device__ uint32_t sub_scan_range(uint32_t* data, uint32_t lo, uint32_t hi, uint32_t unit) {
  __shared__ uint32_t sums[SOLVE_THREADS / 32];  // a slot a warp: each unit uses its own warps' slots
  const uint32_t r = threadIdx.x & (kT - 1u), lane = threadIdx.x & 31u, wl = r >> 5, wbase = unit * (kT / 32u);
  uint32_t carry = 0;
  for (uint32_t base = lo; base < hi; base += kT) {
    const uint32_t i = base + r;
    const uint32_t v = i < hi ? data[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31u) sums[wbase + wl] = x;
    asm volatile("barrier.sync %0, %1;" ::"r"(1u + unit), "r"(kT) : "memory");
    uint32_t before = 0, total = 0;
#pragma unroll
    for (uint32_t k = 0; k < kT / 32u; k++) {
      const uint32_t sk = sums[wbase + k];
      if (k < wl) before += sk;
      total += sk;
    }
    if (i < hi) data[i] = carry + before + x - v;
    carry += total;
    asm volatile("barrier.sync %0, %1;" ::"r"(1u + unit), "r"(kT) : "memory");
  }
  return carry;
}

// A sub-block team of kT threads (a warp, two or four warps): one small world of a batch, a block
// running SOLVE_THREADS / kT worlds at once. Its barriers are __syncwarp or named barrier 1 + unit.
template <uint32_t kT>
struct SubTeam {
  static_assert(kT == 32u || kT == 64u || kT == 128u, "a warp, two or four warps");
  static constexpr bool kDataflow = false;
  static constexpr uint32_t kUnits = SOLVE_THREADS / kT;
  __device__ uint32_t rank() const { return threadIdx.x & (kT - 1u); }
  __device__ uint32_t size() const { return kT; }
  __device__ uint32_t block() const { return 0; }
  __device__ uint32_t blocks() const { return 1; }
  __device__ bool sync() {
    lsync();
    return true;
  }
  __device__ uint32_t unit() const { return threadIdx.x / kT; }
  __device__ uint32_t lrank() const { return rank(); }
  __device__ uint32_t lsize() const { return kT; }
  __device__ void lsync() const {
    if constexpr (kT == 32u) __syncwarp();
    else asm volatile("barrier.sync %0, %1;" ::"r"(1u + unit()), "r"(kT) : "memory");
  }
  __device__ uint32_t scan(uint32_t* data, uint32_t lo, uint32_t hi) const {
    if constexpr (kT == 32u) return warp_scan_range(data, lo, hi);
    else return sub_scan_range<kT>(data, lo, hi, unit());
  }
  __device__ uint32_t laneBudget() const { return SOLVE_THREADS; }
};

// Exclusive scan of data[0, len) across the team; scratch[team.blocks()] receives the total.
template <class Team>
__device__ bool team_scan(uint32_t* data, uint32_t len, uint32_t* scratch, Team& team) {
  const uint32_t nb = team.blocks(), bi = team.block();
  uint32_t chunk = (len + nb - 1) / nb;
  uint32_t lo = min(len, bi * chunk), hi = min(len, lo + chunk);
  uint32_t total = team.scan(data, lo, hi);
  if (team.lrank() == 0) scratch[bi] = total;
  if (!team.sync()) return false;
  if (bi == 0) {
    uint32_t all = team.scan(scratch, 0, nb);
    if (team.lrank() == 0) scratch[nb] = all;
  }
  if (!team.sync()) return false;
  uint32_t add = scratch[bi];
  for (uint32_t i = lo + team.lrank(); i < hi; i += team.lsize()) data[i] += add;
  return team.sync();
}

// --- constraint endpoints and activity (gpu/layout.ts:356-369) ----------------------------------------
__device__ inline bool enabledBody(const DWorld& w, uint32_t i) { return ((uint32_t)w.ipos[i].w & 2u) == 0u; }
__device__ inline bool coldBody(const DWorld& w, uint32_t i) { return ((uint32_t)w.ipos[i].w & 4u) != 0u; }  // layout.ts:31
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

// An adjacency entry of body b for constraint c: its summation-order key (wgsl-topology.ts:116-125:
// joints by slot, then contact pairs by (other body + 2, first point's feature key)), the constraint
// with its row count, and the other body with its dynamic bit.
__device__ inline uint4 adjEntry(const DWorld& w, const StepParams& p, uint32_t b, uint32_t c, int ea, int eb, uint32_t rows) {
  int other = ea == (int)b ? eb : ea;
  uint32_t o = other < 0 ? 0x7fffffffu : ((uint32_t)other | (dynBody(w, other) ? 0x80000000u : 0u));
  if (c < p.nj) return make_uint4(0u, c, c | (rows << 28), o);
  uint4 ids = w.mIds[p.cur][c - p.nj];
  uint32_t feature = __float_as_uint(w.cPt[p.cur][4 * ids.z + K_RA].w) & ~STICK_BIT;
  return make_uint4((uint32_t)other + 2u, feature, c | (rows << 28), o);
}
__device__ inline bool entryLess(uint4 a, uint4 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); }

// --- Jones-Plassmann (wgsl-topology.ts:157-262) ---------------------------------------------------------
__device__ inline uint32_t priority(uint32_t i) { return hash32(i + 0x9e3779b9u); }
__device__ inline bool beats(uint32_t i, uint32_t j) {
  uint32_t pi = priority(i), pj = priority(j);
  return pi > pj || (pi == pj && i > j);
}
// A constraint's other body for the colouring: -1 unless it is dynamic (adjacency entry word w)
__device__ inline int neighbour(const DWorld& w, const StepParams&, uint32_t, uint32_t e) {
  uint32_t o = w.adjList[e].w;
  return (o & 0x80000000u) ? int(o & 0x7fffffffu) : -1;
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

// --- body poses -----------------------------------------------------------------------------------------
// What a contact row needs of a body: its rotation (and step-start rotation, for rolling spheres) and
// its displacement since x- (dlin, dang are kept by the solve, so a partner costs three loads and no
// quaternion division). The solve's unknowns are the displacement from x- and the rotation r since
// x- (q = r q-): both stay precise in f32 wherever the body is, where an absolute position rounds to
// its magnitude's ulp (7.6e-6 m at 100 m) and a difference of two such positions carries that error
// into every constraint value and multiplier. x0 is the step-start position; rw is r's w (its vector
// part is dAng / 2).
struct Pose {
  float3 x0, dLin, dAng;
  float4 q, q0;
  float rw;
};
__device__ inline Pose partnerPose(const DWorld& w, uint32_t i) {
  Pose P;
  P.q = w.rot[i];
  P.dLin = f3(w.dlin[i]);
  P.dAng = f3(w.dang[i]);
  P.x0 = make_float3(0.0f, 0.0f, 0.0f);
  P.q0 = P.q;
  P.rw = 1.0f;
  return P;
}
// r of a body from its dang word, and the dang word of r
__device__ __forceinline__ float4 relRot(float3 dAng, float rw) { return make_float4(dAng.x * 0.5f, dAng.y * 0.5f, dAng.z * 0.5f, rw); }
__device__ __forceinline__ float4 dangWord(float4 r) { return make_float4(r.x * 2.0f, r.y * 2.0f, r.z * 2.0f, r.w); }
__device__ __forceinline__ float4 qnormalize4(float4 q) {
  float l = sqrtf((q.x * q.x + q.y * q.y + q.z * q.z) + q.w * q.w);
  return make_float4(q.x / l, q.y / l, q.z / l, q.w / l);
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

// A point's three rows at once: directions d = n, t1, t2 (signed by sg for body B), stiffnesses k,
// forces F, lever arm r. The rows' outer products sum to M = sum k_i d_i d_i^T (the sign cancels);
// the angular Jacobian rows are [r]x d_i, so the cross block is [r]x M and the angular block
// [r]x M [r]x^T; the gradient is sg sum F_i d_i and r x that.
__device__ inline void addPoint(Acc& A, float3 r, float3 n, float3 t1, float3 t2, float3 k, float3 F, float sg) {
  const float3 a = n * k.x, b = t1 * k.y, c = t2 * k.z;
  const float M00 = a.x * n.x + b.x * t1.x + c.x * t2.x, M01 = a.x * n.y + b.x * t1.y + c.x * t2.y, M02 = a.x * n.z + b.x * t1.z + c.x * t2.z;
  const float M11 = a.y * n.y + b.y * t1.y + c.y * t2.y, M12 = a.y * n.z + b.y * t1.z + c.y * t2.z, M22 = a.z * n.z + b.z * t1.z + c.z * t2.z;
  A.v[0] += M00; A.v[1] += M01; A.v[2] += M02; A.v[3] += M11; A.v[4] += M12; A.v[5] += M22;
  // X = [r]x M (row: angular index)
  const float X00 = r.y * M02 - r.z * M01, X01 = r.y * M12 - r.z * M11, X02 = r.y * M22 - r.z * M12;
  const float X10 = r.z * M00 - r.x * M02, X11 = r.z * M01 - r.x * M12, X12 = r.z * M02 - r.x * M22;
  const float X20 = r.x * M01 - r.y * M00, X21 = r.x * M11 - r.y * M01, X22 = r.x * M12 - r.y * M02;
  A.v[12] += X00; A.v[13] += X01; A.v[14] += X02;
  A.v[15] += X10; A.v[16] += X11; A.v[17] += X12;
  A.v[18] += X20; A.v[19] += X21; A.v[20] += X22;
  // Y = X [r]x^T: Y_jk = sum_m X_jm S_km with S = [r]x
  A.v[6] += r.y * X02 - r.z * X01;
  A.v[7] += r.z * X00 - r.x * X02;
  A.v[8] += r.x * X01 - r.y * X00;
  A.v[9] += r.z * X10 - r.x * X12;
  A.v[10] += r.x * X11 - r.y * X10;
  A.v[11] += r.x * X21 - r.y * X20;
  const float3 gl = (n * F.x + t1 * F.y + t2 * F.z) * sg;
  const float3 ga = cross3(r, gl);
  A.v[21] += gl.x; A.v[22] += gl.y; A.v[23] += gl.z;
  A.v[24] += ga.x; A.v[25] += ga.y; A.v[26] += ga.z;
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
  // Each row's linearised value C0 (1 - alpha) + J dx: the Jacobian terms (rA x d) . dAngA and
  // (rB x -d) . dAngB are d . (dAngA x rA) and -d . (dAngB x rB) (the scalar triple product), so the
  // three rows share the contact point's relative displacement dp
  const float3 dp = (A.dLin - B.dLin) + (cross3(A.dAng, e.rAW) - cross3(B.dAng, e.rBW));
  e.C.x = rb.w * keep + dot3(n, dp);
  e.C.y = pen.w * keep + dot3(t1, dp);
  e.C.z = lam.w * keep + dot3(t2, dp);
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
// Poses of a joint's bodies; `own` is the body being solved (its pose in registers). A position is
// base + disp: the step-start position and the displacement since (at the warm start, `atStart`:
// the positions the step starts from, no displacement), so that two bodies' positions are
// differenced as (base a - base b) + (disp a - disp b), which is exact to the displacements' precision.
struct Bodies2 {
  const DWorld* w;
  uint32_t own;
  const Pose* ownPose;
  bool atStart;
  __device__ inline float3 base(int i) const { return atStart ? f3(w->pos[i]) : (uint32_t)i == own ? ownPose->x0 : f3(w->ipos[i]); }
  __device__ inline float3 disp(int i) const {
    return atStart ? make_float3(0.0f, 0.0f, 0.0f) : (uint32_t)i == own ? ownPose->dLin : f3(w->dlin[i]);
  }
  __device__ inline float4 rot(int i) const { return (uint32_t)i == own ? ownPose->q : w->rot[i]; }
};
__device__ inline float3 jointLinC(const float4* k, int a, int b, const Bodies2& B) {
  float3 rb = qrotate(B.rot(b), f3(k[J_RB]));
  if (a < 0) return ((f3(k[J_RA]) - B.base(b)) - B.disp(b)) - rb;  // a world point against body b
  return ((B.base(a) - B.base(b)) + (B.disp(a) - B.disp(b))) + (qrotate(B.rot(a), f3(k[J_RA])) - rb);
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
    float3 d = ((B.base(a) - B.base(b)) + (B.disp(a) - B.disp(b))) + (rAW - rBW);
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

// --- the 6x6 LDLT with pivot floor (wgsl-solve.ts:504-558): the Newton step (dx, dtheta), which the
// caller subtracts from the body's displacement and rotation -------------------------------------------------
__device__ inline void finishBody(const Acc& acc, float3& dx, float3& dth) {
  const float* v = acc.v;
  float A11 = v[0], A21 = v[1], A22 = v[3], A31 = v[2], A32 = v[4], A33 = v[5];
  float A41 = v[12], A42 = v[13], A43 = v[14], A44 = v[6];
  float A51 = v[15], A52 = v[16], A53 = v[17], A54 = v[7], A55 = v[9];
  float A61 = v[18], A62 = v[19], A63 = v[20], A64 = v[8], A65 = v[10], A66 = v[11];
  // Each pivot is inverted once and multiplied (the reference divides; the results agree to rounding)
  float D1 = A11, i1 = 1.0f / D1;
  float L21 = A21 * i1, L31 = A31 * i1, L41 = A41 * i1, L51 = A51 * i1, L61 = A61 * i1;
  float D2 = fmaxf(A22 - L21 * L21 * D1, A22 * PIVOT_FLOOR), i2 = 1.0f / D2;
  float L32 = (A32 - L21 * L31 * D1) * i2;
  float L42 = (A42 - L21 * L41 * D1) * i2;
  float L52 = (A52 - L21 * L51 * D1) * i2;
  float L62 = (A62 - L21 * L61 * D1) * i2;
  float D3 = fmaxf(A33 - (L31 * L31 * D1 + L32 * L32 * D2), A33 * PIVOT_FLOOR), i3 = 1.0f / D3;
  float L43 = (A43 - L31 * L41 * D1 - L32 * L42 * D2) * i3;
  float L53 = (A53 - L31 * L51 * D1 - L32 * L52 * D2) * i3;
  float L63 = (A63 - L31 * L61 * D1 - L32 * L62 * D2) * i3;
  float D4 = fmaxf(A44 - (L41 * L41 * D1 + L42 * L42 * D2 + L43 * L43 * D3), A44 * PIVOT_FLOOR), i4 = 1.0f / D4;
  float L54 = (A54 - L41 * L51 * D1 - L42 * L52 * D2 - L43 * L53 * D3) * i4;
  float L64 = (A64 - L41 * L61 * D1 - L42 * L62 * D2 - L43 * L63 * D3) * i4;
  float D5 = fmaxf(A55 - (L51 * L51 * D1 + L52 * L52 * D2 + L53 * L53 * D3 + L54 * L54 * D4), A55 * PIVOT_FLOOR), i5 = 1.0f / D5;
  float L65 = (A65 - L51 * L61 * D1 - L52 * L62 * D2 - L53 * L63 * D3 - L54 * L64 * D4) * i5;
  float D6 = fmaxf(A66 - (L61 * L61 * D1 + L62 * L62 * D2 + L63 * L63 * D3 + L64 * L64 * D4 + L65 * L65 * D5), A66 * PIVOT_FLOOR), i6 = 1.0f / D6;
  float y1 = v[21];
  float y2 = v[22] - L21 * y1;
  float y3 = v[23] - L31 * y1 - L32 * y2;
  float y4 = v[24] - L41 * y1 - L42 * y2 - L43 * y3;
  float y5 = v[25] - L51 * y1 - L52 * y2 - L53 * y3 - L54 * y4;
  float y6 = v[26] - L61 * y1 - L62 * y2 - L63 * y3 - L64 * y4 - L65 * y5;
  float w3 = y6 * i6;
  float w2 = y5 * i5 - L65 * w3;
  float w1 = y4 * i4 - L54 * w2 - L64 * w3;
  float v3 = y3 * i3 - L43 * w1 - L53 * w2 - L63 * w3;
  float v2 = y2 * i2 - L32 * v3 - L42 * w1 - L52 * w2 - L62 * w3;
  float v1 = y1 * i1 - L21 * v2 - L31 * v3 - L41 * w1 - L51 * w2 - L61 * w3;
  dx = make_float3(v1, v2, v3);
  dth = make_float3(w1, w2, w3);
}

// One contact row set (a point of a pair) from body i's side
struct PointView {
  float4 ra, rb, pen, lam;
  float3 n, t1, t2;
  float friction;
  bool isA;
  Pose other;
};
__device__ inline void loadPoint(const DWorld& w, const StepParams& p, uint32_t cs, uint32_t i, uint32_t partner, PointView& v) {
  const float4* pt = w.cPt[p.cur] + 4 * cs;
  v.ra = pt[K_RA];
  v.rb = pt[K_RB];
  v.pen = pt[K_PEN];
  v.lam = pt[K_LAM];
  float4 geo = w.mGeo[p.cur][cs / MAX_CONTACTS];
  v.n = f3(geo);
  v.friction = geo.w;
  orthonormal(v.n, v.t1, v.t2);
  v.isA = i > partner;  // a pair's A is its higher index
  v.other = partnerPose(w, partner);
  if ((__float_as_uint(v.ra.w) & ~STICK_BIT) == SPHERE_FEATURE) v.other.q0 = w.irot[partner];
}

__device__ inline void accumulateIncidence(Acc& acc, const DWorld& w, const StepParams& p, uint2 inc, uint32_t i, const Pose& own) {
  uint32_t id = inc.x & ~OWNER_BIT;
  if (id < p.nj) {
    Bodies2 B{&w, i, &own, false};
    addJoint(acc, w, id, p.alpha, i, B);
    return;
  }
  PointView v;
  loadPoint(w, p, id - p.nj, i, inc.y & PARTNER_MASK, v);
  const Pose& A = v.isA ? own : v.other;
  const Pose& B = v.isA ? v.other : own;
  ContactEval e;
  evalContact(v.ra, v.rb, v.pen, v.lam, v.n, v.t1, v.t2, v.friction, A, B, p.alpha, e);
  addPoint(acc, v.isA ? e.rAW : e.rBW, v.n, v.t1, v.t2, make_float3(v.pen.x, v.pen.y, v.pen.z), e.F, v.isA ? 1.0f : -1.0f);
}

// The dual update of one owned incidence (wgsl-solve.ts:562-662)
__device__ inline void dualIncidence(const DWorld& w, const StepParams& p, uint2 inc, uint32_t i, const Pose& own) {
  uint32_t id = inc.x & ~OWNER_BIT;
  if (id < p.nj) {
    Bodies2 B{&w, i, &own, false};
    dualJoint(w, p, id, B);
    return;
  }
  uint32_t cs = id - p.nj;
  PointView v;
  loadPoint(w, p, cs, i, inc.y & PARTNER_MASK, v);
  const Pose& A = v.isA ? own : v.other;
  const Pose& B = v.isA ? v.other : own;
  ContactEval e;
  evalContact(v.ra, v.rb, v.pen, v.lam, v.n, v.t1, v.t2, v.friction, A, B, p.alpha, e);
  float4* pt = w.cPt[p.cur] + 4 * cs;
  pt[K_LAM] = make_float4(e.F.x, e.F.y, e.F.z, v.lam.w);
  float4 pen = v.pen;
  if (e.F.x < 0.0f) pen.x = fminf(pen.x + p.betaLin * fabsf(e.C.x), PENALTY_MAX);
  if (e.frictionScale <= e.bounds) {
    pen.y = fminf(pen.y + p.betaLin * fabsf(e.C.y), PENALTY_MAX);
    pen.z = fminf(pen.z + p.betaLin * fabsf(e.C.z), PENALTY_MAX);
    bool stick = sqrtf(e.C.y * e.C.y + e.C.z * e.C.z) < STICK_THRESH;
    uint32_t key = __float_as_uint(v.ra.w);
    uint32_t nk = (key & ~STICK_BIT) | (stick ? STICK_BIT : 0u);
    if (nk != key) pt[K_RA].w = __uint_as_float(nk);
  }
  pt[K_PEN] = pen;
}

// Lanes per body: `perLane` rows a lane (the colour's rows over the grid's threads, at least one, so a
// colour fills the GPU about once), rounded up to a power of two lanes, up to a warp
__device__ inline uint32_t laneClass(uint32_t rows, uint32_t perLane) {
  uint32_t want = (rows + perLane - 1u) / perLane;
  uint32_t k = 0;
  while (k < 5u && (1u << k) < want) k++;
  return k;
}

// Bucket bookkeeping in w.bucket: counts | starts (+ total) | fill cursors | lane bases | lane totals
constexpr int B_COUNT = 0, B_START = BUCKETS, B_FILL = 2 * BUCKETS + 1, B_LANE = 3 * BUCKETS + 1, B_LANE_TOTAL = 4 * BUCKETS + 1,
              B_ROWS = B_LANE_TOTAL + MAX_COLORS;
static_assert(B_ROWS + MAX_COLORS <= BUCKET_WORDS, "bucket words");

// Waits until a body's count (`flag`: its done or poseDone word, published with release semantics)
// reaches `need`. Bounded: past the clock budget, or once any wait of the launch gave up, it returns
// false.
__device__ inline bool waitDone(const DWorld& w, const uint32_t* flag, uint32_t need) {
  if (ld_acquire_gpu(flag) >= need) return true;
  const long long t0 = clock64();
  for (uint32_t n = 1;; n++) {
    if (n > 64u) __nanosleep(32);
    if (ld_acquire_gpu(flag) >= need) return true;
    if ((n & 15u) == 0u) {
      if (ldv(&w.counters[C_ERROR]) & ERR_DEPENDENCY_TIMEOUT) return false;
      if (clock64() - t0 > BARRIER_CYCLES) {
        atomicOr(&w.counters[C_ERROR], ERR_DEPENDENCY_TIMEOUT);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// What one lane does in a chunk: its group's body, its first row (the group's rows are dealt
// round-robin to the group's L lanes), the end of the body's rows, and its place in the group.
struct LaneJob {
  bool active;
  uint32_t body, e, e1, L, sub;
};
__device__ __forceinline__ LaneJob jobFromEntry(uint4 t, bool active) {
  LaneJob J;
  J.active = active;
  J.body = t.x;
  J.e = t.y;
  J.e1 = t.z;
  J.L = active ? (t.w & 0xffu) : 1u;
  J.sub = active ? (t.w >> 8) : 0u;
  return J;
}

// Lane `base + lane` of colour c's lane space, from the colour's bucket tables: bucket j of the
// colour holds bodies of 32 >> j lanes each.
__device__ __forceinline__ LaneJob laneJob(const DWorld& w, uint32_t c, uint32_t base, const uint32_t* s_lane, const uint32_t* s_start,
                                           const uint32_t* s_total) {
  const uint32_t lam = base + (threadIdx.x & 31u);
  const uint32_t* laneBase = s_lane + c * LANE_CLASSES;
  LaneJob J;
  J.active = lam < s_total[c];
  uint32_t j = 0;
  if (J.active)
    while (j + 1 < (uint32_t)LANE_CLASSES && lam >= laneBase[j + 1]) j++;
  J.L = J.active ? (32u >> j) : 1u;
  const uint32_t local = J.active ? lam - laneBase[j] : 0u;
  J.sub = local & (J.L - 1u);
  J.body = J.e = J.e1 = 0;
  if (J.active) {
    const uint32_t s = s_start[c * LANE_CLASSES + j] + (local >> (5u - j));
    J.body = w.colorBodies[s];
    J.e = w.incStart[s] + J.sub;
    J.e1 = w.incStart[s + 1];
  }
  return J;
}

// The count a lane waits for before reading an incidence's partner (null: a static partner, no
// wait). A partner of an earlier colour must have moved in this iteration: its pose is all this body
// reads of it (their shared rows are this body's to update). One of a later colour must have finished
// the previous iteration, pose and the rows it updates, these among them. A partner of the same colour
// (only where the colour cap forced a clash) is not waited for within the iteration: the
// colour-by-colour sweep runs such pairs side by side too.
__device__ __forceinline__ const uint32_t* partnerFlag(const DWorld& w, uint2 inc, uint32_t it, uint32_t& need) {
  need = 0u;
  if (!(inc.y & PARTNER_DYNAMIC)) return nullptr;
  const uint32_t partner = inc.y & PARTNER_MASK;
  if (inc.y & PARTNER_EARLIER) {
    need = it + 1u;
    return w.poseDone + partner;
  }
  need = it;
  return w.done + partner;
}

// One 32-lane chunk: each group of lanes (one body) accumulates its rows, sums them by butterfly, its
// first lane solves and writes the pose, and the lanes update the rows the body owns. With kWait the
// chunk waits for the partner bodies it reads and afterwards publishes its bodies' iteration count;
// false: a wait gave up (warp-uniform). With kWait the caller runs a chunk on the same warp in every
// iteration, so the chunk's own bodies were last written by this warp (ordered by its __syncwarp)
// and need no wait: their state is loaded first, alongside the first two rows' incidences, and only the
// partners' counts are awaited (those of the first two rows polled together).
template <bool kWait>
__device__ __forceinline__ bool solveLanes(const DWorld& w, const StepParams& p, const LaneJob& J, uint32_t it) {
  const uint32_t lane = threadIdx.x & 31u;
  const float dt2 = p.dt * p.dt;
  const bool active = J.active;
  const uint32_t L = J.L, sub = J.sub, body = J.body, e1 = J.e1;
  const uint32_t leader = lane - sub;
  // the incidence list is fixed for the step: the lane's first two rows are read before any wait
  const uint32_t eB = J.e + L;
  const uint2 inc0 = kWait && active && J.e < e1 ? w.incList[J.e] : make_uint2(0u, 0u);
  const uint2 inc1 = kWait && active && eB < e1 ? w.incList[eB] : make_uint2(0u, 0u);
  Pose own;
  Acc acc;
  accZero(acc);
  if (active) {
    own.x0 = f3(w.ipos[body]);
    own.q = w.rot[body];
    own.q0 = w.irot[body];
    own.dLin = f3(w.dlin[body]);
    const float4 da = w.dang[body];
    own.dAng = f3(da);
    own.rw = da.w;
    if (sub == 0) {
      float m = w.size[body].w / dt2;
      float3 I = f3(w.moment[body]) / dt2;
      acc.v[0] = m;
      acc.v[3] = m;
      acc.v[5] = m;
      acc.v[6] = I.x;
      acc.v[9] = I.y;
      acc.v[11] = I.z;
      // M (x - y) and I qsub(q, y's rotation), both relative to x-: (dlin - ylin) and qsub(r, yang)
      float3 rl = (own.dLin - f3(w.ylin[body])) * m;
      float3 ra = I * qsub(relRot(own.dAng, own.rw), w.yang[body]);
      acc.v[21] = rl.x;
      acc.v[22] = rl.y;
      acc.v[23] = rl.z;
      acc.v[24] = ra.x;
      acc.v[25] = ra.y;
      acc.v[26] = ra.z;
    }
  }
  if constexpr (kWait) {
    bool ok = true;
    uint32_t needA, needB;
    const uint32_t* fA = active && J.e < e1 ? partnerFlag(w, inc0, it, needA) : nullptr;
    const uint32_t* fB = active && eB < e1 ? partnerFlag(w, inc1, it, needB) : nullptr;
    const uint32_t vA = fA ? ld_acquire_gpu(fA) : 0u;
    const uint32_t vB = fB ? ld_acquire_gpu(fB) : 0u;
    if (fA && vA < needA) ok = waitDone(w, fA, needA);
    if (ok && fB && vB < needB) ok = waitDone(w, fB, needB);
    if (active)
      for (uint32_t e = eB + L; e < e1 && ok; e += L) {
        uint32_t need;
        const uint32_t* f = partnerFlag(w, w.incList[e], it, need);
        if (f) ok = waitDone(w, f, need);
      }
    if (__any_sync(0xffffffffu, !ok)) return false;
  }
  if (active)
    for (uint32_t e = J.e; e < e1; e += L) accumulateIncidence(acc, w, p, kWait && e == J.e ? inc0 : kWait && e == eB ? inc1 : w.incList[e], body, own);
  // butterfly over the group: as many rounds as the warp's widest group needs
  const uint32_t Lmax = __reduce_max_sync(0xffffffffu, L);
  for (uint32_t off = Lmax >> 1; off > 0; off >>= 1) {
    const bool take = off < L;
#pragma unroll
    for (int k = 0; k < 27; k++) {
      float o = __shfl_xor_sync(0xffffffffu, acc.v[k], off);
      if (take) acc.v[k] += o;
    }
  }
  float3 dl = own.dLin, da = own.dAng;
  float4 q = own.q;
  if (active && sub == 0) {
    float3 dx, dth;
    finishBody(acc, dx, dth);
    dl = dl - dx;
    const float4 r = qadd(relRot(own.dAng, own.rw), make_float3(-dth.x, -dth.y, -dth.z));
    q = qnormalize4(qmul(r, own.q0));
    const float4 dw = dangWord(r);
    da = f3(dw);
    w.rot[body] = q;
    w.dlin[body] = make_float4(dl.x, dl.y, dl.z, 0.0f);
    w.dang[body] = dw;
    // the pose is final for this iteration: partners of later colours may read it now
    if constexpr (kWait) st_release_gpu(w.poseDone + body, it + 1u);
  }
  own.q = make_float4(__shfl_sync(0xffffffffu, q.x, leader), __shfl_sync(0xffffffffu, q.y, leader), __shfl_sync(0xffffffffu, q.z, leader),
                      __shfl_sync(0xffffffffu, q.w, leader));
  own.dLin = make_float3(__shfl_sync(0xffffffffu, dl.x, leader), __shfl_sync(0xffffffffu, dl.y, leader), __shfl_sync(0xffffffffu, dl.z, leader));
  own.dAng = make_float3(__shfl_sync(0xffffffffu, da.x, leader), __shfl_sync(0xffffffffu, da.y, leader), __shfl_sync(0xffffffffu, da.z, leader));
  if (active) {
    for (uint32_t e = J.e; e < e1; e += L) {
      const uint2 inc = kWait && e == J.e ? inc0 : w.incList[e];
      if (inc.x & OWNER_BIT) dualIncidence(w, p, inc, body, own);
    }
  }
  if constexpr (kWait) {
    // the group's writes (the leader's pose, every lane's rows) are ordered before the leader's
    // release by the warp barrier, as the grid barrier orders a block's writes before its arrival
    __syncwarp();
    if (active && sub == 0) st_release_gpu(w.done + body, it + 1u);
  }
  return true;
}

// --- the wind on sails (wgsl-solve.ts:262-292) ------------------------------------------------------------------
// A sail is a thin plate: pressure drag 1/2 rho C_d A (n.u)|n.u| along its normal n, u the wind
// relative to the plate, and skin friction along the plate at 6 % of that coefficient; the pressure
// term is linearised implicitly in the plate's normal speed (divided by 1 + 2 dt k |n.u|). The wind
// gusts in time and across space: travelling sines in the wind's frame (a downwind, c across, and
// height z), with the reference's frequencies and weights, as a second external acceleration on the
// inertial target. t = step x dt, x the step-start position, v the velocity after damping. Out of
// line: inlined, it changed how the warm start's other sums contract into FMAs in one of the world and
// batch kernels, whose results must agree bit for bit.
__device__ __noinline__ float3 windAccel(const StepParams& p, float t, float3 x, float4 q, float3 v, float4 size) {
  const float3 wv = make_float3(p.windX, p.windY, 0.0f);
  const float speed = len3(wv);
  const float3 d = speed > 1e-6f ? wv * (1.0f / speed) : make_float3(1.0f, 0.0f, 0.0f);
  const float3 side = make_float3(-d.y, d.x, 0.0f);
  const float a = dot3(x, d), c = dot3(x, side);
  const float along = 0.5f * sinf(1.1f * t - 0.35f * a + 0.2f * c) + 0.3f * sinf(2.9f * t - 0.8f * a + 0.6f * x.z) +
                      0.2f * sinf(6.1f * t - 1.7f * a + 1.3f * x.z + 0.9f * c);
  const float across = 0.6f * sinf(1.7f * t - 0.6f * a + 0.4f * x.z) + 0.4f * sinf(4.3f * t - 1.3f * a - 0.7f * x.z);
  const float lift = sinf(2.3f * t - 0.9f * a + 1.1f * c);
  const float g = p.windGust;
  const float3 u = wv * (1.0f + g * along) + (side * (0.25f * across) + make_float3(0.0f, 0.0f, 0.1f * lift)) * (g * speed) - v;
  const float3 n = qrotate(q, make_float3(0.0f, 0.0f, 1.0f));
  const float k = p.windPressure * size.x * size.y / size.w;  // 1/2 rho C_d A / m
  const float un = dot3(u, n);
  const float3 ut = u - n * un;
  return n * (k * un * fabsf(un) / (1.0f + 2.0f * p.dt * k * fabsf(un))) + ut * (0.06f * k * len3(ut));
}

// --- the kernel -----------------------------------------------------------------------------------------------
template <class Team>
__device__ void topologySolve(const DWorld& w, const StepParams& p, Team& team) {
  const uint32_t T = team.size();
  const uint32_t tid = team.rank();
  const uint32_t n = p.n, nj = p.nj;
  uint32_t* ctr = w.counters;
#define GSYNC \
  if (!team.sync()) return;
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
  if (!team_scan(w.adjStart, n + 1, w.scanScratch, team)) return;
  if (tid == 0) ctr[C_ADJ] = w.adjStart[n];
  // B. fill (adjFill zeroed by the host), then each body's list sorted into its summation order and
  // its row count (a joint is one row, a pair one per point)
  for (uint32_t c = tid; c < ncons; c += T) {
    int ea, eb;
    uint32_t cnt;
    if (!endpoints(w, p, c, ea, eb, cnt)) continue;
    if (dynBody(w, ea)) w.adjList[w.adjStart[ea] + atomicAdd(&w.adjFill[ea], 1u)] = adjEntry(w, p, (uint32_t)ea, c, ea, eb, cnt);
    if (dynBody(w, eb)) w.adjList[w.adjStart[eb] + atomicAdd(&w.adjFill[eb], 1u)] = adjEntry(w, p, (uint32_t)eb, c, ea, eb, cnt);
  }
  GSYNC
  for (uint32_t b = tid; b < n; b += T) {
    uint32_t lo = w.adjStart[b], hi = w.adjStart[b + 1];
    uint32_t rows = 0;
    if (hi - lo <= ADJ_SORT_LOCAL) {
      // a short list: every entry loaded at once, sorted in the thread's own (L1-resident) memory,
      // stored at once, instead of a chain of dependent global loads and stores
      uint4 buf[ADJ_SORT_LOCAL];
      const uint32_t d = hi - lo;
      for (uint32_t i = 0; i < d; i++) buf[i] = w.adjList[lo + i];
      for (uint32_t i = 0; i < d; i++) {
        const uint4 ent = buf[i];
        rows += ent.z >> 28;
        uint32_t j = i;
        while (j > 0 && entryLess(ent, buf[j - 1])) {
          buf[j] = buf[j - 1];
          j--;
        }
        buf[j] = ent;
      }
      for (uint32_t i = 0; i < d; i++) w.adjList[lo + i] = buf[i];
    } else {
      for (uint32_t i = lo; i < hi; i++) {
        uint4 ent = w.adjList[i];
        rows += ent.z >> 28;
        if (i == lo) continue;
        uint32_t j = i;
        while (j > lo) {
          uint4 prev = w.adjList[j - 1];
          if (!entryLess(ent, prev)) break;
          w.adjList[j] = prev;
          j--;
        }
        w.adjList[j] = ent;
      }
    }
    w.incCount[b] = rows;
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

  // D. final colours (NO_COLOR -> cap - 1, pending kept and counted), and bodies counted into
  // (colour, lane class) buckets, widest lane class first within a colour. The order of bodies in a
  // bucket does not change any result (a colour's bodies share no row), so the scatter uses atomics.
  // The unit's shared tables: (s_hist, s_base) here, then (s_lane, s_start) in the iterations
  __shared__ uint32_t s_tabs[Team::kUnits][2 * BUCKETS], s_perLaneU[Team::kUnits][MAX_COLORS];
  uint32_t* const s_hist = s_tabs[team.unit()];
  uint32_t* const s_base = s_hist + BUCKETS;
  uint32_t* const s_perLane = s_perLaneU[team.unit()];
  const uint32_t lr = team.lrank(), ls = team.lsize();
  {
    for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls) s_hist[k] = 0;
    team.lsync();
    uint32_t clashes = 0, maxc = 0;
    for (uint32_t b = tid; b < n; b += T) {
      if (!dynBody(w, (int)b)) continue;
      uint32_t s = w.colorA[b];
      uint32_t col = s & 0xffu;
      if (s & PENDING) clashes++;
      if (col == NO_COLOR || col >= (uint32_t)MAX_COLORS) col = cap - 1u;
      w.colorA[b] = col | (s & PENDING);
      maxc = max(maxc, col + 1u);
      atomicAdd(&s_hist[col], w.incCount[b] + 1u);  // the colour's rows (+1: the body's own inertia)
    }
    if (clashes) atomicAdd(&ctr[C_CLASHES], clashes);
    if (maxc) atomicMax(&ctr[C_COLORS], maxc);
    team.lsync();
    for (uint32_t k = lr; k < (uint32_t)MAX_COLORS; k += ls)
      if (s_hist[k]) atomicAdd(&w.bucket[B_ROWS + k], s_hist[k]);
  }
  GSYNC
  {
    const uint32_t budget = team.laneBudget();
    for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls) s_hist[k] = 0;
    for (uint32_t k = lr; k < (uint32_t)MAX_COLORS; k += ls) s_perLane[k] = max(max(1u, p.rowsPerLane), (w.bucket[B_ROWS + k] + budget - 1u) / budget);
    team.lsync();
    for (uint32_t b = tid; b < n; b += T) {
      if (!dynBody(w, (int)b)) continue;
      uint32_t col = w.colorA[b] & 0xffu;
      atomicAdd(&s_hist[col * LANE_CLASSES + (LANE_CLASSES - 1u - laneClass(w.incCount[b], s_perLane[col]))], 1u);
    }
    team.lsync();
    for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls)
      if (s_hist[k]) atomicAdd(&w.bucket[B_COUNT + k], s_hist[k]);
  }
  GSYNC
  if (team.block() == 0) {
    for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls) w.bucket[B_START + k] = w.bucket[B_COUNT + k];
    team.lsync();
    uint32_t total = team.scan(w.bucket + B_START, 0, BUCKETS);
    if (lr == 0) w.bucket[B_START + BUCKETS] = total;
    for (uint32_t c = lr; c < (uint32_t)MAX_COLORS; c += ls) {
      uint32_t lanes = 0;
      for (int j = 0; j < LANE_CLASSES; j++) {
        w.bucket[B_LANE + c * LANE_CLASSES + j] = lanes;
        lanes += w.bucket[B_COUNT + c * LANE_CLASSES + j] * (32u >> j);
      }
      w.bucket[B_LANE_TOTAL + c] = lanes;
    }
    team.lsync();
    for (uint32_t c = lr; c <= (uint32_t)MAX_COLORS; c += ls) w.colorStart[c] = w.bucket[B_START + c * LANE_CLASSES];
  }
  GSYNC
  const uint32_t numDyn = ldv(&w.bucket[B_START + BUCKETS]);
  const uint32_t numColors = ldv(&ctr[C_COLORS]);
  {
    // each unit reserves one range per bucket for its bodies, then places them by shared counters
    for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls) s_hist[k] = 0;
    team.lsync();
    for (uint32_t b = tid; b < n; b += T) {
      if (!dynBody(w, (int)b)) continue;
      uint32_t col = w.colorA[b] & 0xffu;
      atomicAdd(&s_hist[col * LANE_CLASSES + (LANE_CLASSES - 1u - laneClass(w.incCount[b], s_perLane[col]))], 1u);
    }
    team.lsync();
    for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls) {
      s_base[k] = s_hist[k] ? w.bucket[B_START + k] + atomicAdd(&w.bucket[B_FILL + k], s_hist[k]) : 0u;
      s_hist[k] = 0;
    }
    team.lsync();
    for (uint32_t b = tid; b < n; b += T) {
      if (!dynBody(w, (int)b)) continue;
      uint32_t col = w.colorA[b] & 0xffu;
      uint32_t bucket = col * LANE_CLASSES + (LANE_CLASSES - 1u - laneClass(w.incCount[b], s_perLane[col]));
      uint32_t pos = s_base[bucket] + atomicAdd(&s_hist[bucket], 1u);
      w.colorBodies[pos] = b;
      w.incStart[pos] = w.incCount[b];
    }
  }
  if (tid == 0) {
    w.incStart[numDyn] = 0;
    ctr[C_DYN] = numDyn;
  }
  GSYNC

  // E. incidence list: for each colour position s (body b = colorBodies[s]) its rows in summation
  // order, with the partner body and OWNER_BIT where b is the last of the row's dynamic bodies to move
  if (!team_scan(w.incStart, numDyn + 1, w.scanScratch, team)) return;
  const uint32_t totalInc = ldv(&w.scanScratch[team.blocks()]);
  if (tid == 0) ctr[C_INC] = totalInc;
  if (totalInc > p.incCap) {
    if (tid == 0) atomicOr(&ctr[C_ERROR], ERR_INC_OVERFLOW);
    return;  // uniform: every block read the same total after the barrier
  }
  for (uint32_t s = tid; s < numDyn; s += T) {
    uint32_t b = w.colorBodies[s];
    uint32_t colB = w.colorA[b] & 0xffu;
    uint32_t out = w.incStart[s];
    for (uint32_t e = w.adjStart[b]; e < w.adjStart[b + 1]; e++) {
      uint4 ent = w.adjList[e];
      uint32_t c = ent.z & 0x0fffffffu, cnt = ent.z >> 28;
      bool owner = true, earlier = false;
      if (ent.w & 0x80000000u) {
        uint32_t other = ent.w & 0x7fffffffu;
        uint32_t colO = w.colorA[other] & 0xffu;
        earlier = colO < colB;
        owner = earlier || (colO == colB && other < b);
      }
      uint32_t flag = owner ? OWNER_BIT : 0u;
      uint32_t partner = ent.w | (earlier ? PARTNER_EARLIER : 0u);
      if (c < nj) w.incList[out++] = make_uint2(c | flag, partner);
      else
        for (uint32_t k = 0; k < cnt; k++) w.incList[out++] = make_uint2((nj + (c - nj) * MAX_CONTACTS + k) | flag, partner);
    }
  }
  if constexpr (Team::kDataflow) {
    // the lane table of the dataflow sweep: per colour, its lanes in lane-space order, each with its
    // body, first row, the body's row end and (L, sub)
    __shared__ uint32_t s_colOff[MAX_COLORS + 1];
    if (threadIdx.x == 0) {
      uint32_t lanes = 0;
      for (uint32_t c = 0; c <= (uint32_t)MAX_COLORS; c++) {
        s_colOff[c] = lanes;
        if (c < (uint32_t)MAX_COLORS) lanes += w.bucket[B_LANE_TOTAL + c];
      }
    }
    __syncthreads();
    if (s_colOff[MAX_COLORS] > p.incCap) {
      if (tid == 0) atomicOr(&ctr[C_ERROR], ERR_INC_OVERFLOW);
      return;  // uniform: every block sums the same totals
    }
    for (uint32_t s = tid; s < numDyn; s += T) {
      const uint32_t b = w.colorBodies[s];
      const uint32_t col = w.colorA[b] & 0xffu;
      const uint32_t k = laneClass(w.incCount[b], s_perLane[col]);
      const uint32_t bucket = col * LANE_CLASSES + (LANE_CLASSES - 1u - k);
      const uint32_t L = 1u << k;
      const uint32_t first = s_colOff[col] + w.bucket[B_LANE + bucket] + (s - w.bucket[B_START + bucket]) * L;
      const uint32_t e0 = w.incStart[s], e1 = w.incStart[s + 1];
      for (uint32_t q = 0; q < L; q++) w.laneTable[first + q] = make_uint4(b, e0 + q, e1, L | (q << 8));
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
    Bodies2 B{&w, 0xffffffffu, &dummy, true};
    float3 cl = jointLinC(k, a, b, B), ca = jointAngC(k, a, b, B);
    float4* o = w.joint + j * JOINT_VEC4;
    o[J_C0_LIN] = make_float4(cl.x, cl.y, cl.z, 0.0f);
    o[J_C0_ANG] = make_float4(ca.x, ca.y, ca.z, k[J_C0_ANG].w);
    if ((a >= 0 && coldBody(w, (uint32_t)a)) || coldBody(w, (uint32_t)b)) {  // a cold body's joints start afresh (wgsl-solve.ts:247-253)
      const float pl = fminf(PENALTY_MIN, k[J_PEN_LIN].w), pa = fminf(PENALTY_MIN, k[J_PEN_ANG].w);
      o[J_LAM_LIN] = make_float4(0.0f, 0.0f, 0.0f, k[J_LAM_LIN].w);
      o[J_LAM_ANG] = make_float4(0.0f, 0.0f, 0.0f, k[J_LAM_ANG].w);
      o[J_PEN_LIN] = make_float4(pl, pl, pl, k[J_PEN_LIN].w);
      o[J_PEN_ANG] = make_float4(pa, pa, pa, k[J_PEN_ANG].w);
      continue;
    }
    float decay = p.alpha * p.gamma;
    o[J_LAM_LIN] = make_float4(k[J_LAM_LIN].x * decay, k[J_LAM_LIN].y * decay, k[J_LAM_LIN].z * decay, k[J_LAM_LIN].w);
    o[J_LAM_ANG] = make_float4(k[J_LAM_ANG].x * decay, k[J_LAM_ANG].y * decay, k[J_LAM_ANG].z * decay, k[J_LAM_ANG].w);
    float4 pl = k[J_PEN_LIN], pa = k[J_PEN_ANG];
    auto wp = [&](float x, float stiff) { return fminf(fminf(fmaxf(x * p.gamma, PENALTY_MIN), PENALTY_MAX), stiff); };
    o[J_PEN_LIN] = make_float4(wp(pl.x, pl.w), wp(pl.y, pl.w), wp(pl.z, pl.w), pl.w);
    o[J_PEN_ANG] = make_float4(wp(pa.x, pa.w), wp(pa.y, pa.w), wp(pa.z, pa.w), pa.w);
  }
  GSYNC
  const float dt = p.dt, gWorld = p.gravity;
  const float3 up = make_float3(p.upx, p.upy, p.upz);
  const uint32_t stepWord = ldv(&ctr[C_STEP]);  // steps since the world was made, from 1
  for (uint32_t i = tid; i < n; i += T) {
    if constexpr (Team::kDataflow) {
      w.done[i] = 0u;
      w.poseDone[i] = 0u;
    }
    if (!enabledBody(w, i)) continue;
    float4 pos = w.pos[i], rot = w.rot[i], vel = w.vel[i];
    float3 av = f3(w.avel[i]);
    const float av_shape = w.avel[i].w;
    bool dynamic = w.size[i].w > 0.0f;
    // the body's aux record (wgsl-solve.ts:9-20, 297-305): gravity scale, and damping of the
    // incoming velocities, stored so the next step's up-velocity history is this step's start
    const float4 ax = w.aux ? w.aux[i] : make_float4(1.0f, 0.0f, 0.0f, 0.0f);
    const float g = gWorld * ax.x;
    if (dynamic && (ax.y > 0.0f || ax.z > 0.0f)) {
      const float kl = expf(-ax.y * dt), ka = expf(-ax.z * dt);
      vel = make_float4(vel.x * kl, vel.y * kl, vel.z * kl, vel.w);
      av = av * ka;
      w.vel[i] = vel;
      w.avel[i] = make_float4(av.x, av.y, av.z, w.avel[i].w);
    }
    // y - x- and y's rotation relative to q- (the solve's inertial terms), and y itself for readers
    float3 yl = f3(vel) * dt;
    if (dynamic) yl = yl + up * (g * (dt * dt));
    // the wind's push on sails, a second external force (wgsl-solve.ts:310-311)
    if (dynamic && p.windPressure != 0.0f && av_shape == SHAPE_SAIL_F)
      yl = yl + windAccel(p, float(stepWord) * dt, f3(pos), rot, f3(vel), w.size[i]) * (dt * dt);
    const float4 ry = qadd(make_float4(0.0f, 0.0f, 0.0f, 1.0f), av * dt);
    const float3 y = f3(pos) + yl;
    w.ypos[i] = make_float4(y.x, y.y, y.z, w.ypos[i].w);
    w.yrot[i] = qadd(rot, av * dt);
    w.ylin[i] = make_float4(yl.x, yl.y, yl.z, 0.0f);
    w.yang[i] = ry;
    float wgt = 0.0f;
    if (fabsf(g) > 0.0f) wgt = fminf(fmaxf((dot3(f3(vel), up) - vel.w) / dt * (g < 0.0f ? -1.0f : 1.0f) / fabsf(g), 0.0f), 1.0f);
    bool slow = len3(f3(vel)) + len3(av) * w.moment[i].w < REST_SPEED;
    bool atRest = (p.flags & FLAG_START_AT_REST) != 0u && slow;
    w.ipos[i] = make_float4(pos.x, pos.y, pos.z, 0.0f);
    w.irot[i] = rot;
    // the warm-started guess as a displacement dl and a rotation r since x- (q = r q-)
    float3 dl = make_float3(0.0f, 0.0f, 0.0f);
    float4 r = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    bool moved = false;
    if (dynamic && !atRest) {
      dl = f3(vel) * dt + up * (g * (wgt * dt * dt));
      r = ry;
      moved = true;
    }
    if (!dynamic && (vel.x != 0.0f || vel.y != 0.0f || vel.z != 0.0f || av.x != 0.0f || av.y != 0.0f || av.z != 0.0f)) {
      dl = f3(vel) * dt;
      r = ry;
      moved = true;
    }
    const float3 x = f3(pos) + dl;
    const float4 q = moved ? qnormalize4(qmul(r, rot)) : rot;
    w.pos[i] = make_float4(x.x, x.y, x.z, pos.w);
    w.rot[i] = q;
    w.dlin[i] = make_float4(dl.x, dl.y, dl.z, 0.0f);
    w.dang[i] = dangWord(r);
  }
  GSYNC

  // G. iterations: per colour, each body's group of lanes (its lane class) accumulates its rows, the
  // group sums in registers, the first lane solves, and every lane then updates the rows it owns.
  // The colours' lane tables (lane bases, bucket starts, lane totals) are kept in shared memory.
  __shared__ uint32_t s_totalU[Team::kUnits][MAX_COLORS], s_chunk[MAX_COLORS + 1], s_laneOff[MAX_COLORS + 1];
  uint32_t* const s_lane = s_hist;  // the unit's tables, free again since D
  uint32_t* const s_start = s_base;
  uint32_t* const s_total = s_totalU[team.unit()];
  for (uint32_t k = lr; k < (uint32_t)BUCKETS; k += ls) {
    s_lane[k] = w.bucket[B_LANE + k];
    s_start[k] = w.bucket[B_START + k];
  }
  for (uint32_t k = lr; k < (uint32_t)MAX_COLORS; k += ls) s_total[k] = w.bucket[B_LANE_TOTAL + k];
  team.lsync();
  const uint32_t warpGlobal = tid >> 5, nwarps = T >> 5;
  if constexpr (Team::kDataflow) {
    // Dataflow sweep: the iterations' colour passes as one ordered list of 32-lane chunks. A chunk
    // waits only for the partner bodies its rows touch (a body of an earlier colour to finish this
    // iteration, one of a later colour the previous iteration; the body itself ran its previous
    // iteration on the same warp), so every read sees exactly what the colour-by-colour sweep reads,
    // and the colours overlap instead of meeting at grid barriers. Every wait is on chunks earlier in
    // the list, and each warp takes its chunks in list order, so the earliest unfinished chunk can
    // always run.
    if (threadIdx.x == 0) {
      uint32_t acc = 0, lanes = 0;
      for (uint32_t c = 0; c < numColors; c++) {
        s_chunk[c] = acc;
        s_laneOff[c] = lanes;
        acc += (s_total[c] + 31u) / 32u;
        lanes += s_total[c];
      }
      s_chunk[numColors] = acc;
      s_laneOff[numColors] = lanes;
    }
    __syncthreads();
    // Chunk r of every iteration runs on warp r mod (warps): a warp takes its chunks iteration by
    // iteration, in list order, and a body's group of lanes stays on one warp for the whole sweep.
    const uint32_t perIter = s_chunk[numColors];
    const uint32_t mine = warpGlobal < perIter ? (perIter - warpGlobal + nwarps - 1u) / nwarps : 0u;
    const uint32_t items = mine * (uint32_t)max(p.iterations, 0);
    // the warp's j-th chunk's lane entry, fetched one chunk ahead (the lane table is fixed for the step)
    auto entryOf = [&](uint32_t j, bool& active) -> uint4 {
      active = false;
      if (j >= items) return make_uint4(0u, 0u, 0u, 1u);
      const uint32_t r = warpGlobal + (j % mine) * nwarps;
      uint32_t c = 0;
      while (s_chunk[c + 1] <= r) c++;
      const uint32_t lam = (r - s_chunk[c]) * 32u + (threadIdx.x & 31u);
      active = lam < s_total[c];
      return active ? w.laneTable[s_laneOff[c] + lam] : make_uint4(0u, 0u, 0u, 1u);
    };
    bool nextActive;
    uint4 next = entryOf(0u, nextActive);
    for (uint32_t j = 0; j < items; j++) {
      const LaneJob J = jobFromEntry(next, nextActive);
      next = entryOf(j + 1u, nextActive);
      if (!solveLanes<true>(w, p, J, j / mine)) break;
    }
    GSYNC
  } else {
    for (int it = 0; it < p.iterations; it++) {
      for (uint32_t c = 0; c < numColors; c++) {
        for (uint32_t base = warpGlobal * 32u; base < s_total[c]; base += nwarps * 32u)
          solveLanes<false>(w, p, laneJob(w, c, base, s_lane, s_start, s_total), (uint32_t)it);
        GSYNC
      }
    }
  }

  // H. velocities (BDF1)
  for (uint32_t i = tid; i < n; i += T) {
    if (!enabledBody(w, i)) continue;
    float4 vel = w.vel[i];
    float prevUp = dot3(f3(vel), up);
    if (w.size[i].w > 0.0f) {
      // x = x- + the displacement (the sweep keeps only the displacement, which partners read)
      const float3 dl = f3(w.dlin[i]);
      const float3 x = f3(w.ipos[i]) + dl;
      w.pos[i] = make_float4(x.x, x.y, x.z, w.pos[i].w);
      // (x - x-) / dt and qsub(q, q-) / dt: the step's displacement and 2 vec(r)
      float3 v = dl / dt;
      w.vel[i] = make_float4(v.x, v.y, v.z, prevUp);
      float3 av = f3(w.dang[i]) / dt;
      w.avel[i] = make_float4(av.x, av.y, av.z, w.avel[i].w);
    } else {
      w.vel[i] = make_float4(vel.x, vel.y, vel.z, prevUp);
    }
  }
  team.sync();
#undef GSYNC
}

__global__ void __launch_bounds__(SOLVE_THREADS, 2) k_topology_solve(DWorld w, StepParams p) {
  if (threadIdx.x == 0) s_epoch = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    g_clocks = w.clocks;
    w.clocks[0] = 1;
    w.clocks[1] = globaltimer();
  }
  GridTeam team{w.barrier, w.counters};
  topologySolve(w, p, team);
}

// Batched worlds: each block takes worlds from the queue (largest first) and runs the same
// topology + solve code for one world at block scope.
__global__ void __launch_bounds__(SOLVE_THREADS, 2) k_batch_solve(BatchLaunch B) {
  __shared__ uint32_t s_world;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_world = atomicAdd(&B.queue[1], 1u);
    __syncthreads();
    const uint32_t qi = s_world;
    if (qi >= B.nWorlds) return;
    const uint32_t wi = B.order[qi];
    const WorldDesc d = B.worlds[wi];
    const DWorld w = worldView(B.base, d, wi);
    const StepParams p = worldParams(B.p, d);
    for (uint32_t i = threadIdx.x; i <= d.n; i += SOLVE_THREADS) {
      w.adjStart[i] = 0u;
      w.adjFill[i] = 0u;
    }
    for (uint32_t k = threadIdx.x; k < (uint32_t)BUCKET_WORDS; k += SOLVE_THREADS) w.bucket[k] = 0u;
    __syncthreads();
    BlockTeam team;
    topologySolve(w, p, team);
    __syncthreads();
    if (threadIdx.x == 0 && w.counters[C_ERROR]) atomicOr(&B.status[1], w.counters[C_ERROR]);
  }
}

// Batched worlds on part of a block: each team of kT threads (a warp, two or four warps) takes
// worlds from the same queue and runs the topology and barrier sweep with its own barriers, so a block
// steps SOLVE_THREADS / kT worlds at once. Lane classes are sized as a block sizes them
// (SubTeam::laneBudget), so every world's results are bit for bit those of the block-a-world launch.
template <uint32_t kT>
__global__ void __launch_bounds__(SOLVE_THREADS, 2) k_batch_solve_sub(BatchLaunch B) {
  using Team = SubTeam<kT>;
  Team team;
  const uint32_t r = team.rank();
  __shared__ uint32_t s_next[Team::kUnits];
  for (;;) {
    if (r == 0) s_next[team.unit()] = atomicAdd(&B.queue[1], 1u);
    team.lsync();
    const uint32_t qi = s_next[team.unit()];
    if (qi >= B.nWorlds) return;
    const uint32_t wi = B.order[qi];
    const WorldDesc d = B.worlds[wi];
    const DWorld w = worldView(B.base, d, wi);
    const StepParams p = worldParams(B.p, d);
    for (uint32_t i = r; i <= d.n; i += kT) {
      w.adjStart[i] = 0u;
      w.adjFill[i] = 0u;
    }
    for (uint32_t k = r; k < (uint32_t)BUCKET_WORDS; k += kT) w.bucket[k] = 0u;
    team.lsync();
    topologySolve(w, p, team);
    team.lsync();
    if (r == 0 && w.counters[C_ERROR]) atomicOr(&B.status[1], w.counters[C_ERROR]);
  }
}

static_assert(BATCH_SOLVE_THREADS == SOLVE_THREADS, "one solve block size");

int batch_solve_blocks_per_sm(int worldThreads) {
  int perSm = 0;
  if (worldThreads == 32) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_batch_solve_sub<32>, SOLVE_THREADS, 0);
  else if (worldThreads == 64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_batch_solve_sub<64>, SOLVE_THREADS, 0);
  else if (worldThreads == 128) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_batch_solve_sub<128>, SOLVE_THREADS, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_batch_solve, SOLVE_THREADS, 0);
  return perSm;
}

cudaError_t launch_batch_solve(const BatchLaunch& b, int blocks, int worldThreads, cudaStream_t s) {
  if (worldThreads == 32) k_batch_solve_sub<32><<<blocks, SOLVE_THREADS, 0, s>>>(b);
  else if (worldThreads == 64) k_batch_solve_sub<64><<<blocks, SOLVE_THREADS, 0, s>>>(b);
  else if (worldThreads == 128) k_batch_solve_sub<128><<<blocks, SOLVE_THREADS, 0, s>>>(b);
  else k_batch_solve<<<blocks, SOLVE_THREADS, 0, s>>>(b);
  return cudaGetLastError();
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
  cudaMemsetAsync(w.bucket, 0, BUCKET_WORDS * sizeof(uint32_t), s);
  DWorld wc = w;
  StepParams pc = p;
  void* args[] = {&wc, &pc};
  return cudaLaunchCooperativeKernel((const void*)k_topology_solve, dim3(blocks), dim3(SOLVE_THREADS), args, 0, s);
}

}  // namespace avbd
