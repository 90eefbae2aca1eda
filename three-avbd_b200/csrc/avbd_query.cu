// The queries and edits a World runs around the step, on the world's device state:
//
//   impulses on bodies before a step       Pusher (src/lib/push.ts:1-146)
//   contact begin / end events after it    ContactWatch (src/lib/contacts.ts:1-267)
//   nearest hit of each ray                Raycaster (src/lib/raycast.ts:1-251)
//
// All run on the world's stream, in order with its steps. The contact sets and the ray reduction
// are this file's own design: 64-bit keys (a pair of lifetime IDs; a hit's distance bits over its
// body index) that one atomic compare-and-swap or one atomic minimum settles, and a ray's nearest
// hit reduced across a warp by shuffles before one atomic per warp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "avbd_device.cuh"
#include "avbd_host.hpp"

namespace avbd {

namespace {

__device__ __forceinline__ bool bodyDisabled(const DWorld& w, uint32_t i) { return ((uint32_t)w.ipos[i].w & 2u) != 0u; }

// --- impulses -------------------------------------------------------------------------------------------
struct DPush {
  float4 lin;     // xyz: the whole linear impulse, w: the body (bits)
  float4 offLin;  // xyz: the part applied at points
  float4 moment;  // xyz: those parts' moment about the origin, plus angular impulses
};

// Δv = J / m; Δω = I^-1 (L - x × J_off) taken in the body's principal frame, where L is the pushes'
// moment about the origin and x the body's position now (push.ts:23-37)
__global__ void k_apply_pushes(DWorld w, const DPush* pushes, uint32_t n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const DPush P = pushes[k];
  const uint32_t b = __float_as_uint(P.lin.w);
  if (bodyDisabled(w, b)) return;
  const float mass = w.size[b].w;
  if (mass <= 0.0f) return;
  const float4 v = w.vel[b];
  w.vel[b] = make_float4(v.x + P.lin.x / mass, v.y + P.lin.y / mass, v.z + P.lin.z / mass, v.w);
  const float3 L = f3(P.moment) - cross3(f3(w.pos[b]), f3(P.offLin));
  const float4 q = w.rot[b];
  const float3 I = f3(w.moment[b]);
  const float3 Lb = qrotate(qconj(q), L);
  const float3 local = make_float3(Lb.x / fmaxf(I.x, 1e-12f), Lb.y / fmaxf(I.y, 1e-12f), Lb.z / fmaxf(I.z, 1e-12f));
  const float3 dw = qrotate(q, local);
  const float4 av = w.avel[b];
  w.avel[b] = make_float4(av.x + dw.x, av.y + dw.y, av.z + dw.z, av.w);
}

// --- contact events -------------------------------------------------------------------------------------
constexpr unsigned long long EMPTY_KEY = 0ull;

__device__ __forceinline__ unsigned long long pairKey(uint32_t idA, uint32_t idB) { return ((unsigned long long)idA << 32) | idB; }
__device__ __forceinline__ uint32_t keySlot(unsigned long long key, uint32_t mask) {
  // splitmix64's finaliser: consecutive IDs spread over the table
  key ^= key >> 30;
  key *= 0xbf58476d1ce4e5b9ull;
  key ^= key >> 27;
  key *= 0x94d049bb133111ebull;
  key ^= key >> 31;
  return (uint32_t)key & mask;
}
// Inserts `key` (never EMPTY: IDs are nonzero) into a set of mask + 1 slots; false when it is full
__device__ bool setInsert(unsigned long long* set, uint32_t mask, unsigned long long key) {
  uint32_t h = keySlot(key, mask);
  for (uint32_t probe = 0; probe <= mask; probe++) {
    const unsigned long long old = atomicCAS(set + h, EMPTY_KEY, key);
    if (old == EMPTY_KEY || old == key) return true;
    h = (h + 1u) & mask;
  }
  return false;
}
__device__ bool setHas(const unsigned long long* set, uint32_t mask, unsigned long long key) {
  uint32_t h = keySlot(key, mask);
  for (uint32_t probe = 0; probe <= mask; probe++) {
    const unsigned long long k = set[h];
    if (k == EMPTY_KEY) return false;
    if (k == key) return true;
    h = (h + 1u) & mask;
  }
  return false;
}

struct WatchLaunch {
  const uint32_t* watch;          // per body slot: lifetime ID (bits 0..30), reporting (bit 31)
  unsigned long long* now;        // this step's set
  const unsigned long long* old;  // last step's set
  uint32_t mask;                  // slots - 1
  uint32_t* head;                 // [0] events written (may pass the capacity), [1] a set was full
  float4* events;                 // 3 float4 an event
  uint32_t capacity, step;
  float dt;
};

__device__ void emitEvent(const WatchLaunch& L, uint32_t kind, uint32_t a, uint32_t b, float3 point, float impulse, float3 normal) {
  const uint32_t e = atomicAdd(&L.head[0], 1u);
  if (e >= L.capacity) return;
  L.events[3 * e] = make_float4(__uint_as_float(kind), __uint_as_float(a), __uint_as_float(b), __uint_as_float(L.step));
  L.events[3 * e + 1] = make_float4(point.x, point.y, point.z, impulse);
  L.events[3 * e + 2] = make_float4(normal.x, normal.y, normal.z, 0.0f);
}

// Per pair slot of the step just taken: a touching pair with a reporting body goes into this step's
// set, and begins (where: its points' mean on body a; how hard: its normal force over the step; the
// normal) when it is not in last step's set (contacts.ts:93-114)
__global__ void k_watch_touching(DWorld w, int last, uint32_t pairCap, WatchLaunch L) {
  const uint32_t pairs = min(w.counters[C_PAIRS], pairCap);
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < pairs; m += gridDim.x * blockDim.x) {
    const uint4 ids = w.mIds[last][m];
    const uint32_t count = ids.w & 15u;
    if (count == 0u) continue;
    const uint32_t wa = L.watch[ids.x], wb = L.watch[ids.y];
    const uint32_t idA = wa & 0x7fffffffu, idB = wb & 0x7fffffffu;
    if (((wa | wb) & 0x80000000u) == 0u || idA == 0u || idB == 0u) continue;
    const unsigned long long key = pairKey(idA, idB);
    if (!setInsert(L.now, L.mask, key)) atomicOr(&L.head[1], 1u);
    if (setHas(L.old, L.mask, key)) continue;
    const float3 pA = f3(w.pos[ids.x]);
    const float4 qA = w.rot[ids.x];
    float3 point = make_float3(0.0f, 0.0f, 0.0f);
    float force = 0.0f;
    for (uint32_t i = 0; i < count; i++) {
      const float4* c = w.cPt[last] + 4 * (size_t(ids.z) + i);
      point = point + (qrotate(qA, f3(c[K_RA])) + pA);
      force += c[K_LAM].x;
    }
    emitEvent(L, AVBD_CONTACT_BEGIN, idA, idB, point / float(count), fabsf(force) * L.dt, f3(w.mGeo[last][m]));
  }
}

// Per slot of last step's set: the pair ends when it is not in this step's (contacts.ts:117-125)
__global__ void k_watch_ended(WatchLaunch L) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= L.mask; s += gridDim.x * blockDim.x) {
    const unsigned long long key = L.old[s];
    if (key == EMPTY_KEY || setHas(L.now, L.mask, key)) continue;
    emitEvent(L, AVBD_CONTACT_END, uint32_t(key >> 32), uint32_t(key), make_float3(0.0f, 0.0f, 0.0f), 0.0f, make_float3(0.0f, 0.0f, 0.0f));
  }
}

// --- raycasts -------------------------------------------------------------------------------------------
struct DRay {
  float4 o;  // origin, most distance
  float4 d;  // unit direction
};
struct RayLaunch {
  const DRay* rays;
  unsigned long long* best;  // per ray: distance bits << 32 | body (all ones: no hit)
  float4* hits;              // per ray: normal + distance, then body bits
  uint32_t n, bodies, nIgnore, mask;
  uint32_t ignore[AVBD_RAY_MAX_IGNORED];
};
constexpr unsigned long long NO_HIT = ~0ull;

__device__ __forceinline__ bool rayIgnores(const DWorld& w, const RayLaunch& R, uint32_t b) {
  if (bodyDisabled(w, b)) return true;
  if ((w.filters[b].x & R.mask) == 0u) return true;
  for (uint32_t i = 0; i < R.nIgnore; i++)
    if (R.ignore[i] == b) return true;
  return false;
}

// Ray r against body b (raycast.ts:80-150): the distance to its surface (0 from inside, -1 a miss)
// and the normal there in the body's frame. A sphere analytically; a box or hull as the planes of
// its faces: the ray enters through the last plane it crosses inwards and leaves at the first it
// crosses outwards.
__device__ float rayTrace(const DWorld& w, uint32_t b, const DRay& r, float3& n) {
  const float4 q = w.rot[b];
  const float3 size = f3(w.size[b]);
  const float shape = w.avel[b].w;
  const float4 inv = qconj(q);
  const float3 o = qrotate(inv, f3(r.o) - f3(w.pos[b]));
  const float3 d = qrotate(inv, f3(r.d));
  float t;
  if (fabsf(shape - 1.0f) < 0.5f) {
    const float radius = size.x * 0.5f;
    const float bh = dot3(o, d);
    const float c = dot3(o, o) - radius * radius;
    const float disc = bh * bh - c;
    if (disc < 0.0f) return -1.0f;
    t = -bh - sqrtf(disc);
    if (c <= 0.0f) {
      t = 0.0f;
      n = -d;
    } else {
      if (t < 0.0f) return -1.0f;
      const float3 p = o + d * t;
      n = p / len3(p);
    }
  } else {
    float tin = -3.0e38f, tout = 3.0e38f;
    const bool hull = shape > 2.5f && w.hulls;
    uint32_t faces = 6u, fs = 0u;
    if (hull) {
      const uint4 head = w.hulls[(uint32_t)(shape - 3.0f + 0.5f)];
      fs = head.z;
      faces = head.w;
    }
    n = make_float3(0.0f, 0.0f, 0.0f);
    for (uint32_t k = 0; k < faces; k++) {
      float4 plane;
      if (hull) {
        const uint4 u = w.hulls[fs + 2u * k];
        plane = make_float4(__uint_as_float(u.x), __uint_as_float(u.y), __uint_as_float(u.z), __uint_as_float(u.w));
      } else {  // a box's faces +x -x +y -y +z -z, half its size out
        const uint32_t axis = k / 2u;
        const float sgn = (k % 2u == 0u) ? 1.0f : -1.0f;
        const float half = (axis == 0u ? size.x : axis == 1u ? size.y : size.z) * 0.5f;
        plane = make_float4(axis == 0u ? sgn : 0.0f, axis == 1u ? sgn : 0.0f, axis == 2u ? sgn : 0.0f, half);
      }
      const float3 pn = f3(plane);
      const float denom = dot3(pn, d);
      const float dist = plane.w - dot3(pn, o);
      if (fabsf(denom) < 1.0e-12f) {
        if (dist < 0.0f) return -1.0f;
        continue;
      }
      const float s = dist / denom;
      if (denom < 0.0f) {
        if (s > tin) {
          tin = s;
          n = pn;
        }
      } else {
        tout = fminf(tout, s);
      }
      if (tin > tout) return -1.0f;
    }
    if (tout < 0.0f) return -1.0f;
    t = tin;
    if (t <= 0.0f) {
      t = 0.0f;
      n = -d;
    }
  }
  if (t > r.o.w) return -1.0f;
  return t <= 0.0f ? 0.0f : t;  // never -0: its bits would order as a huge distance
}

// One ray (blockIdx.y) against a block of bodies: each warp's least (distance bits, body) by
// shuffles, then one atomic minimum per warp. The least key is the nearest hit, and among hits at
// the same distance the lowest body index, as the reference's two atomic passes find it.
__global__ void __launch_bounds__(256) k_ray_nearest(DWorld w, RayLaunch R) {
  const uint32_t r = blockIdx.y;
  const DRay ray = R.rays[r];
  unsigned long long key = NO_HIT;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < R.bodies; b += gridDim.x * blockDim.x) {
    if (rayIgnores(w, R, b)) continue;
    float3 n;
    const float t = rayTrace(w, b, ray, n);
    if (t >= 0.0f) key = min(key, ((unsigned long long)__float_as_uint(t) << 32) | b);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) key = min(key, __shfl_xor_sync(0xffffffffu, key, off));
  if ((threadIdx.x & 31u) == 0u && key != NO_HIT) atomicMin(R.best + r, key);
}

// Per ray: the nearest hit's normal in world axes, its distance and body (raycast.ts finish)
__global__ void k_ray_finish(DWorld w, RayLaunch R) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R.n) return;
  const unsigned long long key = R.best[r];
  if (key == NO_HIT) {
    R.hits[2 * r] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    R.hits[2 * r + 1] = make_float4(__uint_as_float(0xffffffffu), 0.0f, 0.0f, 0.0f);
    return;
  }
  const uint32_t b = uint32_t(key);
  float3 n;
  const float t = rayTrace(w, b, R.rays[r], n);
  float3 wn = qrotate(w.rot[b], n);
  wn = wn / len3(wn);
  R.hits[2 * r] = make_float4(wn.x, wn.y, wn.z, t);
  R.hits[2 * r + 1] = make_float4(__uint_as_float(b), 0.0f, 0.0f, 0.0f);
}

// Device scratch owned by the world (grown on demand, freed with it)
template <class T>
cudaError_t growBuffer(avbd_world* w, T** p, size_t& cap, size_t want) {
  if (*p && cap >= want) return cudaSuccess;
  if (*p) {
    auto it = std::find(w->allocations.begin(), w->allocations.end(), static_cast<void*>(*p));
    if (it != w->allocations.end()) w->allocations.erase(it);
    cudaStreamSynchronize(w->stream);
    cudaFree(*p);
    *p = nullptr;
  }
  void* ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(want, 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  w->allocations.push_back(ptr);
  *p = static_cast<T*>(ptr);
  cap = want;
  return cudaSuccess;
}

int qfail(avbd_world* w, int code, const std::string& msg) {
  if (w) w->error = msg;
  return code;
}

}  // namespace
}  // namespace avbd

using namespace avbd;

// --- impulses ---------------------------------------------------------------------------------------------
int avbd_apply_pushes(avbd_world* w, const avbd_push* pushes, uint32_t n) {
  if (!w || (n && !pushes)) return AVBD_ERR_INVALID;
  if (n == 0) return AVBD_OK;
  std::vector<char> seen(w->n, 0);
  std::vector<DPush> rec(n);
  for (uint32_t k = 0; k < n; k++) {
    const avbd_push& p = pushes[k];
    if (p.body >= w->n) return qfail(w, AVBD_ERR_INVALID, "push " + std::to_string(k) + ": body " + std::to_string(p.body) + " is not a slot");
    if (seen[p.body]) return qfail(w, AVBD_ERR_INVALID, "push " + std::to_string(k) + ": body " + std::to_string(p.body) + " pushed twice (sum its pushes)");
    seen[p.body] = 1;
    for (int a = 0; a < 3; a++)
      if (!std::isfinite(p.lin[a]) || !std::isfinite(p.off_lin[a]) || !std::isfinite(p.moment[a]))
        return qfail(w, AVBD_ERR_INVALID, "push " + std::to_string(k) + ": non-finite value");
    uint32_t bits = p.body;
    float fb;
    std::memcpy(&fb, &bits, 4);
    rec[k].lin = make_float4(p.lin[0], p.lin[1], p.lin[2], fb);
    rec[k].offLin = make_float4(p.off_lin[0], p.off_lin[1], p.off_lin[2], 0.0f);
    rec[k].moment = make_float4(p.moment[0], p.moment[1], p.moment[2], 0.0f);
  }
  cudaSetDevice(w->device);
  cudaError_t e = growBuffer(w, &w->pushBuf, w->pushCap, 3 * size_t(n));  // three float4 a push
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->pushBuf, rec.data(), n * sizeof(DPush), cudaMemcpyHostToDevice, w->stream);
  if (e == cudaSuccess) {
    k_apply_pushes<<<grid_for(n, 128), 128, 0, w->stream>>>(w->d, reinterpret_cast<const DPush*>(w->pushBuf), n);
    e = cudaGetLastError();
  }
  // the host records must outlive their copy
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) return qfail(w, AVBD_ERR_CUDA, std::string("avbd_apply_pushes: ") + cudaGetErrorString(e));
  return AVBD_OK;
}

// --- contact events -------------------------------------------------------------------------------------------
struct avbd_contact_watch {
  avbd_world* world = nullptr;
  uint32_t slots = 0, capacity = 0, flip = 0;
  uint32_t* watch = nullptr;              // per body slot of the world
  unsigned long long* sets = nullptr;     // two sets of `slots` keys
  uint32_t* head = nullptr;               // 4 words
  float4* events = nullptr;               // 3 float4 an event
  std::string error;
};

static int wfail(avbd_contact_watch* cw, int code, const std::string& msg) {
  if (cw) cw->error = msg;
  return code;
}

int avbd_contact_watch_create(avbd_world* w, uint32_t pairs, uint32_t capacity, avbd_contact_watch** out) {
  if (!w || !out || capacity == 0) return AVBD_ERR_INVALID;
  *out = nullptr;
  auto* cw = new avbd_contact_watch();
  cw->world = w;
  cw->capacity = capacity;
  cw->slots = pow2AtLeast(std::max<uint64_t>(64, 2ull * pairs));
  cudaSetDevice(w->device);
  bool ok = cudaMalloc(&cw->watch, std::max<size_t>(w->bodyCap, 1) * 4) == cudaSuccess &&
            cudaMalloc(&cw->sets, 2ull * cw->slots * sizeof(unsigned long long)) == cudaSuccess && cudaMalloc(&cw->head, 16) == cudaSuccess &&
            cudaMalloc(&cw->events, size_t(capacity) * 3 * sizeof(float4)) == cudaSuccess;
  ok = ok && cudaMemsetAsync(cw->watch, 0, std::max<size_t>(w->bodyCap, 1) * 4, w->stream) == cudaSuccess &&
       cudaMemsetAsync(cw->sets, 0, 2ull * cw->slots * sizeof(unsigned long long), w->stream) == cudaSuccess &&
       cudaMemsetAsync(cw->head, 0, 16, w->stream) == cudaSuccess && cudaStreamSynchronize(w->stream) == cudaSuccess;
  if (!ok) {
    avbd_contact_watch_destroy(cw);
    return qfail(w, AVBD_ERR_CUDA, "avbd_contact_watch_create: device allocation failed");
  }
  *out = cw;
  return AVBD_OK;
}

int avbd_contact_watch_destroy(avbd_contact_watch* cw) {
  if (!cw) return AVBD_OK;
  if (cw->world) {
    cudaSetDevice(cw->world->device);
    cudaStreamSynchronize(cw->world->stream);
  }
  for (void* p : {static_cast<void*>(cw->watch), static_cast<void*>(cw->sets), static_cast<void*>(cw->head), static_cast<void*>(cw->events)})
    if (p) cudaFree(p);
  delete cw;
  return AVBD_OK;
}

const char* avbd_contact_watch_last_error(const avbd_contact_watch* cw) { return cw ? cw->error.c_str() : "no contact watch"; }

int avbd_contact_watch_set(avbd_contact_watch* cw, const uint32_t* indices, const uint32_t* ids, const uint32_t* on, uint32_t n) {
  if (!cw || (n && (!indices || !ids || !on))) return AVBD_ERR_INVALID;
  avbd_world* w = cw->world;
  for (uint32_t k = 0; k < n; k++) {
    if (indices[k] >= w->bodyCap) return wfail(cw, AVBD_ERR_INVALID, "slot " + std::to_string(indices[k]) + " past the world's body capacity");
    if (ids[k] == 0u || ids[k] > 0x7fffffffu) return wfail(cw, AVBD_ERR_INVALID, "lifetime IDs are 1 .. 2^31 - 1");
  }
  cudaSetDevice(w->device);
  for (uint32_t k = 0; k < n; k++) {
    const uint32_t word = ids[k] | (on[k] ? 0x80000000u : 0u);
    if (cudaMemcpyAsync(cw->watch + indices[k], &word, 4, cudaMemcpyHostToDevice, w->stream) != cudaSuccess ||
        cudaStreamSynchronize(w->stream) != cudaSuccess)
      return wfail(cw, AVBD_ERR_CUDA, "avbd_contact_watch_set: copy failed");
  }
  return AVBD_OK;
}

int avbd_contact_watch_run(avbd_contact_watch* cw, uint32_t step, float dt) {
  if (!cw) return AVBD_ERR_INVALID;
  avbd_world* w = cw->world;
  if (w->stepCount == 0) return wfail(cw, AVBD_ERR_INVALID, "the world has not stepped: no contacts to watch");
  cudaSetDevice(w->device);
  cw->flip = 1u - cw->flip;
  WatchLaunch L{};
  L.watch = cw->watch;
  L.now = cw->sets + size_t(cw->flip) * cw->slots;
  L.old = cw->sets + size_t(1u - cw->flip) * cw->slots;
  L.mask = cw->slots - 1u;
  L.head = cw->head;
  L.events = cw->events;
  L.capacity = cw->capacity;
  L.step = step;
  L.dt = dt;
  cudaError_t e = cudaMemsetAsync(L.now, 0, size_t(cw->slots) * sizeof(unsigned long long), w->stream);
  if (e == cudaSuccess) {
    // the step just taken wrote contact buffer 1 - cur (avbd_step flips cur after each step)
    k_watch_touching<<<std::max<uint32_t>(1, std::min<uint32_t>(grid_for(w->pairCap, 256), 1184)), 256, 0, w->stream>>>(w->d, 1 - w->cur, w->pairCap, L);
    k_watch_ended<<<std::max<uint32_t>(1, std::min<uint32_t>(grid_for(cw->slots, 256), 1184)), 256, 0, w->stream>>>(L);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return wfail(cw, AVBD_ERR_CUDA, std::string("avbd_contact_watch_run: ") + cudaGetErrorString(e));
  return AVBD_OK;
}

int avbd_contact_watch_read(avbd_contact_watch* cw, avbd_contact_event* dst, uint32_t cap, uint32_t* n, uint32_t* dropped, uint32_t* full) {
  if (!cw || (cap && !dst)) return AVBD_ERR_INVALID;
  avbd_world* w = cw->world;
  cudaSetDevice(w->device);
  uint32_t head[4];
  std::vector<float4> ev;
  cudaError_t e = cudaStreamSynchronize(w->stream);
  if (e == cudaSuccess) e = copyToHost(head, cw->head, 16, w->stream);
  const uint32_t have = std::min(head[0], cw->capacity);
  if (e == cudaSuccess && have) {
    ev.resize(size_t(have) * 3);
    e = copyToHost(ev.data(), cw->events, ev.size() * sizeof(float4), w->stream);
  }
  if (e == cudaSuccess) e = cudaMemset(cw->head, 0, 16);
  if (e != cudaSuccess) return wfail(cw, AVBD_ERR_CUDA, std::string("avbd_contact_watch_read: ") + cudaGetErrorString(e));
  std::vector<avbd_contact_event> out(have);
  for (uint32_t k = 0; k < have; k++) {
    std::memcpy(&out[k], &ev[3 * k], sizeof(avbd_contact_event));
  }
  // in step order (within a step, as the device wrote them)
  std::stable_sort(out.begin(), out.end(), [](const avbd_contact_event& x, const avbd_contact_event& y) { return x.step < y.step; });
  const uint32_t k = std::min(cap, have);
  if (k) std::memcpy(dst, out.data(), k * sizeof(avbd_contact_event));
  if (n) *n = have;
  if (dropped) *dropped = head[0] - have;
  if (full) *full = head[1] ? 1u : 0u;
  return AVBD_OK;
}

// --- raycasts --------------------------------------------------------------------------------------------------
int avbd_raycast(avbd_world* w, const avbd_ray* rays, uint32_t n, const uint32_t* ignore, uint32_t n_ignore, uint32_t mask, avbd_ray_hit* hits) {
  if (!w || (n && (!rays || !hits)) || (n_ignore && !ignore)) return AVBD_ERR_INVALID;
  if (n > AVBD_RAY_MAX) return qfail(w, AVBD_ERR_INVALID, "avbd_raycast: at most " + std::to_string(AVBD_RAY_MAX) + " rays a call");
  if (n_ignore > AVBD_RAY_MAX_IGNORED) return qfail(w, AVBD_ERR_INVALID, "avbd_raycast: at most " + std::to_string(AVBD_RAY_MAX_IGNORED) + " bodies to ignore");
  if (n == 0) return AVBD_OK;
  std::vector<DRay> rec(n);
  for (uint32_t k = 0; k < n; k++) {
    const avbd_ray& r = rays[k];
    for (int a = 0; a < 3; a++)
      if (!std::isfinite(r.origin[a]) || !std::isfinite(r.direction[a])) return qfail(w, AVBD_ERR_INVALID, "ray " + std::to_string(k) + ": non-finite");
    if (std::isnan(r.max_distance)) return qfail(w, AVBD_ERR_INVALID, "ray " + std::to_string(k) + ": NaN distance");
    // normalised in double (raycast.ts:193-196); a zero direction stays zero
    double l = std::sqrt(double(r.direction[0]) * r.direction[0] + double(r.direction[1]) * r.direction[1] + double(r.direction[2]) * r.direction[2]);
    if (!(l > 0.0)) l = 1.0;
    const float maxd = r.max_distance > 3.0e38f ? 3.0e38f : r.max_distance;
    rec[k].o = make_float4(r.origin[0], r.origin[1], r.origin[2], maxd);
    rec[k].d = make_float4(float(r.direction[0] / l), float(r.direction[1] / l), float(r.direction[2] / l), 0.0f);
  }
  cudaSetDevice(w->device);
  cudaError_t e = growBuffer(w, &w->rayBuf, w->rayCap, size_t(n) * sizeof(DRay) / sizeof(float4));
  if (e == cudaSuccess) e = growBuffer(w, &w->rayBest, w->rayBestCap, n);
  if (e == cudaSuccess) e = growBuffer(w, &w->rayHits, w->rayHitsCap, 2 * size_t(n));
  if (e == cudaSuccess) e = cudaMemcpyAsync(w->rayBuf, rec.data(), n * sizeof(DRay), cudaMemcpyHostToDevice, w->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(w->rayBest, 0xff, n * sizeof(unsigned long long), w->stream);
  if (e == cudaSuccess) {
    RayLaunch R{};
    R.rays = reinterpret_cast<const DRay*>(w->rayBuf);
    R.best = w->rayBest;
    R.hits = w->rayHits;
    R.n = n;
    R.bodies = w->n;
    R.nIgnore = n_ignore;
    R.mask = mask;
    for (uint32_t k = 0; k < n_ignore; k++) R.ignore[k] = ignore[k];
    const uint32_t across = std::max<uint32_t>(1, std::min<uint32_t>(grid_for(w->n, 256), 64));
    if (w->n) k_ray_nearest<<<dim3(across, n), 256, 0, w->stream>>>(w->d, R);
    k_ray_finish<<<grid_for(n, 128), 128, 0, w->stream>>>(w->d, R);
    e = cudaGetLastError();
  }
  std::vector<float4> out(2 * size_t(n));
  if (e == cudaSuccess) e = cudaMemcpyAsync(out.data(), w->rayHits, out.size() * sizeof(float4), cudaMemcpyDeviceToHost, w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) return qfail(w, AVBD_ERR_CUDA, std::string("avbd_raycast: ") + cudaGetErrorString(e));
  for (uint32_t k = 0; k < n; k++) {
    const float4 a = out[2 * k], b = out[2 * k + 1];
    avbd_ray_hit& h = hits[k];
    if (a.w < 0.0f) {
      h.body = -1;
      h.distance = -1.0f;
      std::memset(h.point, 0, sizeof(h.point));
      std::memset(h.normal, 0, sizeof(h.normal));
      continue;
    }
    uint32_t body;
    std::memcpy(&body, &b.x, 4);
    h.body = int32_t(body);
    h.distance = a.w;
    for (int c = 0; c < 3; c++) h.point[c] = (&rec[k].o.x)[c] + (&rec[k].d.x)[c] * a.w;
    h.normal[0] = a.x;
    h.normal[1] = a.y;
    h.normal[2] = a.z;
  }
  return AVBD_OK;
}
