// Batched worlds: many small independent worlds stepped together, one block per world.
//
// The reference steps one world per GpuSolver3D (src/avbd3d/gpu/solver.ts:598) and has no batched
// mode; a batch runs the same step, world by world, with every launch shared:
//   - the worlds' records are concatenated (bodies, joints, pair slots, scratch), and a table of
//     WorldDesc gives each world's slices; a world's indices are local to it;
//   - one launch collides every world (all pairs of a world against the pair rule, then the
//     narrowphase), one launch runs every world's topology, colouring and solve at block scope;
//     blocks take worlds from a queue, largest first;
//   - the step is captured in a CUDA graph per contact-buffer parity;
//   - pair storage grows per world, as a world's does (gpu/solver.ts:2362-2377): the collision
//     kernel flags a world past 80 % or overflowing, and the next step lays the batch out again.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "avbd_host.hpp"
#include "avbd_record.hpp"

using namespace avbd;

struct avbd_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  avbd_params params{};
  uint32_t worldCap = 0, bodyCap = 0, jointCap = 0, pairsPerBody = 6;
  uint32_t n = 0, nj = 0;  // bodies and joints used over all worlds
  std::vector<WorldDesc> worlds;
  std::vector<uint32_t> statics;  // every world's no-collide triples
  DWorld d{};
  float4* staging = nullptr;  // body records for host transfers (10 float4 a body, capacity)
  WorldDesc* dWorlds = nullptr;
  uint32_t *dOrder = nullptr, *dQueue = nullptr, *dStatus = nullptr;
  uint32_t staticsAlloc = 0;
  // pair-dependent storage: allocated entries and entries used by the worlds' slices
  uint64_t pairAlloc = 0, hashAlloc = 0, adjAlloc = 0, incAlloc = 0;
  uint64_t pairUsed = 0, hashUsed = 0, adjUsed = 0, incUsed = 0;
  uint64_t pairReserve = 0;  // the first allocation: pairs_per_body slots for every body of the capacity
  bool tableDirty = true;
  int cur = 0;
  uint32_t stepCount = 0;
  // launch shape (the autotuner's choice)
  int sms = 0, collideThreads = 128, collideBlocks = 0, solveBlocks = 0;
  uint32_t rowsPerLane = 1;  // the solve's least rows a lane (bodies per warp), chosen by the tuner
  int worldThreads = 256;    // the solve's threads a world: 256 (a block) or 32 (a warp), chosen by the tuner
  // status of the last step, copied back asynchronously
  uint32_t* hStatus = nullptr;
  cudaEvent_t statusReady = nullptr;
  bool statusInFlight = false;
  uint32_t relayouts = 0;
  bool useGraphs = true;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  uint64_t graphGen[2] = {0, 0};
  uint64_t configGen = 1;
  std::vector<void*> allocations;
  // the adjoint's recording (avbd_batch_record_start): steps still to append, its device arrays
  struct Recording {
    uint32_t K = 0, done = 0;
    RecordDev d{};
    std::vector<void*> mem;
    std::vector<avbd_body> initial;
    avbd_params params{};
  } rec;
};

namespace {

int bfail(avbd_batch* b, int code, const std::string& msg) {
  if (b) b->error = msg;
  return code;
}

#define BATCH_TRY(b, call)                                                                                   \
  do {                                                                                                       \
    cudaError_t e_ = (call);                                                                                 \
    if (e_ != cudaSuccess) return bfail(b, AVBD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
cudaError_t balloc(avbd_batch* b, T** p, size_t count) {
  void* ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  b->allocations.push_back(ptr);
  *p = static_cast<T*>(ptr);
  return cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), b->stream);
}
void bfree(avbd_batch* b, void* p) {
  if (!p) return;
  auto it = std::find(b->allocations.begin(), b->allocations.end(), p);
  if (it != b->allocations.end()) b->allocations.erase(it);
  cudaFree(p);
}

// A world's pair-dependent slice sizes from its pair capacity (the single world's rule, allocPairs)
void sizeSlices(WorldDesc& w, uint32_t pairCap) {
  w.pairCap = pairCap;
  w.hashMask = pow2AtLeast(2ull * pairCap) - 1u;
  w.adjCap = 2u * (pairCap + w.nj);
  w.incCap = 2u * (pairCap * MAX_CONTACTS + w.nj);
}

// Reallocates the pair-dependent arrays for the worlds' current slices. Last step's manifolds and
// contacts (buffer 1 - cur) move with their world; the rest is scratch.
int layoutPairs(avbd_batch* b, const std::vector<WorldDesc>& old) {
  uint64_t pairs = 0, hash = 0, adj = 0, inc = 0;
  for (auto& w : b->worlds) {
    w.pair = uint32_t(pairs);
    w.hash = uint32_t(hash);
    w.adj = uint32_t(adj);
    w.inc = uint32_t(inc);
    pairs += w.pairCap;
    hash += w.hashMask + 1ull;
    adj += w.adjCap;
    inc += w.incCap;
  }
  if (pairs >= (1ull << 31) / MAX_CONTACTS || inc >= (1ull << 31) || adj >= (1ull << 31) || hash >= (1ull << 31))
    return bfail(b, AVBD_ERR_CAPACITY, "batch pair storage past 2^31 entries");
  b->pairUsed = pairs;
  b->hashUsed = hash;
  b->adjUsed = adj;
  b->incUsed = inc;
  DWorld& d = b->d;
  const int prev = 1 - b->cur;
  bool movePrev = false;
  for (size_t i = 0; i < old.size() && !movePrev; i++) movePrev = old[i].pair != b->worlds[i].pair;
  const bool grow = pairs > b->pairAlloc;
  if (grow || movePrev) {
    uint64_t cap = grow ? std::max<uint64_t>(std::max<uint64_t>(pairs, b->pairAlloc * 3 / 2), b->pairReserve) : b->pairAlloc;
    uint4* ids[2] = {nullptr, nullptr};
    float4* geo[2] = {nullptr, nullptr};
    float4* pts[2] = {nullptr, nullptr};
    for (int k = 0; k < 2; k++) {
      BATCH_TRY(b, balloc(b, &ids[k], cap));
      BATCH_TRY(b, balloc(b, &geo[k], cap));
      BATCH_TRY(b, balloc(b, &pts[k], size_t(cap) * MAX_CONTACTS * 4));
    }
    if (d.mIds[prev] && !movePrev && !old.empty()) {
      // worlds were only appended: the old slices keep their offsets
      const WorldDesc& o = old.back();
      size_t m = size_t(o.pair) + o.pairCap;
      BATCH_TRY(b, cudaMemcpyAsync(ids[prev], d.mIds[prev], m * sizeof(uint4), cudaMemcpyDeviceToDevice, b->stream));
      BATCH_TRY(b, cudaMemcpyAsync(geo[prev], d.mGeo[prev], m * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream));
      BATCH_TRY(b, cudaMemcpyAsync(pts[prev], d.cPt[prev], m * MAX_CONTACTS * 4 * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream));
      BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    } else if (d.mIds[prev]) {
      for (size_t i = 0; i < old.size(); i++) {
        const WorldDesc &o = old[i], &w = b->worlds[i];
        size_t m = std::min(o.pairCap, w.pairCap);
        BATCH_TRY(b, cudaMemcpyAsync(ids[prev] + w.pair, d.mIds[prev] + o.pair, m * sizeof(uint4), cudaMemcpyDeviceToDevice, b->stream));
        BATCH_TRY(b, cudaMemcpyAsync(geo[prev] + w.pair, d.mGeo[prev] + o.pair, m * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream));
        BATCH_TRY(b, cudaMemcpyAsync(pts[prev] + size_t(w.pair) * MAX_CONTACTS * 4, d.cPt[prev] + size_t(o.pair) * MAX_CONTACTS * 4,
                                     m * MAX_CONTACTS * 4 * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream));
      }
      BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    }
    for (int k = 0; k < 2; k++) {
      bfree(b, d.mIds[k]);
      bfree(b, d.mGeo[k]);
      bfree(b, d.cPt[k]);
      d.mIds[k] = ids[k];
      d.mGeo[k] = geo[k];
      d.cPt[k] = pts[k];
    }
    bfree(b, d.pairs);
    BATCH_TRY(b, balloc(b, &d.pairs, cap));
    b->pairAlloc = cap;
  }
  if (hash > b->hashAlloc) {
    bfree(b, d.hash);
    b->hashAlloc = std::max<uint64_t>(hash, b->hashAlloc * 3 / 2);
    BATCH_TRY(b, balloc(b, &d.hash, b->hashAlloc));
  }
  if (adj > b->adjAlloc) {
    bfree(b, d.adjList);
    b->adjAlloc = std::max<uint64_t>(adj, b->adjAlloc * 3 / 2);
    BATCH_TRY(b, balloc(b, &d.adjList, b->adjAlloc));
  }
  if (inc > b->incAlloc) {
    bfree(b, d.incList);
    b->incAlloc = std::max<uint64_t>(inc, b->incAlloc * 3 / 2);
    BATCH_TRY(b, balloc(b, &d.incList, b->incAlloc));
  }
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  b->tableDirty = true;
  b->configGen++;
  return AVBD_OK;
}

// The world table, the queue order (most bodies first) and every world's no-collide triples
int uploadTable(avbd_batch* b) {
  const uint32_t nw = uint32_t(b->worlds.size());
  std::vector<uint32_t> order(nw);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
    const WorldDesc &a = b->worlds[x], &c = b->worlds[y];
    return uint64_t(a.n) + a.nj > uint64_t(c.n) + c.nj;
  });
  if (b->statics.size() > b->staticsAlloc) {
    bfree(b, b->d.nocollide);
    b->staticsAlloc = uint32_t(std::max<size_t>(b->statics.size() * 2, 64));
    BATCH_TRY(b, balloc(b, &b->d.nocollide, b->staticsAlloc));
  }
  if (nw) {
    BATCH_TRY(b, cudaMemcpyAsync(b->dWorlds, b->worlds.data(), nw * sizeof(WorldDesc), cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(b->dOrder, order.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
  }
  if (!b->statics.empty())
    BATCH_TRY(b, cudaMemcpyAsync(b->d.nocollide, b->statics.data(), b->statics.size() * 4, cudaMemcpyHostToDevice, b->stream));
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  b->tableDirty = false;
  b->configGen++;
  return AVBD_OK;
}

// Grows the pair capacity of every world that overflowed or passed 80 % in the last step
int adaptBatch(avbd_batch* b, bool wait) {
  if (!b->statusInFlight) return AVBD_OK;
  if (!wait && cudaEventQuery(b->statusReady) != cudaSuccess) return AVBD_OK;
  BATCH_TRY(b, cudaEventSynchronize(b->statusReady));
  b->statusInFlight = false;
  if (!(b->hStatus[0] & (BATCH_OVERFLOW | BATCH_NEAR_FULL))) return AVBD_OK;
  const uint32_t nw = uint32_t(b->worlds.size());
  std::vector<uint32_t> ctr(size_t(nw) * COUNTER_WORDS);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  BATCH_TRY(b, copyToHost(ctr.data(), b->d.counters, ctr.size() * 4, b->stream));
  std::vector<WorldDesc> old = b->worlds;
  bool any = false;
  for (uint32_t i = 0; i < nw; i++) {
    WorldDesc& w = b->worlds[i];
    const uint32_t* c = ctr.data() + size_t(i) * COUNTER_WORDS;
    uint32_t demand = c[C_PAIRS];
    if ((c[C_OVERFLOW] & 1u) || uint64_t(demand) * 10 > uint64_t(w.pairCap) * 8) {
      uint64_t want = std::min<uint64_t>(std::max<uint64_t>(2ull * demand, uint64_t(w.pairCap) * 5 / 4), 1ull << 24);
      if (want > w.pairCap) {
        sizeSlices(w, uint32_t(want));
        any = true;
      }
    }
  }
  if (!any) return AVBD_OK;
  b->relayouts++;
  return layoutPairs(b, old);
}

void launchShape(avbd_batch* b) {
  const int nw = int(std::max<size_t>(b->worlds.size(), 1));
  int cper = std::max(1, batch_collide_blocks_per_sm(b->collideThreads));
  b->collideBlocks = std::min(nw, b->sms * cper);
  if (b->solveBlocks <= 0) b->solveBlocks = b->sms * std::max(1, batch_solve_blocks_per_sm(b->worldThreads));
}

BatchLaunch makeLaunch(avbd_batch* b) {
  BatchLaunch L{};
  L.base = b->d;
  L.worlds = b->dWorlds;
  L.order = b->dOrder;
  L.nWorlds = uint32_t(b->worlds.size());
  L.queue = b->dQueue;
  L.status = b->dStatus;
  StepParams& p = L.p;
  const avbd_params& a = b->params;
  p.dt = a.dt;
  p.gravity = a.gravity;
  p.alpha = a.alpha;
  p.betaLin = a.beta_lin;
  p.betaAng = a.beta_ang;
  p.gamma = a.gamma;
  p.margin = a.contact_margin;
  p.flags = a.flags;
  p.iterations = a.iterations;
  p.upx = a.up[0];
  p.upy = a.up[1];
  p.upz = a.up[2];
  setWind(p, a);
  p.step = b->stepCount;
  p.colorCap = MAX_COLORS;
  p.rowsPerLane = b->rowsPerLane;
  p.cur = b->cur;
  return L;
}

cudaError_t enqueueStep(avbd_batch* b, const BatchLaunch& L) {
  cudaMemsetAsync(b->dQueue, 0, 2 * sizeof(uint32_t), b->stream);
  cudaMemsetAsync(b->dStatus, 0, 2 * sizeof(uint32_t), b->stream);
  cudaError_t e = launch_batch_collision(L, b->collideBlocks, b->collideThreads, b->stream);
  if (e != cudaSuccess) return e;
  const int worldsPerBlock = BATCH_SOLVE_THREADS / std::max(32, std::min(b->worldThreads, BATCH_SOLVE_THREADS));
  e = launch_batch_solve(L, std::min<int>(b->solveBlocks, (int(L.nWorlds) + worldsPerBlock - 1) / worldsPerBlock), b->worldThreads, b->stream);
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(b->hStatus, b->dStatus, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream);
}

int checkWorld(avbd_batch* b, uint32_t world) {
  if (!b) return AVBD_ERR_INVALID;
  if (world >= b->worlds.size()) return bfail(b, AVBD_ERR_INVALID, "no world " + std::to_string(world) + " in the batch");
  return AVBD_OK;
}

// A new world's slices: bodies and joints appended, pair slices sized from its body count
int appendWorld(avbd_batch* b, uint32_t n, uint32_t nj, uint32_t pairCap, double threshold, const std::vector<NoCollide>& nocollide,
                uint32_t flags, uint32_t* index) {
  WorldDesc w{};
  w.body = b->n;
  w.n = n;
  w.joint = b->nj;
  w.nj = nj;
  w.largeThreshold = float(threshold);
  w.noCollide = uint32_t(b->statics.size());
  w.nNoCollide = uint32_t(nocollide.size());
  w.flags = flags;
  sizeSlices(w, pairCap);
  std::vector<WorldDesc> old = b->worlds;
  b->worlds.push_back(w);
  for (auto& e : nocollide) {
    b->statics.push_back(e.hi);
    b->statics.push_back(e.lo);
    b->statics.push_back(e.slot);
  }
  int r = layoutPairs(b, old);
  if (r) {
    b->worlds.pop_back();
    b->statics.resize(w.noCollide);
    return r;
  }
  b->n += n;
  b->nj += nj;
  if (index) *index = uint32_t(b->worlds.size() - 1);
  return AVBD_OK;
}

void bodiesIn(avbd_batch* b, uint32_t first, const avbd_body* src, uint32_t n, cudaMemcpyKind kind) {
  if (kind == cudaMemcpyHostToDevice && b->staging) {  // one contiguous transfer, then a scatter
    cudaMemcpyAsync(b->staging, src, size_t(n) * sizeof(avbd_body), cudaMemcpyHostToDevice, b->stream);
    unpackBodies(b->d, b->staging, first, n, b->stream);
    return;
  }
  float4* fields[10] = {b->d.pos, b->d.rot, b->d.ipos, b->d.irot, b->d.size, b->d.moment, b->d.ypos, b->d.yrot, b->d.vel, b->d.avel};
  for (int f = 0; f < 10; f++)
    cudaMemcpy2DAsync(fields[f] + first, sizeof(float4), reinterpret_cast<const char*>(src) + f * sizeof(float4), sizeof(avbd_body), sizeof(float4), n, kind,
                      b->stream);
}
void bodiesOut(avbd_batch* b, uint32_t first, avbd_body* dst, uint32_t n) {
  packBodies(b->d, b->staging, first, n, b->stream);  // a gather into records, then one contiguous transfer
  cudaMemcpyAsync(dst, b->staging, size_t(n) * sizeof(avbd_body), cudaMemcpyDeviceToHost, b->stream);
}

void freeRecording(avbd_batch* b) {
  for (void* p : b->rec.mem) cudaFree(p);
  b->rec = avbd_batch::Recording{};
}

template <class T>
bool recAlloc(avbd_batch* b, T** p, size_t count) {
  void* ptr = nullptr;
  if (cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return false;
  b->rec.mem.push_back(ptr);
  *p = static_cast<T*>(ptr);
  return cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), b->stream) == cudaSuccess;
}

}  // namespace

static int takeRecording(avbd_batch* b, RecordingHandoff& out, std::string& why);

int avbd::batch_take_recording(avbd_batch* b, RecordingHandoff& out, std::string& why) {
  if (!b) return AVBD_ERR_INVALID;
  int r = takeRecording(b, out, why);
  if (r) b->error = why;
  return r;
}

static int takeRecording(avbd_batch* b, RecordingHandoff& out, std::string& why) {
  const auto& R = b->rec;
  if (!R.K) {
    why = "the batch holds no recording (avbd_batch_record_start)";
    return AVBD_ERR_INVALID;
  }
  if (R.done < R.K) {
    why = "the recording holds " + std::to_string(R.done) + " of its " + std::to_string(R.K) + " steps";
    return AVBD_ERR_INVALID;
  }
  cudaSetDevice(b->device);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) {
    why = "the batch's stream failed";
    return AVBD_ERR_CUDA;
  }
  uint32_t status[2] = {0, 0};
  unsigned long long totals[2] = {0, 0};
  if (copyToHost(status, R.d.status, sizeof(status), b->stream) != cudaSuccess ||
      copyToHost(totals, R.d.totals, sizeof(totals), b->stream) != cudaSuccess) {
    why = "reading the recording's status failed";
    return AVBD_ERR_CUDA;
  }
  if (status[0] & REC_CAPACITY) {
    why = "the recording ran out of room: start it again with more points per body";
    return AVBD_ERR_CAPACITY;
  }
  if (status[0] & REC_HISTORY) {
    why = "a recorded step warm-started from contacts of a step before the recording (write the bodies again, or record from the first step)";
    return AVBD_ERR_INVALID;
  }
  if (status[0] & REC_SPHERE) {
    why = "the recording holds sphere contacts, which the adjoint does not differentiate";
    return AVBD_ERR_INVALID;
  }
  if (status[0] & (REC_COLORS | REC_ORDER)) {
    why = "the recording holds a step with more than 64 colours or a misordered pair";
    return AVBD_ERR_INVALID;
  }
  out.device = b->device;
  out.K = R.K;
  out.W = R.d.W;
  out.nb = R.d.nb;
  out.maxPts = status[1];
  out.manifolds = totals[0];
  out.points = totals[1];
  out.manFirst = R.d.manFirst;
  out.ptFirst = R.d.ptFirst;
  out.ptMan = R.d.ptMan;
  out.ptPrev = R.d.ptPrev;
  out.color = R.d.color;
  out.ncol = R.d.ncol;
  out.manAB = R.d.manAB;
  out.basis = R.d.basis;
  out.anchors = R.d.anchors;
  out.worldFirst.clear();
  for (auto& w : b->worlds) out.worldFirst.push_back(w.body);
  out.worldFirst.push_back(b->n);
  out.initial = R.initial;
  out.params = R.params;
  out.mem = R.mem;
  b->rec.mem.clear();  // the receiver owns the device arrays now
  b->rec = avbd_batch::Recording{};
  return AVBD_OK;
}

extern "C" {

int avbd_batch_create(const avbd_batch_config* cfg, avbd_batch** out) {
  if (!out || !cfg) return AVBD_ERR_INVALID;
  *out = nullptr;
  if (cfg->world_capacity == 0 || cfg->body_capacity == 0) return AVBD_ERR_INVALID;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return AVBD_ERR_NO_DEVICE;
  if (cfg->device < 0 || cfg->device >= count) return AVBD_ERR_INVALID;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major < 10) return AVBD_ERR_NO_DEVICE;
  cudaSetDevice(cfg->device);
  avbd_batch* b = new avbd_batch();
  b->device = cfg->device;
  b->sms = prop.multiProcessorCount;
  b->worldCap = cfg->world_capacity;
  b->bodyCap = cfg->body_capacity;
  b->jointCap = std::max<uint32_t>(cfg->joint_capacity, 1);
  b->pairsPerBody = cfg->pairs_per_body ? cfg->pairs_per_body : 6;
  b->pairReserve = uint64_t(b->pairsPerBody) * b->bodyCap;
  avbd_default_params(&b->params);
  auto bad = [&](int code) {
    avbd_batch_destroy(b);
    return code;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(AVBD_ERR_CUDA);
  DWorld& d = b->d;
  const size_t B = b->bodyCap, W = b->worldCap;
  bool ok = true;
  auto A = [&](cudaError_t e) { ok = ok && e == cudaSuccess; };
  for (float4** f : {&d.pos, &d.rot, &d.ipos, &d.irot, &d.size, &d.moment, &d.ypos, &d.yrot, &d.vel, &d.avel, &d.dlin, &d.dang, &d.ylin, &d.yang, &d.refPos, &d.refRot, &d.aabb}) A(balloc(b, f, B));
  A(balloc(b, &d.filters, B));
  A(balloc(b, &b->staging, size_t(B) * 10));
  A(balloc(b, &d.cell, B));
  A(balloc(b, &d.colorA, B));
  A(balloc(b, &d.colorB, B));
  A(balloc(b, &d.colorBodies, B));
  A(balloc(b, &d.fixedColor, B));
  A(balloc(b, &d.incCount, B));
  A(balloc(b, &d.adjStart, B + W));
  A(balloc(b, &d.adjFill, B + W));
  A(balloc(b, &d.incStart, B + W));
  A(balloc(b, &d.bucket, W * BUCKET_WORDS));
  A(balloc(b, &d.colorStart, W * (MAX_COLORS + 1)));
  A(balloc(b, &d.scanScratch, W * 2));
  A(balloc(b, &d.counters, W * COUNTER_WORDS));
  A(balloc(b, &d.joint, size_t(b->jointCap) * JOINT_VEC4));
  A(balloc(b, &d.jinfo, b->jointCap));
  A(balloc(b, &b->dWorlds, W));
  A(balloc(b, &b->dOrder, W));
  A(balloc(b, &b->dQueue, 2));
  A(balloc(b, &b->dStatus, 2));
  if (!ok) return bad(AVBD_ERR_CUDA);
  A(cudaMemsetAsync(d.filters, 0xff, B * sizeof(uint2), b->stream));
  A(cudaMallocHost(&b->hStatus, 2 * sizeof(uint32_t)));
  A(cudaEventCreateWithFlags(&b->statusReady, cudaEventDisableTiming));
  A(cudaStreamSynchronize(b->stream));
  if (!ok) return bad(AVBD_ERR_CUDA);
  std::memset(b->hStatus, 0, 2 * sizeof(uint32_t));
  launchShape(b);
  *out = b;
  return AVBD_OK;
}

int avbd_batch_destroy(avbd_batch* b) {
  if (!b) return AVBD_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (void* p : b->allocations) cudaFree(p);
  b->allocations.clear();
  freeRecording(b);
  for (auto& g : b->graph)
    if (g) cudaGraphExecDestroy(g);
  if (b->hStatus) cudaFreeHost(b->hStatus);
  if (b->statusReady) cudaEventDestroy(b->statusReady);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return AVBD_OK;
}

const char* avbd_batch_last_error(const avbd_batch* b) { return b ? b->error.c_str() : "no batch"; }

int avbd_batch_set_params(avbd_batch* b, const avbd_params* p) {
  if (!b || !p) return AVBD_ERR_INVALID;
  if (!(p->dt > 0.0f) || p->iterations < 0 || !std::isfinite(p->gravity)) return bfail(b, AVBD_ERR_INVALID, "dt must be positive, iterations non-negative");
  if (!std::isfinite(p->wind_speed) || !std::isfinite(p->wind_angle) || !std::isfinite(p->wind_gust) || !(p->wind_pressure >= 0.0f) ||
      !std::isfinite(p->wind_pressure))
    return bfail(b, AVBD_ERR_INVALID, "the wind's values must be finite, wind_pressure >= 0");
  b->params = *p;
  b->configGen++;
  return AVBD_OK;
}

int avbd_batch_add_world(avbd_batch* b, const avbd_body* bodies, uint32_t n, const avbd_joint* joints, const avbd_joint_info* info, uint32_t nj,
                         const uint32_t* ignore_ab, uint32_t n_ignore, uint32_t* index) {
  if (!b || !bodies || (nj && (!joints || !info)) || (n_ignore && !ignore_ab)) return AVBD_ERR_INVALID;
  if (n == 0 || n > BATCH_MAX_WORLD_BODIES)
    return bfail(b, AVBD_ERR_INVALID, "a batched world holds 1 to " + std::to_string(BATCH_MAX_WORLD_BODIES) + " bodies");
  if (b->worlds.size() >= b->worldCap) return bfail(b, AVBD_ERR_CAPACITY, "world capacity " + std::to_string(b->worldCap) + " reached");
  if (b->rec.K) return bfail(b, AVBD_ERR_INVALID, "a recording is in progress: adopt it (avbd_adjoint_create_from_batch) before adding worlds");
  if (uint64_t(b->n) + n > b->bodyCap) return bfail(b, AVBD_ERR_CAPACITY, "body capacity " + std::to_string(b->bodyCap) + " reached");
  if (uint64_t(b->nj) + nj > b->jointCap) return bfail(b, AVBD_ERR_CAPACITY, "joint capacity " + std::to_string(b->jointCap) + " reached");
  std::string msg = bodyProblem(bodies, n);
  for (uint32_t i = 0; i < n && msg.empty(); i++)
    if (!(bodies[i].shape == 0.0f || bodies[i].shape == 1.0f || bodies[i].shape == 2.0f)) msg = "batched worlds hold boxes, spheres and sails";
  if (msg.empty()) msg = jointProblem(joints, info, nj, n);
  for (uint32_t i = 0; i < n_ignore && msg.empty(); i++)
    if (ignore_ab[2 * i] >= n || ignore_ab[2 * i + 1] >= n || ignore_ab[2 * i] == ignore_ab[2 * i + 1]) msg = "ignore pair out of range";
  if (!msg.empty()) return bfail(b, AVBD_ERR_INVALID, msg);
  cudaSetDevice(b->device);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  std::vector<double> radii(n);
  for (uint32_t i = 0; i < n; i++) radii[i] = bodies[i].radius;
  std::vector<NoCollide> nocollide;
  for (uint32_t i = 0; i < nj; i++)
    if (info[i].a >= 0 && info[i].type != AVBD_T_NONE) {
      uint32_t a = uint32_t(info[i].a), c = uint32_t(info[i].b);
      nocollide.push_back({std::max(a, c), std::min(a, c), i});
    }
  for (uint32_t i = 0; i < n_ignore; i++)
    nocollide.push_back({std::max(ignore_ab[2 * i], ignore_ab[2 * i + 1]), std::min(ignore_ab[2 * i], ignore_ab[2 * i + 1]), 0xffffffffu});
  std::stable_sort(nocollide.begin(), nocollide.end());
  const uint32_t first = b->n, firstJoint = b->nj;
  int r = appendWorld(b, n, nj, std::max<uint32_t>(32, b->pairsPerBody * n), largeThreshold(radii), nocollide, 0u, index);
  if (r) return r;
  std::vector<avbd_body> copy(bodies, bodies + n);
  for (auto& x : copy) x.flags = float((uint32_t(x.flags) & 6u) | 1u);  // new slots: no contact history
  bodiesIn(b, first, copy.data(), n, cudaMemcpyHostToDevice);
  std::vector<uint32_t> none(n, NO_COLOR);
  BATCH_TRY(b, cudaMemcpyAsync(b->d.colorA + first, none.data(), size_t(n) * 4, cudaMemcpyHostToDevice, b->stream));
  if (nj) {
    BATCH_TRY(b, cudaMemcpyAsync(b->d.joint + size_t(firstJoint) * JOINT_VEC4, joints, size_t(nj) * sizeof(avbd_joint), cudaMemcpyHostToDevice, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(b->d.jinfo + firstJoint, info, size_t(nj) * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
  }
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  return AVBD_OK;
}

int avbd_batch_add_world_from(avbd_batch* b, avbd_world* src, uint32_t* index) {
  if (!b || !src) return AVBD_ERR_INVALID;
  if (src->device != b->device) return bfail(b, AVBD_ERR_INVALID, "the world is on another device");
  if (!src->hullWords.empty()) return bfail(b, AVBD_ERR_INVALID, "batched worlds hold boxes, spheres and sails");
  if (b->rec.K) return bfail(b, AVBD_ERR_INVALID, "a recording is in progress: adopt it (avbd_adjoint_create_from_batch) before adding worlds");
  const uint32_t n = src->n, nj = src->nj;
  if (n == 0 || n > BATCH_MAX_WORLD_BODIES)
    return bfail(b, AVBD_ERR_INVALID, "a batched world holds 1 to " + std::to_string(BATCH_MAX_WORLD_BODIES) + " bodies");
  if (b->worlds.size() >= b->worldCap) return bfail(b, AVBD_ERR_CAPACITY, "world capacity " + std::to_string(b->worldCap) + " reached");
  if (b->rec.K) return bfail(b, AVBD_ERR_INVALID, "a recording is in progress: adopt it (avbd_adjoint_create_from_batch) before adding worlds");
  if (uint64_t(b->n) + n > b->bodyCap) return bfail(b, AVBD_ERR_CAPACITY, "body capacity " + std::to_string(b->bodyCap) + " reached");
  if (uint64_t(b->nj) + nj > b->jointCap) return bfail(b, AVBD_ERR_CAPACITY, "joint capacity " + std::to_string(b->jointCap) + " reached");
  cudaSetDevice(b->device);
  if (avbd_synchronize(src) != AVBD_OK) return bfail(b, AVBD_ERR_CUDA, std::string("source world: ") + src->error);
  if (src->staticsDirty && uploadStatics(src) != AVBD_OK) return bfail(b, AVBD_ERR_CUDA, std::string("source world: ") + src->error);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  // last step's contact pairs (the buffer the next step reads)
  std::vector<uint32_t> ctr(COUNTER_WORDS);
  BATCH_TRY(b, copyToHost(ctr.data(), src->d.counters, COUNTER_WORDS * 4, b->stream));
  const uint32_t prevPairs = std::min(ctr[C_PAIRS], src->pairCap);
  const uint32_t first = b->n, firstJoint = b->nj;
  uint32_t pairCap = std::max<uint32_t>(std::max<uint32_t>(32, b->pairsPerBody * n), 2 * prevPairs);
  int r = appendWorld(b, n, nj, pairCap, src->threshold, src->nocollide, src->fixedColors ? WORLD_FIXED_COLORS : 0u, index);
  if (r) return r;
  const WorldDesc& w = b->worlds.back();
  const DWorld& s = src->d;
  DWorld& d = b->d;
  const float4* sf[10] = {s.pos, s.rot, s.ipos, s.irot, s.size, s.moment, s.ypos, s.yrot, s.vel, s.avel};
  float4* df[10] = {d.pos, d.rot, d.ipos, d.irot, d.size, d.moment, d.ypos, d.yrot, d.vel, d.avel};
  const cudaMemcpyKind DD = cudaMemcpyDeviceToDevice;
  for (int f = 0; f < 10; f++) BATCH_TRY(b, cudaMemcpyAsync(df[f] + first, sf[f], size_t(n) * sizeof(float4), DD, b->stream));
  BATCH_TRY(b, cudaMemcpyAsync(d.filters + first, s.filters, size_t(n) * sizeof(uint2), DD, b->stream));
  BATCH_TRY(b, cudaMemcpyAsync(d.colorA + first, s.colorA, size_t(n) * 4, DD, b->stream));
  BATCH_TRY(b, cudaMemcpyAsync(d.fixedColor + first, s.fixedColor, size_t(n) * 4, DD, b->stream));
  if (nj) {
    BATCH_TRY(b, cudaMemcpyAsync(d.joint + size_t(firstJoint) * JOINT_VEC4, s.joint, size_t(nj) * JOINT_VEC4 * sizeof(float4), DD, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(d.jinfo + firstJoint, s.jinfo, size_t(nj) * sizeof(int4), DD, b->stream));
  }
  const size_t wi = b->worlds.size() - 1;
  BATCH_TRY(b, cudaMemcpyAsync(d.counters + wi * COUNTER_WORDS, s.counters, COUNTER_WORDS * 4, DD, b->stream));
  const int sp = 1 - src->cur, bp = 1 - b->cur;
  if (prevPairs) {
    BATCH_TRY(b, cudaMemcpyAsync(d.mIds[bp] + w.pair, s.mIds[sp], size_t(prevPairs) * sizeof(uint4), DD, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(d.mGeo[bp] + w.pair, s.mGeo[sp], size_t(prevPairs) * sizeof(float4), DD, b->stream));
    BATCH_TRY(b, cudaMemcpyAsync(d.cPt[bp] + size_t(w.pair) * MAX_CONTACTS * 4, s.cPt[sp], size_t(prevPairs) * MAX_CONTACTS * 4 * sizeof(float4), DD,
                                 b->stream));
  }
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  return AVBD_OK;
}

int avbd_batch_world_info(avbd_batch* b, uint32_t world, avbd_batch_world* out) {
  int r = checkWorld(b, world);
  if (r) return r;
  if (!out) return AVBD_ERR_INVALID;
  const WorldDesc& w = b->worlds[world];
  out->first_body = w.body;
  out->bodies = w.n;
  out->first_joint = w.joint;
  out->joints = w.nj;
  out->pair_capacity = w.pairCap;
  out->fixed_colors = (w.flags & WORLD_FIXED_COLORS) ? 1u : 0u;
  return AVBD_OK;
}

int avbd_batch_step(avbd_batch* b, int steps) {
  if (!b || steps < 0) return AVBD_ERR_INVALID;
  if (b->worlds.empty()) return bfail(b, AVBD_ERR_INVALID, "the batch has no worlds");
  cudaSetDevice(b->device);
  for (int s = 0; s < steps; s++) {
    int r = adaptBatch(b, false);
    if (r) return r;
    if (b->tableDirty) {
      r = uploadTable(b);
      if (r) return r;
      launchShape(b);
    }
    b->stepCount++;
    BatchLaunch L = makeLaunch(b);
    bool launched = false;
    if (b->useGraphs) {
      const int c = b->cur;
      if (!b->graph[c] || b->graphGen[c] != b->configGen) {
        if (b->graph[c]) cudaGraphExecDestroy(b->graph[c]);
        b->graph[c] = nullptr;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          cudaError_t le = enqueueStep(b, L);
          e = cudaStreamEndCapture(b->stream, &g);
          if (e == cudaSuccess && le == cudaSuccess) e = cudaGraphInstantiate(&b->graph[c], g, 0);
          else if (e == cudaSuccess) e = le;
          if (g) cudaGraphDestroy(g);
        }
        if (e != cudaSuccess) {
          cudaGetLastError();
          b->useGraphs = false;
          if (b->graph[c]) cudaGraphExecDestroy(b->graph[c]);
          b->graph[c] = nullptr;
        } else {
          b->graphGen[c] = b->configGen;
        }
      }
      if (b->graph[c]) {
        BATCH_TRY(b, cudaGraphLaunch(b->graph[c], b->stream));
        launched = true;
      }
    }
    if (!launched) BATCH_TRY(b, enqueueStep(b, L));
    if (b->rec.done < b->rec.K) {
      BATCH_TRY(b, launch_record_step(L, b->rec.d, b->rec.done, b->sms * 8, b->stream));
      b->rec.done++;
    }
    BATCH_TRY(b, cudaEventRecord(b->statusReady, b->stream));
    b->statusInFlight = true;
    b->cur = 1 - b->cur;
  }
  return AVBD_OK;
}

int avbd_batch_synchronize(avbd_batch* b) {
  if (!b) return AVBD_ERR_INVALID;
  cudaSetDevice(b->device);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  if (b->statusInFlight && b->hStatus[1]) {
    uint32_t bits = b->hStatus[1];
    int r = adaptBatch(b, true);
    if (r) return r;
    return bfail(b, AVBD_ERR_TIMEOUT, "a world's step gave up: error bits " + std::to_string(bits));
  }
  return adaptBatch(b, true);
}

int avbd_batch_read_bodies(avbd_batch* b, uint32_t world, avbd_body* dst, uint32_t cap, uint32_t* n) {
  int r = checkWorld(b, world);
  if (r) return r;
  const WorldDesc& w = b->worlds[world];
  if (n) *n = w.n;
  if (!dst) return AVBD_OK;
  if (cap < w.n) return bfail(b, AVBD_ERR_CAPACITY, "destination holds fewer bodies than the world");
  cudaSetDevice(b->device);
  bodiesOut(b, w.body, dst, w.n);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  return AVBD_OK;
}

int avbd_batch_read_all_bodies_async(avbd_batch* b, avbd_body* dst, uint32_t cap) {
  if (!b || !dst) return AVBD_ERR_INVALID;
  if (cap < b->n) return bfail(b, AVBD_ERR_CAPACITY, "destination holds fewer bodies than the batch");
  cudaSetDevice(b->device);
  bodiesOut(b, 0, dst, b->n);
  BATCH_TRY(b, cudaGetLastError());
  return AVBD_OK;
}

int avbd_batch_write_all_bodies_async(avbd_batch* b, const avbd_body* src, uint32_t n) {
  if (!b || !src) return AVBD_ERR_INVALID;
  if (n != b->n) return bfail(b, AVBD_ERR_INVALID, "one record per body of the batch is needed");
  cudaSetDevice(b->device);
  bodiesIn(b, 0, src, n, cudaMemcpyHostToDevice);
  BATCH_TRY(b, cudaGetLastError());
  return AVBD_OK;
}

int avbd_batch_read_joints(avbd_batch* b, uint32_t world, avbd_joint* dst, avbd_joint_info* info, uint32_t cap, uint32_t* n) {
  int r = checkWorld(b, world);
  if (r) return r;
  const WorldDesc& w = b->worlds[world];
  if (n) *n = w.nj;
  if (!dst && !info) return AVBD_OK;
  if (cap < w.nj) return bfail(b, AVBD_ERR_CAPACITY, "destination holds fewer joints than the world");
  cudaSetDevice(b->device);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  if (dst && w.nj)
    BATCH_TRY(b, copyToHost(dst, b->d.joint + size_t(w.joint) * JOINT_VEC4, size_t(w.nj) * sizeof(avbd_joint), b->stream));
  if (info && w.nj) BATCH_TRY(b, copyToHost(info, b->d.jinfo + w.joint, size_t(w.nj) * sizeof(avbd_joint_info), b->stream));
  return AVBD_OK;
}

int avbd_batch_read_colors(avbd_batch* b, uint32_t world, uint32_t* dst, uint32_t cap, uint32_t* n) {
  int r = checkWorld(b, world);
  if (r) return r;
  const WorldDesc& w = b->worlds[world];
  if (n) *n = w.n;
  if (!dst) return AVBD_OK;
  if (cap < w.n) return bfail(b, AVBD_ERR_CAPACITY, "destination holds fewer entries than the world's bodies");
  cudaSetDevice(b->device);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  BATCH_TRY(b, copyToHost(dst, b->d.colorA + w.body, size_t(w.n) * 4, b->stream));
  return AVBD_OK;
}

int avbd_batch_read_counters(avbd_batch* b, uint32_t world, avbd_counters* out) {
  int r = checkWorld(b, world);
  if (r) return r;
  if (!out) return AVBD_ERR_INVALID;
  cudaSetDevice(b->device);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  uint32_t c[COUNTER_WORDS];
  BATCH_TRY(b, copyToHost(c, b->d.counters + size_t(world) * COUNTER_WORDS, sizeof(c), b->stream));
  std::memset(out, 0, sizeof(*out));
  out->pairs = c[C_PAIRS];
  out->contacts = c[C_CONTACTS];
  out->manifolds = c[C_MANIFOLDS];
  out->overflow = c[C_OVERFLOW];
  out->clashes = c[C_CLASHES];
  out->colors = c[C_COLORS];
  out->rounds = c[C_ROUNDS];
  out->error = c[C_ERROR];
  out->steps = c[C_STEP];
  out->pair_capacity = b->worlds[world].pairCap;
  out->graphs = (b->useGraphs && b->graph[0] != nullptr) || (b->useGraphs && b->graph[1] != nullptr) ? 1u : 0u;
  out->launches = 2;
  return AVBD_OK;
}

int avbd_batch_use_graphs(avbd_batch* b, int enable) {
  if (!b) return AVBD_ERR_INVALID;
  b->useGraphs = enable != 0;
  b->configGen++;
  return AVBD_OK;
}

int avbd_batch_stream(avbd_batch* b, void** stream) {
  if (!b || !stream) return AVBD_ERR_INVALID;
  *stream = b->stream;
  return AVBD_OK;
}

int avbd_batch_tune(avbd_batch* b, int steps, avbd_batch_tuning* out) {
  if (!b || steps <= 0) return AVBD_ERR_INVALID;
  if (b->worlds.empty()) return bfail(b, AVBD_ERR_INVALID, "the batch has no worlds");
  cudaSetDevice(b->device);
  int r = avbd_batch_synchronize(b);
  if (r) return r;
  const int threads[3] = {64, 128, 256};
  avbd_batch_tuning t{};
  cudaEvent_t e0, e1;
  BATCH_TRY(b, cudaEventCreate(&e0));
  BATCH_TRY(b, cudaEventCreate(&e1));
  float best = INFINITY;
  int bestT = b->collideThreads, bestS = b->solveBlocks, bestW = b->worldThreads;
  uint32_t bestR = b->rowsPerLane;
  const bool graphs = b->useGraphs;
  b->useGraphs = false;
  uint32_t k = 0;
  // one candidate: its mean step time over `steps` after one step that settles storage for the shape
  auto trial = [&](int ct, int sb, uint32_t rpl, int wt) -> int {
    if (k >= AVBD_BATCH_TUNE_CANDIDATES) return AVBD_OK;
    b->collideThreads = ct;
    b->solveBlocks = sb;
    b->rowsPerLane = rpl;
    b->worldThreads = wt;
    launchShape(b);
    int rr = avbd_batch_step(b, 1);
    if (!rr) rr = avbd_batch_synchronize(b);
    if (rr) return rr;
    cudaEventRecord(e0, b->stream);
    rr = avbd_batch_step(b, steps);
    cudaEventRecord(e1, b->stream);
    if (!rr) rr = avbd_batch_synchronize(b);
    if (rr) return rr;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= float(steps);
    t.candidate_threads[k] = uint32_t(ct);
    t.candidate_solve_blocks[k] = uint32_t(sb);
    t.candidate_rows_per_lane[k] = rpl;
    t.candidate_world_threads[k] = uint32_t(wt);
    t.candidate_ms[k] = ms;
    k++;
    if (ms < best) {
      best = ms;
      bestT = ct;
      bestS = sb;
      bestR = rpl;
      bestW = wt;
    }
    return AVBD_OK;
  };
  // The collision and the solve are separate launches whose times add, so the collision block size
  // is chosen first (under the starting solve shape), then the solve's shape: a block or a warp a
  // world, resident blocks an SM, and the least rows a lane (1, or 4: bodies per warp).
  const int startS = b->solveBlocks > 0 ? b->solveBlocks : b->sms * std::max(1, batch_solve_blocks_per_sm(b->worldThreads));
  for (int ti = 0; ti < 3 && !r; ti++) r = trial(threads[ti], startS, b->rowsPerLane, b->worldThreads);
  const int collideBest = bestT;
  const int worldThreads[4] = {256, 128, 64, 32};
  for (int wi = 0; wi < 4 && !r; wi++) {
    const int per = std::max(1, batch_solve_blocks_per_sm(worldThreads[wi]));
    for (int sp = 1; sp <= per && !r; sp++) r = trial(collideBest, b->sms * sp, 1, worldThreads[wi]);
  }
  // then bodies per warp: four rows a lane at least, in the fastest scope and block count so far
  if (!r) r = trial(bestT, bestS, 4, bestW);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->useGraphs = graphs;
  b->collideThreads = bestT;
  b->solveBlocks = bestS;
  b->rowsPerLane = bestR;
  b->worldThreads = bestW;
  launchShape(b);
  b->configGen++;
  if (r) return r;
  t.candidates = k;
  t.collide_threads = uint32_t(bestT);
  t.solve_blocks = uint32_t(bestS);
  t.rows_per_lane = bestR;
  t.world_threads = uint32_t(bestW);
  t.ms_per_step = best;
  t.steps_taken = k * uint32_t(steps + 1);
  if (out) *out = t;
  return AVBD_OK;
}

int avbd_batch_record_start(avbd_batch* b, uint32_t steps, uint32_t points_per_body) {
  if (!b || steps == 0) return AVBD_ERR_INVALID;
  if (b->worlds.empty()) return bfail(b, AVBD_ERR_INVALID, "the batch has no worlds");
  if (b->nj) return bfail(b, AVBD_ERR_INVALID, "the adjoint differentiates contacts only: the batch holds joints");
  const avbd_params& P = b->params;
  if (P.flags & (AVBD_FLAG_MATCH_NEAREST | AVBD_FLAG_MASS_PENALTY | AVBD_FLAG_START_AT_REST | AVBD_FLAG_REUSE_CONTACTS))
    return bfail(b, AVBD_ERR_INVALID, "the adjoint follows the default contact rules: no nearest matching, mass penalty, start at rest or contact reuse");
  if (P.up[0] != 0.0f || P.up[1] != 0.0f || P.up[2] != 1.0f) return bfail(b, AVBD_ERR_INVALID, "the adjoint needs up = +z");
  cudaSetDevice(b->device);
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  std::vector<avbd_body> bodies(b->n);
  bodiesOut(b, 0, bodies.data(), b->n);
  if (P.wind_pressure != 0.0f)
    for (const avbd_body& r : bodies)
      if (r.shape == 2.0f && r.mass > 0.0f) return bfail(b, AVBD_ERR_INVALID, "the adjoint does not differentiate the wind: a dynamic sail with wind_pressure > 0");
  BATCH_TRY(b, cudaStreamSynchronize(b->stream));
  for (auto& x : bodies)
    if (x.shape != float(AVBD_SHAPE_BOX)) return bfail(b, AVBD_ERR_INVALID, "the adjoint differentiates boxes only");
  freeRecording(b);
  const uint64_t ppb = points_per_body ? points_per_body : 8u;
  const uint64_t ptCap = uint64_t(steps) * b->n * ppb, manCap = std::max<uint64_t>(ptCap / 2, 1);
  if (ptCap >= (1ull << 31)) return bfail(b, AVBD_ERR_CAPACITY, "a recording holds fewer than 2^31 points");
  auto& R = b->rec;
  RecordDev& d = R.d;
  d.K = steps;
  d.W = uint32_t(b->worlds.size());
  d.nb = b->n;
  d.manCap = manCap;
  d.ptCap = ptCap;
  int2* ab = nullptr;
  bool ok = recAlloc(b, &d.manFirst, size_t(steps) * (d.W + 1)) && recAlloc(b, &d.ptFirst, size_t(steps) * (d.W + 1)) &&
            recAlloc(b, &d.manCount, d.W) && recAlloc(b, &d.ptCount, d.W) && recAlloc(b, &ab, manCap) && recAlloc(b, &d.basis, 9 * manCap) &&
            recAlloc(b, &d.manSlot, manCap) && recAlloc(b, &d.manPt0, manCap) && recAlloc(b, &d.anchors, 6 * ptCap) &&
            recAlloc(b, &d.ptMan, ptCap) && recAlloc(b, &d.ptPrev, ptCap) && recAlloc(b, &d.color, size_t(steps) * b->n) &&
            recAlloc(b, &d.ncol, size_t(steps) * d.W) && recAlloc(b, &d.totals, 2) && recAlloc(b, &d.status, 2);
  d.manAB = ab;
  if (!ok) {
    freeRecording(b);
    return bfail(b, AVBD_ERR_CUDA, "device memory for the recording");
  }
  R.K = steps;
  R.done = 0;
  R.initial = std::move(bodies);
  R.params = P;
  return AVBD_OK;
}

int avbd_batch_record_status(avbd_batch* b, uint32_t* steps, uint64_t* manifolds, uint64_t* points, uint32_t* problems) {
  if (!b) return AVBD_ERR_INVALID;
  uint32_t status[2] = {0, 0};
  unsigned long long totals[2] = {0, 0};
  if (b->rec.K) {
    cudaSetDevice(b->device);
    BATCH_TRY(b, cudaStreamSynchronize(b->stream));
    BATCH_TRY(b, copyToHost(status, b->rec.d.status, sizeof(status), b->stream));
    BATCH_TRY(b, copyToHost(totals, b->rec.d.totals, sizeof(totals), b->stream));
  }
  if (steps) *steps = b->rec.done;
  if (manifolds) *manifolds = totals[0];
  if (points) *points = totals[1];
  if (problems) *problems = status[0];
  return AVBD_OK;
}

int avbd_batch_set_launch(avbd_batch* b, uint32_t collideThreads, uint32_t solveBlocks, uint32_t rowsPerLane, uint32_t worldThreads) {
  if (!b) return AVBD_ERR_INVALID;
  if (collideThreads != 64 && collideThreads != 128 && collideThreads != 256)
    return bfail(b, AVBD_ERR_INVALID, "collision block size must be 64, 128 or 256");
  if (rowsPerLane < 1 || rowsPerLane > 8) return bfail(b, AVBD_ERR_INVALID, "rows per lane must be 1 to 8");
  if (worldThreads != 32 && worldThreads != 64 && worldThreads != 128 && worldThreads != 256)
    return bfail(b, AVBD_ERR_INVALID, "threads a world must be 32, 64, 128 or 256");
  cudaSetDevice(b->device);
  const int per = std::max(1, batch_solve_blocks_per_sm(int(worldThreads)));
  if (solveBlocks > uint32_t(b->sms * per))
    return bfail(b, AVBD_ERR_INVALID, "solve blocks beyond " + std::to_string(b->sms * per) + " (the blocks that fit)");
  int r = avbd_batch_synchronize(b);
  if (r) return r;
  b->collideThreads = int(collideThreads);
  b->solveBlocks = int(solveBlocks);  // 0: as many as fit (launchShape)
  b->rowsPerLane = rowsPerLane;
  b->worldThreads = int(worldThreads);
  launchShape(b);
  b->configGen++;
  return AVBD_OK;
}

int avbd_batch_info(avbd_batch* b, avbd_batch_status* out) {
  if (!b || !out) return AVBD_ERR_INVALID;
  out->worlds = uint32_t(b->worlds.size());
  out->bodies = b->n;
  out->joints = b->nj;
  out->steps = b->stepCount;
  out->pair_slots = b->pairUsed;
  out->relayouts = b->relayouts;
  out->collide_threads = uint32_t(b->collideThreads);
  out->collide_blocks = uint32_t(b->collideBlocks);
  out->solve_blocks = uint32_t(b->solveBlocks);
  out->graphs = b->useGraphs ? 1u : 0u;
  out->rows_per_lane = b->rowsPerLane;
  out->world_threads = uint32_t(b->worldThreads);
  return AVBD_OK;
}

}  // extern "C"
