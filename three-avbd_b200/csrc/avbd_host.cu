// Host side of the B200 AVBD backend: world storage, the step schedule and the C ABI (include/avbd.h).
//
// Mirrors GpuSolver3D (src/avbd3d/gpu/solver.ts): the host keeps what the CPU owns (body radii and
// masses for the broadphase configuration, joint endpoints, the no-collide list) and uploads it
// when it changes (uploadStatics, solver.ts:1263-1318); everything per step runs on the device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "avbd_host.hpp"

using namespace avbd;

namespace avbd {

uint32_t pow2AtLeast(uint64_t n) {
  uint64_t p = 2;
  while (p < n) p <<= 1;
  return (uint32_t)p;
}

// radii.ts:19-55 (selection, not sorting)
double selectKth(std::vector<double>& a, int k) {
  int lo = 0, hi = int(a.size()) - 1;
  while (lo < hi) {
    double pivot = a[k];
    int i = lo, j = hi;
    do {
      while (a[i] < pivot) i++;
      while (pivot < a[j]) j--;
      if (i <= j) {
        std::swap(a[i], a[j]);
        i++;
        j--;
      }
    } while (i <= j);
    if (j < k) lo = i;
    if (k < i) hi = j;
  }
  return a[k];
}
double largestSmall(std::vector<double> radii) {
  const int n = int(radii.size());
  double median = n > 0 ? selectKth(radii, n >> 1) : 1.0;
  double maxSmall = 0.0;
  for (int i = 0; i < n; i++)
    if (radii[i] <= 2.0 * median) maxSmall = std::max(maxSmall, radii[i]);
  if (n > 64) maxSmall = std::max(maxSmall, selectKth(radii, n - 64 - 1));
  return maxSmall;
}


// Bodies above this bounding radius are "large" (tested against every body): halfway between the
// largest small radius and the smallest large one (solver.ts uploadStatics, radii.ts)
double largeThreshold(const std::vector<double>& radii) {
  double maxSmall = largestSmall(radii);
  double minLarge = INFINITY;
  for (double r : radii)
    if (r > maxSmall) minLarge = std::min(minLarge, r);
  return std::isinf(minLarge) ? maxSmall * 1.5 : (maxSmall + minLarge) / 2;
}

std::string bodyProblem(const avbd_body* b, uint32_t n) {
  for (uint32_t i = 0; i < n; i++) {
    const float* f = reinterpret_cast<const float*>(b + i);
    for (int k = 0; k < 40; k++)
      if (!std::isfinite(f[k])) return "body " + std::to_string(i) + ": non-finite value";
    if (b[i].mass < 0.0f || b[i].radius < 0.0f) return "body " + std::to_string(i) + ": negative mass or radius";
  }
  return {};
}

std::string jointProblem(const avbd_joint* j, const avbd_joint_info* info, uint32_t n, uint32_t bodies) {
  for (uint32_t i = 0; i < n; i++) {
    const avbd_joint_info& in = info[i];
    if (in.type != AVBD_T_JOINT && in.type != AVBD_T_SPRING && in.type != AVBD_T_NONE) return "joint " + std::to_string(i) + ": unknown type";
    if (in.b < 0 || uint32_t(in.b) >= bodies || in.a < -1 || (in.a >= 0 && uint32_t(in.a) >= bodies) || in.a == in.b)
      return "joint " + std::to_string(i) + ": bodies must be distinct indices below the body count (a may be -1)";
    if (in.type == AVBD_T_SPRING && in.a < 0) return "joint " + std::to_string(i) + ": a spring joins two bodies";
    const float* f = reinterpret_cast<const float*>(j + i);
    for (int k = 0; k < 40; k++)
      if (std::isnan(f[k])) return "joint " + std::to_string(i) + ": NaN";
  }
  return {};
}

}  // namespace avbd

namespace {

int fail(avbd_world* w, int code, const std::string& msg) {
  if (w) w->error = msg;
  return code;
}

#define CUDA_TRY(w, call)                                                                    \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) return fail(w, AVBD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
cudaError_t dalloc(avbd_world* w, T** p, size_t count) {
  void* ptr = nullptr;
  cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess) return e;
  w->allocations.push_back(ptr);
  *p = static_cast<T*>(ptr);
  return cudaMemsetAsync(ptr, 0, std::max<size_t>(count, 1) * sizeof(T), w->stream);
}
void dfree(avbd_world* w, void* p) {
  if (!p) return;
  auto it = std::find(w->allocations.begin(), w->allocations.end(), p);
  if (it != w->allocations.end()) w->allocations.erase(it);
  cudaFree(p);
}

// Pair-dependent storage (pairs, both manifold/contact buffers, hash, adjacency and incidence
// lists). On growth last step's buffer (1 - cur) is carried over, so warm starts survive.
int allocPairs(avbd_world* w, uint32_t cap) {
  DWorld& d = w->d;
  const uint32_t oldCap = w->pairCap;
  const int prev = 1 - w->cur;
  uint4* oldIds = d.mIds[prev];
  float4* oldGeo = d.mGeo[prev];
  float4* oldPt = d.cPt[prev];
  uint4* keepIds[2] = {d.mIds[0], d.mIds[1]};
  float4* keepGeo[2] = {d.mGeo[0], d.mGeo[1]};
  float4* keepPt[2] = {d.cPt[0], d.cPt[1]};
  dfree(w, d.pairs);
  dfree(w, d.hash);
  dfree(w, d.adjList);
  dfree(w, d.incList);
  dfree(w, d.laneTable);
  dfree(w, d.hullPairs);
  w->pairCap = cap;
  w->configGen++;
  w->hashSize = pow2AtLeast(2ull * cap);
  w->adjCap = 2u * (cap + w->jointCap);
  w->incCap = 2u * (cap * MAX_CONTACTS + w->jointCap);
  CUDA_TRY(w, dalloc(w, &d.pairs, cap));
  CUDA_TRY(w, dalloc(w, &d.hullPairs, cap));
  CUDA_TRY(w, dalloc(w, &d.hash, w->hashSize));
  CUDA_TRY(w, dalloc(w, &d.adjList, w->adjCap));
  CUDA_TRY(w, dalloc(w, &d.incList, w->incCap));
  CUDA_TRY(w, dalloc(w, &d.laneTable, w->incCap));
  for (int b = 0; b < 2; b++) {
    CUDA_TRY(w, dalloc(w, &d.mIds[b], cap));
    CUDA_TRY(w, dalloc(w, &d.mGeo[b], cap));
    CUDA_TRY(w, dalloc(w, &d.cPt[b], size_t(cap) * MAX_CONTACTS * 4));
  }
  if (oldIds) {
    size_t m = std::min(oldCap, cap);
    CUDA_TRY(w, cudaMemcpyAsync(d.mIds[prev], oldIds, m * sizeof(uint4), cudaMemcpyDeviceToDevice, w->stream));
    CUDA_TRY(w, cudaMemcpyAsync(d.mGeo[prev], oldGeo, m * sizeof(float4), cudaMemcpyDeviceToDevice, w->stream));
    CUDA_TRY(w, cudaMemcpyAsync(d.cPt[prev], oldPt, m * MAX_CONTACTS * 4 * sizeof(float4), cudaMemcpyDeviceToDevice, w->stream));
    CUDA_TRY(w, cudaStreamSynchronize(w->stream));
    for (int b = 0; b < 2; b++) {
      dfree(w, keepIds[b]);
      dfree(w, keepGeo[b]);
      dfree(w, keepPt[b]);
    }
  }
  // the clears above run on the world's stream; host copies that follow use the default stream
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  return AVBD_OK;
}

int allocJoints(avbd_world* w, uint32_t cap) {
  DWorld& d = w->d;
  float4* oldJ = d.joint;
  int4* oldI = d.jinfo;
  float4* nj = nullptr;
  int4* ni = nullptr;
  CUDA_TRY(w, dalloc(w, &nj, size_t(cap) * JOINT_VEC4));
  CUDA_TRY(w, dalloc(w, &ni, cap));
  if (oldJ) {
    CUDA_TRY(w, cudaMemcpyAsync(nj, oldJ, size_t(w->nj) * JOINT_VEC4 * sizeof(float4), cudaMemcpyDeviceToDevice, w->stream));
    CUDA_TRY(w, cudaMemcpyAsync(ni, oldI, size_t(w->nj) * sizeof(int4), cudaMemcpyDeviceToDevice, w->stream));
    CUDA_TRY(w, cudaStreamSynchronize(w->stream));
    dfree(w, oldJ);
    dfree(w, oldI);
  }
  d.joint = nj;
  d.jinfo = ni;
  w->jointCap = cap;
  w->configGen++;
  // adjacency and incidence lists are sized by the joint capacity too
  dfree(w, d.adjList);
  dfree(w, d.incList);
  dfree(w, d.laneTable);
  w->adjCap = 2u * (w->pairCap + w->jointCap);
  w->incCap = 2u * (w->pairCap * MAX_CONTACTS + w->jointCap);
  CUDA_TRY(w, dalloc(w, &d.adjList, w->adjCap));
  CUDA_TRY(w, dalloc(w, &d.incList, w->incCap));
  CUDA_TRY(w, dalloc(w, &d.laneTable, w->incCap));
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  return AVBD_OK;
}

StepParams makeParams(avbd_world* w) {
  StepParams p{};
  const avbd_params& a = w->params;
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
  p.cellSize = w->cellSize;
  p.largeThreshold = w->threshold;
  p.tableMask = w->tableSize - 1;
  p.nLarge = w->nLarge;
  p.nNoCollide = w->nNoCollide;
  p.anyDynamicLarge = w->anyDynamicLarge;
  p.n = w->n;
  p.nj = w->nj;
  p.pairCap = w->pairCap;
  p.hashMask = w->hashSize - 1;
  p.incCap = w->incCap;
  p.adjCap = w->adjCap;
  p.step = w->stepCount;
  p.fixedColors = w->fixedColors ? 1u : 0u;
  p.colorCap = MAX_COLORS;
  p.cur = w->cur;
  return p;
}

// Storage grows past 80 % use or on overflow, to twice the demand (solver.ts:2362-2377).
int adaptCapacity(avbd_world* w, bool wait) {
  if (!w->countersInFlight) return AVBD_OK;
  if (!wait && cudaEventQuery(w->countersReady) != cudaSuccess) return AVBD_OK;
  CUDA_TRY(w, cudaEventSynchronize(w->countersReady));
  w->countersInFlight = false;
  const uint32_t* c = w->hCounters;
  uint32_t demand = c[C_PAIRS];
  if ((c[C_OVERFLOW] & 1u) || uint64_t(demand) * 10 > uint64_t(w->pairCap) * 8) {
    uint64_t want = std::max<uint64_t>(2ull * demand, uint64_t(w->pairCap) * 5 / 4);
    want = std::min<uint64_t>(want, 1ull << 26);
    if (want > w->pairCap) {
      CUDA_TRY(w, cudaStreamSynchronize(w->stream));
      int r = allocPairs(w, uint32_t(want));
      if (r) return r;
    }
  }
  return AVBD_OK;
}

void copyBodiesIn(avbd_world* w, uint32_t first, const avbd_body* b, uint32_t n, cudaMemcpyKind kind) {
  if (kind == cudaMemcpyHostToDevice && w->staging) {  // one contiguous transfer, then a scatter
    cudaMemcpyAsync(w->staging, b, size_t(n) * sizeof(avbd_body), cudaMemcpyHostToDevice, w->stream);
    unpackBodies(w->d, w->staging, first, n, w->stream);
    return;
  }
  float4* fields[10] = {w->d.pos, w->d.rot, w->d.ipos, w->d.irot, w->d.size, w->d.moment, w->d.ypos, w->d.yrot, w->d.vel, w->d.avel};
  for (int f = 0; f < 10; f++)
    cudaMemcpy2DAsync(fields[f] + first, sizeof(float4), reinterpret_cast<const char*>(b) + f * sizeof(float4), sizeof(avbd_body), sizeof(float4), n, kind,
                      w->stream);
}
void copyBodiesOut(avbd_world* w, avbd_body* b, uint32_t n) {
  packBodies(w->d, w->staging, 0, n, w->stream);  // a gather into records, then one contiguous transfer
  cudaMemcpyAsync(b, w->staging, size_t(n) * sizeof(avbd_body), cudaMemcpyDeviceToHost, w->stream);
}

bool finite(float x) { return std::isfinite(x); }

}  // namespace

namespace avbd {

// Body records between the device's field arrays and a contiguous staging array of records, so that
// a host copy is one contiguous transfer (a strided 2D copy moves one 16-byte field per row)
__device__ inline float4* bodyField(const DWorld& d, uint32_t f) {
  switch (f) {
    case 0: return d.pos;
    case 1: return d.rot;
    case 2: return d.ipos;
    case 3: return d.irot;
    case 4: return d.size;
    case 5: return d.moment;
    case 6: return d.ypos;
    case 7: return d.yrot;
    case 8: return d.vel;
    default: return d.avel;
  }
}
static_assert(sizeof(avbd_body) == 10 * sizeof(float4), "a body record is its ten device fields in order");
__global__ void k_pack_bodies(DWorld d, float4* out, uint32_t first, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 10u * n) out[i] = bodyField(d, i % 10u)[first + i / 10u];
}
__global__ void k_unpack_bodies(DWorld d, const float4* in, uint32_t first, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 10u * n) bodyField(d, i % 10u)[first + i / 10u] = in[i];
}
void packBodies(const DWorld& d, float4* staging, uint32_t first, uint32_t n, cudaStream_t s) {
  if (n) k_pack_bodies<<<grid_for(10u * n, 256), 256, 0, s>>>(d, staging, first, n);
}
void unpackBodies(const DWorld& d, const float4* staging, uint32_t first, uint32_t n, cudaStream_t s) {
  if (n) k_unpack_bodies<<<grid_for(10u * n, 256), 256, 0, s>>>(d, staging, first, n);
}


// uploadStatics (solver.ts:1263-1318): large bodies, cell size, sorted no-collide triples
int uploadStatics(avbd_world* w) {
  const uint32_t n = w->n;
  std::vector<double> radii(n);
  for (uint32_t i = 0; i < n; i++) radii[i] = w->radius[i];
  double maxSmall = largestSmall(radii);
  w->threshold = float(largeThreshold(radii));
  w->cellSize = float(std::max(2.0 * maxSmall * (1 + 1e-4), 1e-3));
  std::vector<uint32_t> data;
  w->anyDynamicLarge = 0;
  for (uint32_t i = 0; i < n; i++)
    if (w->radius[i] > w->threshold) {
      data.push_back(i);
      if (w->dynamic[i]) w->anyDynamicLarge = 1;
    }
  w->nLarge = uint32_t(data.size());
  std::stable_sort(w->nocollide.begin(), w->nocollide.end());
  for (auto& e : w->nocollide) {
    data.push_back(e.hi);
    data.push_back(e.lo);
    data.push_back(e.slot);
  }
  w->nNoCollide = uint32_t(w->nocollide.size());
  w->configGen++;
  if (data.size() > w->staticsWords) {
    dfree(w, w->d.large);
    w->staticsWords = uint32_t(std::max<size_t>(data.size() * 2, 64));
    CUDA_TRY(w, dalloc(w, &w->d.large, w->staticsWords));
  }
  if (!data.empty()) CUDA_TRY(w, cudaMemcpyAsync(w->d.large, data.data(), data.size() * 4, cudaMemcpyHostToDevice, w->stream));
  // keep the upload's source alive until it lands (pageable copies are staged synchronously)
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  w->d.nocollide = w->d.large + w->nLarge;
  w->staticsDirty = false;
  return AVBD_OK;
}

}  // namespace avbd

extern "C" {

int avbd_abi_version(void) { return AVBD_ABI_VERSION; }

int avbd_device_info(int device, char* name, size_t cap, int* sms) {
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return AVBD_ERR_NO_DEVICE;
  if (name && cap) {
    std::strncpy(name, prop.name, cap - 1);
    name[cap - 1] = 0;
  }
  if (sms) *sms = prop.multiProcessorCount;
  return AVBD_OK;
}

int avbd_default_params(avbd_params* p) {
  if (!p) return AVBD_ERR_INVALID;
  p->dt = 1.0f / 60.0f;
  p->gravity = -10.0f;
  p->alpha = 0.99f;
  p->beta_lin = 10000.0f;
  p->beta_ang = 100.0f;
  p->gamma = 0.999f;
  p->contact_margin = 0.01f;
  p->iterations = 10;
  p->flags = 0;
  p->up[0] = 0.0f;
  p->up[1] = 0.0f;
  p->up[2] = 1.0f;
  p->wind_speed = 0.0f;
  p->wind_angle = 0.0f;
  p->wind_gust = 0.4f;
  p->wind_pressure = 0.0f;
  return AVBD_OK;
}

int avbd_world_params(avbd_params* p) {
  if (!p) return AVBD_ERR_INVALID;
  avbd_default_params(p);
  p->flags = AVBD_FLAG_MATCH_NEAREST | AVBD_FLAG_FACE_BIAS | AVBD_FLAG_REUSE_CONTACTS | AVBD_FLAG_START_AT_REST | AVBD_FLAG_MASS_PENALTY;
  p->up[0] = 0.0f;
  p->up[1] = 1.0f;
  p->up[2] = 0.0f;
  p->wind_pressure = 0.72f;  // gpu/solver.ts:226-229
  return AVBD_OK;
}

int avbd_world_create(const avbd_config* cfg, avbd_world** out) {
  if (!out) return AVBD_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return AVBD_ERR_NO_DEVICE;
  avbd_world* w = new avbd_world();
  w->device = cfg ? cfg->device : 0;
  if (w->device < 0 || w->device >= count) {
    delete w;
    return AVBD_ERR_INVALID;
  }
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, w->device);
  if (prop.major < 10) {
    delete w;
    return AVBD_ERR_NO_DEVICE;
  }
  cudaSetDevice(w->device);
  avbd_default_params(&w->params);
  w->bodyCap = cfg && cfg->body_capacity ? cfg->body_capacity : 1024;
  if (w->bodyCap > (1u << 30)) {  // body indices share a word with two flag bits in the incidence list
    delete w;
    return AVBD_ERR_INVALID;
  }
  w->jointCap = cfg && cfg->joint_capacity ? cfg->joint_capacity : 256;
  uint32_t pairCap = cfg && cfg->pair_capacity ? cfg->pair_capacity : std::max<uint32_t>(65536, 8 * w->bodyCap);
  auto bad = [&](int code) {
    avbd_world_destroy(w);
    return code;
  };
  if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess) return bad(AVBD_ERR_CUDA);
  DWorld& d = w->d;
  const uint32_t B = w->bodyCap;
  w->tableSize = pow2AtLeast(2ull * B);
  w->sortTiles = (B + 8191) / 8192;
  w->solveBlocks = w->maxSolveBlocks = solve_grid_blocks(w->device);
  bool ok = true;
  auto A = [&](cudaError_t e) { ok = ok && e == cudaSuccess; };
  for (float4** f : {&d.pos, &d.rot, &d.ipos, &d.irot, &d.size, &d.moment, &d.ypos, &d.yrot, &d.vel, &d.avel}) A(dalloc(w, f, B));
  A(dalloc(w, &w->staging, size_t(B) * 10));
  A(dalloc(w, &d.aux, B));
  if (ok) {  // every slot at the default aux record: gravity scale 1, no damping
    std::vector<float4> aux(B, make_float4(1.0f, 0.0f, 0.0f, 0.0f));
    A(copyToDevice(d.aux, aux.data(), size_t(B) * sizeof(float4), w->stream));
  }
  A(dalloc(w, &d.filters, B));
  A(dalloc(w, &d.keyA, B));
  A(dalloc(w, &d.keyB, B));
  A(dalloc(w, &d.valA, B));
  A(dalloc(w, &d.valB, B));
  A(dalloc(w, &d.radixHist, size_t(w->tableSize) / 4096 + 2));
  A(dalloc(w, &d.cell, B));
  A(dalloc(w, &d.sortedPR, B));
  A(dalloc(w, &d.sortedCell, B));
  A(dalloc(w, &d.aabb, B));
  A(dalloc(w, &d.sortedAabb, B));
  A(dalloc(w, &d.cellStart, w->tableSize));
  A(dalloc(w, &d.cellEnd, w->tableSize));
  A(dalloc(w, &d.adjStart, B + 1));
  A(dalloc(w, &d.adjFill, B + 1));
  A(dalloc(w, &d.colorA, B));
  A(dalloc(w, &d.colorB, B));
  A(dalloc(w, &d.colorHist, size_t(MAX_COLORS) * w->solveBlocks + 1));
  A(dalloc(w, &d.colorStart, MAX_COLORS + 1));
  A(dalloc(w, &d.colorBodies, B));
  A(dalloc(w, &d.fixedColor, B));
  A(dalloc(w, &d.incStart, B + 1));
  A(dalloc(w, &d.incCount, B));
  A(dalloc(w, &d.bucket, BUCKET_WORDS));
  A(dalloc(w, &d.dlin, B));
  A(dalloc(w, &d.dang, B));
  A(dalloc(w, &d.ylin, B));
  A(dalloc(w, &d.yang, B));
  A(dalloc(w, &d.refPos, B));
  A(dalloc(w, &d.refRot, B));
  A(dalloc(w, &d.done, B));
  A(dalloc(w, &d.poseDone, B));
  A(dalloc(w, &d.scanScratch, w->solveBlocks + 1));
  A(dalloc(w, &d.counters, COUNTER_WORDS));
  A(dalloc(w, &d.barrier, 2));
  A(dalloc(w, &d.clocks, CLOCK_WORDS));
  if (!ok) return bad(AVBD_ERR_CUDA);
  // every body in every group, colliding with every group; colours start unset
  A(cudaMemsetAsync(d.filters, 0xff, size_t(B) * sizeof(uint2), w->stream));
  A(cudaStreamSynchronize(w->stream));
  {
    std::vector<uint32_t> none(B, NO_COLOR);
    A(copyToDevice(d.colorA, none.data(), size_t(B) * 4, w->stream));
  }
  if (!ok) return bad(AVBD_ERR_CUDA);
  w->pairCap = 0;
  if (allocPairs(w, pairCap) != AVBD_OK) return bad(AVBD_ERR_CUDA);
  if (allocJoints(w, w->jointCap) != AVBD_OK) return bad(AVBD_ERR_CUDA);
  if (uploadStatics(w) != AVBD_OK) return bad(AVBD_ERR_CUDA);
  if (cudaMallocHost(&w->hCounters, COUNTER_WORDS * sizeof(uint32_t)) != cudaSuccess) return bad(AVBD_ERR_CUDA);
  std::memset(w->hCounters, 0, COUNTER_WORDS * sizeof(uint32_t));
  if (cudaEventCreateWithFlags(&w->countersReady, cudaEventDisableTiming) != cudaSuccess) return bad(AVBD_ERR_CUDA);
  if (cudaStreamSynchronize(w->stream) != cudaSuccess) return bad(AVBD_ERR_CUDA);
  *out = w;
  return AVBD_OK;
}

int avbd_world_destroy(avbd_world* w) {
  if (!w) return AVBD_OK;
  cudaSetDevice(w->device);
  if (w->stream) cudaStreamSynchronize(w->stream);
  for (void* p : w->allocations) cudaFree(p);
  w->allocations.clear();
  if (w->hCounters) cudaFreeHost(w->hCounters);
  for (auto& gk : w->graph)
    for (auto& g : gk)
      if (g) cudaGraphExecDestroy(g);
  if (w->countersReady) cudaEventDestroy(w->countersReady);

  if (w->stream) cudaStreamDestroy(w->stream);
  delete w;
  return AVBD_OK;
}

const char* avbd_last_error(const avbd_world* w) { return w ? w->error.c_str() : "no world"; }

int avbd_set_params(avbd_world* w, const avbd_params* p) {
  if (!w || !p) return AVBD_ERR_INVALID;
  if (!(p->dt > 0.0f) || !finite(p->dt) || !finite(p->gravity) || !finite(p->alpha) || !finite(p->gamma) || p->iterations < 0 ||
      !(p->contact_margin >= 0.0f) || !finite(p->contact_margin) || !finite(p->wind_speed) || !finite(p->wind_angle) || !finite(p->wind_gust) ||
      !(p->wind_pressure >= 0.0f) || !finite(p->wind_pressure))
    return fail(w, AVBD_ERR_INVALID, "invalid params (dt > 0, finite values, iterations >= 0, contact_margin >= 0, wind_pressure >= 0)");
  w->params = *p;
  w->configGen++;
  return AVBD_OK;
}

int avbd_get_params(const avbd_world* w, avbd_params* p) {
  if (!w || !p) return AVBD_ERR_INVALID;
  *p = w->params;
  return AVBD_OK;
}

static int checkBodies(avbd_world* w, const avbd_body* b, uint32_t n) {
  std::string msg = bodyProblem(b, n);
  if (!msg.empty()) return fail(w, AVBD_ERR_INVALID, msg);
  // a shape code is a box, sphere or sail, or SHAPE_HULL + the header offset of a hull of this world
  for (uint32_t i = 0; i < n; i++) {
    float s = b[i].shape;
    if (s == 0.0f || s == 1.0f || s == 2.0f) continue;
    float h = s - float(AVBD_SHAPE_HULL);
    if (!(h >= 0.0f) || h != std::floor(h) || !w->hullStarts.count(uint32_t(h)))
      return fail(w, AVBD_ERR_INVALID, "body " + std::to_string(i) + ": shape " + std::to_string(s) + " is no box, sphere, sail or hull of this world");
  }
  return AVBD_OK;
}

// A packed hull record (header at vec4 0): counts within the narrowphase's limits, every block and
// index inside the record, finite planes and vertices
static std::string hullProblem(const uint32_t* u, uint32_t vec4s) {
  if (vec4s < 2) return "a hull record holds at least its header";
  const uint32_t vs = u[0], nv = u[1], fs = u[2], nf = u[3], es = u[4], ne = u[5], is = u[6];
  if (nv < 4 || nv > AVBD_MAX_HULL_VERTICES || nf < 4 || nf > 255 || ne < 6 || ne > 255) return "hull counts out of range";
  auto inside = [&](uint64_t start, uint64_t count) { return start >= 2 && start + count <= vec4s; };
  if (!inside(vs, nv) || !inside(fs, 2ull * nf) || !inside(es, ne) || !(is >= 2 && is < vec4s)) return "hull blocks outside the record";
  auto finite = [&](uint32_t word) {
    float f;
    std::memcpy(&f, &u[word], 4);
    return std::isfinite(f);
  };
  for (uint32_t v = 0; v < nv; v++)
    for (int k = 0; k < 3; k++)
      if (!finite((vs + v) * 4 + k)) return "hull vertex not finite";
  for (uint32_t f = 0; f < nf; f++) {
    const uint32_t o = (fs + 2 * f) * 4;
    for (int k = 0; k < 4; k++)
      if (!finite(o + k)) return "hull face plane not finite";
    const uint32_t first = u[o + 4], count = u[o + 5];
    if (count < 3 || count > nv || uint64_t(is) * 4 + first + count > uint64_t(vec4s) * 4) return "hull face indices outside the record";
    for (uint32_t j = 0; j < count; j++)
      if (u[is * 4 + first + j] >= nv) return "hull face vertex out of range";
  }
  for (uint32_t e = 0; e < ne; e++) {
    const uint32_t* q = u + (es + e) * 4;
    if (q[0] >= nv || q[1] >= nv || q[2] >= nf || q[3] >= nf) return "hull edge out of range";
  }
  return {};
}

int avbd_add_bodies(avbd_world* w, const avbd_body* bodies, uint32_t n, uint32_t* first) {
  if (!w || (!bodies && n)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (uint64_t(w->n) + n > w->bodyCap) return fail(w, AVBD_ERR_CAPACITY, "body capacity " + std::to_string(w->bodyCap) + " reached");
  int r = checkBodies(w, bodies, n);
  if (r) return r;
  uint32_t at = w->n;
  if (first) *first = at;
  if (n == 0) return AVBD_OK;
  return avbd_write_bodies(w, at, bodies, n, 0) == AVBD_OK ? AVBD_OK : AVBD_ERR_CUDA;
}

int avbd_write_bodies(avbd_world* w, uint32_t first, const avbd_body* bodies, uint32_t n, int keep_contacts) {
  if (!w || (!bodies && n)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (uint64_t(first) + n > w->bodyCap || first > w->n) return fail(w, AVBD_ERR_INVALID, "body range outside the world");
  int r = checkBodies(w, bodies, n);
  if (r) return r;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  std::vector<avbd_body> copy(bodies, bodies + n);
  for (auto& b : copy) {
    uint32_t flags = uint32_t(b.flags) & 6u;
    b.flags = float(keep_contacts ? flags : (flags | 1u));
  }
  copyBodiesIn(w, first, copy.data(), n, cudaMemcpyHostToDevice);
  if (!keep_contacts) {
    std::vector<uint32_t> none(n, NO_COLOR);
    CUDA_TRY(w, cudaMemcpyAsync(w->d.colorA + first, none.data(), size_t(n) * 4, cudaMemcpyHostToDevice, w->stream));
  }
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (w->radius.size() < first + n) {
    w->radius.resize(first + n);
    w->dynamic.resize(first + n);
  }
  for (uint32_t i = 0; i < n; i++) {
    if (w->radius[first + i] != bodies[i].radius || w->dynamic[first + i] != (bodies[i].mass > 0.0f)) w->staticsDirty = true;
    w->radius[first + i] = bodies[i].radius;
    w->dynamic[first + i] = bodies[i].mass > 0.0f;
  }
  if (first + n > w->n) {
    w->n = first + n;
    w->staticsDirty = true;
  }
  return AVBD_OK;
}

// rewriteBodies(indices, bodies) (gpu/solver.ts:1774-1784): every record checked first, then one
// write per run of consecutive slots, each slot starting afresh (no contact history, no colour)
int avbd_write_bodies_at(avbd_world* w, const uint32_t* indices, const avbd_body* bodies, uint32_t n) {
  if (!w || (n && (!indices || !bodies))) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  for (uint32_t k = 0; k < n; k++)
    if (indices[k] >= w->n) return fail(w, AVBD_ERR_INVALID, "rewriteBodies: slot " + std::to_string(indices[k]) + " is not a body of the world");
  int r = checkBodies(w, bodies, n);
  if (r) return r;
  for (uint32_t k = 0; k < n;) {
    uint32_t e = k + 1;
    while (e < n && indices[e] == indices[e - 1] + 1) e++;
    r = avbd_write_bodies(w, indices[k], bodies + k, e - k, 0);
    if (r) return r;
    k = e;
  }
  return AVBD_OK;
}

static int checkJoints(avbd_world* w, const avbd_joint* j, const avbd_joint_info* info, uint32_t n) {
  std::string msg = jointProblem(j, info, n, w->n);
  return msg.empty() ? AVBD_OK : fail(w, AVBD_ERR_INVALID, msg);
}

int avbd_write_joints(avbd_world* w, uint32_t first, const avbd_joint* joints, const avbd_joint_info* info, uint32_t n) {
  if (!w || (n && (!joints || !info))) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (uint64_t(first) + n > w->nj) return fail(w, AVBD_ERR_INVALID, "joint range outside the world's slots");
  int r = checkJoints(w, joints, info, n);
  if (r) return r;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  CUDA_TRY(w, copyToDevice(w->d.joint + size_t(first) * JOINT_VEC4, joints, size_t(n) * sizeof(avbd_joint), w->stream));
  CUDA_TRY(w, copyToDevice(w->d.jinfo + first, info, size_t(n) * sizeof(int4), w->stream));
  for (uint32_t i = 0; i < n; i++) w->info[first + i] = info[i];
  // a released slot rewritten with a live joint is taken again
  w->freeSlots.erase(std::remove_if(w->freeSlots.begin(), w->freeSlots.end(),
                                    [&](uint32_t s) { return s >= first && s - first < n && w->info[s].type != AVBD_T_NONE; }),
                     w->freeSlots.end());
  return AVBD_OK;
}

int avbd_add_joints(avbd_world* w, const avbd_joint* joints, const avbd_joint_info* info, uint32_t n, uint32_t* first) {
  if (!w || (n && (!joints || !info))) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  int r = checkJoints(w, joints, info, n);
  if (r) return r;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (uint64_t(w->nj) + n > w->jointCap) {
    uint64_t cap = std::max<uint64_t>(uint64_t(w->nj) + n + 256, uint64_t(w->jointCap) * 2);
    r = allocJoints(w, uint32_t(cap));
    if (r) return r;
  }
  uint32_t at = w->nj;
  if (first) *first = at;
  w->nj += n;
  w->info.resize(w->nj);
  r = avbd_write_joints(w, at, joints, info, n);
  if (r) {
    w->nj -= n;
    return r;
  }
  for (uint32_t i = 0; i < n; i++)
    if (info[i].a >= 0 && info[i].type != AVBD_T_NONE) {
      uint32_t a = uint32_t(info[i].a), b = uint32_t(info[i].b);
      w->nocollide.push_back({std::max(a, b), std::min(a, b), at + i});
    }
  w->staticsDirty = true;
  return AVBD_OK;
}

// appendConstraints (gpu/solver.ts:1709-1738): released slots first, lowest first, then new slots
// at the end; each record and info written, each joint's pair kept out of the broadphase
int avbd_append_joints(avbd_world* w, const avbd_joint* joints, const avbd_joint_info* info, uint32_t n, uint32_t* slots) {
  if (!w || (n && (!joints || !info || !slots))) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  int r = checkJoints(w, joints, info, n);
  if (r) return r;
  if (!n) return AVBD_OK;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  std::sort(w->freeSlots.begin(), w->freeSlots.end(), std::greater<uint32_t>());
  const uint32_t reused = std::min<uint32_t>(n, uint32_t(w->freeSlots.size()));
  const uint32_t fresh = n - reused;
  if (uint64_t(w->nj) + fresh > w->jointCap) {
    const uint64_t cap = std::max<uint64_t>(uint64_t(w->nj) + fresh + 256, uint64_t(w->jointCap) * 2);
    r = allocJoints(w, uint32_t(cap));
    if (r) return r;
  }
  for (uint32_t k = 0; k < reused; k++) {
    slots[k] = w->freeSlots.back();
    w->freeSlots.pop_back();
  }
  for (uint32_t k = 0; k < fresh; k++) slots[reused + k] = w->nj + k;
  w->nj += fresh;
  w->info.resize(w->nj);
  for (uint32_t k = 0; k < n;) {  // one copy per run of consecutive slots
    uint32_t e = k + 1;
    while (e < n && slots[e] == slots[e - 1] + 1) e++;
    CUDA_TRY(w, copyToDevice(w->d.joint + size_t(slots[k]) * JOINT_VEC4, joints + k, size_t(e - k) * sizeof(avbd_joint), w->stream));
    CUDA_TRY(w, copyToDevice(w->d.jinfo + slots[k], info + k, size_t(e - k) * sizeof(int4), w->stream));
    k = e;
  }
  for (uint32_t k = 0; k < n; k++) {
    w->info[slots[k]] = info[k];
    if (info[k].a >= 0 && info[k].type != AVBD_T_NONE) {
      const uint32_t a = uint32_t(info[k].a), b = uint32_t(info[k].b);
      w->nocollide.push_back({std::max(a, b), std::min(a, b), slots[k]});
    }
  }
  w->staticsDirty = true;
  return AVBD_OK;
}

// releaseJoints (gpu/solver.ts:1745-1771): slots in range and not yet released stop acting, their
// records zeroed and their info T_NONE; their pairs collide again (their no-collide entries go, so a
// reused slot keeps only its new pair's); the slots go to the free list
int avbd_release_joints(avbd_world* w, const uint32_t* slots, uint32_t n) {
  if (!w || (n && !slots)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  std::vector<uint32_t> order;
  for (uint32_t i = 0; i < n; i++)
    if (slots[i] < w->nj && w->info[slots[i]].type != AVBD_T_NONE) order.push_back(slots[i]);
  std::sort(order.begin(), order.end());
  order.erase(std::unique(order.begin(), order.end()), order.end());
  if (order.empty()) return AVBD_OK;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  const avbd_joint_info none{AVBD_T_NONE, -1, -1, 0};
  for (size_t k = 0; k < order.size();) {
    size_t e = k + 1;
    while (e < order.size() && order[e] == order[e - 1] + 1) e++;
    const std::vector<avbd_joint> zeros(e - k);
    const std::vector<avbd_joint_info> infos(e - k, none);
    CUDA_TRY(w, copyToDevice(w->d.joint + size_t(order[k]) * JOINT_VEC4, zeros.data(), zeros.size() * sizeof(avbd_joint), w->stream));
    CUDA_TRY(w, copyToDevice(w->d.jinfo + order[k], infos.data(), infos.size() * sizeof(int4), w->stream));
    k = e;
  }
  for (uint32_t s : order) {
    w->info[s] = none;
    w->freeSlots.push_back(s);
  }
  w->nocollide.erase(std::remove_if(w->nocollide.begin(), w->nocollide.end(),
                                    [&](const NoCollide& c) { return c.slot != 0xffffffffu && std::binary_search(order.begin(), order.end(), c.slot); }),
                     w->nocollide.end());
  w->staticsDirty = true;
  return AVBD_OK;
}

int avbd_disable_joints(avbd_world* w, const uint32_t* slots, uint32_t n) {
  if (!w || (n && !slots)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  for (uint32_t i = 0; i < n; i++)
    if (slots[i] >= w->nj) return fail(w, AVBD_ERR_INVALID, "joint slot " + std::to_string(slots[i]) + " out of range");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  const float zeros[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t i = 0; i < n; i++) {
    float* rec = reinterpret_cast<float*>(w->d.joint + size_t(slots[i]) * JOINT_VEC4);
    CUDA_TRY(w, copyToDevice(rec, zeros, 8 * sizeof(float), w->stream));        // penalties and stiffnesses
    CUDA_TRY(w, copyToDevice(rec + 8, zeros, 3 * sizeof(float), w->stream));    // lam_lin (fracture kept)
    CUDA_TRY(w, copyToDevice(rec + 12, zeros, 3 * sizeof(float), w->stream));   // lam_ang (torque arm kept)
  }
  return AVBD_OK;
}

int avbd_add_ignore_pairs(avbd_world* w, const uint32_t* ab, uint32_t n) {
  if (!w || (n && !ab)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  for (uint32_t i = 0; i < n; i++)
    if (ab[2 * i] >= w->n || ab[2 * i + 1] >= w->n || ab[2 * i] == ab[2 * i + 1]) return fail(w, AVBD_ERR_INVALID, "ignore pair out of range");
  for (uint32_t i = 0; i < n; i++) w->nocollide.push_back({std::max(ab[2 * i], ab[2 * i + 1]), std::min(ab[2 * i], ab[2 * i + 1]), 0xffffffffu});
  w->staticsDirty = true;
  return AVBD_OK;
}

// setFilters(indices, groups, collidesWith) (gpu/solver.ts:1791-1801): one write per run of
// consecutive slots
int avbd_set_filters_at(avbd_world* w, const uint32_t* indices, const uint32_t* groups, const uint32_t* collides_with, uint32_t n) {
  if (!w || (n && (!indices || !groups || !collides_with))) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  for (uint32_t k = 0; k < n; k++)
    if (indices[k] >= w->n) return fail(w, AVBD_ERR_INVALID, "setFilters: slot " + std::to_string(indices[k]) + " is not a body of the world");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  for (uint32_t k = 0; k < n;) {
    uint32_t e = k + 1;
    while (e < n && indices[e] == indices[e - 1] + 1) e++;
    std::vector<uint2> run(e - k);
    for (uint32_t i = k; i < e; i++) run[i - k] = make_uint2(groups[i], collides_with[i]);
    CUDA_TRY(w, copyToDevice(w->d.filters + indices[k], run.data(), run.size() * sizeof(uint2), w->stream));
    k = e;
  }
  return AVBD_OK;
}

int avbd_set_filters(avbd_world* w, uint32_t first, const uint32_t* gm, uint32_t n) {
  if (!w || (n && !gm)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (uint64_t(first) + n > w->n) return fail(w, AVBD_ERR_INVALID, "setFilters: slots outside the world's bodies");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  CUDA_TRY(w, copyToDevice(w->d.filters + first, gm, size_t(n) * sizeof(uint2), w->stream));
  return AVBD_OK;
}

int avbd_set_body_aux(avbd_world* w, const uint32_t* indices, uint32_t n, const float* scales, const float* linear, const float* angular) {
  if (!w || (n && (!indices || !scales))) return AVBD_ERR_INVALID;
  if ((linear == nullptr) != (angular == nullptr)) return fail(w, AVBD_ERR_INVALID, "pass both damping rate arrays or neither");
  for (uint32_t k = 0; k < n; k++) {
    if (indices[k] >= w->bodyCap) return fail(w, AVBD_ERR_INVALID, "slot " + std::to_string(indices[k]) + " is outside the body capacity");
    if (!std::isfinite(scales[k])) return fail(w, AVBD_ERR_INVALID, "scales must be finite");
    if (linear && !(std::isfinite(linear[k]) && linear[k] >= 0.0f && std::isfinite(angular[k]) && angular[k] >= 0.0f))
      return fail(w, AVBD_ERR_INVALID, "damping rates must be finite and at least 0");
  }
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  // As setBodyAux writes them (gpu/solver.ts:1826-1845): a lone slot without rates changes only its
  // gravity scale; otherwise each run of consecutive slots gets whole records, with the default
  // rates (0) where none are given
  for (uint32_t k = 0; k < n;) {
    uint32_t e = k + 1;
    while (e < n && indices[e] == indices[e - 1] + 1) e++;
    if (e - k == 1 && !linear) {
      float4 rec;
      CUDA_TRY(w, copyToHost(&rec, w->d.aux + indices[k], sizeof(float4), w->stream));
      rec.x = scales[k];
      CUDA_TRY(w, copyToDevice(w->d.aux + indices[k], &rec, sizeof(float4), w->stream));
    } else {
      std::vector<float4> run(e - k);
      for (uint32_t i = k; i < e; i++) run[i - k] = make_float4(scales[i], linear ? linear[i] : 0.0f, linear ? angular[i] : 0.0f, 0.0f);
      CUDA_TRY(w, copyToDevice(w->d.aux + indices[k], run.data(), run.size() * sizeof(float4), w->stream));
    }
    k = e;
  }
  return AVBD_OK;
}

int avbd_read_body_aux(avbd_world* w, uint32_t first, float* aux4, uint32_t n) {
  if (!w || (n && !aux4)) return AVBD_ERR_INVALID;
  if (uint64_t(first) + n > w->bodyCap) return fail(w, AVBD_ERR_INVALID, "aux records outside the body capacity");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  CUDA_TRY(w, copyToHost(aux4, w->d.aux + first, size_t(n) * sizeof(float4), w->stream));
  return AVBD_OK;
}

int avbd_set_lifecycle(avbd_world* w, uint32_t index, uint32_t bits) {
  if (!w) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (index >= w->n || (bits & ~6u)) return fail(w, AVBD_ERR_INVALID, "Invalid body lifecycle flags/index");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  // the lifecycle word is the initial pose's w (layout.ts:17-19); a rewritten slot has no contact history
  float4 ip;
  CUDA_TRY(w, copyToHost(&ip, w->d.ipos + index, sizeof(float4), w->stream));
  ip.w = float(1u | bits);
  CUDA_TRY(w, copyToDevice(w->d.ipos + index, &ip, sizeof(float4), w->stream));
  const uint32_t none = NO_COLOR;
  CUDA_TRY(w, copyToDevice(w->d.colorA + index, &none, sizeof(uint32_t), w->stream));
  return AVBD_OK;
}

int avbd_seed_contacts(avbd_world* w, const avbd_manifold* m, uint32_t nm, const avbd_contact* c, uint32_t nc) {
  if (!w || (nm && !m) || (nc && !c)) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  for (uint32_t i = 0; i < nm; i++) {
    if (m[i].count > MAX_CONTACTS || uint64_t(m[i].first) + m[i].count > nc || m[i].a >= w->n || m[i].b >= w->n)
      return fail(w, AVBD_ERR_INVALID, "manifold " + std::to_string(i) + ": bad bodies or contact range");
  }
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (nm > w->pairCap) {
    int r = allocPairs(w, pow2AtLeast(nm));
    if (r) return r;
  }
  const int prev = 1 - w->cur;
  std::vector<uint4> ids(nm);
  std::vector<float4> geo(nm);
  std::vector<avbd_contact> pts(size_t(nm) * MAX_CONTACTS);
  std::memset(pts.data(), 0, pts.size() * sizeof(avbd_contact));
  for (uint32_t i = 0; i < nm; i++) {
    ids[i] = make_uint4(m[i].a, m[i].b, i * MAX_CONTACTS, m[i].count);
    geo[i] = make_float4(m[i].normal[0], m[i].normal[1], m[i].normal[2], m[i].friction);
    for (uint32_t k = 0; k < m[i].count; k++) pts[size_t(i) * MAX_CONTACTS + k] = c[m[i].first + k];
  }
  DWorld& d = w->d;
  if (nm) {
    CUDA_TRY(w, copyToDevice(d.mIds[prev], ids.data(), nm * sizeof(uint4), w->stream));
    CUDA_TRY(w, copyToDevice(d.mGeo[prev], geo.data(), nm * sizeof(float4), w->stream));
    CUDA_TRY(w, copyToDevice(d.cPt[prev], pts.data(), pts.size() * sizeof(avbd_contact), w->stream));
  }
  uint32_t pairs = nm;
  CUDA_TRY(w, copyToDevice(d.counters + C_PAIRS, &pairs, 4, w->stream));
  w->countersInFlight = false;
  return AVBD_OK;
}

int avbd_set_fixed_colors(avbd_world* w, const uint32_t* colors, uint32_t n) {
  if (!w) return AVBD_ERR_INVALID;
  w->configGen++;
  if (!colors) {
    w->fixedColors = false;
    return AVBD_OK;
  }
  if (n < w->n) return fail(w, AVBD_ERR_INVALID, "one colour per body is needed");
  for (uint32_t i = 0; i < w->n; i++)
    if (colors[i] != NO_COLOR && colors[i] >= uint32_t(MAX_COLORS)) return fail(w, AVBD_ERR_INVALID, "colours are below 64 (or 255: none)");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  CUDA_TRY(w, copyToDevice(w->d.fixedColor, colors, size_t(w->n) * 4, w->stream));
  w->fixedColors = true;
  return AVBD_OK;
}

int avbd_step(avbd_world* w, int n) { return avbd_step_with(w, n, nullptr); }

int avbd_step_with(avbd_world* w, int n, const avbd_step_options* opts) {
  if (!w || n < 0) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  for (int s = 0; s < n; s++) {
    // last step's manifolds are kept only while they are valid (gpu/solver.ts:2121)
    const bool reuse = opts && opts->reuse_manifolds && w->manifoldsValid;
    int r = adaptCapacity(w, false);
    if (r) return r;
    if (w->staticsDirty) {
      r = uploadStatics(w);
      if (r) return r;
    }
    w->stepCount++;
    StepParams p = makeParams(w);
    auto enqueue = [&]() -> cudaError_t {
      uint32_t launches = launch_collision(w->d, p, w->tableSize, reuse, w->stream) + 1;
      cudaError_t le = launch_topology_solve(w->d, p, w->solveBlocks, w->stream);
      if (w->statsCap) launch_step_stats(w->d, launches + 1, w->stream);
      w->launchesPerStep = launches + (w->statsCap ? 1 : 0);
      cudaMemcpyAsync(w->hCounters, w->d.counters, COUNTER_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost, w->stream);
      return le;
    };
    bool launched = false;
    if (w->useGraphs) {
      const int c = w->cur;
      cudaGraphExec_t& graph = w->graph[reuse ? 1 : 0][c];
      uint64_t& graphGen = w->graphGen[reuse ? 1 : 0][c];
      if (!graph || graphGen != w->configGen) {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          cudaError_t le = enqueue();
          e = cudaStreamEndCapture(w->stream, &g);
          if (e == cudaSuccess && le == cudaSuccess) e = cudaGraphInstantiate(&graph, g, 0);
          else if (e == cudaSuccess) e = le;
          if (g) cudaGraphDestroy(g);
        }
        if (e != cudaSuccess) {
          // capture is not available here: launch directly from now on
          cudaGetLastError();
          w->useGraphs = false;
          w->graphNote = std::string("graph capture failed: ") + cudaGetErrorString(e);
          if (graph) cudaGraphExecDestroy(graph);
          graph = nullptr;
        } else {
          graphGen = w->configGen;
        }
      }
      if (graph) {
        CUDA_TRY(w, cudaGraphLaunch(graph, w->stream));
        launched = true;
      }
    }
    if (!launched) {
      cudaError_t le = enqueue();
      CUDA_TRY(w, cudaGetLastError());
      CUDA_TRY(w, le);
    }
    if (w->statsCap) w->statsCount++;
    CUDA_TRY(w, cudaEventRecord(w->countersReady, w->stream));
    w->countersInFlight = true;
    w->cur = 1 - w->cur;
    w->manifoldsValid = true;
  }
  return AVBD_OK;
}

int avbd_read_reuse_state(avbd_world* w, float* ref_poses, uint32_t body_cap, uint32_t* n_bodies, uint32_t* generations, uint32_t manifold_cap,
                          uint32_t* n_manifolds) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (n_bodies) *n_bodies = w->n;
  const uint32_t nb = std::min(body_cap, w->n);
  if (nb && !ref_poses) return AVBD_ERR_INVALID;
  if (nb) {
    std::vector<float4> pos(nb), rot(nb);
    CUDA_TRY(w, copyToHost(pos.data(), w->d.refPos, nb * sizeof(float4), w->stream));
    CUDA_TRY(w, copyToHost(rot.data(), w->d.refRot, nb * sizeof(float4), w->stream));
    for (uint32_t i = 0; i < nb; i++) {
      std::memcpy(ref_poses + 8 * size_t(i), &pos[i], sizeof(float4));
      std::memcpy(ref_poses + 8 * size_t(i) + 4, &rot[i], sizeof(float4));
    }
  }
  uint32_t pairs = 0;
  CUDA_TRY(w, copyToHost(&pairs, w->d.counters + C_PAIRS, 4, w->stream));
  pairs = std::min(pairs, w->pairCap);
  std::vector<uint4> ids(pairs);
  if (pairs) CUDA_TRY(w, copyToHost(ids.data(), w->d.mIds[1 - w->cur], pairs * sizeof(uint4), w->stream));
  uint32_t mi = 0;
  for (uint32_t p = 0; p < pairs; p++) {
    if (!(ids[p].w & 15u)) continue;
    if (generations && mi < manifold_cap) generations[mi] = ids[p].w >> 4;
    mi++;
  }
  if (n_manifolds) *n_manifolds = mi;
  return AVBD_OK;
}

int avbd_synchronize(avbd_world* w) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (w->countersInFlight) {
    CUDA_TRY(w, cudaEventSynchronize(w->countersReady));
    w->countersInFlight = false;
    if (w->hCounters[C_ERROR]) return fail(w, AVBD_ERR_TIMEOUT, "the step gave up: error bits " + std::to_string(w->hCounters[C_ERROR]));
  }
  return AVBD_OK;
}

int avbd_read_bodies(avbd_world* w, avbd_body* dst, uint32_t cap, uint32_t* n) {
  if (!w) return AVBD_ERR_INVALID;
  if (n) *n = w->n;
  uint32_t k = std::min(cap, w->n);
  if (k && !dst) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  if (k) copyBodiesOut(w, dst, k);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  return AVBD_OK;
}

int avbd_read_bodies_async(avbd_world* w, avbd_body* dst, uint32_t cap) {
  if (!w) return AVBD_ERR_INVALID;
  uint32_t k = std::min(cap, w->n);
  if (k && !dst) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  if (k) copyBodiesOut(w, dst, k);
  CUDA_TRY(w, cudaGetLastError());
  return AVBD_OK;
}

int avbd_read_joints(avbd_world* w, avbd_joint* dst, avbd_joint_info* info, uint32_t cap, uint32_t* n) {
  if (!w) return AVBD_ERR_INVALID;
  if (n) *n = w->nj;
  uint32_t k = std::min(cap, w->nj);
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (k && dst) CUDA_TRY(w, copyToHost(dst, w->d.joint, size_t(k) * sizeof(avbd_joint), w->stream));
  if (k && info) std::memcpy(info, w->info.data(), size_t(k) * sizeof(avbd_joint_info));
  return AVBD_OK;
}

int avbd_read_counters(avbd_world* w, avbd_counters* out) {
  if (!w || !out) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  uint32_t c[COUNTER_WORDS];
  CUDA_TRY(w, copyToHost(c, w->d.counters, sizeof(c), w->stream));
  std::memset(out, 0, sizeof(*out));
  out->pairs = c[C_PAIRS];
  out->contacts = c[C_CONTACTS];
  out->manifolds = c[C_MANIFOLDS];
  out->overflow = c[C_OVERFLOW];
  out->clashes = c[C_CLASHES];
  out->colors = c[C_COLORS];
  out->rounds = c[C_ROUNDS];
  out->error = c[C_ERROR];
  out->steps = w->stepCount;
  out->graphs = w->useGraphs ? 1u : 0u;
  out->launches = w->launchesPerStep;
  out->pair_capacity = w->pairCap;
  return AVBD_OK;
}

int avbd_read_contacts(avbd_world* w, avbd_manifold* mout, uint32_t mcap, uint32_t* nm, avbd_contact* cout, uint32_t ccap, uint32_t* nc) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  uint32_t pairs = 0;
  CUDA_TRY(w, copyToHost(&pairs, w->d.counters + C_PAIRS, 4, w->stream));
  pairs = std::min(pairs, w->pairCap);
  const int last = 1 - w->cur;
  std::vector<uint4> ids(pairs);
  std::vector<float4> geo(pairs);
  if (pairs) {
    CUDA_TRY(w, copyToHost(ids.data(), w->d.mIds[last], pairs * sizeof(uint4), w->stream));
    CUDA_TRY(w, copyToHost(geo.data(), w->d.mGeo[last], pairs * sizeof(float4), w->stream));
  }
  std::vector<avbd_contact> pts;
  if (pairs) {
    pts.resize(size_t(pairs) * MAX_CONTACTS);
    CUDA_TRY(w, copyToHost(pts.data(), w->d.cPt[last], pts.size() * sizeof(avbd_contact), w->stream));
  }
  uint32_t mi = 0, ci = 0;
  for (uint32_t p = 0; p < pairs; p++) {
    uint32_t count = ids[p].w & 15u;
    if (!count) continue;
    if (mout && mi < mcap) {
      avbd_manifold& m = mout[mi];
      m.a = ids[p].x;
      m.b = ids[p].y;
      m.first = ci;
      m.count = count;
      m.normal[0] = geo[p].x;
      m.normal[1] = geo[p].y;
      m.normal[2] = geo[p].z;
      m.friction = geo[p].w;
    }
    for (uint32_t k = 0; k < count; k++) {
      if (cout && ci + k < ccap) cout[ci + k] = pts[size_t(p) * MAX_CONTACTS + k];
    }
    mi++;
    ci += count;
  }
  if (nm) *nm = mi;
  if (nc) *nc = ci;
  return AVBD_OK;
}

int avbd_read_pairs(avbd_world* w, uint32_t* dst, uint32_t cap, uint32_t* n) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  uint32_t pairs = 0;
  CUDA_TRY(w, copyToHost(&pairs, w->d.counters + C_PAIRS, 4, w->stream));
  pairs = std::min(pairs, w->pairCap);
  if (n) *n = pairs;
  uint32_t k = std::min(cap, pairs);
  if (k && dst) CUDA_TRY(w, copyToHost(dst, w->d.pairs, size_t(k) * sizeof(uint2), w->stream));
  return AVBD_OK;
}

int avbd_read_colors(avbd_world* w, uint32_t* dst, uint32_t cap, uint32_t* n) {
  if (!w) return AVBD_ERR_INVALID;
  if (n) *n = w->n;
  uint32_t k = std::min(cap, w->n);
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (k && dst) CUDA_TRY(w, copyToHost(dst, w->d.colorA, size_t(k) * 4, w->stream));
  return AVBD_OK;
}

int avbd_enable_step_stats(avbd_world* w, uint32_t capacity) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  dfree(w, w->d.statsRing);
  w->d.statsRing = nullptr;
  w->d.statsCap = 0;
  w->statsCap = capacity;
  w->statsCount = 0;
  w->configGen++;
  if (!capacity) return AVBD_OK;
  CUDA_TRY(w, dalloc(w, &w->d.statsRing, size_t(capacity) * STAT_WORDS));
  w->d.statsCap = capacity;
  uint32_t zero = 0;
  CUDA_TRY(w, cudaMemcpyAsync(w->d.counters + C_STATS_NEXT, &zero, 4, cudaMemcpyHostToDevice, w->stream));
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  return AVBD_OK;
}

int avbd_read_step_stats(avbd_world* w, avbd_step_stats* dst, uint32_t cap, uint32_t* n) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  uint32_t have = std::min(w->statsCount, w->statsCap);
  if (n) *n = have;
  if (!dst || !have) return AVBD_OK;
  std::vector<uint32_t> r(size_t(w->statsCap) * STAT_WORDS);
  CUDA_TRY(w, copyToHost(r.data(), w->d.statsRing, r.size() * 4, w->stream));
  uint32_t first = w->statsCount - have;
  for (uint32_t k = 0; k < have && k < cap; k++) {
    const uint32_t* q = &r[size_t((first + k) % w->statsCap) * STAT_WORDS];
    avbd_step_stats& s = dst[k];
    s.collision_ms = float(q[0] * 1e-6);
    s.solve_ms = float(q[1] * 1e-6);
    s.pairs = q[2];
    s.contacts = q[3];
    s.manifolds = q[4];
    s.adjacency = q[5];
    s.incidences = q[6];
    s.dynamic_bodies = q[7];
    s.colors = q[8];
    s.rounds = q[9];
    s.launches = q[10];
    s.error = q[11];
  }
  return AVBD_OK;
}

int avbd_read_phase_clocks(avbd_world* w, double* dst, uint32_t cap, uint32_t* n) {
  if (!w) return AVBD_ERR_INVALID;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  std::vector<unsigned long long> ck(CLOCK_WORDS);
  CUDA_TRY(w, copyToHost(ck.data(), w->d.clocks, ck.size() * 8, w->stream));
  uint32_t k = uint32_t(std::min<unsigned long long>(ck[0], MAX_CLOCKS));
  if (n) *n = k;
  for (uint32_t i = 0; i < k && i < cap && dst; i++) dst[i] = double(ck[1 + i] - ck[1]) * 1e-6;
  return AVBD_OK;
}

int avbd_use_graphs(avbd_world* w, int enable) {
  if (!w) return AVBD_ERR_INVALID;
  w->useGraphs = enable != 0;
  w->configGen++;
  return AVBD_OK;
}

int avbd_set_solve_blocks(avbd_world* w, int blocks) {
  if (!w || blocks < 0) return AVBD_ERR_INVALID;
  if (blocks > w->maxSolveBlocks) return fail(w, AVBD_ERR_INVALID, "at most " + std::to_string(w->maxSolveBlocks) + " co-resident solve blocks");
  w->solveBlocks = blocks ? blocks : w->maxSolveBlocks;
  w->configGen++;
  return AVBD_OK;
}

int avbd_add_hull(avbd_world* w, const uint32_t* packed, uint32_t vec4s, uint32_t* offset) {
  if (!w || !packed || !offset) return AVBD_ERR_INVALID;
  std::string msg = hullProblem(packed, vec4s);
  if (!msg.empty()) return fail(w, AVBD_ERR_INVALID, msg);
  // the first released run that fits (as acquireHull takes a free block, gpu/solver.ts:1389-1399), else the top
  uint32_t at = uint32_t(w->hullWords.size() / 4);
  bool reused = false;
  for (auto it = w->hullFree.begin(); it != w->hullFree.end(); ++it)
    if (it->second >= vec4s) {
      at = it->first;
      const uint32_t rest = it->second - vec4s;
      w->hullFree.erase(it);
      if (rest) w->hullFree[at + vec4s] = rest;
      reused = true;
      break;
    }
  if (uint64_t(at) + vec4s + AVBD_SHAPE_HULL >= (1ull << 24)) return fail(w, AVBD_ERR_CAPACITY, "hull buffer beyond 2^24 vec4s (f32 shape codes)");
  std::vector<uint32_t> rec(packed, packed + size_t(vec4s) * 4);
  for (int k : {0, 2, 4, 6}) rec[k] += at;
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  if (reused) std::copy(rec.begin(), rec.end(), w->hullWords.begin() + size_t(at) * 4);
  else w->hullWords.insert(w->hullWords.end(), rec.begin(), rec.end());
  const uint32_t total = uint32_t(w->hullWords.size() / 4);
  if (total > w->hullCapVec4) {
    uint32_t cap = std::max<uint32_t>(4096, std::max(total, 2 * w->hullCapVec4));
    uint4* fresh = nullptr;
    cudaError_t e = dalloc(w, &fresh, cap);
    if (e != cudaSuccess) {
      w->hullWords.resize(size_t(at) * 4);
      return fail(w, AVBD_ERR_CUDA, std::string("hull buffer: ") + cudaGetErrorString(e));
    }
    dfree(w, w->d.hulls);
    w->d.hulls = fresh;
    w->hullCapVec4 = cap;
    w->configGen++;  // the step graphs hold the buffer's address
    CUDA_TRY(w, copyToDevice(w->d.hulls, w->hullWords.data(), w->hullWords.size() * 4, w->stream));
  } else {
    CUDA_TRY(w, copyToDevice(w->d.hulls + at, rec.data(), rec.size() * 4, w->stream));
  }
  w->hullStarts.insert(at);
  w->hullSize[at] = vec4s;
  *offset = at;
  return AVBD_OK;
}

int avbd_release_hull(avbd_world* w, uint32_t offset) {
  if (!w) return AVBD_ERR_INVALID;
  if (!w->hullStarts.count(offset)) return fail(w, AVBD_ERR_INVALID, "no hull record at offset " + std::to_string(offset));
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  // a record some body still names stays (its shape code would point into whatever reuses the run)
  std::vector<float4> avel(w->n);
  if (w->n) CUDA_TRY(w, copyToHost(avel.data(), w->d.avel, size_t(w->n) * sizeof(float4), w->stream));
  const float code = float(AVBD_SHAPE_HULL + offset);
  for (uint32_t i = 0; i < w->n; i++)
    if (avel[i].w == code) return fail(w, AVBD_ERR_INVALID, "body " + std::to_string(i) + " uses the hull at offset " + std::to_string(offset));
  const uint32_t size = w->hullSize[offset];
  w->hullStarts.erase(offset);
  w->hullSize.erase(offset);
  // free run, merged with its neighbours (releaseHull / mergeFree, gpu/solver.ts:1408-1414)
  uint32_t start = offset, len = size;
  auto next = w->hullFree.find(offset + size);
  if (next != w->hullFree.end()) {
    len += next->second;
    w->hullFree.erase(next);
  }
  auto prev = w->hullFree.lower_bound(offset);
  if (prev != w->hullFree.begin()) {
    --prev;
    if (prev->first + prev->second == offset) {
      start = prev->first;
      len += prev->second;
      w->hullFree.erase(prev);
    }
  }
  w->hullFree[start] = len;
  return AVBD_OK;
}

int avbd_hull_storage(const avbd_world* w, uint32_t* top, uint32_t* capacity, uint32_t* largest_free) {
  if (!w) return AVBD_ERR_INVALID;
  uint32_t big = 0;
  for (auto& f : w->hullFree) big = std::max(big, f.second);
  if (top) *top = uint32_t(w->hullWords.size() / 4);
  if (capacity) *capacity = w->hullCapVec4;
  if (largest_free) *largest_free = big;
  return AVBD_OK;
}

int avbd_broadphase_radii(const double* radii, uint32_t n, double* largest_small, double* large_threshold) {
  if (n && !radii) return AVBD_ERR_INVALID;
  std::vector<double> r(radii, radii + n);
  for (double x : r)
    if (!std::isfinite(x) || x < 0.0) return AVBD_ERR_INVALID;
  if (largest_small) *largest_small = largestSmall(r);
  if (large_threshold) *large_threshold = largeThreshold(r);
  return AVBD_OK;
}

int avbd_world_stream(avbd_world* w, void** stream) {
  if (!w || !stream) return AVBD_ERR_INVALID;
  *stream = (void*)w->stream;
  return AVBD_OK;
}

int avbd_write_bodies_async(avbd_world* w, uint32_t first, const avbd_body* bodies, uint32_t n) {
  if (!w || (!bodies && n) || uint64_t(first) + n > w->n) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  cudaSetDevice(w->device);
  if (n) copyBodiesIn(w, first, bodies, n, cudaMemcpyHostToDevice);
  CUDA_TRY(w, cudaGetLastError());
  return AVBD_OK;
}

// appendWorldJoint, 'legacy' policy (gpu/solver.ts:1592-1623): the record of freshJoint (:132-138)
// with a hard linear stiffness, the world point in r_a, the body point in r_b and the torque arm of
// the body's size; no angular stiffness, so the joint holds the point and leaves the turn free.
int avbd_add_world_joint(avbd_world* w, uint32_t body, const float anchor_world[3], const float anchor_body[3], uint32_t* slot) {
  if (!w || !anchor_world || !anchor_body) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (body >= w->n) return fail(w, AVBD_ERR_INVALID, "appendWorldJoint: body " + std::to_string(body) + " is not a body of the world");
  for (int k = 0; k < 3; k++)
    if (!std::isfinite(anchor_world[k]) || !std::isfinite(anchor_body[k]))
      return fail(w, AVBD_ERR_INVALID, "appendWorldJoint: anchors need three finite f32 numbers");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  float4 size;
  CUDA_TRY(w, copyToHost(&size, w->d.size + body, sizeof(float4), w->stream));
  const float arm = size.x * size.x + size.y * size.y + size.z * size.z;
  if (!std::isfinite(arm)) return fail(w, AVBD_ERR_INVALID, "appendWorldJoint: torque arm must be finite as f32");
  avbd_joint j{};
  j.stiffness_lin = AVBD_BIG;
  j.fracture = AVBD_BIG;
  j.yield_force = AVBD_BIG;
  j.break_bend = AVBD_BIG;
  j.rest[3] = 1.0f;
  j.rest_start[3] = 1.0f;
  j.torque_arm = arm;
  for (int k = 0; k < 3; k++) {
    j.r_a[k] = anchor_world[k];
    j.r_b[k] = anchor_body[k];
  }
  const avbd_joint_info info{AVBD_T_JOINT, -1, int32_t(body), 0};
  uint32_t at = 0;
  const int r = avbd_append_joints(w, &j, &info, 1, &at);
  if (!r && slot) *slot = at;
  return r;
}

// setWorldAnchor (gpu/solver.ts:1937-1939): the slot's r_a, in place before the next step
int avbd_set_world_anchor(avbd_world* w, uint32_t slot, const float p[3]) {
  if (!w || !p) return AVBD_ERR_INVALID;
  w->manifoldsValid = false;
  if (slot >= w->nj) return fail(w, AVBD_ERR_INVALID, "setWorldAnchor: joint slot " + std::to_string(slot) + " out of range");
  for (int k = 0; k < 3; k++)
    if (!std::isfinite(p[k])) return fail(w, AVBD_ERR_INVALID, "setWorldAnchor: the anchor needs three finite f32 numbers");
  cudaSetDevice(w->device);
  CUDA_TRY(w, cudaStreamSynchronize(w->stream));
  float* rec = reinterpret_cast<float*>(w->d.joint + size_t(slot) * JOINT_VEC4 + J_RA);
  CUDA_TRY(w, copyToDevice(rec, p, 3 * sizeof(float), w->stream));
  return AVBD_OK;
}

int avbd_body_storage(avbd_world* w, avbd_body_view* out) {
  if (!w || !out) return AVBD_ERR_INVALID;
  float4* const fields[10] = {w->d.pos, w->d.rot, w->d.ipos, w->d.irot, w->d.size, w->d.moment, w->d.ypos, w->d.yrot, w->d.vel, w->d.avel};
  for (int f = 0; f < 10; f++) out->fields[f] = fields[f];
  out->count = w->n;
  out->capacity = w->bodyCap;
  return AVBD_OK;
}

int avbd_contact_storage(avbd_world* w, uint32_t which, avbd_contact_view* out) {
  if (!w || !out || which > 1u) return AVBD_ERR_INVALID;
  const int buf = which == 0u ? 1 - w->cur : w->cur;  // avbd_step flips cur after each step
  out->pairs = w->d.mIds[buf];
  out->normals = w->d.mGeo[buf];
  out->points = w->d.cPt[buf];
  out->counters = w->d.counters;
  out->count_word = which == 0u ? uint32_t(C_PAIRS) : uint32_t(C_PREV_PAIRS);
  out->pair_capacity = w->pairCap;
  return AVBD_OK;
}

}  // extern "C"
