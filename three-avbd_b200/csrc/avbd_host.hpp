// Host-side state shared by the single-world and batched entry points (avbd_host.cu, avbd_batch.cu).
#pragma once
#include <cmath>
#include <cstdint>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "avbd.h"
#include "avbd_device.cuh"

namespace avbd {

uint32_t pow2AtLeast(uint64_t n);
// The largest "small" bounding radius of a body set (radii.ts:19-55): the broadphase classification
double largestSmall(std::vector<double> radii);
double largeThreshold(const std::vector<double>& radii);
// Why a set of records is invalid (empty: valid)
std::string bodyProblem(const avbd_body* b, uint32_t n);
std::string jointProblem(const avbd_joint* j, const avbd_joint_info* info, uint32_t n, uint32_t bodies);

// Body records between the field arrays and a staging array of records (10 float4 a body), on `s`
void packBodies(const DWorld& d, float4* staging, uint32_t first, uint32_t n, cudaStream_t s);
void unpackBodies(const DWorld& d, const float4* staging, uint32_t first, uint32_t n, cudaStream_t s);

struct NoCollide {
  uint32_t hi, lo, slot;
  bool operator<(const NoCollide& o) const { return hi < o.hi || (hi == o.hi && lo < o.lo); }
};

}  // namespace avbd

// One simulation world (GpuSolver3D's state, gpu/solver.ts:598-700)
struct avbd_world {
  using DWorld = avbd::DWorld;
  using NoCollide = avbd::NoCollide;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  avbd_params params{};
  uint32_t bodyCap = 0, n = 0, jointCap = 0, nj = 0, pairCap = 0, tableSize = 0, hashSize = 0, incCap = 0, adjCap = 0;
  uint32_t sortTiles = 0;
  DWorld d{};
  float4* staging = nullptr;  // body records for host transfers (10 float4 a body, capacity)
  int solveBlocks = 0, maxSolveBlocks = 0;  // the cooperative solve's grid (maxSolveBlocks: all co-resident)
  int cur = 0;
  uint32_t stepCount = 0;
  bool fixedColors = false;
  // host mirrors
  std::vector<float> radius;
  std::vector<char> dynamic;
  std::vector<avbd_joint_info> info;
  std::vector<uint32_t> freeSlots;  // released joint slots, taken again by avbd_append_joints
  std::vector<NoCollide> nocollide;
  bool staticsDirty = true;
  float threshold = 0.0f, cellSize = 1.0f;
  uint32_t nLarge = 0, nNoCollide = 0, anyDynamicLarge = 0;
  uint32_t staticsWords = 0;
  // counters of the last step, copied back asynchronously
  uint32_t* hCounters = nullptr;
  cudaEvent_t countersReady = nullptr;
  bool countersInFlight = false;
  // per-step statistics: a device ring written by the step itself (graph-compatible)
  uint32_t statsCap = 0, statsCount = 0;
  uint32_t launchesPerStep = 0;
  // The step as CUDA graphs, one per contact-buffer parity and per kind (detecting, or keeping last
  // step's manifolds), rebuilt when anything baked into their launches changes (configGen)
  bool useGraphs = true;
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  uint64_t graphGen[2][2] = {{0, 0}, {0, 0}};
  // last step's manifolds may be kept by the next step (reuseManifolds): a step ran and nothing
  // that changes bodies, joints, filters or contacts happened since (gpu/solver.ts manifoldsValid)
  bool manifoldsValid = false;
  uint64_t configGen = 1;
  std::string graphNote;
  std::vector<void*> allocations;
  // scratch of the queries around the step (avbd_query.cu), grown on demand: pushes, rays, the
  // rays' nearest keys and their hits
  float4 *pushBuf = nullptr, *rayBuf = nullptr, *rayHits = nullptr;
  unsigned long long* rayBest = nullptr;
  size_t pushCap = 0, rayCap = 0, rayBestCap = 0, rayHitsCap = 0;
  // hull buffer: host copy of every record (wgsl-hull.ts layout), header offsets, device capacity
  std::vector<uint32_t> hullWords;
  std::set<uint32_t> hullStarts;
  std::map<uint32_t, uint32_t> hullSize;  // header offset -> vec4s of each resident record
  std::map<uint32_t, uint32_t> hullFree;  // released runs: offset -> vec4s (merged with neighbours)
  uint32_t hullCapVec4 = 0;
};

namespace avbd {
// Uploads the world's large-body list and sorted no-collide triples when they changed
int uploadStatics(avbd_world* w);

// The wind's step parameters: its velocity from speed and angle, as gpu/solver.ts:1994-1998 packs it
inline void setWind(StepParams& p, const avbd_params& a) {
  p.windX = float(double(a.wind_speed) * std::cos(double(a.wind_angle)));
  p.windY = float(double(a.wind_speed) * std::sin(double(a.wind_angle)));
  p.windGust = a.wind_gust;
  p.windPressure = a.wind_pressure;
}

// Copies between host and device, ordered on stream s and complete when they return. A plain
// cudaMemcpy runs on the legacy default stream, which the worlds' non-blocking streams do not wait
// on, and from pageable memory it returns before its DMA has landed: a kernel launched next on the
// world's stream could read the old bytes. The async copy stages pageable memory before returning,
// so the host buffer may go as soon as these return.
inline cudaError_t copyToDevice(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return cudaSuccess;
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}
inline cudaError_t copyToHost(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return cudaSuccess;
  const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}
}  // namespace avbd
