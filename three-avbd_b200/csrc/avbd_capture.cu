// Pose capture: the frames of the pose cache (src/bake/pose-cache.ts, frame layout: u32 step, then
// per body slot position xyz and rotation xyzw as f32) gathered on the device. The host enqueues one
// kernel per frame on the world's stream and keeps the frame count itself (frames are enqueued in
// order), so a capture every k-th step adds one launch and no synchronisation; the step word is read
// on the device when the frame runs. The CRC-32s, chunking and manifest are the host codec's.

#include <cstring>
#include <string>
#include <vector>

#include "avbd_device.cuh"
#include "avbd_host.hpp"

struct avbd_pose_capture {
  avbd_world* world = nullptr;
  uint32_t n = 0, maxFrames = 0, frames = 0, dropped = 0;
  uint32_t* slots = nullptr;  // device, n
  uint32_t* steps = nullptr;  // device, maxFrames
  float* poses = nullptr;     // device, maxFrames x n x 7
};

namespace avbd {
namespace {

// One frame: thread i writes slot i's pose (+0 for a disabled slot); thread 0 the step word
__global__ void k_pose_capture(DWorld w, const uint32_t* slots, uint32_t n, uint32_t frame, uint32_t* steps, float* poses) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) steps[frame] = w.counters[C_STEP];
  if (i >= n) return;
  const uint32_t b = slots[i];
  float* o = poses + (size_t(frame) * n + i) * 7;
  if (((uint32_t)w.ipos[b].w & 2u) != 0u) {
    for (int k = 0; k < 7; k++) o[k] = 0.0f;
    return;
  }
  const float4 p = w.pos[b], q = w.rot[b];
  o[0] = p.x, o[1] = p.y, o[2] = p.z;
  o[3] = q.x, o[4] = q.y, o[5] = q.z, o[6] = q.w;
}

int wfail(avbd_world* w, int code, const std::string& m) {
  if (w) w->error = m;
  return code;
}
int cfail(avbd_pose_capture* c, int code, const std::string& m) { return wfail(c ? c->world : nullptr, code, m); }

}  // namespace
}  // namespace avbd

using namespace avbd;

extern "C" int avbd_pose_capture_create(avbd_world* w, const uint32_t* slots, uint32_t n, uint32_t max_frames, avbd_pose_capture** out) {
  if (!w || !out || (n && !slots)) return AVBD_ERR_INVALID;
  *out = nullptr;
  if (n == 0 || max_frames == 0) return wfail(w, AVBD_ERR_INVALID, "a capture needs at least one slot and one frame");
  for (uint32_t i = 0; i < n; i++)
    if (slots[i] >= w->n) return wfail(w, AVBD_ERR_INVALID, "slot " + std::to_string(slots[i]) + " is not a body of the world");
  if (uint64_t(max_frames) * n * 7 * sizeof(float) > (uint64_t(1) << 36)) return wfail(w, AVBD_ERR_CAPACITY, "a capture holds at most 64 GiB of poses");
  cudaSetDevice(w->device);
  auto* c = new avbd_pose_capture();
  c->world = w;
  c->n = n;
  c->maxFrames = max_frames;
  bool ok = cudaMalloc(&c->slots, size_t(n) * 4) == cudaSuccess && cudaMalloc(&c->steps, size_t(max_frames) * 4) == cudaSuccess &&
            cudaMalloc(&c->poses, size_t(max_frames) * n * 7 * sizeof(float)) == cudaSuccess &&
            copyToDevice(c->slots, slots, size_t(n) * 4, w->stream) == cudaSuccess;
  if (!ok) {
    avbd_pose_capture_destroy(c);
    return wfail(w, AVBD_ERR_CUDA, "pose capture: device allocation failed");
  }
  *out = c;
  return AVBD_OK;
}

extern "C" int avbd_pose_capture_frame(avbd_pose_capture* c) {
  if (!c) return AVBD_ERR_INVALID;
  avbd_world* w = c->world;
  if (c->frames >= c->maxFrames) {
    c->dropped++;
    return AVBD_OK;
  }
  cudaSetDevice(w->device);
  k_pose_capture<<<grid_for(c->n, 256), 256, 0, w->stream>>>(w->d, c->slots, c->n, c->frames, c->steps, c->poses);
  if (cudaGetLastError() != cudaSuccess) return cfail(c, AVBD_ERR_CUDA, "pose capture: launch failed");
  c->frames++;
  return AVBD_OK;
}

extern "C" int avbd_pose_capture_read(avbd_pose_capture* c, uint32_t* steps, float* poses, uint32_t cap, uint32_t* frames, uint32_t* dropped) {
  if (!c || (cap && (!steps || !poses))) return AVBD_ERR_INVALID;
  avbd_world* w = c->world;
  cudaSetDevice(w->device);
  const uint32_t k = cap < c->frames ? cap : c->frames;
  if (copyToHost(steps, c->steps, size_t(k) * 4, w->stream) != cudaSuccess ||
      copyToHost(poses, c->poses, size_t(k) * c->n * 7 * sizeof(float), w->stream) != cudaSuccess ||
      cudaStreamSynchronize(w->stream) != cudaSuccess)
    return cfail(c, AVBD_ERR_CUDA, "pose capture: read failed");
  if (frames) *frames = c->frames;
  if (dropped) *dropped = c->dropped;
  return AVBD_OK;
}

extern "C" int avbd_pose_capture_reset(avbd_pose_capture* c) {
  if (!c) return AVBD_ERR_INVALID;
  c->frames = c->dropped = 0;
  return AVBD_OK;
}

extern "C" int avbd_pose_capture_destroy(avbd_pose_capture* c) {
  if (!c) return AVBD_OK;
  if (c->world) cudaSetDevice(c->world->device);
  if (c->world) cudaStreamSynchronize(c->world->stream);
  cudaFree(c->slots);
  cudaFree(c->steps);
  cudaFree(c->poses);
  delete c;
  return AVBD_OK;
}
