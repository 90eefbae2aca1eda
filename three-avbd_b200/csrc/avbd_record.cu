// Recording a batched rollout's contact structure for the adjoint, on the device, after each step.
//
// The adjoint differentiates the step with its contact structure frozen: per step the manifolds
// (bodies, normal basis), each point's body-frame anchors and the last-step point it warm-started
// from, and the colouring. After a batched step these live in the step's pair slots (mIds, mGeo,
// cPt of the buffer the step wrote) and colour words; three launches append them to the recording
// in the adjoint's layout: per world counts, one scan over the worlds for global offsets, then a
// block per world writing its records in slot order. The warm-start source of a point is found as
// the narrowphase found it (writeManifold): the last step's manifold of the same pair through the
// pair hash, then the first of its points with the same feature key.
#include <algorithm>

#include "avbd_device.cuh"

namespace avbd {
namespace {

constexpr int REC_THREADS = 128;

// Block-wide exclusive scan of two counters (REC_THREADS threads); returns the block totals
__device__ inline void scan2(int a, int b, int& ea, int& eb, int& ta, int& tb) {
  __shared__ int s_a[REC_THREADS / 32], s_b[REC_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int ia = a, ib = b;
  for (int o = 1; o < 32; o <<= 1) {
    int xa = __shfl_up_sync(0xffffffffu, ia, o), xb = __shfl_up_sync(0xffffffffu, ib, o);
    if (lane >= o) {
      ia += xa;
      ib += xb;
    }
  }
  if (lane == 31) {
    s_a[warp] = ia;
    s_b[warp] = ib;
  }
  __syncthreads();
  int ba = 0, bb = 0;
  ta = tb = 0;
  for (int k = 0; k < REC_THREADS / 32; k++) {
    if (k < warp) {
      ba += s_a[k];
      bb += s_b[k];
    }
    ta += s_a[k];
    tb += s_b[k];
  }
  ea = ba + ia - a;
  eb = bb + ib - b;
  __syncthreads();
}

__device__ inline uint32_t slotCount(uint4 ids) { return min(ids.w & 15u, (uint32_t)MAX_CONTACTS); }

// The last step's manifold of pair (a, b): its slot, or -1 (hashFind of the narrowphase)
__device__ inline int prevSlot(const DWorld& w, uint32_t hashMask, int prev, uint32_t a, uint32_t b) {
  uint32_t h = pairHash(a, b) & hashMask;
  for (uint32_t probe = 0; probe <= hashMask; probe++) {
    uint32_t v = w.hash[h];
    if (v == 0u) return -1;
    uint4 ids = w.mIds[prev][v - 1u];
    if (ids.x == a && ids.y == b) return int(v - 1u);
    h = (h + 1u) & hashMask;
  }
  return -1;
}

__global__ void __launch_bounds__(REC_THREADS) k_rec_count(BatchLaunch L, RecordDev R) {
  for (uint32_t wi = blockIdx.x; wi < L.nWorlds; wi += gridDim.x) {
    const WorldDesc d = L.worlds[wi];
    const DWorld w = worldView(L.base, d, wi);
    const uint32_t pairs = min(w.counters[C_PAIRS], d.pairCap);
    int man = 0, pts = 0;
    for (uint32_t m = threadIdx.x; m < pairs; m += blockDim.x) {
      uint32_t c = slotCount(w.mIds[L.p.cur][m]);
      man += c > 0u;
      pts += int(c);
    }
    int ea, eb, ta, tb;
    scan2(man, pts, ea, eb, ta, tb);
    if (threadIdx.x == 0) {
      R.manCount[wi] = ta;
      R.ptCount[wi] = tb;
    }
  }
}

// One block of 1024 threads: global first indices of every world's records of step s
__global__ void __launch_bounds__(1024) k_rec_scan(RecordDev R, uint32_t s) {
  __shared__ unsigned long long s_wm[32], s_wp[32];
  __shared__ unsigned long long s_carry[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    s_carry[0] = R.totals[0];
    s_carry[1] = R.totals[1];
  }
  __syncthreads();
  int most = 0;
  for (uint32_t c0 = 0; c0 < R.W; c0 += blockDim.x) {
    const uint32_t i = c0 + threadIdx.x;
    const unsigned long long m = i < R.W ? (unsigned long long)R.manCount[i] : 0ull, p = i < R.W ? (unsigned long long)R.ptCount[i] : 0ull;
    if (i < R.W) most = max(most, int(p));
    unsigned long long im = m, ip = p;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long xm = __shfl_up_sync(0xffffffffu, im, o), xp = __shfl_up_sync(0xffffffffu, ip, o);
      if (lane >= o) {
        im += xm;
        ip += xp;
      }
    }
    if (lane == 31) {
      s_wm[warp] = im;
      s_wp[warp] = ip;
    }
    __syncthreads();
    unsigned long long bm = s_carry[0], bp = s_carry[1], tm = 0, tp = 0;
    for (int k = 0; k < int(blockDim.x >> 5); k++) {
      if (k < warp) {
        bm += s_wm[k];
        bp += s_wp[k];
      }
      tm += s_wm[k];
      tp += s_wp[k];
    }
    if (i < R.W) {
      R.manFirst[size_t(s) * (R.W + 1) + i] = int(min(bm + im - m, (unsigned long long)R.manCap));
      R.ptFirst[size_t(s) * (R.W + 1) + i] = int(min(bp + ip - p, (unsigned long long)R.ptCap));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry[0] += tm;
      s_carry[1] += tp;
    }
    __syncthreads();
  }
  if (most) atomicMax(&R.status[1], uint32_t(most));
  if (threadIdx.x == 0) {
    unsigned long long tm = s_carry[0], tp = s_carry[1];
    if (tm > R.manCap || tp > R.ptCap) atomicOr(&R.status[0], REC_CAPACITY);
    R.manFirst[size_t(s) * (R.W + 1) + R.W] = int(min(tm, (unsigned long long)R.manCap));
    R.ptFirst[size_t(s) * (R.W + 1) + R.W] = int(min(tp, (unsigned long long)R.ptCap));
    R.totals[0] = min(tm, (unsigned long long)R.manCap);
    R.totals[1] = min(tp, (unsigned long long)R.ptCap);
  }
}

// A block per world: its manifolds and points in slot order, the warm-start sources, the colours
__global__ void __launch_bounds__(REC_THREADS) k_rec_fill(BatchLaunch L, RecordDev R, uint32_t s) {
  __shared__ int s_carry[2];
  const int cur = L.p.cur, prev = 1 - cur;
  for (uint32_t wi = blockIdx.x; wi < L.nWorlds; wi += gridDim.x) {
    const WorldDesc d = L.worlds[wi];
    const DWorld w = worldView(L.base, d, wi);
    const uint32_t pairs = min(w.counters[C_PAIRS], d.pairCap);
    const size_t row = size_t(s) * (R.W + 1) + wi;
    const int mBase = R.manFirst[row], pBase = R.ptFirst[row];
    // a world whose records would pass the capacity writes none (the recording is marked invalid)
    const bool room = uint64_t(mBase) + uint64_t(R.manCount[wi]) <= R.manCap && uint64_t(pBase) + uint64_t(R.ptCount[wi]) <= R.ptCap;
    const int prevM0 = s > 0 ? R.manFirst[row - (R.W + 1)] : 0, prevM1 = s > 0 ? R.manFirst[row - (R.W + 1) + 1] : 0;
    if (threadIdx.x == 0) s_carry[0] = s_carry[1] = 0;
    __syncthreads();
    for (uint32_t base = 0; base < pairs; base += blockDim.x) {
      const uint32_t m = base + threadIdx.x;
      const uint4 ids = m < pairs ? w.mIds[cur][m] : make_uint4(0, 0, 0, 0);
      const int cnt = m < pairs ? int(slotCount(ids)) : 0;
      int om, op, tm, tp;
      scan2(cnt > 0, cnt, om, op, tm, tp);
      if (cnt > 0 && room) {
        const int gm = mBase + s_carry[0] + om, k0 = pBase + s_carry[1] + op;
        if (ids.x <= ids.y) atomicOr(&R.status[0], REC_ORDER);
        R.manAB[gm] = make_int2(int(ids.x), int(ids.y));
        R.manSlot[gm] = int(m);
        R.manPt0[gm] = k0;
        float3 n = f3(w.mGeo[cur][m]), t1, t2;
        orthonormal(n, t1, t2);
        double* B = R.basis + 9 * size_t(gm);
        B[0] = n.x, B[1] = n.y, B[2] = n.z, B[3] = t1.x, B[4] = t1.y, B[5] = t1.z, B[6] = t2.x, B[7] = t2.y, B[8] = t2.z;
        // the last step's manifold of the pair, and its record
        uint32_t prevFirst = 0, prevCount = 0;
        int prevPt0 = -1;
        const int pm = prevSlot(w, d.hashMask, prev, ids.x, ids.y);
        if (pm >= 0) {
          const uint4 pid = w.mIds[prev][pm];
          prevFirst = pid.z;
          prevCount = slotCount(pid);
          int lo = prevM0, hi = prevM1;  // manSlot ascends within the world's last step
          while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (R.manSlot[mid] < pm) lo = mid + 1;
            else hi = mid;
          }
          if (lo < prevM1 && R.manSlot[lo] == pm) prevPt0 = R.manPt0[lo];
        }
        for (int j = 0; j < cnt; j++) {
          const float4* q = w.cPt[cur] + 4 * size_t(ids.z + j);
          const float4 ra = q[K_RA], rb = q[K_RB];
          const uint32_t key = __float_as_uint(ra.w) & ~STICK_BIT;
          if (key == SPHERE_FEATURE) atomicOr(&R.status[0], REC_SPHERE);
          int src = -1;
          for (uint32_t c = prevFirst; c < prevFirst + prevCount; c++)
            if ((__float_as_uint(w.cPt[prev][4 * size_t(c) + K_RA].w) & ~STICK_BIT) == key) {
              // the step warm-started from this point: the recording must hold it
              if (prevPt0 >= 0) src = prevPt0 + int(c - prevFirst);
              else atomicOr(&R.status[0], REC_HISTORY);
              break;
            }
          double* A = R.anchors + 6 * size_t(k0 + j);
          A[0] = ra.x, A[1] = ra.y, A[2] = ra.z, A[3] = rb.x, A[4] = rb.y, A[5] = rb.z;
          R.ptMan[k0 + j] = gm;
          R.ptPrev[k0 + j] = src;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        s_carry[0] += tm;
        s_carry[1] += tp;
      }
      __syncthreads();
    }
    for (uint32_t b = threadIdx.x; b < d.n; b += blockDim.x)
      R.color[size_t(s) * R.nb + d.body + b] = w.size[b].w > 0.0f ? int(w.colorA[b]) : -1;
    if (threadIdx.x == 0) {
      const uint32_t nc = w.counters[C_COLORS];
      if (nc > uint32_t(MAX_COLORS)) atomicOr(&R.status[0], REC_COLORS);
      R.ncol[size_t(s) * R.W + wi] = int(nc);
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t launch_record_step(const BatchLaunch& L, const RecordDev& R, uint32_t s, int blocks, cudaStream_t st) {
  const int g = std::max(1, std::min<int>(blocks, int(L.nWorlds)));
  k_rec_count<<<g, REC_THREADS, 0, st>>>(L, R);
  k_rec_scan<<<1, 1024, 0, st>>>(R, s);
  k_rec_fill<<<g, REC_THREADS, 0, st>>>(L, R, s);
  return cudaGetLastError();
}

}  // namespace avbd
