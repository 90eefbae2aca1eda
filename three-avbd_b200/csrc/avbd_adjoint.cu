// The adjoint of the step (batched worlds, double precision): gradients of a pose loss with respect
// to every body's initial linear and angular velocity, mass and friction coefficient.
//
// The step is differentiated with its contact structure frozen from a recorded rollout: per step,
// the pairs with their normals, each point's body-frame anchors and the last-step point it warm-
// starts from, and the colouring. Everything else is differentiated: C(x-) from the poses, the warm
// starts, the inertial targets and the accelerated warm-start guess, the coloured Gauss-Seidel
// primal solves (6x6 LDLT), the duals (lambda, penalty ramps, friction cone) and the velocities.
// The replay forward keeps the state every `checkpoint` steps; the reverse pass recomputes a
// segment from its checkpoint, then each step with per-iteration snapshots, and sweeps the step
// backwards: velocities, then per iteration the duals and the colours in reverse, then the warm
// starts. One block per world; a thread per body (primal) or per point (duals, warm starts).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "avbd.h"
#include "avbd_adjoint_math.cuh"
#include "avbd_record.hpp"

using namespace avbd::adj;

namespace {

constexpr int ADJ_MAX_BODIES = 128;  // bodies of a world at most
constexpr int ADJ_BLOCK = 64;        // threads a world (a block): bodies and points are strided over them
constexpr int ADJ_MAX_POINTS = 1024;  // points of a world in one step at most
constexpr int ADJ_BLOCKS_PER_SM = 8;  // worlds in flight per SM in the replay: registers capped at 128 a thread
constexpr double PEN_MIN = 1.0, PEN_MAX = 1e10, PIVOT = 1e-5;

// A body's primal solve at one iteration, kept by the segment recompute for the reverse sweep: its
// factorization (L's lower triangle, D, 1/D), right-hand side, step and floored pivots
struct FactRec {
  double L[15], D[6], invD[6], rhs[6], delta[6];
  int floored;
};
// x = H^-1 b from a kept factorization, read in place (L's row i, column j < i at i (i - 1) / 2 + j):
// solve6's operations in solve6's order
__device__ inline void solvePacked(const FactRec& fr, const double* b, double* x) {
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    double s = b[i];
#pragma unroll
    for (int k = 0; k < i; k++) s -= fr.L[i * (i - 1) / 2 + k] * y[k];
    y[i] = s;
  }
#pragma unroll
  for (int i = 5; i >= 0; i--) {
    double s = y[i] * fr.invD[i];
#pragma unroll
    for (int k = i + 1; k < 6; k++) s -= fr.L[k * (k - 1) / 2 + i] * x[k];
    x[i] = s;
  }
}

struct AdjDev {
  int W, K, I, ck;
  double dt, g, alpha, gamma, beta, margin;
  const int* bodyFirst;  // W + 1
  const D3* pos0;
  const D4* rot0;
  const double* prevVz0;
  const D3* unitMoment;
  const int* dynamic;
  const double* fricStatic;
  const int* manFirst;  // K x (W + 1), global manifold index
  const int* ptFirst;   // K x (W + 1)
  const int2* manAB;    // world-local bodies
  const D3* basis;      // 3 rows per manifold
  const D3* anchor;   // 2 per point: rA, rB in the bodies' frames
  const int* ptMan;   // global manifold index
  const int* ptPrev;  // global index into the previous step's points, or -1
  const int* color;   // K x bodies (-1: static)
  const int* ncol;    // K x W
  int nb, maxPts;
  // params (8 per body), target (7 per body)
  const double* params;
  const double* target;
  // state (per body) and per-world point buffers
  D3 *pos, *vel, *ang, *ipos, *ypos;
  D4 *rot, *irot, *yrot;
  QInv *irotI, *yrotI;  // the step-start and inertial rotations prepared for qsub
  double* pvz;
  D3 *lam, *pen, *lamP, *penP, *C0;  // world w's points at w * maxPts
  // checkpoints: every ck steps, the body state and the last step's points
  D3 *ckPos, *ckVel, *ckAng, *ckLam, *ckPen;
  D4* ckRot;
  double* ckPvz;
  // segment: the start state of each step of a segment
  D3 *sgPos, *sgVel, *sgAng, *sgLam, *sgPen;
  D4* sgRot;
  double* sgPvz;
  // per step of a segment: its per-iteration snapshots (I + 1), start poses, inertial targets, C0
  D3 *snPos, *snLam, *snPen;
  D4* snRot;
  D3 *stIpos, *stYpos, *stC0;
  D4 *stIrot, *stYrot;
  FactRec* snFact;  // I x bodies per step
  // cotangents
  D3 *gPos, *gVel, *gAng, *gIpos, *gYpos;
  D4 *gRot, *gIrot, *gYrot;
  double *gPvz, *gMass, *gMu;
  D3 *gLam, *gPen, *gLamP, *gPenP, *gC0;
  double* loss;  // per world
  double* finalPose;
  double* floorWork;  // per world, ADJ_GROUP x (H's cotangent 36, L's 36): a floored factorization's reverse
};

__device__ inline void atomicAdd3(D3* a, D3 v) {
  atomicAdd(&a->x, v.x);
  atomicAdd(&a->y, v.y);
  atomicAdd(&a->z, v.z);
}
__device__ inline void atomicAdd4(D4* a, D4 v) {
  atomicAdd(&a->x, v.x);
  atomicAdd(&a->y, v.y);
  atomicAdd(&a->z, v.z);
  atomicAdd(&a->w, v.w);
}

// The world's view of step s: its manifolds, points and incidence (CSR in shared memory)
struct StepView {
  int m0, m1, p0, p1, b0, nb, ncol;
  const int* color;
};
__device__ inline StepView viewOf(const AdjDev& D, int s, int w) {
  StepView v;
  v.m0 = D.manFirst[s * (D.W + 1) + w];
  v.m1 = D.manFirst[s * (D.W + 1) + w + 1];
  v.p0 = D.ptFirst[s * (D.W + 1) + w];
  v.p1 = D.ptFirst[s * (D.W + 1) + w + 1];
  v.b0 = D.bodyFirst[w];
  v.nb = D.bodyFirst[w + 1] - v.b0;
  v.ncol = D.ncol[s * D.W + w];
  v.color = D.color + (size_t)s * D.nb + v.b0;
  return v;
}

constexpr int ADJ_MAX_COLORS = 64;
constexpr int ADJ_GROUP = 16;  // bodies of one colour solved together, a thread each
constexpr int ADJ_ROW = 27;    // an incidence's share of its body's system: H's lower triangle, g

// The step's solve positions: its dynamic coloured bodies by colour, then by index; a colour's
// bodies are positions s_colStart[c] .. s_colStart[c + 1], and their incidences (local point |
// position << 16) are contiguous in s_inc, position p's at s_incStart[p] .. s_incStart[p + 1].
__shared__ int s_colStart[ADJ_MAX_COLORS + 1];
__shared__ int s_colBody[ADJ_MAX_BODIES];
__shared__ int s_posOf[ADJ_MAX_BODIES];
__shared__ int s_nSolved;
__shared__ int s_incStart[ADJ_MAX_BODIES + 1];
__shared__ int s_inc[2 * ADJ_MAX_POINTS];
__shared__ int s_color[ADJ_MAX_BODIES];
// Dynamic shared memory: a chunk of incidences, a row each (its share of the body's system, or its
// own-body cotangents), then, in the reverse sweep, a group's bodies: step, cotangent of g, and for a
// floored factorization the cotangents of H and L
struct BodyVjp {
  double delta[6], w[6];
  int floored;
};
extern __shared__ __align__(16) double s_dyn[];
constexpr size_t ADJ_SMEM_ROWS = sizeof(double) * ADJ_BLOCK * ADJ_ROW;
constexpr size_t ADJ_SMEM_FORWARD = ADJ_SMEM_ROWS, ADJ_SMEM_BACKWARD = ADJ_SMEM_ROWS + sizeof(BodyVjp) * ADJ_GROUP;
__device__ inline double* rowOf(int i) { return s_dyn + size_t(i) * ADJ_ROW; }
// In the reverse sweep an incidence's row is its own body's cotangents (14); a group slot's sums of
// them follow the rows, so that they stay in shared memory rather than registers across the
// incidences' long evaluation
constexpr int ADJ_OWN = 14;
__device__ inline double* ownRow(int i) { return s_dyn + size_t(i) * ADJ_OWN; }
__device__ inline double* ownSum(int slot) { return s_dyn + size_t(ADJ_BLOCK) * ADJ_OWN + size_t(slot) * ADJ_OWN; }
static_assert(size_t(ADJ_BLOCK + ADJ_GROUP) * ADJ_OWN <= size_t(ADJ_BLOCK) * ADJ_ROW, "the reverse rows and sums fit in the rows");
__device__ inline BodyVjp* bodyVjp() { return reinterpret_cast<BodyVjp*>(s_dyn + size_t(ADJ_BLOCK) * ADJ_ROW); }
// While the incidence is built the rows are free: the step's points' bodies (world-local) go there
__device__ inline int2* pointBodies() { return reinterpret_cast<int2*>(s_dyn); }
static_assert(sizeof(int2) * ADJ_MAX_POINTS <= ADJ_SMEM_ROWS, "a step's point bodies fit in the rows");
// Group slot i's floored-factorization cotangents (H's, then L's): global, as floored pivots are rare
__device__ inline double* floorHb(const AdjDev& D, int i) { return D.floorWork + (size_t(blockIdx.x) * ADJ_GROUP + i) * 72; }

__device__ void buildIncidence(const AdjDev& D, const StepView& v) {
  const int tid = threadIdx.x;
  for (int i = tid; i <= ADJ_MAX_COLORS; i += blockDim.x) s_colStart[i] = 0;
  for (int b = tid; b < v.nb; b += blockDim.x) s_color[b] = v.color[b];
  __syncthreads();
  for (int b = tid; b < v.nb; b += blockDim.x) {
    const int c = s_color[b];
    if (c >= 0 && c < v.ncol) atomicAdd(&s_colStart[c + 1], 1);
  }
  __syncthreads();
  if (tid == 0) {
    for (int c = 0; c < ADJ_MAX_COLORS; c++) s_colStart[c + 1] += s_colStart[c];
    s_nSolved = s_colStart[ADJ_MAX_COLORS];
  }
  __syncthreads();
  // a colour's bodies by index: a body's position is its colour's start + the bodies of its colour
  // before it
  for (int b = tid; b < v.nb; b += blockDim.x) {
    const int c = s_color[b];
    int pos = -1;
    if (c >= 0 && c < v.ncol) {
      int r = 0;
      for (int j = 0; j < b; j++) r += s_color[j] == c;
      pos = s_colStart[c] + r;
      s_colBody[pos] = b;
    }
    s_posOf[b] = pos;
  }
  for (int i = tid; i <= s_nSolved; i += blockDim.x) s_incStart[i] = 0;
  // the step's points' bodies, once, for the counts and the per-body fill
  const int np = v.p1 - v.p0;
  int2* s_ptAB = pointBodies();
  for (int lk = tid; lk < np; lk += blockDim.x) s_ptAB[lk] = D.manAB[D.ptMan[v.p0 + lk]];
  __syncthreads();
  for (int lk = tid; lk < np; lk += blockDim.x) {
    const int2 ab = s_ptAB[lk];
    const int pa = s_posOf[ab.x], pb = s_posOf[ab.y];
    if (pa >= 0) atomicAdd(&s_incStart[pa + 1], 1);
    if (pb >= 0) atomicAdd(&s_incStart[pb + 1], 1);
  }
  __syncthreads();
  if (tid == 0)
    for (int i = 0; i < s_nSolved; i++) s_incStart[i + 1] += s_incStart[i];
  __syncthreads();
  // fill in point order per body (deterministic)
  for (int p = tid; p < s_nSolved; p += blockDim.x) {
    const int lb = s_colBody[p];
    int o = s_incStart[p];
    for (int lk = 0; lk < np; lk++) {
      const int2 ab = s_ptAB[lk];
      if (ab.x == lb || ab.y == lb) s_inc[o++] = lk | (p << 16);
    }
  }
  __syncthreads();
}

__device__ inline double mu(const AdjDev& D, int gb) { return D.dynamic[gb] ? D.params[8 * gb + 7] : D.fricStatic[gb]; }
__device__ inline double mass(const AdjDev& D, int gb) { return D.params[8 * gb + 6]; }

// C, F of point k (manifold.ts:139-168 with the GPU's rules) at poses (xa, qa), (xb, qb) and the
// step-start poses; lam, pen the point's current values
struct PointEval {
  D3 rAW, rBW, dAL, dAA, dBL, dBA, C, Fraw, F;
  double fs, bd, fr;
  bool clamped;
};
__device__ inline void evalPoint(const AdjDev& D, int k, D3 xa, D4 qa, D3 xa0, const QInv& qa0, D3 xb, D4 qb, D3 xb0, const QInv& qb0, D3 c0, D3 lam, D3 pen, double fr,
                                 PointEval& e) {
  const D3* B = D.basis + 3 * D.ptMan[k];
  e.rAW = rotate(qa, D.anchor[2 * k]);
  e.rBW = rotate(qb, D.anchor[2 * k + 1]);
  e.dAL = xa - xa0;
  e.dAA = qsubI(qa, qa0);
  e.dBL = xb - xb0;
  e.dBA = qsubI(qb, qb0);
  for (int c = 0; c < 3; c++) {
    D3 bk = B[c];
    double v = comp(c0, c) * (1.0 - D.alpha);
    v = v + dot(bk, e.dAL) - dot(bk, e.dBL) + dot(cross(e.rAW, bk), e.dAA) + dot(cross(e.rBW, -bk), e.dBA);
    setComp(e.C, c, v);
    setComp(e.Fraw, c, comp(pen, c) * v + comp(lam, c));
  }
  e.F = e.Fraw;
  e.F.x = fmin(e.F.x, 0.0);
  e.fr = fr;
  e.bd = fabs(e.F.x) * fr;
  e.fs = sqrt(e.F.y * e.F.y + e.F.z * e.F.z);
  e.clamped = e.fs > e.bd && e.fs > 0.0;
  if (e.clamped) {
    e.F.y = e.F.y * (e.bd / e.fs);
    e.F.z = e.F.z * (e.bd / e.fs);
  }
}

// The cotangents of (C, lam, pen, friction) from the cotangent of F
__device__ inline void evalFVjp(const PointEval& e, D3 lam, D3 pen, D3 gF, D3& gC, D3& gLam, D3& gPen, double& gFr) {
  D3 gRaw{0, 0, 0};
  double gFx = gF.x;  // of the min'd normal force
  if (e.clamped) {
    double s = e.bd / e.fs;
    double dotFR = gF.y * e.Fraw.y + gF.z * e.Fraw.z;
    gRaw.y = s * gF.y - (e.bd / (e.fs * e.fs * e.fs)) * dotFR * e.Fraw.y;
    gRaw.z = s * gF.z - (e.bd / (e.fs * e.fs * e.fs)) * dotFR * e.Fraw.z;
    double gBd = dotFR / e.fs;
    gFr += gBd * fabs(e.F.x);
    gFx += gBd * e.fr * (e.F.x < 0.0 ? -1.0 : 1.0);
  } else {
    gRaw.y = gF.y;
    gRaw.z = gF.z;
  }
  gRaw.x = e.Fraw.x < 0.0 ? gFx : 0.0;  // min(raw, 0)
  for (int c = 0; c < 3; c++) {
    double r = comp(gRaw, c);
    setComp(gC, c, comp(gC, c) + comp(pen, c) * r);
    setComp(gPen, c, comp(gPen, c) + comp(e.C, c) * r);
    setComp(gLam, c, comp(gLam, c) + r);
  }
}

// The cotangents of the poses, step-start poses and C0 from the cotangent of C
__device__ inline void evalCVjp(const AdjDev& D, int k, D4 qa, D4 qa0, const QInv& ia0, D4 qb, D4 qb0, const QInv& ib0, const PointEval& e, D3 gC, D3& gXa, D4& gQa, D3& gXa0, D4& gQa0,
                                D3& gXb, D4& gQb, D3& gXb0, D4& gQb0, D3& gC0) {
  const D3* B = D.basis + 3 * D.ptMan[k];
  D3 gdAL{0, 0, 0}, gdAA{0, 0, 0}, gdBL{0, 0, 0}, gdBA{0, 0, 0}, grA{0, 0, 0}, grB{0, 0, 0};
  for (int c = 0; c < 3; c++) {
    double g = comp(gC, c);
    D3 bk = B[c];
    setComp(gC0, c, comp(gC0, c) + g * (1.0 - D.alpha));
    gdAL += bk * g;
    gdBL -= bk * g;
    gdAA += cross(e.rAW, bk) * g;
    gdBA += cross(e.rBW, -bk) * g;
    grA += cross(bk, e.dAA) * g;
    grB += cross(-bk, e.dBA) * g;
  }
  gXa += gdAL;
  gXa0 -= gdAL;
  gXb += gdBL;
  gXb0 -= gdBL;
  qsubVjpI(qa, qa0, ia0, gdAA, gQa, gQa0);
  qsubVjpI(qb, qb0, ib0, gdBA, gQb, gQb0);
  gQa += rotateVjpQ(qa, D.anchor[2 * k], grA);
  gQb += rotateVjpQ(qb, D.anchor[2 * k + 1], grB);
}

// Incidence `entry`'s share of its body's system at the poses poseOf gives: H's lower triangle (21,
// row-major) and g (6), into row
template <class PoseOf>
__device__ inline void incidenceRows(const AdjDev& D, const StepView& v, int wpt, int entry, const D3* lamCur, const D3* penCur, PoseOf poseOf,
                                     double* row) {
  const int lk = entry & 0xffff, k = v.p0 + lk;
  const int gb = v.b0 + s_colBody[entry >> 16];
  const int2 ab = D.manAB[D.ptMan[k]];
  const int a = v.b0 + ab.x, b = v.b0 + ab.y;
  D3 xa, xb;
  D4 qa, qb;
  poseOf(a, xa, qa);
  poseOf(b, xb, qb);
  PointEval e;
  evalPoint(D, k, xa, qa, D.ipos[a], D.irotI[a], xb, qb, D.ipos[b], D.irotI[b], D.C0[wpt + lk], lamCur[wpt + lk], penCur[wpt + lk],
            sqrt(mu(D, a) * mu(D, b)), e);
  const double sg = gb == a ? 1.0 : -1.0;
  const D3 rr = gb == a ? e.rAW : e.rBW;
  const D3* B = D.basis + 3 * D.ptMan[k];
  double h[21], r[6];
  for (int i = 0; i < 21; i++) h[i] = 0.0;
  for (int i = 0; i < 6; i++) r[i] = 0.0;
  for (int c = 0; c < 3; c++) {
    const D3 l = B[c] * sg;
    const D3 aa = cross(rr, l);
    const double kk = comp(penCur[wpt + lk], c), F = comp(e.F, c);
    const double J[6] = {l.x, l.y, l.z, aa.x, aa.y, aa.z};
    int o = 0;
    for (int i = 0; i < 6; i++)
      for (int j = 0; j <= i; j++) h[o++] += kk * J[i] * J[j];
    for (int i = 0; i < 6; i++) r[i] += J[i] * F;
  }
  for (int i = 0; i < 21; i++) row[i] = h[i];
  for (int i = 0; i < 6; i++) row[21 + i] = r[i];
}

// The bodies at positions g0..g1 (thread tid: position g0 + tid) sum their incidences' rows, a chunk
// of incidences at a time (one per thread), in incidence order
template <class PoseOf>
__device__ inline void groupRows(const AdjDev& D, const StepView& v, int wpt, int g0, int g1, const D3* lamCur, const D3* penCur, PoseOf poseOf,
                                 double* acc) {
  const int tid = threadIdx.x;
  for (int i = 0; i < ADJ_ROW; i++) acc[i] = 0.0;
  const int i0 = s_incStart[g0], i1 = s_incStart[g1];
  for (int ch = i0; ch < i1; ch += blockDim.x) {
    if (ch + tid < i1) incidenceRows(D, v, wpt, s_inc[ch + tid], lamCur, penCur, poseOf, rowOf(tid));
    __syncthreads();
    if (tid < g1 - g0) {
      const int p = g0 + tid;
      const int u0 = max(s_incStart[p], ch), u1 = min(s_incStart[p + 1], ch + int(blockDim.x));
      for (int u = u0; u < u1; u++)
        for (int i = 0; i < ADJ_ROW; i++) acc[i] += rowOf(u - ch)[i];
    }
    __syncthreads();
  }
}

// Body gb's system: its rows' sums and its inertia (solver.ts:300-318)
template <class PoseOf>
__device__ inline void bodySystem(const AdjDev& D, int gb, const double* acc, PoseOf poseOf, Sys6& S, double* g) {
  int o = 0;
  for (int i = 0; i < 6; i++)
    for (int j = 0; j <= i; j++) S.A[i][j] = acc[o++];
  for (int i = 0; i < 6; i++) g[i] = acc[21 + i];
  const double dt2 = D.dt * D.dt, m = mass(D, gb) / dt2;
  const D3 I = D.unitMoment[gb] * m;
  D3 x;
  D4 q;
  poseOf(gb, x, q);
  S.A[0][0] += m;
  S.A[1][1] += m;
  S.A[2][2] += m;
  S.A[3][3] += I.x;
  S.A[4][4] += I.y;
  S.A[5][5] += I.z;
  const D3 gl = (x - D.ypos[gb]) * m, qd = qsubI(q, D.yrotI[gb]);
  g[0] += gl.x;
  g[1] += gl.y;
  g[2] += gl.z;
  g[3] += I.x * qd.x;
  g[4] += I.y * qd.y;
  g[5] += I.z * qd.z;
}

// One step of the replay (the oracle's stepGpu with the recorded structure). With snapshots, the
// poses after the warm start and after each iteration, and the points after each dual, are kept.
__device__ void stepForward(const AdjDev& D, int s, int w, int slot) {
  const bool snapshots = slot >= 0;
  const size_t snB = snapshots ? (size_t)slot * (D.I + 1) * D.nb : 0, snP = snapshots ? (size_t)slot * (D.I + 1) * D.W * D.maxPts : 0;
  const StepView v = viewOf(D, s, w);
  const int wpt = w * D.maxPts;
  const int np = v.p1 - v.p0;
  const double dt = D.dt;
  buildIncidence(D, v);
  // points: warm starts and C(x-)
  for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
    int k = v.p0 + lk;
    int pv = D.ptPrev[k];
    D3 l{0, 0, 0}, pe{0, 0, 0};
    if (pv >= 0) {
      int plk = pv - D.ptFirst[(s - 1) * (D.W + 1) + w];
      l = D.lamP[wpt + plk];
      pe = D.penP[wpt + plk];
    }
    D3 lw = l * (D.alpha * D.gamma), pw;
    for (int c = 0; c < 3; c++) setComp(pw, c, fmin(fmax(comp(pe, c) * D.gamma, PEN_MIN), PEN_MAX));
    int2 ab = D.manAB[D.ptMan[k]];
    int a = v.b0 + ab.x, b = v.b0 + ab.y;
    D3 d = (rotate(D.rot[a], D.anchor[2 * k]) + D.pos[a]) - (rotate(D.rot[b], D.anchor[2 * k + 1]) + D.pos[b]);
    const D3* B = D.basis + 3 * D.ptMan[k];
    D3 c0{dot(B[0], d) + D.margin, dot(B[1], d), dot(B[2], d)};
    D.lam[wpt + lk] = lw;
    D.pen[wpt + lk] = pw;
    D.C0[wpt + lk] = c0;
  }
  __syncthreads();
  // bodies: inertial targets and the warm-start guess (solver.ts:273-295, up = z)
  for (int bi = threadIdx.x; bi < v.nb; bi += blockDim.x) {
    int gb = v.b0 + bi;
    D.ipos[gb] = D.pos[gb];
    D.irot[gb] = D.rot[gb];
    D.irotI[gb] = qinv(D.rot[gb]);
    if (D.dynamic[gb]) {
      D3 x = D.pos[gb], u = D.vel[gb];
      D4 q = D.rot[gb];
      D3 y = x + u * dt;
      y.z = y.z + D.g * (dt * dt);
      D.ypos[gb] = y;
      D4 qt = qaddv(q, D.ang[gb] * dt);
      D.yrot[gb] = qt;
      D.yrotI[gb] = qinv(qt);
      double sgn = D.g < 0 ? -1.0 : (D.g > 0 ? 1.0 : 0.0);
      double accelExt = (u.z - D.pvz[gb]) / dt * sgn;
      double wgt = fmin(fmax(accelExt / fabs(D.g), 0.0), 1.0);
      D3 xn = x + u * dt;
      xn.z = xn.z + D.g * (wgt * dt * dt);
      D.pos[gb] = xn;
      D.rot[gb] = qt;
    }
    if (snapshots) {
      D.snPos[snB + gb] = D.pos[gb];
      D.snRot[snB + gb] = D.rot[gb];
      D.stIpos[(size_t)slot * D.nb + gb] = D.ipos[gb];
      D.stIrot[(size_t)slot * D.nb + gb] = D.irot[gb];
      D.stYpos[(size_t)slot * D.nb + gb] = D.ypos[gb];
      D.stYrot[(size_t)slot * D.nb + gb] = D.yrot[gb];
    }
  }
  if (snapshots)
    for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
      D.snLam[snP + wpt + lk] = D.lam[wpt + lk];
      D.snPen[snP + wpt + lk] = D.pen[wpt + lk];
      D.stC0[(size_t)slot * D.W * D.maxPts + wpt + lk] = D.C0[wpt + lk];
    }
  __syncthreads();
  auto livePose = [&](int b, D3& x, D4& q) {
    x = D.pos[b];
    q = D.rot[b];
  };
  for (int it = 0; it < D.I; it++) {
    for (int c = 0; c < v.ncol; c++) {  // the colour's bodies in groups, a thread each
      for (int g0 = s_colStart[c]; g0 < s_colStart[c + 1]; g0 += ADJ_GROUP) {
        const int g1 = min(g0 + ADJ_GROUP, s_colStart[c + 1]);
        double acc[ADJ_ROW];
        groupRows(D, v, wpt, g0, g1, D.lam, D.pen, livePose, acc);
        if (threadIdx.x < g1 - g0) {
          const int gb = v.b0 + s_colBody[g0 + threadIdx.x];
          Sys6 S;
          double rhs[6], dx[6];
          bodySystem(D, gb, acc, livePose, S, rhs);
          LDLT6 F;
          const int floored = factor6(S, F, PIVOT);
          solve6(F, rhs, dx);
          D.pos[gb] = D.pos[gb] - D3{dx[0], dx[1], dx[2]};
          D.rot[gb] = qaddv(D.rot[gb], D3{-dx[3], -dx[4], -dx[5]});
          if (snapshots) {
            FactRec& fr = D.snFact[(size_t(slot) * D.I + it) * D.nb + gb];
            int o = 0;
            for (int i = 1; i < 6; i++)
              for (int j = 0; j < i; j++) fr.L[o++] = F.L[i][j];
            for (int i = 0; i < 6; i++) {
              fr.D[i] = F.D[i];
              fr.invD[i] = F.invD[i];
              fr.rhs[i] = rhs[i];
              fr.delta[i] = dx[i];
            }
            fr.floored = floored;
          }
        }
        __syncthreads();
      }
    }
    // duals (manifold.ts:202-217)
    for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
      int k = v.p0 + lk;
      int2 ab = D.manAB[D.ptMan[k]];
      int a = v.b0 + ab.x, b = v.b0 + ab.y;
      PointEval e;
      evalPoint(D, k, D.pos[a], D.rot[a], D.ipos[a], D.irotI[a], D.pos[b], D.rot[b], D.ipos[b], D.irotI[b], D.C0[wpt + lk], D.lam[wpt + lk], D.pen[wpt + lk],
                sqrt(mu(D, a) * mu(D, b)), e);
      D3 pen = D.pen[wpt + lk];
      if (e.F.x < 0.0) pen.x = fmin(pen.x + D.beta * fabs(e.C.x), PEN_MAX);
      if (e.fs <= e.bd) {
        pen.y = fmin(pen.y + D.beta * fabs(e.C.y), PEN_MAX);
        pen.z = fmin(pen.z + D.beta * fabs(e.C.z), PEN_MAX);
      }
      D.lam[wpt + lk] = e.F;
      D.pen[wpt + lk] = pen;
    }
    __syncthreads();
    if (snapshots) {
      for (int bi = threadIdx.x; bi < v.nb; bi += blockDim.x) {
        int gb = v.b0 + bi;
        D.snPos[snB + (size_t)(it + 1) * D.nb + gb] = D.pos[gb];
        D.snRot[snB + (size_t)(it + 1) * D.nb + gb] = D.rot[gb];
      }
      for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
        D.snLam[snP + (size_t)(it + 1) * D.W * D.maxPts + wpt + lk] = D.lam[wpt + lk];
        D.snPen[snP + (size_t)(it + 1) * D.W * D.maxPts + wpt + lk] = D.pen[wpt + lk];
      }
      __syncthreads();
    }
  }
  // velocities (solver.ts:328-334)
  for (int bi = threadIdx.x; bi < v.nb; bi += blockDim.x) {
    int gb = v.b0 + bi;
    D.pvz[gb] = D.vel[gb].z;
    if (D.dynamic[gb]) {
      D.vel[gb] = (D.pos[gb] - D.ipos[gb]) * (1.0 / dt);
      D.ang[gb] = qsub(D.rot[gb], D.irot[gb]) * (1.0 / dt);
    }
  }
  // this step's points become the last step's
  for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
    D.lamP[wpt + lk] = D.lam[wpt + lk];
    D.penP[wpt + lk] = D.pen[wpt + lk];
  }
  __syncthreads();
}

__device__ void loadInitial(const AdjDev& D, int w) {
  const int b0 = D.bodyFirst[w], nb = D.bodyFirst[w + 1] - b0;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    int gb = b0 + bi;
    const double* q = D.params + 8 * gb;
    D.pos[gb] = D.pos0[gb];
    D.rot[gb] = D.rot0[gb];
    D.vel[gb] = D.dynamic[gb] ? D3{q[0], q[1], q[2]} : D3{0, 0, 0};
    D.ang[gb] = D.dynamic[gb] ? D3{q[3], q[4], q[5]} : D3{0, 0, 0};
    D.pvz[gb] = D.prevVz0[gb];
  }
  __syncthreads();
}

// State copies: `bodies and last step's points` to/from a checkpoint or segment slot
__device__ void saveState(const AdjDev& D, int w, int np, D3* P, D4* R, D3* V, D3* A, double* Z, D3* L, D3* N, size_t slot) {
  const int b0 = D.bodyFirst[w], nb = D.bodyFirst[w + 1] - b0;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    int gb = b0 + bi;
    size_t o = slot * D.nb + gb;
    P[o] = D.pos[gb];
    R[o] = D.rot[gb];
    V[o] = D.vel[gb];
    A[o] = D.ang[gb];
    Z[o] = D.pvz[gb];
  }
  for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
    size_t o = slot * D.W * D.maxPts + w * D.maxPts + lk;
    L[o] = D.lamP[w * D.maxPts + lk];
    N[o] = D.penP[w * D.maxPts + lk];
  }
  __syncthreads();
}
__device__ void loadState(const AdjDev& D, int w, int np, const D3* P, const D4* R, const D3* V, const D3* A, const double* Z, const D3* L, const D3* N,
                          size_t slot) {
  const int b0 = D.bodyFirst[w], nb = D.bodyFirst[w + 1] - b0;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    int gb = b0 + bi;
    size_t o = slot * D.nb + gb;
    D.pos[gb] = P[o];
    D.rot[gb] = R[o];
    D.vel[gb] = V[o];
    D.ang[gb] = A[o];
    D.pvz[gb] = Z[o];
  }
  for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
    size_t o = slot * D.W * D.maxPts + w * D.maxPts + lk;
    D.lamP[w * D.maxPts + lk] = L[o];
    D.penP[w * D.maxPts + lk] = N[o];
  }
  __syncthreads();
}
__device__ inline int pointsBefore(const AdjDev& D, int s, int w) {  // the last step's point count (step s's input)
  if (s == 0) return 0;
  return D.ptFirst[(s - 1) * (D.W + 1) + w + 1] - D.ptFirst[(s - 1) * (D.W + 1) + w];
}

__device__ void worldLoss(const AdjDev& D, int w) {
  const int b0 = D.bodyFirst[w], nb = D.bodyFirst[w + 1] - b0;
  __shared__ double s_loss[ADJ_BLOCK];
  double l = 0.0;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    int gb = b0 + bi;
    const double* t = D.target + 7 * gb;
    D3 x = D.pos[gb];
    D4 q = D.rot[gb];
    if (D.dynamic[gb]) {
      double d[7] = {x.x - t[0], x.y - t[1], x.z - t[2], q.x - t[3], q.y - t[4], q.z - t[5], q.w - t[6]};
      for (int k = 0; k < 7; k++) l += d[k] * d[k];
    }
    if (D.finalPose) {
      double* o = D.finalPose + 7 * gb;
      o[0] = x.x; o[1] = x.y; o[2] = x.z; o[3] = q.x; o[4] = q.y; o[5] = q.z; o[6] = q.w;
    }
  }
  s_loss[threadIdx.x] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < (int)blockDim.x; i++) s += s_loss[i];
    D.loss[w] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(ADJ_BLOCK, ADJ_BLOCKS_PER_SM) k_adj_forward(AdjDev D) {
  const int w = blockIdx.x;
  loadInitial(D, w);
  for (int s = 0; s < D.K; s++) {
    if (s % D.ck == 0) saveState(D, w, pointsBefore(D, s, w), D.ckPos, D.ckRot, D.ckVel, D.ckAng, D.ckPvz, D.ckLam, D.ckPen, s / D.ck);
    stepForward(D, s, w, -1);
  }
  worldLoss(D, w);
}

// --- reverse ------------------------------------------------------------------------------------------
// Incidence `entry` of a body in the reverse sweep (its body's step, cotangent of g and floored
// reverse in the group's BodyVjp): the cotangents from its rows go to its partner's pose and step-start pose,
// its point's lambda, penalty and C0 and the friction coefficients (atomically), and to its own
// body's pose and step-start pose, returned in out (gX 3, gQ 4, gX0 3, gQ0 4).
template <class PoseOf>
__device__ inline void incidenceVjp(const AdjDev& D, const StepView& v, int wpt, int entry, int g0, const D3* lamIn, const D3* penIn, PoseOf poseOf,
                                    double* out) {
  const int lk = entry & 0xffff, k = v.p0 + lk, pos = entry >> 16;
  const int gb = v.b0 + s_colBody[pos];
  const BodyVjp& bv = bodyVjp()[pos - g0];
  const D3 dL{bv.delta[0], bv.delta[1], bv.delta[2]}, dA{bv.delta[3], bv.delta[4], bv.delta[5]};
  const D3 wl{bv.w[0], bv.w[1], bv.w[2]}, wa{bv.w[3], bv.w[4], bv.w[5]};
  const int floored = bv.floored;
  const int2 ab = D.manAB[D.ptMan[k]];
  const int a = v.b0 + ab.x, b = v.b0 + ab.y;
  D3 xa, xb;
  D4 qa, qb;
  poseOf(a, xa, qa);
  poseOf(b, xb, qb);
  const double fr = sqrt(mu(D, a) * mu(D, b));
  PointEval e;
  const D3 lamv = lamIn[wpt + lk], penv = penIn[wpt + lk];
  evalPoint(D, k, xa, qa, D.ipos[a], D.irotI[a], xb, qb, D.ipos[b], D.irotI[b], D.C0[wpt + lk], lamv, penv, fr, e);
  const bool isA = gb == a;
  const double sg = isA ? 1.0 : -1.0;
  const D3 r = isA ? e.rAW : e.rBW;
  const D3* B = D.basis + 3 * D.ptMan[k];
  D3 gF{0, 0, 0}, gPen{0, 0, 0}, gr{0, 0, 0};
  for (int cc = 0; cc < 3; cc++) {
    const D3 l = B[cc] * sg;
    const D3 aa = cross(r, l);
    const double kk = comp(penv, cc);
    const double wJ = dot(wl, l) + dot(wa, aa);
    double kb;
    D3 gAa;  // cotangent of a (the angular Jacobian row): F_c w_a from g, k (Hb + Hb^T) J from H
    if (!floored) {  // Hb = -(w delta^T) symmetrised
      const double dJ = dot(dL, l) + dot(dA, aa);
      kb = -wJ * dJ;
      gAa = wa * comp(e.F, cc) - (wa * dJ + dA * wJ) * kk;
    } else {
      const double J[6] = {l.x, l.y, l.z, aa.x, aa.y, aa.z};
      double MJ[3] = {0.0, 0.0, 0.0};
      kb = 0.0;
      for (int i = 0; i < 6; i++)
        for (int j = 0; j <= i; j++) {
          const double hb = floorHb(D, pos - g0)[6 * i + j];
          kb += hb * J[i] * J[j];
          if (i >= 3) MJ[i - 3] += hb * J[j];
          if (j >= 3) MJ[j - 3] += hb * J[i];
        }
      gAa = wa * comp(e.F, cc) + D3{MJ[0], MJ[1], MJ[2]} * kk;
    }
    setComp(gF, cc, wJ);
    setComp(gPen, cc, kb);
    gr += cross(l, gAa);
  }
  D3 gC{0, 0, 0}, gLam{0, 0, 0};
  double gFr = 0.0;
  evalFVjp(e, lamv, penv, gF, gC, gLam, gPen, gFr);
  D3 gXa{0, 0, 0}, gXb{0, 0, 0}, gXa0{0, 0, 0}, gXb0{0, 0, 0}, gC0{0, 0, 0};
  D4 gQa{0, 0, 0, 0}, gQb{0, 0, 0, 0}, gQa0{0, 0, 0, 0}, gQb0{0, 0, 0, 0};
  evalCVjp(D, k, qa, D.irot[a], D.irotI[a], qb, D.irot[b], D.irotI[b], e, gC, gXa, gQa, gXa0, gQa0, gXb, gQb, gXb0, gQb0, gC0);
  // the lever arm r = R(q_own) r_local
  if (isA) gQa += rotateVjpQ(qa, D.anchor[2 * k], gr);
  else gQb += rotateVjpQ(qb, D.anchor[2 * k + 1], gr);
  const D3 oX = isA ? gXa : gXb, oX0 = isA ? gXa0 : gXb0;
  const D4 oQ = isA ? gQa : gQb, oQ0 = isA ? gQa0 : gQb0;
  const int other = isA ? b : a;
  if (D.dynamic[other]) {
    atomicAdd3(&D.gPos[other], isA ? gXb : gXa);
    atomicAdd4(&D.gRot[other], isA ? gQb : gQa);
    atomicAdd3(&D.gIpos[other], isA ? gXb0 : gXa0);
    atomicAdd4(&D.gIrot[other], isA ? gQb0 : gQa0);
  }
  atomicAdd3(&D.gLam[wpt + lk], gLam);
  atomicAdd3(&D.gPen[wpt + lk], gPen);
  atomicAdd3(&D.gC0[wpt + lk], gC0);
  if (gFr != 0.0 && fr > 0.0) {
    double ma = mu(D, a), mb = mu(D, b);
    if (D.dynamic[a]) atomicAdd(&D.gMu[a], gFr * mb / (2.0 * fr));
    if (D.dynamic[b]) atomicAdd(&D.gMu[b], gFr * ma / (2.0 * fr));
  }
  out[0] = oX.x, out[1] = oX.y, out[2] = oX.z;
  out[3] = oQ.x, out[4] = oQ.y, out[5] = oQ.z, out[6] = oQ.w;
  out[7] = oX0.x, out[8] = oX0.y, out[9] = oX0.z;
  out[10] = oQ0.x, out[11] = oQ0.y, out[12] = oQ0.z, out[13] = oQ0.w;
}

// The primal updates of colour c's bodies at positions g0..g1 at iteration it, reversed (poses read
// from the snapshots the sweep read: partners of earlier colours at iteration it, the rest at
// it - 1; the points' values after the dual of iteration it - 1). Thread tid < g1 - g0 owns body
// position g0 + tid; the incidences are spread over all threads.
__device__ void primalGroupVjp(const AdjDev& D, const StepView& v, int wpt, int it, int c, int g0, int g1) {
  const int tid = threadIdx.x, nbg = g1 - g0;
  const double dt2 = D.dt * D.dt;
  const size_t prevSn = (size_t)it * D.nb, curSn = (size_t)(it + 1) * D.nb;
  const D3* lamIn = D.snLam + (size_t)it * D.W * D.maxPts;
  const D3* penIn = D.snPen + (size_t)it * D.W * D.maxPts;
  auto poseOf = [&](int b, D3& x, D4& q) {
    const size_t o = D.dynamic[b] && v.color[b - v.b0] < c ? curSn : prevSn;
    x = D.snPos[o + b];
    q = D.snRot[o + b];
  };
  if (tid < nbg) {
    const int gb = v.b0 + s_colBody[g0 + tid];
    // the forward's factorization and step, as the segment recompute kept them
    const FactRec& fr = D.snFact[size_t(it) * D.nb + gb];
    double delta[6];
#pragma unroll
    for (int i = 0; i < 6; i++) delta[i] = fr.delta[i];
    const int floored = fr.floored;
    // the new pose's cotangent: x' = x - delta_lin, q' = qaddv(q, -delta_ang)
    D3 x;
    D4 q;
    poseOf(gb, x, q);
    const D3 gXn = D.gPos[gb];
    const D4 gQn = D.gRot[gb];
    D4 gQ{0, 0, 0, 0};
    D3 gV{0, 0, 0};
    qaddvVjp(q, D3{-delta[3], -delta[4], -delta[5]}, gQn, gQ, gV);
    double gDelta[6] = {-gXn.x, -gXn.y, -gXn.z, -gV.x, -gV.y, -gV.z};
    BodyVjp& bv = bodyVjp()[tid];
    // the cotangent of g is w = H^-1 gDelta; that of H is -w delta^T symmetrised, or, through a
    // floored pivot, Hb from the factorization's reverse
    if (!floored) {
      solvePacked(fr, gDelta, bv.w);
    } else {
      LDLT6 F;
      double rhs[6];
      int o = 0;
      for (int i = 0; i < 6; i++) {
        for (int j = 0; j < i; j++) F.L[i][j] = fr.L[o++];
        F.L[i][i] = 1.0;
        F.D[i] = fr.D[i];
        F.invD[i] = fr.invD[i];
        rhs[i] = fr.rhs[i];
      }
      ldltVjpMasked(F, floored, PIVOT, rhs, delta, gDelta, bv.w, floorHb(D, tid) + 36, floorHb(D, tid));
    }
    for (int i = 0; i < 6; i++) bv.delta[i] = delta[i];
    bv.floored = floored;
  }
  __syncthreads();
  // the incidences' cotangents; each body sums its own
  if (tid < nbg)
    for (int i = 0; i < ADJ_OWN; i++) ownSum(tid)[i] = 0.0;
  const int i0 = s_incStart[g0], i1 = s_incStart[g1];
  for (int ch = i0; ch < i1; ch += blockDim.x) {
    if (ch + tid < i1) incidenceVjp(D, v, wpt, s_inc[ch + tid], g0, lamIn, penIn, poseOf, ownRow(tid));
    __syncthreads();
    if (tid < nbg) {
      const int p = g0 + tid;
      const int u0 = max(s_incStart[p], ch), u1 = min(s_incStart[p + 1], ch + int(blockDim.x));
      double* own = ownSum(tid);
      for (int u = u0; u < u1; u++)
        for (int i = 0; i < ADJ_OWN; i++) own[i] += ownRow(u - ch)[i];
    }
    __syncthreads();
  }
  if (tid < nbg) {
    const double* own = ownSum(tid);
    const int gb = v.b0 + s_colBody[g0 + tid];
    const BodyVjp& bv = bodyVjp()[tid];
    D3 x;
    D4 q;
    poseOf(gb, x, q);
    const double m = mass(D, gb) / dt2;
    const D3 Iu = D.unitMoment[gb];
    const D3 I = Iu * m;
    const D3 gXn = D.gPos[gb];
    const D4 gQn = D.gRot[gb];
    D4 gQ{0, 0, 0, 0};
    D3 gV{0, 0, 0};
    qaddvVjp(q, D3{-bv.delta[3], -bv.delta[4], -bv.delta[5]}, gQn, gQ, gV);
    const D3 wl{bv.w[0], bv.w[1], bv.w[2]}, wa{bv.w[3], bv.w[4], bv.w[5]};
    // inertia: g_lin = (x - y) m, g_ang = I qsub(q, y_rot); H_lin = m, H_ang = I (m, I over dt^2)
    const D3 gX = gXn + wl * m + D3{own[0], own[1], own[2]};
    const D3 gY = wl * (-m);
    const D3 gqd{I.x * wa.x, I.y * wa.y, I.z * wa.z};
    D4 gYq{0, 0, 0, 0};
    qsubVjpI(q, D.yrot[gb], D.yrotI[gb], gqd, gQ, gYq);
    const D3 xy = x - D.ypos[gb];
    const D3 qd = qsubI(q, D.yrotI[gb]);
    double dH, dHa;
    if (!bv.floored) {
      dH = -(bv.w[0] * bv.delta[0] + bv.w[1] * bv.delta[1] + bv.w[2] * bv.delta[2]);
      dHa = -bv.w[3] * bv.delta[3] * Iu.x - bv.w[4] * bv.delta[4] * Iu.y - bv.w[5] * bv.delta[5] * Iu.z;
    } else {
      const double* Hb = floorHb(D, tid);
      dH = Hb[0] + Hb[7] + Hb[14];
      dHa = Hb[21] * Iu.x + Hb[28] * Iu.y + Hb[35] * Iu.z;
    }
    const double gM = (dH + dot(wl, xy) + dHa + wa.x * Iu.x * qd.x + wa.y * Iu.y * qd.y + wa.z * Iu.z * qd.z) / dt2;
    D.gPos[gb] = gX;
    D.gRot[gb] = gQ + D4{own[3], own[4], own[5], own[6]};
    D.gYpos[gb] += gY;
    D.gYrot[gb] += gYq;
    D.gIpos[gb] += D3{own[7], own[8], own[9]};
    D.gIrot[gb] += D4{own[10], own[11], own[12], own[13]};
    D.gMass[gb] += gM;
  }
  __syncthreads();
}

// Point k's dual at iteration it: lambda' = F, the penalty ramps
__device__ void dualVjp(const AdjDev& D, const StepView& v, int wpt, int it, int k) {
  const int lk = k - v.p0;
  const size_t sn = (size_t)(it + 1) * D.nb;
  const D3* lamIn = D.snLam + (size_t)it * D.W * D.maxPts;
  const D3* penIn = D.snPen + (size_t)it * D.W * D.maxPts;
  int2 ab = D.manAB[D.ptMan[k]];
  int a = v.b0 + ab.x, b = v.b0 + ab.y;
  D3 xa = D.snPos[sn + a], xb = D.snPos[sn + b];
  D4 qa = D.snRot[sn + a], qb = D.snRot[sn + b];
  double fr = sqrt(mu(D, a) * mu(D, b));
  D3 lamv = lamIn[wpt + lk], penv = penIn[wpt + lk];
  PointEval e;
  evalPoint(D, k, xa, qa, D.ipos[a], D.irotI[a], xb, qb, D.ipos[b], D.irotI[b], D.C0[wpt + lk], lamv, penv, fr, e);
  D3 gLamOut = D.gLam[wpt + lk], gPenOut = D.gPen[wpt + lk];
  D3 gPen{0, 0, 0}, gC{0, 0, 0}, gLam{0, 0, 0};
  // pen' = min(pen + beta |C|, MAX) where the ramp applies, else pen
  auto ramp = [&](int c, bool on) {
    double go = comp(gPenOut, c);
    if (!on) {
      setComp(gPen, c, comp(gPen, c) + go);
      return;
    }
    double raw = comp(penv, c) + D.beta * fabs(comp(e.C, c));
    if (raw < PEN_MAX) {
      setComp(gPen, c, comp(gPen, c) + go);
      setComp(gC, c, comp(gC, c) + go * D.beta * (comp(e.C, c) < 0.0 ? -1.0 : 1.0));
    }
  };
  ramp(0, e.F.x < 0.0);
  ramp(1, e.fs <= e.bd);
  ramp(2, e.fs <= e.bd);
  double gFr = 0.0;
  evalFVjp(e, lamv, penv, gLamOut, gC, gLam, gPen, gFr);
  D3 gXa{0, 0, 0}, gXb{0, 0, 0}, gXa0{0, 0, 0}, gXb0{0, 0, 0}, gC0{0, 0, 0};
  D4 gQa{0, 0, 0, 0}, gQb{0, 0, 0, 0}, gQa0{0, 0, 0, 0}, gQb0{0, 0, 0, 0};
  evalCVjp(D, k, qa, D.irot[a], D.irotI[a], qb, D.irot[b], D.irotI[b], e, gC, gXa, gQa, gXa0, gQa0, gXb, gQb, gXb0, gQb0, gC0);
  if (D.dynamic[a]) {
    atomicAdd3(&D.gPos[a], gXa);
    atomicAdd4(&D.gRot[a], gQa);
    atomicAdd3(&D.gIpos[a], gXa0);
    atomicAdd4(&D.gIrot[a], gQa0);
  }
  if (D.dynamic[b]) {
    atomicAdd3(&D.gPos[b], gXb);
    atomicAdd4(&D.gRot[b], gQb);
    atomicAdd3(&D.gIpos[b], gXb0);
    atomicAdd4(&D.gIrot[b], gQb0);
  }
  D.gLam[wpt + lk] = gLam;  // the value before this dual
  D.gPen[wpt + lk] = gPen;
  D.gC0[wpt + lk] += gC0;
  if (gFr != 0.0 && fr > 0.0) {
    double ma = mu(D, a), mb = mu(D, b);
    if (D.dynamic[a]) atomicAdd(&D.gMu[a], gFr * mb / (2.0 * fr));
    if (D.dynamic[b]) atomicAdd(&D.gMu[b], gFr * ma / (2.0 * fr));
  }
}

// Step s backwards. On entry its start state is in segment slot `slot` and loaded (pos.., lamP/
// penP), and the cotangents of its outputs (the bodies' state, its points' lambda and penalty) are
// in gPos.. and gLam/gPen; on exit gPos.. hold those of its inputs and gLamP/gPenP those of the last
// step's points.
__device__ void stepBackward(const AdjDev& D0, int s, int w, size_t slot) {
  // this step's stored intermediates in place of the working arrays
  AdjDev D = D0;
  D.ipos = D0.stIpos + slot * D0.nb;
  D.irot = D0.stIrot + slot * D0.nb;
  D.ypos = D0.stYpos + slot * D0.nb;
  D.yrot = D0.stYrot + slot * D0.nb;
  D.C0 = D0.stC0 + slot * D0.W * D0.maxPts;
  D.snPos = D0.snPos + slot * (D0.I + 1) * D0.nb;
  D.snRot = D0.snRot + slot * (D0.I + 1) * D0.nb;
  D.snLam = D0.snLam + slot * (D0.I + 1) * D0.W * D0.maxPts;
  D.snPen = D0.snPen + slot * (D0.I + 1) * D0.W * D0.maxPts;
  D.snFact = D0.snFact + slot * D0.I * D0.nb;
  const StepView v = viewOf(D, s, w);
  const int wpt = w * D.maxPts;
  const int np = v.p1 - v.p0;
  const double dt = D.dt;
  for (int bi = threadIdx.x; bi < v.nb; bi += blockDim.x) {  // the stored step's rotations prepared for qsub
    const int gb = v.b0 + bi;
    D.irotI[gb] = qinv(D.irot[gb]);
    if (D.dynamic[gb]) D.yrotI[gb] = qinv(D.yrot[gb]);
  }
  buildIncidence(D, v);
  // velocities: v' = (x - x0)/dt, w' = qsub(q, q0)/dt, prevVz' = v_old.z
  for (int bi = threadIdx.x; bi < v.nb; bi += blockDim.x) {
    int gb = v.b0 + bi;
    D3 gv = D.gVel[gb], gw = D.gAng[gb];
    double gz = D.gPvz[gb];
    D.gIpos[gb] = D3{0, 0, 0};
    D.gIrot[gb] = D4{0, 0, 0, 0};
    D.gYpos[gb] = D3{0, 0, 0};
    D.gYrot[gb] = D4{0, 0, 0, 0};
    if (D.dynamic[gb]) {
      D4 q = D.snRot[(size_t)D.I * D.nb + gb];
      D.gPos[gb] += gv * (1.0 / dt);
      D.gIpos[gb] -= gv * (1.0 / dt);
      D4 gq{0, 0, 0, 0}, gq0{0, 0, 0, 0};
      qsubVjp(q, D.irot[gb], gw * (1.0 / dt), gq, gq0);
      D.gRot[gb] += gq;
      D.gIrot[gb] += gq0;
    } else {
      D.gPos[gb] = D3{0, 0, 0};
      D.gRot[gb] = D4{0, 0, 0, 0};
    }
    D.gVel[gb] = D3{0, 0, gz};  // the input velocity feeds prevVz'
    D.gAng[gb] = D3{0, 0, 0};
    D.gPvz[gb] = 0.0;
  }
  for (int lk = threadIdx.x; lk < np; lk += blockDim.x) D.gC0[wpt + lk] = D3{0, 0, 0};
  __syncthreads();
  for (int it = D.I - 1; it >= 0; it--) {
    for (int lk = threadIdx.x; lk < np; lk += blockDim.x) dualVjp(D, v, wpt, it, v.p0 + lk);
    __syncthreads();
    for (int c = v.ncol - 1; c >= 0; c--)  // the colour's bodies in groups (order within a colour is free)
      for (int g0 = s_colStart[c]; g0 < s_colStart[c + 1]; g0 += ADJ_GROUP) primalGroupVjp(D, v, wpt, it, c, g0, min(g0 + ADJ_GROUP, s_colStart[c + 1]));
  }
  // points' warm starts and C(x-) (the start poses' cotangents gather in gIpos/gIrot)
  const int prevFirst = s > 0 ? D.ptFirst[(s - 1) * (D.W + 1) + w] : 0;
  for (int lk = threadIdx.x; lk < np; lk += blockDim.x) {
    int k = v.p0 + lk;
    int pv = D.ptPrev[k];
    if (pv >= 0) {
      int plk = pv - prevFirst;
      D3 gl = D.gLam[wpt + lk], gp = D.gPen[wpt + lk];
      D3 pe = D.sgPen[slot * D.W * D.maxPts + wpt + plk];
      D3 gpp{0, 0, 0};
      for (int c = 0; c < 3; c++) {
        double x = comp(pe, c) * D.gamma;
        if (x > PEN_MIN && x < PEN_MAX) setComp(gpp, c, comp(gp, c) * D.gamma);
      }
      atomicAdd3(&D.gLamP[wpt + plk], gl * (D.alpha * D.gamma));  // two points may warm-start from one
      atomicAdd3(&D.gPenP[wpt + plk], gpp);
    }
    int2 ab = D.manAB[D.ptMan[k]];
    int a = v.b0 + ab.x, b = v.b0 + ab.y;
    const D3* B = D.basis + 3 * D.ptMan[k];
    D3 gc0 = D.gC0[wpt + lk];
    D3 gd = B[0] * gc0.x + B[1] * gc0.y + B[2] * gc0.z;
    if (D.dynamic[a]) {
      atomicAdd3(&D.gIpos[a], gd);
      atomicAdd4(&D.gIrot[a], rotateVjpQ(D.irot[a], D.anchor[2 * k], gd));
    }
    if (D.dynamic[b]) {
      atomicAdd3(&D.gIpos[b], -gd);
      atomicAdd4(&D.gIrot[b], rotateVjpQ(D.irot[b], D.anchor[2 * k + 1], -gd));
    }
  }
  __syncthreads();
  // bodies: the warm-start guess and the inertial targets (solver.ts:273-295)
  for (int bi = threadIdx.x; bi < v.nb; bi += blockDim.x) {
    int gb = v.b0 + bi;
    if (D.dynamic[gb]) {
      const size_t o = slot * D.nb + gb;
      const D3 u = D.sgVel[o], om = D.sgAng[o];
      const double pvz = D.sgPvz[o];
      const D4 q0 = D.irot[gb];
      D3 gxg = D.gPos[gb];  // the guess: the pose iteration 0 starts from
      D4 gqg = D.gRot[gb];
      D3 gY = D.gYpos[gb];
      D4 gYq = D.gYrot[gb];
      D3 gX0 = gxg + gY + D.gIpos[gb];
      D4 gQ0 = D.gIrot[gb];
      D3 gU = (gxg + gY) * dt;
      double sgn = D.g < 0 ? -1.0 : (D.g > 0 ? 1.0 : 0.0);
      double accelExt = (u.z - pvz) / dt * sgn;
      double wgt = accelExt / fabs(D.g);
      double gPvz = 0.0;
      if (wgt > 0.0 && wgt < 1.0) {
        double gW = gxg.z * D.g * dt * dt;
        double gA = gW / fabs(D.g);
        gU.z += gA * sgn / dt;
        gPvz = -gA * sgn / dt;
      }
      D3 gOm{0, 0, 0};
      qaddvVjp(q0, om * dt, D4{gqg.x + gYq.x, gqg.y + gYq.y, gqg.z + gYq.z, gqg.w + gYq.w}, gQ0, gOm);
      D.gPos[gb] = gX0;
      D.gRot[gb] = gQ0;
      D.gVel[gb] += gU;
      D.gAng[gb] = gOm * dt;
      D.gPvz[gb] = gPvz;
    }
  }
  __syncthreads();
}

// The reverse sweep's incidence cotangents hold more live state than 128 registers: 4 worlds an SM
// at up to 255 registers beat 8 at 128 with spills
__global__ void __launch_bounds__(ADJ_BLOCK, 4) k_adj_backward(const AdjDev D) {
  const int w = blockIdx.x;
  const int b0 = D.bodyFirst[w], nb = D.bodyFirst[w + 1] - b0;
  const int wpt = w * D.maxPts;
  for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {
    int gb = b0 + bi;
    D.gVel[gb] = D.gAng[gb] = D3{0, 0, 0};
    D.gPvz[gb] = 0.0;
    D.gMass[gb] = D.gMu[gb] = 0.0;
  }
  for (int lk = threadIdx.x; lk < D.maxPts; lk += blockDim.x) {
    D.gLam[wpt + lk] = D.gPen[wpt + lk] = D.gLamP[wpt + lk] = D.gPenP[wpt + lk] = D3{0, 0, 0};
  }
  __syncthreads();
  const int segments = (D.K + D.ck - 1) / D.ck;
  for (int sg = segments - 1; sg >= 0; sg--) {
    const int s0 = sg * D.ck, s1 = min(D.K, s0 + D.ck);
    loadState(D, w, pointsBefore(D, s0, w), D.ckPos, D.ckRot, D.ckVel, D.ckAng, D.ckPvz, D.ckLam, D.ckPen, sg);
    for (int s = s0; s < s1; s++) {
      saveState(D, w, pointsBefore(D, s, w), D.sgPos, D.sgRot, D.sgVel, D.sgAng, D.sgPvz, D.sgLam, D.sgPen, s - s0);
      stepForward(D, s, w, s - s0);
    }
    if (sg == segments - 1) {
      worldLoss(D, w);
      for (int bi = threadIdx.x; bi < nb; bi += blockDim.x) {  // the loss's cotangent: 2 (pose - target)
        int gb = b0 + bi;
        const double* t = D.target + 7 * gb;
        D3 x = D.pos[gb];
        D4 q = D.rot[gb];
        bool dyn = D.dynamic[gb];
        D.gPos[gb] = dyn ? D3{2 * (x.x - t[0]), 2 * (x.y - t[1]), 2 * (x.z - t[2])} : D3{0, 0, 0};
        D.gRot[gb] = dyn ? D4{2 * (q.x - t[3]), 2 * (q.y - t[4]), 2 * (q.z - t[5]), 2 * (q.w - t[6])} : D4{0, 0, 0, 0};
      }
      __syncthreads();
    }
    for (int s = s1 - 1; s >= s0; s--) {
      stepBackward(D, s, w, s - s0);
      // the last step's points' cotangents become the outputs' of step s - 1. They are copied, not
      // swapped: the buffers stay fixed in the struct the step functions take by reference.
      const int npv = pointsBefore(D, s, w);
      for (int lk = threadIdx.x; lk < D.maxPts; lk += blockDim.x) {
        const bool live = lk < npv;
        D.gLam[wpt + lk] = live ? D.gLamP[wpt + lk] : D3{0, 0, 0};
        D.gPen[wpt + lk] = live ? D.gPenP[wpt + lk] : D3{0, 0, 0};
        D.gLamP[wpt + lk] = D.gPenP[wpt + lk] = D3{0, 0, 0};
      }
      __syncthreads();
    }
  }
}

}  // namespace

struct avbd_adjoint {
  int device = 0;
  std::string error;
  AdjDev d{};
  std::vector<void*> allocations;
  int W = 0, nb = 0;
  std::vector<double> nominal;        // 8 per body when built from a batch recording
  uint64_t manifolds = 0, points = 0;
  bool forwardDone = false;  // the checkpoints hold the forward of lastParams
  std::vector<double> lastParams;
};

namespace {

int afail(avbd_adjoint* a, int code, const std::string& m) {
  if (a) a->error = m;
  return code;
}
template <class T>
bool aalloc(avbd_adjoint* a, T** p, size_t n) {
  void* ptr = nullptr;
  if (cudaMalloc(&ptr, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return false;
  cudaMemset(ptr, 0, std::max<size_t>(n, 1) * sizeof(T));
  a->allocations.push_back(ptr);
  *p = static_cast<T*>(ptr);
  return true;
}
template <class T>
bool aupload(avbd_adjoint* a, const T** dst, const T* src, size_t n) {
  T* p = nullptr;
  if (!aalloc(a, &p, n)) return false;
  if (n && cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return false;
  *dst = p;
  return true;
}

// The replay's working buffers, checkpoints, snapshots and cotangents (D's sizes set)
bool adjAllocWork(avbd_adjoint* a) {
  AdjDev& D = a->d;
  // shared memory sized for the blocks of several worlds on one SM
  if (cudaFuncSetAttribute(k_adj_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ADJ_SMEM_FORWARD)) != cudaSuccess ||
      cudaFuncSetAttribute(k_adj_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ADJ_SMEM_BACKWARD)) != cudaSuccess ||
      cudaFuncSetAttribute(k_adj_forward, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
      cudaFuncSetAttribute(k_adj_backward, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
    return false;
  const size_t W = size_t(D.W), K = size_t(D.K), nb = size_t(D.nb);
  bool ok = true;
  const size_t WP = W * size_t(D.maxPts), segs = (K + D.ck - 1) / D.ck, I1 = size_t(D.I) + 1;
  double* prm = nullptr;
  double* tgt = nullptr;
  ok = ok && aalloc(a, &prm, 8 * size_t(nb)) && aalloc(a, &tgt, 7 * size_t(nb));
  D.params = prm;
  D.target = tgt;
  for (D3** p : {&D.pos, &D.vel, &D.ang, &D.ipos, &D.ypos, &D.gPos, &D.gVel, &D.gAng, &D.gIpos, &D.gYpos}) ok = ok && aalloc(a, p, nb);
  for (D4** p : {&D.rot, &D.irot, &D.yrot, &D.gRot, &D.gIrot, &D.gYrot}) ok = ok && aalloc(a, p, nb);
  ok = ok && aalloc(a, &D.irotI, nb) && aalloc(a, &D.yrotI, nb);
  for (double** p : {&D.pvz, &D.gPvz, &D.gMass, &D.gMu}) ok = ok && aalloc(a, p, nb);
  for (D3** p : {&D.lam, &D.pen, &D.lamP, &D.penP, &D.C0, &D.gLam, &D.gPen, &D.gLamP, &D.gPenP, &D.gC0}) ok = ok && aalloc(a, p, WP);
  ok = ok && aalloc(a, &D.ckPos, segs * nb) && aalloc(a, &D.ckVel, segs * nb) && aalloc(a, &D.ckAng, segs * nb) && aalloc(a, &D.ckRot, segs * nb) &&
       aalloc(a, &D.ckPvz, segs * nb) && aalloc(a, &D.ckLam, segs * WP) && aalloc(a, &D.ckPen, segs * WP);
  ok = ok && aalloc(a, &D.sgPos, size_t(D.ck) * nb) && aalloc(a, &D.sgVel, size_t(D.ck) * nb) && aalloc(a, &D.sgAng, size_t(D.ck) * nb) &&
       aalloc(a, &D.sgRot, size_t(D.ck) * nb) && aalloc(a, &D.sgPvz, size_t(D.ck) * nb) && aalloc(a, &D.sgLam, size_t(D.ck) * WP) &&
       aalloc(a, &D.sgPen, size_t(D.ck) * WP);
  const size_t CK = size_t(D.ck);
  ok = ok && aalloc(a, &D.snPos, CK * I1 * nb) && aalloc(a, &D.snRot, CK * I1 * nb) && aalloc(a, &D.snLam, CK * I1 * WP) && aalloc(a, &D.snPen, CK * I1 * WP);
  ok = ok && aalloc(a, &D.snFact, CK * size_t(std::max(D.I, 1)) * nb);
  ok = ok && aalloc(a, &D.stIpos, CK * nb) && aalloc(a, &D.stIrot, CK * nb) && aalloc(a, &D.stYpos, CK * nb) && aalloc(a, &D.stYrot, CK * nb) &&
       aalloc(a, &D.stC0, CK * WP);
  double* loss = nullptr;
  double* fin = nullptr;
  double* fw = nullptr;
  ok = ok && aalloc(a, &loss, W) && aalloc(a, &fin, 7 * size_t(nb)) && aalloc(a, &fw, size_t(W) * ADJ_GROUP * 72);
  D.loss = loss;
  D.finalPose = fin;
  D.floorWork = fw;
  return ok;
}

}  // namespace

extern "C" {

int avbd_adjoint_create(const avbd_adjoint_desc* desc, avbd_adjoint** out) {
  if (!desc || !out) return AVBD_ERR_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return AVBD_ERR_NO_DEVICE;
  if (desc->device < 0 || desc->device >= count) return AVBD_ERR_INVALID;
  const uint32_t W = desc->worlds, K = desc->steps;
  if (W == 0 || K == 0 || !desc->world_first_body || !desc->bodies || !desc->step_first_manifold || !desc->step_first_point || !desc->colors ||
      !desc->color_counts)
    return AVBD_ERR_INVALID;
  const uint32_t nb = desc->world_first_body[W];
  for (uint32_t w = 0; w < W; w++)
    if (desc->world_first_body[w + 1] < desc->world_first_body[w] || desc->world_first_body[w + 1] - desc->world_first_body[w] > ADJ_MAX_BODIES)
      return AVBD_ERR_CAPACITY;  // a world holds at most 128 bodies
  const uint32_t nm = desc->step_first_manifold[K * (W + 1) - 1], npts = desc->step_first_point[K * (W + 1) - 1];
  int maxPts = 1;
  for (uint32_t s = 0; s < K; s++)
    for (uint32_t w = 0; w < W; w++) {
      int c = int(desc->step_first_point[s * (W + 1) + w + 1]) - int(desc->step_first_point[s * (W + 1) + w]);
      if (c < 0) return AVBD_ERR_INVALID;
      maxPts = std::max(maxPts, c);
    }
  if (maxPts > ADJ_MAX_POINTS) return AVBD_ERR_CAPACITY;
  // every index inside its own world and step: manifolds' bodies, points' manifolds and sources
  for (uint32_t s = 0; s < K; s++)
    for (uint32_t w = 0; w < W; w++) {
      const uint32_t m0 = desc->step_first_manifold[s * (W + 1) + w], m1 = desc->step_first_manifold[s * (W + 1) + w + 1];
      const uint32_t p0 = desc->step_first_point[s * (W + 1) + w], p1 = desc->step_first_point[s * (W + 1) + w + 1];
      const int nbw = int(desc->world_first_body[w + 1] - desc->world_first_body[w]);
      if (m1 < m0 || m1 > nm || p1 > npts) return AVBD_ERR_INVALID;
      for (uint32_t m = m0; m < m1; m++) {
        int a = desc->manifold_bodies[2 * m], b = desc->manifold_bodies[2 * m + 1];
        if (a < 0 || b < 0 || a >= nbw || b >= nbw || a == b) return AVBD_ERR_INVALID;
      }
      for (uint32_t k = p0; k < p1; k++) {
        int m = desc->point_manifold[k], pv = desc->point_prev[k];
        if (m < int(m0) || m >= int(m1)) return AVBD_ERR_INVALID;
        if (pv >= 0) {
          if (s == 0) return AVBD_ERR_INVALID;
          const int q0 = int(desc->step_first_point[(s - 1) * (W + 1) + w]), q1 = int(desc->step_first_point[(s - 1) * (W + 1) + w + 1]);
          if (pv < q0 || pv >= q1) return AVBD_ERR_INVALID;
        }
      }
      if (desc->color_counts[s * W + w] < 0 || desc->color_counts[s * W + w] > 64) return AVBD_ERR_INVALID;
    }
  cudaSetDevice(desc->device);
  auto* a = new avbd_adjoint();
  a->device = desc->device;
  a->W = int(W);
  a->nb = int(nb);
  a->manifolds = nm;
  a->points = npts;
  AdjDev& D = a->d;
  D.W = int(W);
  D.K = int(K);
  D.I = int(desc->iterations);
  D.ck = desc->checkpoint ? int(desc->checkpoint) : 10;
  D.dt = desc->dt;
  D.g = desc->gravity;
  D.alpha = desc->alpha;
  D.gamma = desc->gamma;
  D.beta = desc->beta_lin;
  D.margin = desc->contact_margin;
  D.nb = int(nb);
  D.maxPts = maxPts;
  // host-side unpacking of the body records (13 doubles each)
  std::vector<D3> pos0(nb), um(nb);
  std::vector<D4> rot0(nb);
  std::vector<double> pvz(nb), fs(nb);
  std::vector<int> dyn(nb), fb(desc->world_first_body, desc->world_first_body + W + 1);
  for (uint32_t b = 0; b < nb; b++) {
    const double* r = desc->bodies + 13 * b;
    pos0[b] = D3{r[0], r[1], r[2]};
    rot0[b] = D4{r[3], r[4], r[5], r[6]};
    pvz[b] = r[7];
    um[b] = D3{r[8], r[9], r[10]};
    dyn[b] = r[11] != 0.0;
    fs[b] = r[12];
  }
  std::vector<int> mf(desc->step_first_manifold, desc->step_first_manifold + K * (W + 1));
  std::vector<int> pf(desc->step_first_point, desc->step_first_point + K * (W + 1));
  std::vector<int2> ab(nm);
  std::vector<D3> basis(3 * size_t(nm)), anchors(2 * size_t(npts));
  for (uint32_t m = 0; m < nm; m++) {
    ab[m] = make_int2(desc->manifold_bodies[2 * m], desc->manifold_bodies[2 * m + 1]);
    for (int c = 0; c < 3; c++) basis[3 * m + c] = D3{desc->manifold_basis[9 * m + 3 * c], desc->manifold_basis[9 * m + 3 * c + 1], desc->manifold_basis[9 * m + 3 * c + 2]};
  }
  for (uint32_t k = 0; k < npts; k++) {
    const double* r = desc->point_anchors + 6 * k;
    anchors[2 * k] = D3{r[0], r[1], r[2]};
    anchors[2 * k + 1] = D3{r[3], r[4], r[5]};
  }
  bool ok = aupload(a, &D.bodyFirst, fb.data(), fb.size()) && aupload(a, &D.pos0, pos0.data(), nb) && aupload(a, &D.rot0, rot0.data(), nb) &&
            aupload(a, &D.prevVz0, pvz.data(), nb) && aupload(a, &D.unitMoment, um.data(), nb) && aupload(a, &D.dynamic, dyn.data(), nb) &&
            aupload(a, &D.fricStatic, fs.data(), nb) && aupload(a, &D.manFirst, mf.data(), mf.size()) && aupload(a, &D.ptFirst, pf.data(), pf.size()) &&
            aupload(a, &D.manAB, ab.data(), nm) && aupload(a, &D.basis, basis.data(), basis.size()) && aupload(a, &D.anchor, anchors.data(), anchors.size()) && aupload(a, &D.ptMan, desc->point_manifold, npts) && aupload(a, &D.ptPrev, desc->point_prev, npts) &&
            aupload(a, &D.color, desc->colors, size_t(K) * nb) && aupload(a, &D.ncol, desc->color_counts, size_t(K) * W);
  ok = ok && adjAllocWork(a);
  if (!ok) {
    avbd_adjoint_destroy(a);
    return AVBD_ERR_CUDA;
  }
  *out = a;
  return AVBD_OK;
}

int avbd_adjoint_create_from_batch(avbd_batch* batch, uint32_t checkpoint, avbd_adjoint** out) {
  if (!batch || !out) return AVBD_ERR_INVALID;
  *out = nullptr;
  avbd::RecordingHandoff h;
  std::string why;
  int r = avbd::batch_take_recording(batch, h, why);
  if (r) return r;
  cudaSetDevice(h.device);
  auto* a = new avbd_adjoint();
  a->device = h.device;
  a->allocations = h.mem;  // adopted: freed with the adjoint
  const uint32_t W = h.W, nb = h.nb;
  for (uint32_t w = 0; w < W; w++)
    if (h.worldFirst[w + 1] - h.worldFirst[w] > uint32_t(ADJ_MAX_BODIES)) {
      avbd_adjoint_destroy(a);
      return AVBD_ERR_CAPACITY;  // a world holds at most 128 bodies
    }
  if (h.maxPts > uint32_t(ADJ_MAX_POINTS)) {
    avbd_adjoint_destroy(a);
    return AVBD_ERR_CAPACITY;
  }
  a->W = int(W);
  a->nb = int(nb);
  a->manifolds = h.manifolds;
  a->points = h.points;
  AdjDev& D = a->d;
  D.W = int(W);
  D.K = int(h.K);
  D.I = h.params.iterations;
  D.ck = checkpoint ? int(checkpoint) : 10;
  D.dt = h.params.dt;
  D.g = h.params.gravity;
  D.alpha = h.params.alpha;
  D.gamma = h.params.gamma;
  D.beta = h.params.beta_lin;
  D.margin = h.params.contact_margin;
  D.nb = int(nb);
  D.maxPts = std::max<int>(1, int(h.maxPts));
  D.manFirst = h.manFirst;
  D.ptFirst = h.ptFirst;
  D.manAB = static_cast<const int2*>(h.manAB);
  D.basis = reinterpret_cast<const D3*>(h.basis);
  D.anchor = reinterpret_cast<const D3*>(h.anchors);
  D.ptMan = h.ptMan;
  D.ptPrev = h.ptPrev;
  D.color = h.color;
  D.ncol = h.ncol;
  std::vector<D3> pos0(nb), um(nb);
  std::vector<D4> rot0(nb);
  std::vector<double> pvz(nb), fs(nb);
  std::vector<int> dyn(nb), fb(h.worldFirst.begin(), h.worldFirst.end());
  a->nominal.assign(8 * size_t(nb), 0.0);
  for (uint32_t b = 0; b < nb; b++) {
    const avbd_body& x = h.initial[b];
    const bool d = x.mass > 0.0f;
    pos0[b] = D3{x.pos[0], x.pos[1], x.pos[2]};
    rot0[b] = D4{x.rot[0], x.rot[1], x.rot[2], x.rot[3]};
    pvz[b] = x.prev_up_vel;
    um[b] = d ? D3{double(x.moment[0]) / x.mass, double(x.moment[1]) / x.mass, double(x.moment[2]) / x.mass} : D3{0, 0, 0};
    dyn[b] = d;
    fs[b] = x.friction;
    double* q = a->nominal.data() + 8 * size_t(b);
    if (d) {
      for (int k = 0; k < 3; k++) {
        q[k] = x.vel[k];
        q[3 + k] = x.ang_vel[k];
      }
      q[6] = x.mass;
    }
    q[7] = x.friction;
  }
  bool ok = aupload(a, &D.bodyFirst, fb.data(), fb.size()) && aupload(a, &D.pos0, pos0.data(), nb) && aupload(a, &D.rot0, rot0.data(), nb) &&
            aupload(a, &D.prevVz0, pvz.data(), nb) && aupload(a, &D.unitMoment, um.data(), nb) && aupload(a, &D.dynamic, dyn.data(), nb) &&
            aupload(a, &D.fricStatic, fs.data(), nb);
  ok = ok && adjAllocWork(a);
  if (!ok) {
    avbd_adjoint_destroy(a);
    return AVBD_ERR_CUDA;
  }
  *out = a;
  return AVBD_OK;
}

int avbd_adjoint_nominal(const avbd_adjoint* a, double* params) {
  if (!a || !params) return AVBD_ERR_INVALID;
  if (a->nominal.empty()) std::memset(params, 0, sizeof(double) * 8 * size_t(a->nb));
  else std::memcpy(params, a->nominal.data(), sizeof(double) * a->nominal.size());
  return AVBD_OK;
}

int avbd_adjoint_info(const avbd_adjoint* a, uint32_t* worlds, uint32_t* steps, uint32_t* bodies, uint32_t* max_points, uint64_t* manifolds,
                      uint64_t* points) {
  if (!a) return AVBD_ERR_INVALID;
  if (worlds) *worlds = uint32_t(a->W);
  if (steps) *steps = uint32_t(a->d.K);
  if (bodies) *bodies = uint32_t(a->nb);
  if (max_points) *max_points = uint32_t(a->d.maxPts);
  if (manifolds) *manifolds = a->manifolds;
  if (points) *points = a->points;
  return AVBD_OK;
}

int avbd_adjoint_read_recording(const avbd_adjoint* a, double* bodies, int32_t* step_first_manifold, int32_t* step_first_point, int32_t* manifold_bodies,
                                double* manifold_basis, double* point_anchors, int32_t* point_manifold, int32_t* point_prev, int32_t* colors,
                                int32_t* color_counts) {
  if (!a || !bodies || !step_first_manifold || !step_first_point || !colors || !color_counts) return AVBD_ERR_INVALID;
  if ((a->manifolds && (!manifold_bodies || !manifold_basis)) || (a->points && (!point_anchors || !point_manifold || !point_prev)))
    return AVBD_ERR_INVALID;
  cudaSetDevice(a->device);
  if (cudaDeviceSynchronize() != cudaSuccess) return AVBD_ERR_CUDA;
  const AdjDev& D = a->d;
  const size_t nb = size_t(a->nb), K = size_t(D.K), W = size_t(D.W);
  std::vector<D3> pos(nb), um(nb);
  std::vector<D4> rot(nb);
  std::vector<double> pvz(nb), fs(nb);
  std::vector<int> dyn(nb);
  bool ok = cudaMemcpy(pos.data(), D.pos0, nb * sizeof(D3), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(rot.data(), D.rot0, nb * sizeof(D4), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(pvz.data(), D.prevVz0, nb * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(um.data(), D.unitMoment, nb * sizeof(D3), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(dyn.data(), D.dynamic, nb * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(fs.data(), D.fricStatic, nb * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(step_first_manifold, D.manFirst, K * (W + 1) * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(step_first_point, D.ptFirst, K * (W + 1) * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(colors, D.color, K * nb * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
            cudaMemcpy(color_counts, D.ncol, K * W * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (ok && a->manifolds)
    ok = cudaMemcpy(manifold_bodies, D.manAB, a->manifolds * sizeof(int2), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(manifold_basis, D.basis, a->manifolds * 3 * sizeof(D3), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (ok && a->points)
    ok = cudaMemcpy(point_anchors, D.anchor, a->points * 2 * sizeof(D3), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(point_manifold, D.ptMan, a->points * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess &&
         cudaMemcpy(point_prev, D.ptPrev, a->points * sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (!ok) return AVBD_ERR_CUDA;
  for (size_t b = 0; b < nb; b++) {
    double* r = bodies + 13 * b;
    r[0] = pos[b].x, r[1] = pos[b].y, r[2] = pos[b].z;
    r[3] = rot[b].x, r[4] = rot[b].y, r[5] = rot[b].z, r[6] = rot[b].w;
    r[7] = pvz[b];
    r[8] = um[b].x, r[9] = um[b].y, r[10] = um[b].z;
    r[11] = dyn[b] ? 1.0 : 0.0;
    r[12] = fs[b];
  }
  return AVBD_OK;
}

int avbd_adjoint_destroy(avbd_adjoint* a) {
  if (!a) return AVBD_OK;
  cudaSetDevice(a->device);
  cudaDeviceSynchronize();
  for (void* p : a->allocations) cudaFree(p);
  delete a;
  return AVBD_OK;
}

const char* avbd_adjoint_last_error(const avbd_adjoint* a) { return a ? a->error.c_str() : "no adjoint"; }

int avbd_adjoint_set_target(avbd_adjoint* a, const double* target) {
  if (!a || !target) return AVBD_ERR_INVALID;
  cudaSetDevice(a->device);
  if (cudaMemcpy(const_cast<double*>(a->d.target), target, 7 * size_t(a->nb) * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return afail(a, AVBD_ERR_CUDA, "target upload");
  return AVBD_OK;
}

static int adjParams(avbd_adjoint* a, const double* params) {
  if (!params) return afail(a, AVBD_ERR_INVALID, "params");
  for (int b = 0; b < a->nb; b++)
    for (int k = 0; k < 8; k++)
      if (!std::isfinite(params[8 * b + k])) return afail(a, AVBD_ERR_INVALID, "params not finite");
  if (cudaMemcpy(const_cast<double*>(a->d.params), params, 8 * size_t(a->nb) * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return afail(a, AVBD_ERR_CUDA, "params upload");
  return AVBD_OK;
}

int avbd_adjoint_forward(avbd_adjoint* a, const double* params, double* loss, double* final_pose) {
  if (!a) return AVBD_ERR_INVALID;
  cudaSetDevice(a->device);
  int r = adjParams(a, params);
  if (r) return r;
  k_adj_forward<<<a->W, ADJ_BLOCK, ADJ_SMEM_FORWARD>>>(a->d);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return afail(a, AVBD_ERR_CUDA, std::string("replay launch: ") + cudaGetErrorString(e));
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return afail(a, AVBD_ERR_CUDA, cudaGetErrorString(e));
  if (loss) cudaMemcpy(loss, a->d.loss, sizeof(double) * a->W, cudaMemcpyDeviceToHost);
  if (final_pose) cudaMemcpy(final_pose, a->d.finalPose, sizeof(double) * 7 * a->nb, cudaMemcpyDeviceToHost);
  a->forwardDone = true;
  a->lastParams.assign(params, params + 8 * size_t(a->nb));
  return AVBD_OK;
}

int avbd_adjoint_backward(avbd_adjoint* a, const double* params, double* grad, double* loss) {
  if (!a || !grad) return AVBD_ERR_INVALID;
  cudaSetDevice(a->device);
  if (a->forwardDone && (!params || std::memcmp(params, a->lastParams.data(), a->lastParams.size() * sizeof(double)) != 0)) a->forwardDone = false;
  int r = adjParams(a, params);
  if (r) return r;
  if (!a->forwardDone) {  // the checkpoints come from a forward with these params
    k_adj_forward<<<a->W, ADJ_BLOCK, ADJ_SMEM_FORWARD>>>(a->d);
    cudaError_t e0 = cudaGetLastError();
    if (e0 != cudaSuccess) return afail(a, AVBD_ERR_CUDA, std::string("replay launch: ") + cudaGetErrorString(e0));
  }
  a->forwardDone = false;
  k_adj_backward<<<a->W, ADJ_BLOCK, ADJ_SMEM_BACKWARD>>>(a->d);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return afail(a, AVBD_ERR_CUDA, std::string("reverse launch: ") + cudaGetErrorString(e));
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return afail(a, AVBD_ERR_CUDA, cudaGetErrorString(e));
  std::vector<D3> gv(a->nb), ga(a->nb);
  std::vector<double> gm(a->nb), gu(a->nb);
  cudaMemcpy(gv.data(), a->d.gVel, sizeof(D3) * a->nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(ga.data(), a->d.gAng, sizeof(D3) * a->nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(gm.data(), a->d.gMass, sizeof(double) * a->nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(gu.data(), a->d.gMu, sizeof(double) * a->nb, cudaMemcpyDeviceToHost);
  for (int b = 0; b < a->nb; b++) {
    double* o = grad + 8 * b;
    o[0] = gv[b].x; o[1] = gv[b].y; o[2] = gv[b].z;
    o[3] = ga[b].x; o[4] = ga[b].y; o[5] = ga[b].z;
    o[6] = gm[b];
    o[7] = gu[b];
  }
  if (loss) cudaMemcpy(loss, a->d.loss, sizeof(double) * a->W, cudaMemcpyDeviceToHost);
  return AVBD_OK;
}

}  // extern "C"
