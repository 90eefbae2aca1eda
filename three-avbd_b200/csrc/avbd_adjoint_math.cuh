// Double-precision vector and quaternion helpers for the adjoint, with their vector-Jacobian
// products (the reverse-mode derivative of each operation, written out by hand).
#pragma once
#include <cuda_runtime.h>

namespace avbd {
namespace adj {

struct D3 {
  double x, y, z;
};
struct D4 {
  double x, y, z, w;
};
__host__ __device__ inline D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__host__ __device__ inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline D3 operator-(D3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline D3& operator+=(D3& a, D3 b) {
  a = a + b;
  return a;
}
__host__ __device__ inline D3& operator-=(D3& a, D3 b) {
  a = a - b;
  return a;
}
__host__ __device__ inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__host__ __device__ inline double comp(D3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
__host__ __device__ inline void setComp(D3& v, int k, double s) {
  if (k == 0) v.x = s;
  else if (k == 1) v.y = s;
  else v.z = s;
}
__host__ __device__ inline D4 operator+(D4 a, D4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
__host__ __device__ inline D4 operator*(D4 a, double s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
__host__ __device__ inline D4& operator+=(D4& a, D4 b) {
  a = a + b;
  return a;
}
__host__ __device__ inline double dot4(D4 a, D4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__host__ __device__ inline D4 conj(D4 q) { return {-q.x, -q.y, -q.z, q.w}; }
__host__ __device__ inline D4 qmul(D4 a, D4 b) {  // ref/math.ts:57-67
  return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
          a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
// rotate (ref/math.ts:115-126): t = 2 u x v; v + w t + u x t
__host__ __device__ inline D3 rotate(D4 q, D3 v) {
  D3 u{q.x, q.y, q.z};
  D3 t = cross(u, v) * 2.0;
  return v + t * q.w + cross(u, t);
}
// its cotangent with respect to q (v is a constant body-frame vector)
__host__ __device__ inline D4 rotateVjpQ(D4 q, D3 v, D3 g) {
  D3 u{q.x, q.y, q.z};
  D3 t = cross(u, v) * 2.0;
  D3 tb = g * q.w + cross(g, u);  // cotangent of t
  D3 ub = cross(t, g) + cross(v, tb) * 2.0;
  return {ub.x, ub.y, ub.z, dot(g, t)};
}
// qsub (ref/math.ts:86-89): 2 vec(a b^-1), b^-1 = conj(b) / |b|^2
__host__ __device__ inline D3 qsub(D4 a, D4 b) {
  double l = (b.x * b.x + b.y * b.y + b.z * b.z) + b.w * b.w;
  D4 inv{-b.x / l, -b.y / l, -b.z / l, b.w / l};
  D4 s = qmul(a, inv);
  return {s.x * 2.0, s.y * 2.0, s.z * 2.0};
}
__host__ __device__ inline void qsubVjp(D4 a, D4 b, D3 g, D4& ga, D4& gb) {
  double l = (b.x * b.x + b.y * b.y + b.z * b.z) + b.w * b.w;
  D4 inv{-b.x / l, -b.y / l, -b.z / l, b.w / l};
  D4 sb{2.0 * g.x, 2.0 * g.y, 2.0 * g.z, 0.0};  // cotangent of s = a inv
  ga += qmul(sb, conj(inv));                  // right multiplication's transpose
  D4 ib = qmul(conj(a), sb);                  // left multiplication's transpose
  // inv = conj(b) / l, l = |b|^2
  D4 cb = conj(ib) * (1.0 / l);
  double dl = -(dot4(ib, conj(b))) / (l * l);
  gb += cb + b * (2.0 * dl);
}
// A rotation prepared for qsub against it: conj(b) / |b|^2 and 1 / |b|^2 (one division)
struct QInv {
  D4 inv;
  double il;
};
__host__ __device__ inline QInv qinv(D4 b) {
  const double il = 1.0 / ((b.x * b.x + b.y * b.y + b.z * b.z) + b.w * b.w);
  return {D4{-b.x * il, -b.y * il, -b.z * il, b.w * il}, il};
}
__host__ __device__ inline D3 qsubI(D4 a, const QInv& bi) {
  D4 s = qmul(a, bi.inv);
  return {s.x * 2.0, s.y * 2.0, s.z * 2.0};
}
__host__ __device__ inline void qsubVjpI(D4 a, D4 b, const QInv& bi, D3 g, D4& ga, D4& gb) {
  D4 sb{2.0 * g.x, 2.0 * g.y, 2.0 * g.z, 0.0};
  ga += qmul(sb, conj(bi.inv));
  D4 ib = qmul(conj(a), sb);
  D4 cb = conj(ib) * bi.il;
  double dl = -(dot4(ib, conj(b))) * (bi.il * bi.il);
  gb += cb + b * (2.0 * dl);
}
// qaddv (ref/math.ts:109-113): normalize(a + (v, 0) a / 2)
__host__ __device__ inline D4 qaddv(D4 a, D3 v) {
  D4 s = qmul(D4{v.x, v.y, v.z, 0.0}, a);
  D4 q{a.x + s.x * 0.5, a.y + s.y * 0.5, a.z + s.z * 0.5, a.w + s.w * 0.5};
  double il = 1.0 / sqrt((q.x * q.x + q.y * q.y + q.z * q.z) + q.w * q.w);
  return {q.x * il, q.y * il, q.z * il, q.w * il};
}
__host__ __device__ inline void qaddvVjp(D4 a, D3 v, D4 g, D4& ga, D3& gv) {
  D4 V{v.x, v.y, v.z, 0.0};
  D4 s = qmul(V, a);
  D4 p{a.x + s.x * 0.5, a.y + s.y * 0.5, a.z + s.z * 0.5, a.w + s.w * 0.5};
  double l = sqrt(dot4(p, p));
  D4 o = p * (1.0 / l);
  D4 pb = (g + o * (-dot4(o, g))) * (1.0 / l);
  ga += pb;
  ga += qmul(conj(V), pb) * 0.5;
  D4 Vb = qmul(pb, conj(a)) * 0.5;
  gv += D3{Vb.x, Vb.y, Vb.z};
}

// The 6x6 system of one body: lin and ang 3x3 blocks, the cross block (row: angular, column:
// linear), as the solver builds them; LDLT with the pivot floor (math.ts:244-302 solve6, floored)
struct Sys6 {
  double A[6][6];
};
struct LDLT6 {
  double L[6][6], D[6], invD[6];
};
// returns the mask of pivots the floor replaced
__host__ __device__ inline int factor6(const Sys6& S, LDLT6& F, double floor) {
  int floored = 0;
  for (int j = 0; j < 6; j++) {
    double d = S.A[j][j];
    for (int k = 0; k < j; k++) d -= F.L[j][k] * F.L[j][k] * F.D[k];
    if (j > 0 && d < S.A[j][j] * floor) {
      d = S.A[j][j] * floor;
      floored |= 1 << j;
    }
    F.D[j] = d;
    F.invD[j] = 1.0 / d;
    F.L[j][j] = 1.0;
    for (int i = j + 1; i < 6; i++) {
      double s = S.A[i][j];
      for (int k = 0; k < j; k++) s -= F.L[i][k] * F.L[j][k] * F.D[k];
      F.L[i][j] = s * F.invD[j];
    }
  }
  return floored;
}
__host__ __device__ inline void forwardSub6(const LDLT6& F, const double* b, double* y) {
  for (int i = 0; i < 6; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= F.L[i][k] * y[k];
    y[i] = s;
  }
}
__host__ __device__ inline void solve6(const LDLT6& F, const double* b, double* x) {
  double y[6];
  forwardSub6(F, b, y);
  for (int i = 5; i >= 0; i--) {
    double s = y[i] * F.invD[i];
    for (int k = i + 1; k < 6; k++) s -= F.L[k][i] * x[k];
    x[i] = s;
  }
}

// The reverse of x = solve6(factor6(A), b) with the pivot floor: from the cotangent xb of x, the
// cotangents of b (bb) and of A's lower triangle (Ab[i][j], i >= j: factor6 reads only those; the
// upper triangle is left zero). A floored pivot D_j = floor A_jj passes its cotangent to A_jj alone,
// as the forward's max took that branch. Without a floored pivot bb = A^-1 xb and
// Ab = -(bb x^T + x bb^T) on the lower triangle (-bb_i x_i on the diagonal).
__host__ __device__ inline void ldltVjp(const Sys6& S, const LDLT6& F, double floor, const double* b, const double* x, const double* xb, double* bb,
                                        double Ab[6][6]) {
  double y[6], yb[6], xbar[6], Lb[6][6], Db[6];
  forwardSub6(F, b, y);
  for (int i = 0; i < 6; i++) {
    xbar[i] = xb[i];
    Db[i] = 0.0;
    for (int j = 0; j < 6; j++) Lb[i][j] = Ab[i][j] = 0.0;
  }
  // back substitution (the forward ran i = 5..0: x_i = y_i / D_i - sum_{k>i} L_ki x_k)
  for (int i = 0; i < 6; i++) {
    yb[i] = xbar[i] / F.D[i];
    Db[i] -= xbar[i] * y[i] / (F.D[i] * F.D[i]);
    for (int k = i + 1; k < 6; k++) {
      Lb[k][i] -= xbar[i] * x[k];
      xbar[k] -= xbar[i] * F.L[k][i];
    }
  }
  // forward substitution (y_i = b_i - sum_{k<i} L_ik y_k)
  for (int i = 5; i >= 0; i--) {
    bb[i] = yb[i];
    for (int k = 0; k < i; k++) {
      Lb[i][k] -= yb[i] * y[k];
      yb[k] -= yb[i] * F.L[i][k];
    }
  }
  // the factorization, column by column from the last
  for (int j = 5; j >= 0; j--) {
    const double d = F.D[j];
    for (int i = j + 1; i < 6; i++) {  // L_ij = s / d, s = A_ij - sum_{k<j} L_ik L_jk D_k
      double sb = Lb[i][j] / d;
      Db[j] -= Lb[i][j] * F.L[i][j] / d;
      Ab[i][j] += sb;
      for (int k = 0; k < j; k++) {
        Lb[i][k] -= sb * F.L[j][k] * F.D[k];
        Lb[j][k] -= sb * F.L[i][k] * F.D[k];
        Db[k] -= sb * F.L[i][k] * F.L[j][k];
      }
    }
    double raw = S.A[j][j];
    for (int k = 0; k < j; k++) raw -= F.L[j][k] * F.L[j][k] * F.D[k];
    const double db = Db[j];
    if (j > 0 && raw < S.A[j][j] * floor) {
      Ab[j][j] += db * floor;
    } else {
      Ab[j][j] += db;
      for (int k = 0; k < j; k++) {
        Lb[j][k] -= db * 2.0 * F.L[j][k] * F.D[k];
        Db[k] -= db * F.L[j][k] * F.L[j][k];
      }
    }
  }
}

// ldltVjp with the floored pivots given by factor6's mask and its 6x6 work arrays (Lb, Hb: 36
// doubles each, row-major) supplied by the caller, for instance in shared memory
__host__ __device__ inline void ldltVjpMasked(const LDLT6& F, int floored, double floor, const double* b, const double* x, const double* xb, double* bb,
                                              double* Lb, double* Hb) {
  double y[6], yb[6], xbar[6], Db[6];
  forwardSub6(F, b, y);
  for (int i = 0; i < 6; i++) {
    xbar[i] = xb[i];
    Db[i] = 0.0;
  }
  for (int i = 0; i < 36; i++) Lb[i] = Hb[i] = 0.0;
  for (int i = 0; i < 6; i++) {
    yb[i] = xbar[i] * F.invD[i];
    Db[i] -= xbar[i] * y[i] * (F.invD[i] * F.invD[i]);
    for (int k = i + 1; k < 6; k++) {
      Lb[6 * k + i] -= xbar[i] * x[k];
      xbar[k] -= xbar[i] * F.L[k][i];
    }
  }
  for (int i = 5; i >= 0; i--) {
    bb[i] = yb[i];
    for (int k = 0; k < i; k++) {
      Lb[6 * i + k] -= yb[i] * y[k];
      yb[k] -= yb[i] * F.L[i][k];
    }
  }
  for (int j = 5; j >= 0; j--) {
    const double id = F.invD[j];
    for (int i = j + 1; i < 6; i++) {
      double sb = Lb[6 * i + j] * id;
      Db[j] -= Lb[6 * i + j] * F.L[i][j] * id;
      Hb[6 * i + j] += sb;
      for (int k = 0; k < j; k++) {
        Lb[6 * i + k] -= sb * F.L[j][k] * F.D[k];
        Lb[6 * j + k] -= sb * F.L[i][k] * F.D[k];
        Db[k] -= sb * F.L[i][k] * F.L[j][k];
      }
    }
    const double db = Db[j];
    if (floored & (1 << j)) {
      Hb[6 * j + j] += db * floor;
    } else {
      Hb[6 * j + j] += db;
      for (int k = 0; k < j; k++) {
        Lb[6 * j + k] -= db * 2.0 * F.L[j][k] * F.D[k];
        Db[k] -= db * F.L[j][k] * F.L[j][k];
      }
    }
  }
}

}  // namespace adj
}  // namespace avbd
