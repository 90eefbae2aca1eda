// CPU oracle for the 3D AVBD step: TEST INFRASTRUCTURE ONLY.
//
// A C++ restatement of three-avbd's CPU reference (src/avbd3d/ref/*.ts), templated on the
// floating type. The CUDA backend is compared against it in the tests; nothing in the product
// links, includes or calls it. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
// leg load it (through ctypes).
//
//   * Upstream mode (`orc_step`): src/avbd3d/ref/solver.ts:137-223 operation for operation, in
//     double, compiled with -ffp-contract=off. Pinned against the reference's golden trajectories
//     tests/fixtures/oracle3d/scene-{0..13}.json (upstream avbd-demo3d in double, no FMA) at 1e-9.
//   * GPU mode (`orc_step_gpu`): the same constraint maths with the WebGPU solver's rules
//     (src/avbd3d/gpu/wgsl-collision.ts, wgsl-solve.ts, src/avbd2d/gpu/wgsl-topology.ts): pairs
//     from the grid rule, fresh manifolds warm-started by (pair, feature), sphere shapes, the
//     incremental Jones-Plassmann colouring, bodies swept colour by colour, LDLT pivot floor.
//   * FP32 predicates (`T = float`): the broadphase pair tests and the box/sphere narrowphase in
//     the WGSL's operation order, so pair sets and feature keys compare bit for bit.
//
// Every function names the reference lines it restates.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <unordered_map>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif


// ---------------------------------------------------------------------------------------------
// Reverse-mode scalar for the FP64 CPU adjoint (test infrastructure): every operation on AD values
// appends a node (two parents and their partial derivatives) to a tape; sweeping the tape backwards
// gives the gradient of one output with respect to every input. Comparisons and selections act on
// the values, so a derivative follows the branch the forward took.
// ---------------------------------------------------------------------------------------------
namespace orc {
struct ADNode { int a, b; double da, db; };
inline std::vector<ADNode>& adTape() {
  static std::vector<ADNode> tape;
  return tape;
}
struct AD {
  double v = 0;
  int i = -1;
  AD() {}
  AD(double x) : v(x) {}
  static AD node(double v, int a, double da, int b = -1, double db = 0) {
    AD r(v);
    if (a < 0 && b < 0) return r;
    adTape().push_back({a, b, da, db});
    r.i = int(adTape().size()) - 1;
    return r;
  }
  static AD input(double v) {
    AD r(v);
    adTape().push_back({-1, -1, 0, 0});
    r.i = int(adTape().size()) - 1;
    return r;
  }
  explicit operator double() const { return v; }
  explicit operator float() const { return float(v); }
  AD& operator+=(const AD& o);
  AD& operator-=(const AD& o);
  AD& operator*=(const AD& o);
  AD& operator/=(const AD& o);
};
inline AD operator+(const AD& x, const AD& y) { return AD::node(x.v + y.v, x.i, 1.0, y.i, 1.0); }
inline AD operator-(const AD& x, const AD& y) { return AD::node(x.v - y.v, x.i, 1.0, y.i, -1.0); }
inline AD operator*(const AD& x, const AD& y) { return AD::node(x.v * y.v, x.i, y.v, y.i, x.v); }
inline AD operator/(const AD& x, const AD& y) { return AD::node(x.v / y.v, x.i, 1.0 / y.v, y.i, -x.v / (y.v * y.v)); }
inline AD operator-(const AD& x) { return AD::node(-x.v, x.i, -1.0); }
inline AD& AD::operator+=(const AD& o) { return *this = *this + o; }
inline AD& AD::operator-=(const AD& o) { return *this = *this - o; }
inline AD& AD::operator*=(const AD& o) { return *this = *this * o; }
inline AD& AD::operator/=(const AD& o) { return *this = *this / o; }
inline bool operator<(const AD& x, const AD& y) { return x.v < y.v; }
inline bool operator>(const AD& x, const AD& y) { return x.v > y.v; }
inline bool operator<=(const AD& x, const AD& y) { return x.v <= y.v; }
inline bool operator>=(const AD& x, const AD& y) { return x.v >= y.v; }
inline bool operator==(const AD& x, const AD& y) { return x.v == y.v; }
inline bool operator!=(const AD& x, const AD& y) { return x.v != y.v; }
}  // namespace orc
namespace std {
inline orc::AD sqrt(const orc::AD& x) {
  double r = std::sqrt(x.v);
  return orc::AD::node(r, x.i, r > 0 ? 0.5 / r : 0.0);
}
inline orc::AD fabs(const orc::AD& x) { return orc::AD::node(std::fabs(x.v), x.i, x.v < 0 ? -1.0 : 1.0); }
inline bool isfinite(const orc::AD& x) { return std::isfinite(x.v); }
}  // namespace std
namespace orc {

// ---------------------------------------------------------------------------------------------
// Maths: src/avbd3d/ref/math.ts (row-major 3x3, quaternions xyzw), every expression in order.
// ---------------------------------------------------------------------------------------------

template <class T> using V3 = std::array<T, 3>;
template <class T> using Q4 = std::array<T, 4>;
template <class T> using M3 = std::array<T, 9>;

template <class T> inline T dot(const V3<T>& a, const V3<T>& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }  // math.ts:22
template <class T> inline T lengthSq(const V3<T>& v) { return dot(v, v); }
template <class T> inline T length(const V3<T>& v) { return std::sqrt(lengthSq(v)); }
template <class T> inline V3<T> add3(const V3<T>& a, const V3<T>& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
template <class T> inline V3<T> sub3(const V3<T>& a, const V3<T>& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
template <class T> inline V3<T> scale3(const V3<T>& a, T s) { return {a[0] * s, a[1] * s, a[2] * s}; }
template <class T> inline V3<T> div3(const V3<T>& a, T s) { return {a[0] / s, a[1] / s, a[2] / s}; }
template <class T> inline V3<T> neg3(const V3<T>& a) { return {-a[0], -a[1], -a[2]}; }
template <class T> inline V3<T> abs3(const V3<T>& a) { return {std::fabs(a[0]), std::fabs(a[1]), std::fabs(a[2])}; }
// math.ts:40 out = a + b * s
template <class T> inline V3<T> addScaled3(const V3<T>& a, const V3<T>& b, T s) { return {a[0] + b[0] * s, a[1] + b[1] * s, a[2] + b[2] * s}; }
template <class T> inline V3<T> normalize3(const V3<T>& v) { return div3(v, length(v)); }
template <class T> inline V3<T> cross(const V3<T>& a, const V3<T>& b) {  // math.ts:44
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
template <class T> inline Q4<T> qmul(const Q4<T>& a, const Q4<T>& b) {  // math.ts:57-67
  T ax = a[0], ay = a[1], az = a[2], aw = a[3];
  T bx = b[0], by = b[1], bz = b[2], bw = b[3];
  return {aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw,
          aw * bw - ax * bx - ay * by - az * bz};
}
template <class T> inline Q4<T> conjugate(const Q4<T>& q) { return {-q[0], -q[1], -q[2], q[3]}; }
template <class T> inline T qlengthSq(const Q4<T>& q) { return (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) + q[3] * q[3]; }  // math.ts:70
template <class T> inline Q4<T> qinverse(const Q4<T>& q) {  // math.ts:72-75
  T l = qlengthSq(q);
  return {-q[0] / l, -q[1] / l, -q[2] / l, q[3] / l};
}
template <class T> inline Q4<T> qnormalize(const Q4<T>& q) {  // math.ts:77-80
  T l = std::sqrt(qlengthSq(q));
  return {q[0] / l, q[1] / l, q[2] / l, q[3] / l};
}
template <class T> inline V3<T> qsub(const Q4<T>& a, const Q4<T>& b) {  // math.ts:86-89
  Q4<T> s = qmul(a, qinverse(b));
  return {s[0] * 2, s[1] * 2, s[2] * 2};
}
template <class T> inline T qangle(const Q4<T>& a, const Q4<T>& b) {  // math.ts:97-106
  if (a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3]) return 0;
  T ax = -a[0], ay = -a[1], az = -a[2], aw = a[3];
  T bx = b[0], by = b[1], bz = b[2], bw = b[3];
  T x = aw * bx + ax * bw + ay * bz - az * by;
  T y = aw * by - ax * bz + ay * bw + az * bx;
  T z = aw * bz + ax * by - ay * bx + az * bw;
  T w = aw * bw - ax * bx - ay * by - az * bz;
  return 2 * std::atan2(std::sqrt(x * x + y * y + z * z), std::fabs(w));
}
template <class T> inline Q4<T> qaddv(const Q4<T>& a, const V3<T>& b) {  // math.ts:109-113
  Q4<T> s = qmul(Q4<T>{b[0], b[1], b[2], T(0)}, a);
  return qnormalize(Q4<T>{a[0] + s[0] * T(0.5), a[1] + s[1] * T(0.5), a[2] + s[2] * T(0.5), a[3] + s[3] * T(0.5)});
}
template <class T> inline V3<T> rotate(const Q4<T>& q, const V3<T>& v) {  // math.ts:115-126
  T ux = q[0], uy = q[1], uz = q[2], w = q[3];
  T tx = (uy * v[2] - uz * v[1]) * 2;
  T ty = (uz * v[0] - ux * v[2]) * 2;
  T tz = (ux * v[1] - uy * v[0]) * 2;
  return {v[0] + tx * w + (uy * tz - uz * ty), v[1] + ty * w + (uz * tx - ux * tz), v[2] + tz * w + (ux * ty - uy * tx)};
}
template <class T> inline V3<T> transform(const V3<T>& p, const Q4<T>& q, const V3<T>& v) { return add3(rotate(q, v), p); }  // math.ts:130
template <class T> inline V3<T> rotateInv(const Q4<T>& q, const V3<T>& v) { return rotate(conjugate(q), v); }
template <class T> inline M3<T> diagonal(T a, T b, T c) { return {a, 0, 0, 0, b, 0, 0, 0, c}; }
template <class T> inline M3<T> skew(const V3<T>& r) { return {0, -r[2], r[1], r[2], 0, -r[0], -r[1], r[0], 0}; }  // math.ts:150
template <class T> inline M3<T> transpose(const M3<T>& a) { return {a[0], a[3], a[6], a[1], a[4], a[7], a[2], a[5], a[8]}; }
template <class T> inline M3<T> mul(const M3<T>& a, const M3<T>& b) {  // math.ts:178-191
  return {a[0] * b[0] + a[1] * b[3] + a[2] * b[6], a[0] * b[1] + a[1] * b[4] + a[2] * b[7], a[0] * b[2] + a[1] * b[5] + a[2] * b[8],
          a[3] * b[0] + a[4] * b[3] + a[5] * b[6], a[3] * b[1] + a[4] * b[4] + a[5] * b[7], a[3] * b[2] + a[4] * b[5] + a[5] * b[8],
          a[6] * b[0] + a[7] * b[3] + a[8] * b[6], a[6] * b[1] + a[7] * b[4] + a[8] * b[7], a[6] * b[2] + a[7] * b[5] + a[8] * b[8]};
}
template <class T> inline V3<T> mulv(const M3<T>& a, const V3<T>& v) {  // math.ts:193-196
  T x = v[0], y = v[1], z = v[2];
  return {a[0] * x + a[1] * y + a[2] * z, a[3] * x + a[4] * y + a[5] * z, a[6] * x + a[7] * y + a[8] * z};
}
template <class T> inline void addm(M3<T>& out, const M3<T>& a) { for (int i = 0; i < 9; i++) out[i] += a[i]; }
template <class T> inline M3<T> scalem(const M3<T>& a, T s) { M3<T> o; for (int i = 0; i < 9; i++) o[i] = a[i] * s; return o; }
template <class T> inline M3<T> negm(const M3<T>& a) { M3<T> o; for (int i = 0; i < 9; i++) o[i] = -a[i]; return o; }
template <class T> inline M3<T> outer(const V3<T>& a, const V3<T>& b) {  // math.ts:214-217
  M3<T> o;
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) o[i * 3 + j] = b[j] * a[i];
  return o;
}
template <class T> inline M3<T> diagonalize(const M3<T>& m) {  // math.ts:220-225
  T c0 = std::sqrt(m[0] * m[0] + m[3] * m[3] + m[6] * m[6]);
  T c1 = std::sqrt(m[1] * m[1] + m[4] * m[4] + m[7] * m[7]);
  T c2 = std::sqrt(m[2] * m[2] + m[5] * m[5] + m[8] * m[8]);
  return diagonal(c0, c1, c2);
}
template <class T> inline M3<T> orthonormal(const V3<T>& n) {  // math.ts:228-238
  V3<T> t1 = std::fabs(n[0]) > std::fabs(n[2]) ? V3<T>{-n[1], n[0], 0} : V3<T>{0, -n[2], n[1]};
  t1 = normalize3(t1);
  V3<T> t2 = cross(n, t1);
  return {n[0], n[1], n[2], t1[0], t1[1], t1[2], t2[0], t2[1], t2[2]};
}
template <class T> inline T tmin(T a, T b) { return a < b ? a : b; }  // math.ts:16-18
template <class T> inline T tmax(T a, T b) { return a > b ? a : b; }
template <class T> inline T clampv(T x, T a, T b) { return tmax(a, tmin(b, x)); }
template <class T> inline T signv(T x) { return x < 0 ? T(-1) : x > 0 ? T(1) : T(0); }

// solve6 (math.ts:244-302); `floor` > 0 adds the GPU's pivot floor (wgsl-solve.ts:519-539).
template <class T>
void solve6(const M3<T>& aLin, const M3<T>& aAng, const M3<T>& aCross, const V3<T>& bLin, const V3<T>& bAng, V3<T>& xLin, V3<T>& xAng,
            T floor = 0) {
  const T A11 = aLin[0];
  const T A21 = aLin[3], A22 = aLin[4];
  const T A31 = aLin[6], A32 = aLin[7], A33 = aLin[8];
  const T A41 = aCross[0], A42 = aCross[1], A43 = aCross[2], A44 = aAng[0];
  const T A51 = aCross[3], A52 = aCross[4], A53 = aCross[5], A54 = aAng[3], A55 = aAng[4];
  const T A61 = aCross[6], A62 = aCross[7], A63 = aCross[8], A64 = aAng[6], A65 = aAng[7], A66 = aAng[8];
  auto fl = [&](T d, T diag) { return floor > 0 ? tmax(d, diag * floor) : d; };
  const T L21 = A21 / A11, L31 = A31 / A11, L41 = A41 / A11, L51 = A51 / A11, L61 = A61 / A11;
  const T D1 = A11;
  const T D2 = fl(A22 - L21 * L21 * D1, A22);
  const T L32 = (A32 - L21 * L31 * D1) / D2;
  const T L42 = (A42 - L21 * L41 * D1) / D2;
  const T L52 = (A52 - L21 * L51 * D1) / D2;
  const T L62 = (A62 - L21 * L61 * D1) / D2;
  const T D3 = fl(A33 - (L31 * L31 * D1 + L32 * L32 * D2), A33);
  const T L43 = (A43 - L31 * L41 * D1 - L32 * L42 * D2) / D3;
  const T L53 = (A53 - L31 * L51 * D1 - L32 * L52 * D2) / D3;
  const T L63 = (A63 - L31 * L61 * D1 - L32 * L62 * D2) / D3;
  const T D4 = fl(A44 - (L41 * L41 * D1 + L42 * L42 * D2 + L43 * L43 * D3), A44);
  const T L54 = (A54 - L41 * L51 * D1 - L42 * L52 * D2 - L43 * L53 * D3) / D4;
  const T L64 = (A64 - L41 * L61 * D1 - L42 * L62 * D2 - L43 * L63 * D3) / D4;
  const T D5 = fl(A55 - (L51 * L51 * D1 + L52 * L52 * D2 + L53 * L53 * D3 + L54 * L54 * D4), A55);
  const T L65 = (A65 - L51 * L61 * D1 - L52 * L62 * D2 - L53 * L63 * D3 - L54 * L64 * D4) / D5;
  const T D6 = fl(A66 - (L61 * L61 * D1 + L62 * L62 * D2 + L63 * L63 * D3 + L64 * L64 * D4 + L65 * L65 * D5), A66);
  const T y1 = bLin[0];
  const T y2 = bLin[1] - L21 * y1;
  const T y3 = bLin[2] - L31 * y1 - L32 * y2;
  const T y4 = bAng[0] - L41 * y1 - L42 * y2 - L43 * y3;
  const T y5 = bAng[1] - L51 * y1 - L52 * y2 - L53 * y3 - L54 * y4;
  const T y6 = bAng[2] - L61 * y1 - L62 * y2 - L63 * y3 - L64 * y4 - L65 * y5;
  const T z1 = y1 / D1, z2 = y2 / D2, z3 = y3 / D3, z4 = y4 / D4, z5 = y5 / D5, z6 = y6 / D6;
  xAng[2] = z6;
  xAng[1] = z5 - L65 * xAng[2];
  xAng[0] = z4 - L54 * xAng[1] - L64 * xAng[2];
  xLin[2] = z3 - L43 * xAng[0] - L53 * xAng[1] - L63 * xAng[2];
  xLin[1] = z2 - L32 * xLin[2] - L42 * xAng[0] - L52 * xAng[1] - L62 * xAng[2];
  xLin[0] = z1 - L21 * xLin[1] - L31 * xLin[2] - L41 * xAng[0] - L51 * xAng[1] - L61 * xAng[2];
}

// ---------------------------------------------------------------------------------------------
// Constants: src/avbd3d/ref/body.ts:8-11, src/avbd3d/gpu/layout.ts:130-170, avbd2d/gpu/layout.ts:99-100
// ---------------------------------------------------------------------------------------------
const double PENALTY_MIN = 1.0, PENALTY_MAX = 1e10, COLLISION_MARGIN = 0.01, STICK_THRESH = 1e-5;
const uint32_t STICK_BIT = 0x80000000u, SPHERE_FEATURE = 3u << 24;
const int SHAPE_BOX = 0, SHAPE_SPHERE = 1, SHAPE_SAIL = 2, SHAPE_HULL = 3;  // layout.ts:143-151 (a hull: SHAPE_HULL + header offset)
const int MAX_COLORS = 64;
const uint32_t NO_COLOR = 255, PENDING = 256;
const double PIVOT_FLOOR = 1e-5;
const double NEAREST_FRACTION = 0.05;
enum { FLAG_MATCH_NEAREST = 1, FLAG_FACE_BIAS = 2, FLAG_REUSE_CONTACTS = 4, FLAG_START_AT_REST = 8, FLAG_MASS_PENALTY = 16 };
// Contact reuse tolerances (gpu/layout.ts:174-175)
const float REUSE_LIN_TOL = 0.002f, REUSE_ANG_TOL = 0.002f;
const double REST_SPEED = 0.1;

template <class T> struct Solver;

// Rigid (ref/body.ts:13-62): indices into the solver's body vector.
template <class T> struct Force;
template <class T> struct Body {
  V3<T> pos{}, initPos{}, inertialPos{}, vel{}, angVel{}, prevVel{}, size{}, moment{};
  Q4<T> rot{0, 0, 0, 1}, initRot{0, 0, 0, 1}, inertialRot{0, 0, 0, 1};
  T mass = 0, friction = 0, radius = 0;
  int shape = SHAPE_BOX;
  uint32_t groups = 0xffffffffu, mask = 0xffffffffu;
  uint32_t color = NO_COLOR;  // GPU-mode colour state (colour | PENDING)
  // GPU-mode body aux record (gpu/layout.ts:33-46): gravity scale, damping rates (1/s)
  T gravityScale = 1, linDamp = 0, angDamp = 0;
  uint32_t lifecycle = 0;  // GPU-mode lifecycle bits (layout.ts:17-19): 4 cold
  // GPU-mode contact reuse (wgsl-collision.ts:20-44): the reference pose (f32, as the device keeps
  // it; a zero rotation: none yet) and the step at which the body last moved past the tolerances
  V3<float> refPos{0, 0, 0};
  Q4<float> refRot{0, 0, 0, 0};
  uint32_t movedStep = 0;
  std::vector<Force<T>*> forces;
};

template <class T> struct BodySystem { M3<T> lhsLin{}, lhsAng{}, lhsCross{}; V3<T> rhsLin{}, rhsAng{}; };

enum ForceKind { K_MANIFOLD = 0, K_JOINT = 1, K_SPRING = 2, K_IGNORE = 3 };

template <class T> struct Force {  // ref/body.ts:76-112
  Solver<T>* solver;
  int bodyA, bodyB;  // bodyA -1: the world
  int kind;
  Force(Solver<T>* s, int a, int b, int k) : solver(s), bodyA(a), bodyB(b), kind(k) {}
  virtual ~Force() {}
  virtual bool initialize() = 0;
  virtual void updatePrimal(int body, T alpha, BodySystem<T>& sys) = 0;
  virtual void updateDual(T alpha) = 0;
};

// ---------------------------------------------------------------------------------------------
// Narrowphase: box-box SAT + clipping (ref/collide.ts:67-345, wgsl-collision.ts:385-683), sphere
// contacts (wgsl-collision.ts:601-654). Works on world points; rA/rB are made body-local at the end.
// ---------------------------------------------------------------------------------------------

template <class T> struct OBB { V3<T> c, h; V3<T> ax[3]; };
template <class T> struct Sat { int type = 0, ia = 0, ib = 0; T sep = 0; V3<T> n{}; bool valid = false; };
template <class T> struct Found { uint32_t feature[8]; V3<T> xA[8], xB[8]; int count = 0; };
const int MAX_CONTACTS = 8;
const double SAT_AXIS_EPSILON = 1.0e-6, PLANE_EPSILON = 1.0e-5, CONTACT_MERGE_DIST_SQ = 1.0e-6;
const int AXIS_FACE_A = 0, AXIS_FACE_B = 1, AXIS_EDGE = 2;

template <class T> OBB<T> makeOBB(const V3<T>& c, const Q4<T>& q, const V3<T>& size) {  // collide.ts:285-292
  OBB<T> b;
  b.c = c;
  b.h = scale3(size, T(0.5));
  b.ax[0] = rotate(q, V3<T>{1, 0, 0});
  b.ax[1] = rotate(q, V3<T>{0, 1, 0});
  b.ax[2] = rotate(q, V3<T>{0, 0, 1});
  return b;
}
template <class T> inline T projRadius(const OBB<T>& b, const V3<T>& n) {  // collide.ts:399 / wgsl-collision.ts:427
  return b.h[0] * std::fabs(dot(n, b.ax[0])) + b.h[1] * std::fabs(dot(n, b.ax[1])) + b.h[2] * std::fabs(dot(n, b.ax[2]));
}
template <class T> V3<T> support(const OBB<T>& b, const V3<T>& dir) {  // collide.ts:296-303
  T sx = dot(dir, b.ax[0]) >= 0 ? T(1) : T(-1);
  T sy = dot(dir, b.ax[1]) >= 0 ? T(1) : T(-1);
  T sz = dot(dir, b.ax[2]) >= 0 ? T(1) : T(-1);
  V3<T> p = addScaled3(b.c, b.ax[0], b.h[0] * sx);
  p = addScaled3(p, b.ax[1], b.h[1] * sy);
  return addScaled3(p, b.ax[2], b.h[2] * sz);
}
template <class T> void addFound(Found<T>& f, const V3<T>& xA, const V3<T>& xB, uint32_t feature) {  // collide.ts:376-387
  V3<T> mid = scale3(add3(xA, xB), T(0.5));
  for (int i = 0; i < f.count; i++) {
    V3<T> m = scale3(add3(f.xA[i], f.xB[i]), T(0.5));
    if (lengthSq(sub3(mid, m)) < T(CONTACT_MERGE_DIST_SQ)) return;
  }
  if (f.count >= MAX_CONTACTS) return;
  f.feature[f.count] = feature;
  f.xA[f.count] = xA;
  f.xB[f.count] = xB;
  f.count++;
}
template <class T> bool testAxis(const OBB<T>& A, const OBB<T>& B, const V3<T>& delta, const V3<T>& axis, int type, int ia, int ib,
                                 Sat<T>& best) {  // collide.ts:390-414
  T lenSq = lengthSq(axis);
  if (lenSq < T(SAT_AXIS_EPSILON)) return true;
  T invLen = T(1) / std::sqrt(lenSq);
  V3<T> n = scale3(axis, invLen);
  if (dot(n, delta) < 0) n = neg3(n);
  T distance = std::fabs(dot(delta, n));
  T rA = projRadius(A, n);
  T rB = projRadius(B, n);
  T separation = distance - (rA + rB);
  if (separation > 0) return false;
  if (!best.valid || separation > best.sep) {
    best.valid = true;
    best.type = type;
    best.ia = ia;
    best.ib = ib;
    best.sep = separation;
    best.n = n;
  }
  return true;
}
template <class T> int clipPoly(const V3<T>* in, int n, V3<T>* out, const V3<T>& pn, T offset) {  // collide.ts:343-363
  int count = 0;
  if (n == 0) return 0;
  V3<T> a = in[n - 1];
  T da = dot(pn, a) - offset;
  for (int i = 0; i < n; i++) {
    V3<T> b = in[i];
    T db = dot(pn, b) - offset;
    bool aIn = da <= T(PLANE_EPSILON), bIn = db <= T(PLANE_EPSILON);
    if (aIn != bIn) {
      T t = 0;
      T denom = da - db;
      if (std::fabs(denom) > T(SAT_AXIS_EPSILON)) t = clampv(da / denom, T(0), T(1));
      if (count < 16) out[count++] = addScaled3(a, sub3(b, a), t);
    }
    if (bIn && count < 16) out[count++] = b;
    a = b;
    da = db;
  }
  return count;
}
inline int faceU(int k) { return k == 0 ? 1 : 0; }
inline int faceV(int k) { return k != 2 ? 2 : 1; }

template <class T> Found<T> faceManifold(const OBB<T>& A, const OBB<T>& B, bool refIsA, int refAxis, const V3<T>& nAB) {  // collide.ts:464-510
  Found<T> found;
  const OBB<T>& R = refIsA ? A : B;
  const OBB<T>& I = refIsA ? B : A;
  V3<T> outward = refIsA ? nAB : neg3(nAB);
  T rs = dot(outward, R.ax[refAxis]) >= 0 ? T(1) : T(-1);
  V3<T> rn = scale3(R.ax[refAxis], rs);
  V3<T> rc = addScaled3(R.c, rn, R.h[refAxis]);
  V3<T> ru = R.ax[faceU(refAxis)], rv = R.ax[faceV(refAxis)];
  T eu = R.h[faceU(refAxis)], ev = R.h[faceV(refAxis)];
  int incAxis = 0;
  T bestDot = T(-3.4028234663852886e38);
  for (int k = 0; k < 3; k++) {
    T d = std::fabs(dot(I.ax[k], rn));
    if (d > bestDot) { bestDot = d; incAxis = k; }
  }
  T is = dot(I.ax[incAxis], rn) > 0 ? T(-1) : T(1);
  V3<T> fn = scale3(I.ax[incAxis], is);
  V3<T> fc = addScaled3(I.c, fn, I.h[incAxis]);
  V3<T> u = I.ax[faceU(incAxis)], v = I.ax[faceV(incAxis)];
  T eU = I.h[faceU(incAxis)], eV = I.h[faceV(incAxis)];
  auto vert = [&](T su, T sv) { V3<T> p = addScaled3(fc, u, su * eU); return addScaled3(p, v, sv * eV); };
  V3<T> poly[16], tmp[16];
  poly[0] = vert(1, 1); poly[1] = vert(-1, 1); poly[2] = vert(-1, -1); poly[3] = vert(1, -1);
  int n = 4;
  V3<T> nru = neg3(ru), nrv = neg3(rv);
  n = clipPoly(poly, n, tmp, ru, dot(ru, rc) + eu);
  if (!n) return found;
  n = clipPoly(tmp, n, poly, nru, dot(nru, rc) + eu);
  if (!n) return found;
  n = clipPoly(poly, n, tmp, rv, dot(rv, rc) + ev);
  if (!n) return found;
  n = clipPoly(tmp, n, poly, nrv, dot(nrv, rc) + ev);
  if (!n) return found;
  uint32_t prefix = (uint32_t(refIsA ? AXIS_FACE_A : AXIS_FACE_B) << 24) | (uint32_t(refAxis & 0xff) << 16) | (uint32_t(incAxis & 0xff) << 8);
  for (int i = 0; i < n && found.count < MAX_CONTACTS; i++) {
    V3<T> p = poly[i];
    T dist = dot(sub3(p, rc), rn);
    if (dist > T(PLANE_EPSILON)) continue;
    V3<T> onRef = addScaled3(p, rn, -dist);
    addFound(found, refIsA ? onRef : p, refIsA ? p : onRef, prefix | uint32_t(i & 0xff));
  }
  if (found.count == 0) addFound(found, support(A, nAB), support(B, neg3(nAB)), prefix);
  return found;
}
template <class T> void supportEdge(const OBB<T>& b, int k, const V3<T>& dir, V3<T>& e0, V3<T>& e1) {  // collide.ts:416-425
  int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
  T s1 = dot(dir, b.ax[k1]) >= 0 ? T(1) : T(-1);
  T s2 = dot(dir, b.ax[k2]) >= 0 ? T(1) : T(-1);
  V3<T> c = addScaled3(b.c, b.ax[k1], b.h[k1] * s1);
  c = addScaled3(c, b.ax[k2], b.h[k2] * s2);
  V3<T> e = scale3(b.ax[k], b.h[k]);
  e0 = sub3(c, e);
  e1 = add3(c, e);
}
template <class T> Found<T> edgeContact(const OBB<T>& A, const OBB<T>& B, int ia, int ib, const V3<T>& nAB) {  // collide.ts:427-462,512-524
  Found<T> found;
  V3<T> p0, p1, q0, q1;
  supportEdge(A, ia, nAB, p0, p1);
  supportEdge(B, ib, neg3(nAB), q0, q1);
  V3<T> d1 = sub3(p1, p0), d2 = sub3(q1, q0), r = sub3(p0, q0);
  T a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  T s = 0, t = 0;
  const T eps = T(SAT_AXIS_EPSILON);
  if (a <= eps && e <= eps) {
  } else if (a <= eps) {
    t = clampv(f / e, T(0), T(1));
  } else {
    T c = dot(d1, r);
    if (e <= eps) {
      s = clampv(-c / a, T(0), T(1));
    } else {
      T b = dot(d1, d2);
      T denom = a * e - b * b;
      if (std::fabs(denom) > eps) s = clampv((b * f - c * e) / denom, T(0), T(1));
      t = (b * s + f) / e;
      if (t < 0) { t = 0; s = clampv(-c / a, T(0), T(1)); }
      else if (t > 1) { t = 1; s = clampv((b - c) / a, T(0), T(1)); }
    }
  }
  uint32_t key = (uint32_t(AXIS_EDGE) << 24) | (uint32_t(ia & 0xff) << 8) | uint32_t(ib & 0xff);
  addFound(found, addScaled3(p0, d1, s), addScaled3(q0, d2, t), key);
  if (found.count == 0) addFound(found, support(A, nAB), support(B, neg3(nAB)), key);
  return found;
}
// collide.ts:530-563 (faceBias: wgsl-collision.ts:674-679). sat.n points from A towards B.
template <class T> Found<T> collideBoxes(const OBB<T>& A, const OBB<T>& B, bool faceBias, Sat<T>& out) {
  Found<T> none;
  V3<T> delta = sub3(B.c, A.c);
  Sat<T> face, edge;
  for (int i = 0; i < 3; i++) if (!testAxis(A, B, delta, A.ax[i], AXIS_FACE_A, i, 0, face)) return none;
  for (int i = 0; i < 3; i++) if (!testAxis(A, B, delta, B.ax[i], AXIS_FACE_B, 0, i, face)) return none;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      if (!testAxis(A, B, delta, cross(A.ax[i], B.ax[j]), AXIS_EDGE, i, j, edge)) return none;
  if (!face.valid) return none;
  Sat<T> best = face;
  if (edge.valid) {
    bool edgeWins = T(0.95) * edge.sep > face.sep + T(0.01);
    if (faceBias) edgeWins = edge.sep > T(0.95) * face.sep + T(0.01);
    if (edgeWins) best = edge;
  }
  out = best;
  if (best.type == AXIS_EDGE) return edgeContact(A, B, best.ia, best.ib, best.n);
  return faceManifold(A, B, best.type == AXIS_FACE_A, best.type == AXIS_FACE_A ? best.ia : best.ib, best.n);
}
// wgsl-collision.ts:604-614
template <class T> Found<T> sphereSphere(const OBB<T>& A, const OBB<T>& B, Sat<T>& sat) {
  Found<T> found;
  V3<T> d = sub3(B.c, A.c);
  T dist = length(d);
  if (dist > A.h[0] + B.h[0]) return found;
  V3<T> n{0, 0, 1};
  if (dist > 0) n = div3(d, dist);
  sat.n = n;
  addFound(found, addScaled3(A.c, n, A.h[0]), sub3(B.c, scale3(n, B.h[0])), SPHERE_FEATURE);
  return found;
}
// wgsl-collision.ts:616-653: S a sphere, X a box turned by qX. n points from the sphere to the box.
template <class T> bool sphereBox(const OBB<T>& S, const OBB<T>& X, const Q4<T>& qX, V3<T>& onSphere, V3<T>& onBox, V3<T>& nOut) {
  V3<T> p = rotate(conjugate(qX), sub3(S.c, X.c));
  V3<T> q{clampv(p[0], -X.h[0], X.h[0]), clampv(p[1], -X.h[1], X.h[1]), clampv(p[2], -X.h[2], X.h[2])};
  T r = S.h[0];
  V3<T> nLocal{};
  V3<T> ob = q;
  if (p[0] != q[0] || p[1] != q[1] || p[2] != q[2]) {
    V3<T> d = sub3(p, q);
    T dist = length(d);
    if (dist > r) return false;
    nLocal = div3(d, dist);
  } else {
    V3<T> depth = sub3(X.h, abs3(p));
    int k = 0;
    if (depth[1] < depth[k]) k = 1;
    if (depth[2] < depth[k]) k = 2;
    T s = p[k] >= 0 ? T(1) : T(-1);
    nLocal = V3<T>{0, 0, 0};
    nLocal[k] = s;
    ob[k] = s * X.h[k];
  }
  V3<T> n = rotate(qX, nLocal);
  nOut = neg3(n);
  onBox = add3(X.c, rotate(qX, ob));
  onSphere = sub3(S.c, scale3(n, r));
  return true;
}

// ---------------------------------------------------------------------------------------------
// Convex hulls (src/avbd3d/gpu/wgsl-hull.ts), restated from the WGSL in its operation order. The
// hull buffer is the reference's packed layout (gpu/solver.ts:313-338): 4 words per vec4; a body's
// shape code is SHAPE_HULL + its header offset. A box takes part with its own topology.
// ---------------------------------------------------------------------------------------------
const uint32_t NO_HULL = 0xffffffffu;
const int MAX_CLIP = 64;
const uint32_t BOX_FACE_VERTS[24] = {1, 3, 7, 5, 0, 2, 6, 4, 2, 3, 7, 6, 0, 1, 5, 4, 4, 5, 7, 6, 0, 1, 3, 2};  // wgsl-hull.ts:37
const uint32_t BOX_EDGES[12][4] = {{0, 1, 3, 5}, {2, 3, 2, 5}, {4, 5, 3, 4}, {6, 7, 2, 4}, {0, 2, 1, 5}, {1, 3, 0, 5},
                                   {4, 6, 1, 4}, {5, 7, 0, 4}, {0, 4, 1, 3}, {1, 5, 0, 3}, {2, 6, 1, 2}, {3, 7, 0, 2}};  // :38-41

template <class T> struct PolyShape {  // wgsl-hull.ts:27-33 (Poly)
  V3<T> c, h;
  Q4<T> q;
  uint32_t hull = NO_HULL, vs = 0, nv = 8, fs = 0, nf = 6, es = 0, ne = 12, is = 0;
  const uint32_t* buf = nullptr;
};
inline float wordf(const uint32_t* b, uint32_t word) {
  float f;
  std::memcpy(&f, b + word, 4);
  return f;
}
template <class T> PolyShape<T> polyOf(const Body<T>& body, const uint32_t* buf) {  // wgsl-hull.ts:47-63
  PolyShape<T> P;
  P.c = body.pos;
  P.q = body.rot;
  P.h = scale3(body.size, T(0.5));
  P.buf = buf;
  if (body.shape >= SHAPE_HULL) {
    uint32_t h = uint32_t(body.shape - SHAPE_HULL);
    P.hull = h;
    P.vs = buf[4 * h]; P.nv = buf[4 * h + 1]; P.fs = buf[4 * h + 2]; P.nf = buf[4 * h + 3];
    P.es = buf[4 * h + 4]; P.ne = buf[4 * h + 5]; P.is = buf[4 * h + 6];
  }
  return P;
}
template <class T> V3<T> vertLocal(const PolyShape<T>& P, uint32_t v) {  // :65-70
  if (P.hull == NO_HULL) return {(v & 1u) ? P.h[0] : -P.h[0], (v & 2u) ? P.h[1] : -P.h[1], (v & 4u) ? P.h[2] : -P.h[2]};
  uint32_t o = 4 * (P.vs + v);
  return {T(wordf(P.buf, o)), T(wordf(P.buf, o + 1)), T(wordf(P.buf, o + 2))};
}
template <class T> V3<T> vertOf(const PolyShape<T>& P, uint32_t v) { return add3(P.c, rotate(P.q, vertLocal(P, v))); }  // :72-74
template <class T> V3<T> faceNormalLocal(const PolyShape<T>& P, uint32_t f) {  // :149-157
  if (P.hull == NO_HULL) {
    V3<T> n{0, 0, 0};
    n[f / 2u] = (f & 1u) ? T(-1) : T(1);
    return n;
  }
  uint32_t o = 4 * (P.fs + 2 * f);
  return {T(wordf(P.buf, o)), T(wordf(P.buf, o + 1)), T(wordf(P.buf, o + 2))};
}
template <class T> Q4<T> facePlane(const PolyShape<T>& P, uint32_t f) {  // :77-92 (normal, offset)
  V3<T> nl = faceNormalLocal(P, f);
  T d = P.hull == NO_HULL ? P.h[f / 2u] : T(wordf(P.buf, 4 * (P.fs + 2 * f) + 3));
  V3<T> n = rotate(P.q, nl);
  return {n[0], n[1], n[2], d + dot(n, P.c)};
}
template <class T> V3<T> planeN(const Q4<T>& p) { return {p[0], p[1], p[2]}; }
template <class T> uint32_t faceVertCount(const PolyShape<T>& P, uint32_t f) { return P.hull == NO_HULL ? 4u : P.buf[4 * (P.fs + 2 * f + 1) + 1]; }
template <class T> uint32_t faceVert(const PolyShape<T>& P, uint32_t f, uint32_t j) {  // :99-103
  if (P.hull == NO_HULL) return BOX_FACE_VERTS[f * 4 + j];
  uint32_t k = P.buf[4 * (P.fs + 2 * f + 1)] + j;
  return P.buf[4 * (P.is + k / 4) + k % 4];
}
template <class T> std::array<uint32_t, 4> edgeOf(const PolyShape<T>& P, uint32_t e) {  // :105-108
  if (P.hull == NO_HULL) return {BOX_EDGES[e][0], BOX_EDGES[e][1], BOX_EDGES[e][2], BOX_EDGES[e][3]};
  const uint32_t* q = P.buf + 4 * (P.es + e);
  return {q[0], q[1], q[2], q[3]};
}
template <class T> V3<T> polySupport(const PolyShape<T>& P, const V3<T>& dir) {  // :110-121
  V3<T> l = rotate(conjugate(P.q), dir);
  if (P.hull == NO_HULL) return add3(P.c, rotate(P.q, V3<T>{l[0] >= 0 ? P.h[0] : -P.h[0], l[1] >= 0 ? P.h[1] : -P.h[1], l[2] >= 0 ? P.h[2] : -P.h[2]}));
  T best = T(-3.4e38);
  V3<T> at{0, 0, 0};
  for (uint32_t v = 0; v < P.nv; v++) {
    V3<T> p = vertLocal(P, v);
    T s = dot(p, l);
    if (s > best) { best = s; at = p; }
  }
  return add3(P.c, rotate(P.q, at));
}
template <class T> void queryFaces(const PolyShape<T>& A, const PolyShape<T>& B, T& sep, uint32_t& face) {  // :126-134
  sep = T(-3.4e38);
  face = 0;
  for (uint32_t f = 0; f < A.nf; f++) {
    Q4<T> p = facePlane(A, f);
    T s = dot(planeN(p), polySupport(B, neg3(planeN(p)))) - p[3];
    if (s > sep) { sep = s; face = f; }
  }
}
template <class T> bool minkowskiFace(const V3<T>& a, const V3<T>& b, const V3<T>& c, const V3<T>& d) {  // :137-146
  V3<T> bxa = cross(b, a), dxc = cross(d, c);
  T cba = dot(c, bxa), dba = dot(d, bxa), adc = dot(a, dxc), bdc = dot(b, dxc);
  return cba * dba < 0 && adc * bdc < 0 && cba * bdc > 0;
}
template <class T> struct EdgeQuery { T sep; uint32_t ea = 0, eb = 0; V3<T> n{}; bool valid = false; };
template <class T> EdgeQuery<T> queryEdges(const PolyShape<T>& A, const PolyShape<T>& B) {  // :159-188
  EdgeQuery<T> out;
  out.sep = T(-3.4e38);
  Q4<T> toB = qmul(conjugate(B.q), A.q);
  for (uint32_t i = 0; i < A.ne; i++) {
    auto ea = edgeOf(A, i);
    V3<T> a = rotate(toB, faceNormalLocal(A, ea[2]));
    V3<T> b = rotate(toB, faceNormalLocal(A, ea[3]));
    for (uint32_t j = 0; j < B.ne; j++) {
      auto eb = edgeOf(B, j);
      if (!minkowskiFace(a, b, neg3(faceNormalLocal(B, eb[2])), neg3(faceNormalLocal(B, eb[3])))) continue;
      V3<T> pa = vertOf(A, ea[0]), qa = vertOf(A, ea[1]), pb = vertOf(B, eb[0]), qb = vertOf(B, eb[1]);
      V3<T> n = cross(sub3(qa, pa), sub3(qb, pb));
      T l = length(n);
      if (l < T(1e-5) * length(sub3(qa, pa)) * length(sub3(qb, pb))) continue;
      n = div3(n, l);
      if (dot(n, sub3(pa, A.c)) < 0) n = neg3(n);
      T s = dot(n, sub3(pb, pa));
      if (s > out.sep) { out.sep = s; out.ea = i; out.eb = j; out.n = n; out.valid = true; }
    }
  }
  return out;
}
template <class T> int clipHull(const V3<T>* src, int n, V3<T>* dst, const V3<T>& pn, T offset) {  // :191-211
  if (n == 0) return 0;
  int count = 0;
  V3<T> a = src[n - 1];
  T da = dot(pn, a) - offset;
  for (int i = 0; i < n; i++) {
    V3<T> b = src[i];
    T db = dot(pn, b) - offset;
    if ((da <= T(PLANE_EPSILON)) != (db <= T(PLANE_EPSILON))) {
      T t = 0;
      if (std::fabs(da - db) > T(SAT_AXIS_EPSILON)) t = clampv(da / (da - db), T(0), T(1));
      if (count < MAX_CLIP) dst[count++] = add3(a, scale3(sub3(b, a), t));
    }
    if (db <= T(PLANE_EPSILON) && count < MAX_CLIP) dst[count++] = b;
    a = b;
    da = db;
  }
  return count;
}
template <class T> Found<T> hullFaceContact(const PolyShape<T>& A, const PolyShape<T>& B, bool refIsA, uint32_t refFace) {  // :214-291
  Found<T> found;
  const PolyShape<T>& R = refIsA ? A : B;
  const PolyShape<T>& I = refIsA ? B : A;
  Q4<T> plane = facePlane(R, refFace);
  V3<T> rn = planeN(plane);
  uint32_t deepest = 0;
  T low = T(3.4e38);
  for (uint32_t v = 0; v < I.nv; v++) {
    T d = dot(vertOf(I, v), rn);
    if (d < low) { low = d; deepest = v; }
  }
  uint32_t inc = 0;
  T least = T(3.4e38);
  for (uint32_t f = 0; f < I.nf; f++) {
    bool touches = false;
    for (uint32_t j = 0; j < faceVertCount(I, f); j++)
      if (faceVert(I, f, j) == deepest) { touches = true; break; }
    if (!touches) continue;
    T d = dot(planeN(facePlane(I, f)), rn);
    if (d < least) { least = d; inc = f; }
  }
  V3<T> poly[MAX_CLIP], tmp[MAX_CLIP];
  int n = int(std::min<uint32_t>(faceVertCount(I, inc), MAX_CLIP));
  for (int j = 0; j < n; j++) poly[j] = vertOf(I, faceVert(I, inc, uint32_t(j)));
  uint32_t k = faceVertCount(R, refFace);
  V3<T> centre{0, 0, 0};
  for (uint32_t j = 0; j < k; j++) centre = add3(centre, vertOf(R, faceVert(R, refFace, j)));
  centre = div3(centre, T(k));
  for (uint32_t j = 0; j < k && n > 0; j++) {
    V3<T> v0 = vertOf(R, faceVert(R, refFace, j));
    V3<T> v1 = vertOf(R, faceVert(R, refFace, (j + 1) % k));
    V3<T> sd = cross(sub3(v1, v0), rn);
    T l = length(sd);
    if (l < T(SAT_AXIS_EPSILON)) continue;
    sd = div3(sd, l);
    if (dot(sd, sub3(centre, v0)) > 0) sd = neg3(sd);
    n = clipHull(poly, n, tmp, sd, dot(sd, v0));
    for (int m = 0; m < n; m++) poly[m] = tmp[m];
  }
  T depth[MAX_CLIP];
  uint32_t index[MAX_CLIP];
  bool chosen[MAX_CLIP] = {};
  int keep = 0;
  for (int m = 0; m < n; m++) {
    T dist = dot(rn, poly[m]) - plane[3];
    if (dist <= T(PLANE_EPSILON)) { tmp[keep] = poly[m]; depth[keep] = dist; index[keep] = uint32_t(m); keep++; }
  }
  uint32_t prefix = (uint32_t(refIsA ? AXIS_FACE_A : AXIS_FACE_B) << 24) | (std::min<uint32_t>(refFace, 255) << 16) | (std::min<uint32_t>(inc, 255) << 8);
  for (int c = 0; c < std::min(keep, MAX_CONTACTS); c++) {
    int pick = 0;
    T bestScore = T(-3.4e38);
    for (int m = 0; m < keep; m++) {
      if (chosen[m]) continue;
      T score = -depth[m];
      if (c > 0) {
        score = T(3.4e38);
        for (int o = 0; o < keep; o++)
          if (chosen[o]) score = tmin(score, dot(sub3(tmp[m], tmp[o]), sub3(tmp[m], tmp[o])));
      }
      if (score > bestScore) { bestScore = score; pick = m; }
    }
    chosen[pick] = true;
    V3<T> p = tmp[pick];
    V3<T> onRef = sub3(p, scale3(rn, depth[pick]));
    addFound(found, refIsA ? onRef : p, refIsA ? p : onRef, prefix | std::min<uint32_t>(index[pick], 255));
  }
  if (found.count == 0) {
    V3<T> nAB = refIsA ? rn : neg3(rn);
    addFound(found, polySupport(A, nAB), polySupport(B, neg3(nAB)), prefix);
  }
  return found;
}
template <class T> Found<T> hullEdgeContact(const PolyShape<T>& A, const PolyShape<T>& B, const EdgeQuery<T>& q) {  // :293-315
  Found<T> found;
  auto ea = edgeOf(A, q.ea);
  auto eb = edgeOf(B, q.eb);
  V3<T> p0 = vertOf(A, ea[0]), q0 = vertOf(B, eb[0]);
  V3<T> d1 = sub3(vertOf(A, ea[1]), p0), d2 = sub3(vertOf(B, eb[1]), q0);
  V3<T> r = sub3(p0, q0);
  T a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r), c = dot(d1, r), b = dot(d1, d2);
  T denom = a * e - b * b;
  T s = 0;
  if (std::fabs(denom) > T(SAT_AXIS_EPSILON) * a * e) s = clampv((b * f - c * e) / denom, T(0), T(1));
  T t = (b * s + f) / tmax(e, T(SAT_AXIS_EPSILON));
  if (t < 0) { t = 0; s = clampv(-c / tmax(a, T(SAT_AXIS_EPSILON)), T(0), T(1)); }
  else if (t > 1) { t = 1; s = clampv((b - c) / tmax(a, T(SAT_AXIS_EPSILON)), T(0), T(1)); }
  addFound(found, add3(p0, scale3(d1, s)), add3(q0, scale3(d2, t)), (uint32_t(AXIS_EDGE) << 24) | (std::min<uint32_t>(q.ea, 255) << 8) | std::min<uint32_t>(q.eb, 255));
  return found;
}
template <class T> Found<T> collidePoly(const PolyShape<T>& A, const PolyShape<T>& B, bool faceBias, Sat<T>& sat) {  // :318-341
  Found<T> none;
  T faSep, fbSep;
  uint32_t faFace, fbFace;
  queryFaces(A, B, faSep, faFace);
  if (faSep > 0) return none;
  queryFaces(B, A, fbSep, fbFace);
  if (fbSep > 0) return none;
  EdgeQuery<T> eq = queryEdges(A, B);
  if (eq.valid && eq.sep > 0) return none;
  T faceSep = tmax(faSep, fbSep);
  bool edgeWins = eq.valid && eq.sep > T(0.95) * faceSep + T(0.01);
  if (!faceBias) edgeWins = eq.valid && T(0.95) * eq.sep > faceSep + T(0.01);
  if (edgeWins) {
    sat.type = AXIS_EDGE; sat.ia = int(eq.ea); sat.ib = int(eq.eb); sat.sep = eq.sep; sat.n = eq.n; sat.valid = true;
    return hullEdgeContact(A, B, eq);
  }
  if (fbSep > faSep) {
    sat.type = AXIS_FACE_B; sat.ia = 0; sat.ib = int(fbFace); sat.sep = fbSep; sat.n = neg3(planeN(facePlane(B, fbFace))); sat.valid = true;
    return hullFaceContact(A, B, false, fbFace);
  }
  sat.type = AXIS_FACE_A; sat.ia = int(faFace); sat.ib = 0; sat.sep = faSep; sat.n = planeN(facePlane(A, faFace)); sat.valid = true;
  return hullFaceContact(A, B, true, faFace);
}
template <class T> V3<T> segmentPoint(const V3<T>& a, const V3<T>& b, const V3<T>& p) {  // :344-347
  V3<T> d = sub3(b, a);
  return add3(a, scale3(d, clampv(dot(sub3(p, a), d) / tmax(dot(d, d), T(1e-20)), T(0), T(1))));
}
// wgsl-hull.ts:350-405: n from the sphere towards X
template <class T> bool sphereHull(const V3<T>& c, T r, const PolyShape<T>& X, V3<T>& onSphere, V3<T>& onHull, V3<T>& nOut) {
  T deepest = T(-3.4e38);
  uint32_t deepFace = 0;
  for (uint32_t f = 0; f < X.nf; f++) {
    T s = dot(planeN(facePlane(X, f)), c) - facePlane(X, f)[3];
    if (s > deepest) { deepest = s; deepFace = f; }
  }
  if (deepest > r) return false;
  if (deepest <= 0) {
    V3<T> n = planeN(facePlane(X, deepFace));
    nOut = neg3(n);
    onHull = sub3(c, scale3(n, deepest));
    onSphere = sub3(c, scale3(n, r));
    return true;
  }
  V3<T> best{0, 0, 0};
  T bestDist = T(3.4e38);
  for (uint32_t f = 0; f < X.nf; f++) {
    Q4<T> plane = facePlane(X, f);
    T s = dot(planeN(plane), c) - plane[3];
    if (s <= 0) continue;
    V3<T> p = sub3(c, scale3(planeN(plane), s));
    uint32_t k = faceVertCount(X, f);
    V3<T> centre{0, 0, 0};
    for (uint32_t j = 0; j < k; j++) centre = add3(centre, vertOf(X, faceVert(X, f, j)));
    centre = div3(centre, T(k));
    bool inside = true;
    V3<T> edgeBest{0, 0, 0};
    T edgeDist = T(3.4e38);
    for (uint32_t j = 0; j < k; j++) {
      V3<T> v0 = vertOf(X, faceVert(X, f, j));
      V3<T> v1 = vertOf(X, faceVert(X, f, (j + 1) % k));
      V3<T> side = cross(sub3(v1, v0), planeN(plane));
      if (dot(side, sub3(centre, v0)) > 0) side = neg3(side);
      if (dot(side, sub3(p, v0)) > 0) inside = false;
      V3<T> q = segmentPoint(v0, v1, c);
      T dq = dot(sub3(q, c), sub3(q, c));
      if (dq < edgeDist) { edgeDist = dq; edgeBest = q; }
    }
    if (!inside) p = edgeBest;
    T dist = length(sub3(p, c));
    if (dist < bestDist) { bestDist = dist; best = p; }
  }
  if (bestDist > r) return false;
  V3<T> n{0, 0, 1};
  if (bestDist > 0) n = div3(sub3(c, best), bestDist);
  nOut = neg3(n);
  onHull = best;
  onSphere = sub3(c, scale3(n, r));
  return true;
}

// One pair's contacts (wgsl-collision.ts:767-811). Returns the manifold normal (B to A) in `normal`.
template <class T> Found<T> narrowphase(const Body<T>& a, const Body<T>& b, bool faceBias, V3<T>& normal, const uint32_t* hulls = nullptr) {
  OBB<T> A = makeOBB(a.pos, a.rot, a.size), B = makeOBB(b.pos, b.rot, b.size);
  Sat<T> sat;
  Found<T> found;
  bool sA = a.shape == SHAPE_SPHERE, sB = b.shape == SHAPE_SPHERE;
  if (sA && sB) {
    found = sphereSphere(A, B, sat);
  } else if (hulls && (a.shape >= SHAPE_HULL || b.shape >= SHAPE_HULL)) {  // wgsl-collision.ts:781-796
    if (sA || sB) {
      V3<T> onS, onX, n;
      if (sA) {
        bool hit = sphereHull(A.c, A.h[0], polyOf(b, hulls), onS, onX, n);
        sat.n = n;
        if (hit) addFound(found, onS, onX, SPHERE_FEATURE);
      } else {
        bool hit = sphereHull(B.c, B.h[0], polyOf(a, hulls), onS, onX, n);
        sat.n = neg3(n);
        if (hit) addFound(found, onX, onS, SPHERE_FEATURE);
      }
    } else {
      found = collidePoly(polyOf(a, hulls), polyOf(b, hulls), faceBias, sat);
    }
  } else if (sA || sB) {
    V3<T> onS, onX, n;
    if (sA) {
      bool hit = sphereBox(A, B, b.rot, onS, onX, n);
      sat.n = n;
      if (hit) addFound(found, onS, onX, SPHERE_FEATURE);
    } else {
      bool hit = sphereBox(B, A, a.rot, onS, onX, n);
      sat.n = neg3(n);
      if (hit) addFound(found, onX, onS, SPHERE_FEATURE);
    }
  } else {
    found = collideBoxes(A, B, faceBias, sat);
  }
  normal = neg3(sat.n);
  return found;
}

// ---------------------------------------------------------------------------------------------
// Manifold (ref/manifold.ts:81-217)
// ---------------------------------------------------------------------------------------------
template <class T> struct Contact { uint32_t feature = 0; V3<T> rA{}, rB{}, C0{}, penalty{}, lambda{}; bool stick = false; };

template <class T> struct Manifold : Force<T> {
  std::vector<Contact<T>> contacts;
  M3<T> basis{};
  T friction = 0;
  uint32_t generated = 0;  // GPU mode: the step whose narrowphase made its contact points
  // GPU mode: which rule set, and the manifold of the same pair last step (warm start)
  Manifold(Solver<T>* s, int a, int b) : Force<T>(s, a, b, K_MANIFOLD) {}

  bool initialize() override {  // manifold.ts:95-133
    Body<T>& A = this->solver->bodies[this->bodyA];
    Body<T>& B = this->solver->bodies[this->bodyB];
    Solver<T>& solver = *this->solver;
    friction = std::sqrt(A.friction * B.friction);
    std::vector<Contact<T>> old = std::move(contacts);
    contacts.clear();
    OBB<T> oa = makeOBB(A.pos, A.rot, A.size), ob = makeOBB(B.pos, B.rot, B.size);
    Sat<T> sat;
    Found<T> f = collideBoxes(oa, ob, false, sat);
    if (f.count) basis = orthonormal(neg3(sat.n));  // collide.ts:558: the basis is written once a face axis is valid
    for (int i = 0; i < f.count; i++) {
      Contact<T> c;
      c.feature = f.feature[i];
      c.rA = rotateInv(A.rot, sub3(f.xA[i], A.pos));
      c.rB = rotateInv(B.rot, sub3(f.xB[i], B.pos));
      const Contact<T>* prev = nullptr;
      for (auto& o : old) if (o.feature == c.feature) { prev = &o; break; }
      if (prev) {
        if (prev->stick) { c.rA = prev->rA; c.rB = prev->rB; }
        c.penalty = prev->penalty;
        c.lambda = prev->lambda;
        c.stick = prev->stick;
      }
      contacts.push_back(c);
    }
    for (auto& c : contacts) {
      V3<T> xA = transform(A.pos, A.rot, c.rA);
      V3<T> xB = transform(B.pos, B.rot, c.rB);
      c.C0 = mulv(basis, sub3(xA, xB));
      c.C0[0] += T(COLLISION_MARGIN);
      for (int i = 0; i < 3; i++) {
        c.lambda[i] = c.lambda[i] * solver.alpha * solver.gamma;
        c.penalty[i] = clampv(c.penalty[i] * solver.gamma, T(PENALTY_MIN), T(PENALTY_MAX));
      }
    }
    return !contacts.empty();
  }

  // manifold.ts:139-168; GPU mode evaluates sphere contacts' lever arms at the step-start
  // rotation (wgsl-solve.ts:197-206).
  void evaluate(const Contact<T>& c, T alpha, const V3<T>& dqALin, const V3<T>& dqAAng, const V3<T>& dqBLin, const V3<T>& dqBAng,
                V3<T>& C, V3<T>& F, T& frictionScale, T& bounds, M3<T>& jBLin, M3<T>& jAAng, M3<T>& jBAng) const {
    const Body<T>& A = this->solver->bodies[this->bodyA];
    const Body<T>& B = this->solver->bodies[this->bodyB];
    bool rolling = this->solver->gpuMode && (c.feature & ~STICK_BIT) == SPHERE_FEATURE;
    V3<T> rAWorld = rotate(rolling ? A.initRot : A.rot, c.rA);
    V3<T> rBWorld = rotate(rolling ? B.initRot : B.rot, c.rB);
    jBLin = negm(basis);
    for (int k = 0; k < 3; k++) {
      V3<T> r1 = cross(rAWorld, V3<T>{basis[k * 3], basis[k * 3 + 1], basis[k * 3 + 2]});
      V3<T> r2 = cross(rBWorld, V3<T>{jBLin[k * 3], jBLin[k * 3 + 1], jBLin[k * 3 + 2]});
      for (int j = 0; j < 3; j++) { jAAng[k * 3 + j] = r1[j]; jBAng[k * 3 + j] = r2[j]; }
    }
    M3<T> K = diagonal(c.penalty[0], c.penalty[1], c.penalty[2]);
    C = scale3(c.C0, T(1) - alpha);
    C = addScaled3(C, mulv(basis, dqALin), T(1));
    C = addScaled3(C, mulv(jBLin, dqBLin), T(1));
    C = addScaled3(C, mulv(jAAng, dqAAng), T(1));
    C = addScaled3(C, mulv(jBAng, dqBAng), T(1));
    F = mulv(K, C);
    F = addScaled3(F, c.lambda, T(1));
    F[0] = tmin(F[0], T(0));
    bounds = std::fabs(F[0]) * friction;
    frictionScale = std::sqrt(F[1] * F[1] + F[2] * F[2]);
    if (frictionScale > bounds && frictionScale > 0) {
      F[1] *= bounds / frictionScale;
      F[2] *= bounds / frictionScale;
    }
  }
  void displacements(V3<T>& aL, V3<T>& aA, V3<T>& bL, V3<T>& bA) const {  // manifold.ts:170-177
    const Body<T>& A = this->solver->bodies[this->bodyA];
    const Body<T>& B = this->solver->bodies[this->bodyB];
    aL = sub3(A.pos, A.initPos);
    aA = qsub(A.rot, A.initRot);
    bL = sub3(B.pos, B.initPos);
    bA = qsub(B.rot, B.initRot);
  }
  void updatePrimal(int body, T alpha, BodySystem<T>& sys) override {  // manifold.ts:179-200
    V3<T> aL, aA, bL, bA;
    displacements(aL, aA, bL, bA);
    bool isA = body == this->bodyA;
    for (auto& c : contacts) {
      V3<T> C, F;
      T fs, bd;
      M3<T> jBLin, jAAng, jBAng;
      evaluate(c, alpha, aL, aA, bL, bA, C, F, fs, bd, jBLin, jAAng, jBAng);
      const M3<T>& jLin = isA ? basis : jBLin;
      const M3<T>& jAng = isA ? jAAng : jBAng;
      M3<T> K = diagonal(c.penalty[0], c.penalty[1], c.penalty[2]);
      M3<T> jLinT = transpose(jLin), jAngT = transpose(jAng);
      M3<T> jAngTk = mul(jAngT, K);
      addm(sys.lhsLin, mul(mul(jLinT, K), jLin));
      addm(sys.lhsAng, mul(jAngTk, jAng));
      addm(sys.lhsCross, mul(jAngTk, jLin));
      sys.rhsLin = addScaled3(sys.rhsLin, mulv(jLinT, F), T(1));
      sys.rhsAng = addScaled3(sys.rhsAng, mulv(jAngT, F), T(1));
    }
  }
  void updateDual(T alpha) override {  // manifold.ts:202-217
    V3<T> aL, aA, bL, bA;
    displacements(aL, aA, bL, bA);
    Solver<T>& solver = *this->solver;
    for (auto& c : contacts) {
      V3<T> C, F;
      T fs, bd;
      M3<T> jBLin, jAAng, jBAng;
      evaluate(c, alpha, aL, aA, bL, bA, C, F, fs, bd, jBLin, jAAng, jBAng);
      c.lambda = F;
      if (F[0] < 0) c.penalty[0] = tmin(c.penalty[0] + solver.betaLin * std::fabs(C[0]), T(PENALTY_MAX));
      if (fs <= bd) {
        c.penalty[1] = tmin(c.penalty[1] + solver.betaLin * std::fabs(C[1]), T(PENALTY_MAX));
        c.penalty[2] = tmin(c.penalty[2] + solver.betaLin * std::fabs(C[2]), T(PENALTY_MAX));
        c.stick = std::sqrt(C[1] * C[1] + C[2] * C[2]) < T(STICK_THRESH);
      }
    }
  }
};

// ---------------------------------------------------------------------------------------------
// Joint, Spring, IgnoreCollision (ref/forces.ts:61-390)
// ---------------------------------------------------------------------------------------------
const double INF = std::numeric_limits<double>::infinity();

template <class T> M3<T> geometricStiffnessBallSocket(int k, const V3<T>& v) {  // forces.ts:62-68
  M3<T> o = diagonal(-v[k], -v[k], -v[k]);
  o[k] += v[0];
  o[3 + k] += v[1];
  o[6 + k] += v[2];
  return o;
}
template <class T> V3<T> componentMin(const V3<T>& a, T b) { return {tmin(a[0], b), tmin(a[1], b), tmin(a[2], b)}; }

template <class T> struct Joint : Force<T> {
  V3<T> rA{}, rB{}, C0Lin{}, C0Ang{}, penaltyLin{}, penaltyAng{}, lambdaLin{}, lambdaAng{};
  T stiffnessLin = INF, stiffnessAng = 0, fracture = INF, torqueArm = 0;
  bool broken = false, fractureLinear = false;
  bool hasRest = false, hasRestStart = false;
  Q4<T> rest{0, 0, 0, 1}, restStart{0, 0, 0, 1};
  T yield = INF, breakBend = INF;

  Joint(Solver<T>* s, int a, int b, V3<T> ra, V3<T> rb, T sl, T sa, T fr) : Force<T>(s, a, b, K_JOINT) {  // forces.ts:129-147
    rA = ra; rB = rb; stiffnessLin = sl; stiffnessAng = sa; fracture = fr;
    V3<T> sz = a >= 0 ? s->bodies[a].size : V3<T>{0, 0, 0};
    const V3<T>& bs = s->bodies[b].size;
    torqueArm = lengthSq(V3<T>{sz[0] + bs[0], sz[1] + bs[1], sz[2] + bs[2]});
  }
  V3<T> evaluateLin() const {  // forces.ts:150-155
    V3<T> pA = this->bodyA >= 0 ? transform(this->solver->bodies[this->bodyA].pos, this->solver->bodies[this->bodyA].rot, rA) : rA;
    const Body<T>& B = this->solver->bodies[this->bodyB];
    return sub3(pA, transform(B.pos, B.rot, rB));
  }
  V3<T> evaluateAng() const {  // forces.ts:165-172
    Q4<T> rotA = this->bodyA >= 0 ? this->solver->bodies[this->bodyA].rot : Q4<T>{0, 0, 0, 1};
    const Q4<T>& rotB = this->solver->bodies[this->bodyB].rot;
    Q4<T> target = hasRest ? qmul(rotA, rest) : rotA;
    V3<T> out = qsub(target, rotB);
    if (target[0] * rotB[0] + target[1] * rotB[1] + target[2] * rotB[2] + target[3] * rotB[3] < 0) out = neg3(out);
    return scale3(out, torqueArm);
  }
  void holdCurrentRotation() {  // forces.ts:175-179
    Q4<T> rotA = this->bodyA >= 0 ? this->solver->bodies[this->bodyA].rot : Q4<T>{0, 0, 0, 1};
    rest = qnormalize(qmul(conjugate(rotA), this->solver->bodies[this->bodyB].rot));
    hasRest = true;
  }
  T bend() const { return hasRestStart ? qangle(restStart, hasRest ? rest : Q4<T>{0, 0, 0, 1}) : T(0); }  // forces.ts:182-184
  bool initialize() override {  // forces.ts:186-203
    Solver<T>& s = *this->solver;
    C0Lin = evaluateLin();
    C0Ang = evaluateAng();
    const bool cold = (this->bodyA >= 0 && (s.bodies[this->bodyA].lifecycle & 4u)) || (s.bodies[this->bodyB].lifecycle & 4u);
    if (cold) {  // a cold body's joints start afresh (wgsl-solve.ts:247-253)
      for (int i = 0; i < 3; i++) {
        lambdaLin[i] = lambdaAng[i] = T(0);
        penaltyLin[i] = tmin(T(PENALTY_MIN), stiffnessLin);
        penaltyAng[i] = tmin(T(PENALTY_MIN), stiffnessAng);
      }
      return !broken;
    }
    for (int i = 0; i < 3; i++) {
      lambdaLin[i] = lambdaLin[i] * s.alpha * s.gamma;
      lambdaAng[i] = lambdaAng[i] * s.alpha * s.gamma;
      penaltyLin[i] = clampv(penaltyLin[i] * s.gamma, T(PENALTY_MIN), T(PENALTY_MAX));
      penaltyAng[i] = clampv(penaltyAng[i] * s.gamma, T(PENALTY_MIN), T(PENALTY_MAX));
    }
    penaltyLin = componentMin(penaltyLin, stiffnessLin);
    penaltyAng = componentMin(penaltyAng, stiffnessAng);
    return !broken;
  }
  void updatePrimal(int body, T alpha, BodySystem<T>& sys) override {  // forces.ts:205-263
    bool isA = body == this->bodyA;
    if (lengthSq(penaltyLin) > 0) {
      M3<T> K = diagonal(penaltyLin[0], penaltyLin[1], penaltyLin[2]);
      V3<T> C = evaluateLin();
      if (stiffnessLin == T(INF)) C = addScaled3(C, C0Lin, -alpha);
      V3<T> F = mulv(K, C);
      F = addScaled3(F, lambdaLin, T(1));
      T sgn = isA ? T(1) : T(-1);
      M3<T> jLin = diagonal(sgn, sgn, sgn);
      M3<T> jAng = isA ? skew(neg3(rotate(this->solver->bodies[this->bodyA].rot, rA))) : skew(rotate(this->solver->bodies[this->bodyB].rot, rB));
      M3<T> jLinT = transpose(jLin), jAngT = transpose(jAng);
      M3<T> jAngTk = mul(jAngT, K);
      addm(sys.lhsLin, mul(mul(jLinT, K), jLin));
      addm(sys.lhsAng, mul(jAngTk, jAng));
      addm(sys.lhsCross, mul(jAngTk, jLin));
      V3<T> r = isA ? rotate(this->solver->bodies[this->bodyA].rot, rA) : neg3(rotate(this->solver->bodies[this->bodyB].rot, rB));
      M3<T> H = scalem(geometricStiffnessBallSocket(0, r), F[0]);
      addm(H, scalem(geometricStiffnessBallSocket(1, r), F[1]));
      addm(H, scalem(geometricStiffnessBallSocket(2, r), F[2]));
      addm(sys.lhsAng, diagonalize(H));
      sys.rhsLin = addScaled3(sys.rhsLin, mulv(jLinT, F), T(1));
      sys.rhsAng = addScaled3(sys.rhsAng, mulv(jAngT, F), T(1));
    }
    if (lengthSq(penaltyAng) > 0) {
      M3<T> K = diagonal(penaltyAng[0], penaltyAng[1], penaltyAng[2]);
      V3<T> C = evaluateAng();
      if (stiffnessAng == T(INF)) C = addScaled3(C, C0Ang, -alpha);
      V3<T> F = mulv(K, C);
      F = addScaled3(F, lambdaAng, T(1));
      T s = (isA ? T(1) : T(-1)) * torqueArm;
      M3<T> jAng = diagonal(s, s, s);
      M3<T> jAngT = transpose(jAng);
      addm(sys.lhsAng, mul(mul(jAngT, K), jAng));
      sys.rhsAng = addScaled3(sys.rhsAng, mulv(jAngT, F), T(1));
    }
  }
  void updateDual(T alpha) override {  // forces.ts:265-321
    Solver<T>& s = *this->solver;
    if (lengthSq(penaltyLin) > 0) {
      M3<T> K = diagonal(penaltyLin[0], penaltyLin[1], penaltyLin[2]);
      V3<T> C = evaluateLin();
      if (stiffnessLin == T(INF)) {
        C = addScaled3(C, C0Lin, -alpha);
        V3<T> F = mulv(K, C);
        lambdaLin = addScaled3(F, lambdaLin, T(1));
      }
      penaltyLin = addScaled3(penaltyLin, abs3(C), s.betaLin);
      penaltyLin = componentMin(penaltyLin, tmin(stiffnessLin, T(PENALTY_MAX)));
    }
    bool yielded = false;
    if (lengthSq(penaltyAng) > 0) {
      M3<T> K = diagonal(penaltyAng[0], penaltyAng[1], penaltyAng[2]);
      V3<T> C = evaluateAng();
      if (stiffnessAng == T(INF)) {
        C = addScaled3(C, C0Ang, -alpha);
        V3<T> F = mulv(K, C);
        lambdaAng = addScaled3(F, lambdaAng, T(1));
        T force2 = lengthSq(lambdaAng);
        if (force2 > yield * yield && force2 <= fracture * fracture) {
          if (!hasRestStart) { restStart = hasRest ? rest : Q4<T>{0, 0, 0, 1}; hasRestStart = true; }
          holdCurrentRotation();
          C0Ang = V3<T>{0, 0, 0};
          lambdaAng = scale3(lambdaAng, yield / std::sqrt(force2));
          yielded = true;
        }
      }
      if (!yielded) {
        penaltyAng = addScaled3(penaltyAng, abs3(C), s.betaAng);
        penaltyAng = componentMin(penaltyAng, tmin(stiffnessAng, T(PENALTY_MAX)));
      }
    }
    if (lengthSq(lambdaAng) > fracture * fracture || (fractureLinear && lengthSq(lambdaLin) > fracture * fracture) ||
        (yielded && bend() > breakBend)) {
      penaltyLin = penaltyAng = lambdaLin = lambdaAng = V3<T>{0, 0, 0};
      broken = true;
    }
  }
};

template <class T> struct Spring : Force<T> {  // forces.ts:325-381
  V3<T> rA{}, rB{};
  T rest = -1, stiffness = 0;
  Spring(Solver<T>* s, int a, int b, V3<T> ra, V3<T> rb, T k, T r) : Force<T>(s, a, b, K_SPRING) {
    rA = ra; rB = rb; stiffness = k; rest = r;
    if (rest < 0) {
      V3<T> pA = transform(s->bodies[a].pos, s->bodies[a].rot, rA);
      V3<T> pB = transform(s->bodies[b].pos, s->bodies[b].rot, rB);
      rest = length(sub3(pA, pB));
    }
  }
  bool initialize() override { return true; }
  void updatePrimal(int body, T, BodySystem<T>& sys) override {
    const Body<T>& A = this->solver->bodies[this->bodyA];
    const Body<T>& B = this->solver->bodies[this->bodyB];
    V3<T> pA = transform(A.pos, A.rot, rA), pB = transform(B.pos, B.rot, rB);
    V3<T> d = sub3(pA, pB);
    T dLen = length(d);
    if (dLen <= T(1.0e-6)) return;
    V3<T> n = div3(d, dLen);
    T c = dLen - rest;
    T f = stiffness * c;
    V3<T> jl, ja;
    if (body == this->bodyA) {
      V3<T> r = rotate(A.rot, rA);
      jl = n;
      ja = cross(r, n);
    } else {
      V3<T> r = rotate(B.rot, rB);
      jl = neg3(n);
      ja = neg3(cross(r, n));
    }
    addm(sys.lhsLin, scalem(outer(jl, jl), stiffness));
    addm(sys.lhsAng, scalem(outer(ja, ja), stiffness));
    addm(sys.lhsCross, scalem(outer(ja, jl), stiffness));
    sys.rhsLin = addScaled3(sys.rhsLin, scale3(jl, f), T(1));
    sys.rhsAng = addScaled3(sys.rhsAng, scale3(ja, f), T(1));
  }
  void updateDual(T) override {}
};

template <class T> struct Ignore : Force<T> {  // forces.ts:384-390
  Ignore(Solver<T>* s, int a, int b) : Force<T>(s, a, b, K_IGNORE) {}
  bool initialize() override { return true; }
  void updatePrimal(int, T, BodySystem<T>&) override {}
  void updateDual(T) override {}
};

// ---------------------------------------------------------------------------------------------
// Broadphase pair rule of the GPU (wgsl-collision.ts:109-323, radii.ts:12-55,
// solver.ts:1263-1318), with the probing body's perspective kept so the f32 tests round the same.
// ---------------------------------------------------------------------------------------------

inline double selectKth(std::vector<double>& a, int k) {  // radii.ts:19-41 (Wirth)
  int lo = 0, hi = int(a.size()) - 1;
  while (lo < hi) {
    double pivot = a[k];
    int i = lo, j = hi;
    do {
      while (a[i] < pivot) i++;
      while (pivot < a[j]) j--;
      if (i <= j) { std::swap(a[i], a[j]); i++; j--; }
    } while (i <= j);
    if (j < k) lo = i;
    if (k < i) hi = j;
  }
  return a[k];
}
inline double largestSmall(std::vector<double> radii) {  // radii.ts:47-55
  int n = int(radii.size());
  double median = n > 0 ? selectKth(radii, n >> 1) : 1;
  double maxSmall = 0;
  for (int i = 0; i < n; i++) if (radii[i] <= 2 * median) maxSmall = std::max(maxSmall, radii[i]);
  if (n > 64) maxSmall = std::max(maxSmall, selectKth(radii, n - 64 - 1));
  return maxSmall;
}

struct BroadConfig { float threshold; double maxSmall; };
// solver.ts:1265-1275 (radii as the GPU stores them, f32)
inline BroadConfig broadConfig(const std::vector<float>& r32) {
  std::vector<double> radii(r32.begin(), r32.end());
  double maxSmall = largestSmall(radii);
  double minLarge = INF;
  for (double r : radii) if (r > maxSmall) minLarge = std::min(minLarge, r);
  double threshold = minLarge == INF ? maxSmall * 1.5 : (maxSmall + minLarge) / 2;
  return BroadConfig{float(threshold), maxSmall};
}

struct Shape32 { V3<float> ax[3]; V3<float> h; bool sphere; };
inline Shape32 shapeOf32(const Q4<float>& q, const V3<float>& size, bool sphere) {  // wgsl-collision.ts:157-166
  Shape32 s;
  s.h = scale3(size, 0.5f);
  s.sphere = sphere;
  s.ax[0] = rotate(q, V3<float>{1, 0, 0});
  s.ax[1] = rotate(q, V3<float>{0, 1, 0});
  s.ax[2] = rotate(q, V3<float>{0, 0, 1});
  return s;
}
inline float extent32(const Shape32& s, const V3<float>& n) {  // :169-172
  if (s.sphere) return s.h[0];
  return s.h[0] * std::fabs(dot(n, s.ax[0])) + s.h[1] * std::fabs(dot(n, s.ax[1])) + s.h[2] * std::fabs(dot(n, s.ax[2]));
}
inline V3<float> aabbHalf32(const Shape32& s) {  // :175-178
  if (s.sphere) return V3<float>{s.h[0], s.h[0], s.h[0]};
  V3<float> a0 = abs3(s.ax[0]), a1 = abs3(s.ax[1]), a2 = abs3(s.ax[2]);
  return add3(add3(scale3(a0, s.h[0]), scale3(a1, s.h[1])), scale3(a2, s.h[2]));
}
inline bool faceSeparated32(const Shape32& A, const Shape32& B, const V3<float>& d) {  // :185-191
  for (int k = 0; k < 3; k++) {
    if (std::fabs(dot(d, A.ax[k])) - extent32(A, A.ax[k]) - extent32(B, A.ax[k]) > 1e-3f) return true;
    if (std::fabs(dot(d, B.ax[k])) - extent32(A, B.ax[k]) - extent32(B, B.ax[k]) > 1e-3f) return true;
  }
  return false;
}

// The GPU record of a body, as the pair test reads it (f32).
struct Rec32 { V3<float> pos; Q4<float> rot; V3<float> size; float mass, radius; bool sphere; uint32_t groups, mask; };

// testPair (wgsl-collision.ts:208-234) from probing body p against j, before the ignore check.
inline bool pairTest32(const Rec32& P, const Rec32& J) {
  if (!(P.mass > 0) && J.mass <= 0) return false;
  if ((P.groups & J.mask) == 0 || (J.groups & P.mask) == 0) return false;
  V3<float> d = sub3(P.pos, J.pos);
  float r = P.radius + J.radius;
  if (dot(d, d) > r * r) return false;
  Shape32 sp = shapeOf32(P.rot, P.size, P.sphere), sj = shapeOf32(J.rot, J.size, J.sphere);
  V3<float> ap = aabbHalf32(sp), aj = aabbHalf32(sj);
  for (int k = 0; k < 3; k++) if (std::fabs(d[k]) > ap[k] + aj[k] + 1e-4f) return false;
  if (faceSeparated32(sp, sj, d)) return false;
  return true;
}

// All pairs (hi, lo) the GPU broadphase reports, sorted. `ignored(hi, lo)` is the no-collide rule.
template <class Ign> std::vector<std::pair<uint32_t, uint32_t>> gpuPairs(const std::vector<Rec32>& B, Ign ignored) {
  int n = int(B.size());
  std::vector<float> radii(n);
  for (int i = 0; i < n; i++) radii[i] = B[i].radius;
  BroadConfig cfg = broadConfig(radii);
  std::vector<char> large(n);
  std::vector<int> largeList;
  for (int i = 0; i < n; i++) { large[i] = B[i].radius > cfg.threshold; if (large[i]) largeList.push_back(i); }
  double cell = std::max(2 * cfg.maxSmall * (1 + 1e-4), 1e-3);
  // Any complete candidate search gives the same set; this one hashes exact cells.
  std::unordered_map<uint64_t, std::vector<int>> grid;
  auto cellOf = [&](int i) { return std::array<int64_t, 3>{(int64_t)std::floor(double(B[i].pos[0]) / cell), (int64_t)std::floor(double(B[i].pos[1]) / cell), (int64_t)std::floor(double(B[i].pos[2]) / cell)}; };
  auto key = [](int64_t x, int64_t y, int64_t z) { return (uint64_t(x & 0x1fffff) << 42) | (uint64_t(y & 0x1fffff) << 21) | uint64_t(z & 0x1fffff); };
  for (int i = 0; i < n; i++) if (!large[i]) { auto c = cellOf(i); grid[key(c[0], c[1], c[2])].push_back(i); }
  std::vector<std::pair<uint32_t, uint32_t>> out;
  // Which body probes (findPairs / findFixedLarge ownership, wgsl-collision.ts:243-323)
  auto prober = [&](int i, int j) -> int {
    bool di = B[i].mass > 0, dj = B[j].mass > 0;
    if (di && dj) {
      if (!large[i] && !large[j]) return std::max(i, j);
      if (large[i] != large[j]) return large[i] ? j : i;
      return std::min(i, j);
    }
    int dyn = di ? i : j, fix = di ? j : i;
    if (!large[fix] && large[dyn]) return fix;  // findFixedLarge
    return dyn;
  };
#pragma omp parallel
  {
    std::vector<std::pair<uint32_t, uint32_t>> local;
    auto emit = [&](int p, int j) {
      if (!pairTest32(B[p], B[j])) return;
      uint32_t a = std::max(p, j), b = std::min(p, j);
      if (ignored(a, b)) return;
      local.push_back({a, b});
    };
#pragma omp for schedule(dynamic, 256)
    for (int i = 0; i < n; i++) {
      if (large[i]) continue;
      auto c = cellOf(i);
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            auto it = grid.find(key(c[0] + dx, c[1] + dy, c[2] + dz));
            if (it == grid.end()) continue;
            for (int j : it->second)
              if (j < i) {
                int p = prober(i, j);
                emit(p, p == i ? j : i);
              }
          }
    }
#pragma omp for schedule(dynamic, 1)
    for (int li = 0; li < int(largeList.size()); li++) {
      int l = largeList[li];
      for (int j = 0; j < n; j++) {
        if (j == l || (large[j] && j > l)) continue;  // large-large once
        int p = prober(l, j);
        emit(p, p == l ? j : l);
      }
    }
#pragma omp critical
    out.insert(out.end(), local.begin(), local.end());
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// ---------------------------------------------------------------------------------------------
// Jones-Plassmann colouring of the GPU (avbd2d/gpu/wgsl-topology.ts:155-328 with the 3D
// pending-colour rule; CPU model avbd2d/soa/coloring.ts), rounds run until nothing is pending.
// ---------------------------------------------------------------------------------------------
inline uint32_t hash32(uint32_t x) {  // avbd2d/gpu/layout.ts:107-115
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}
inline uint32_t priority(uint32_t i) { return hash32(i + 0x9e3779b9u); }
inline bool beats(uint32_t i, uint32_t j) { uint32_t pi = priority(i), pj = priority(j); return pi > pj || (pi == pj && i > j); }

struct ColorResult { int rounds = 0; int clashes = 0; int colors = 0; };

// state: per body colour | PENDING (input: last step's, output: this step's). nbr: CSR of dynamic
// neighbours (duplicates allowed). cap: colour cap (<= 64). maxRounds: even.
inline ColorResult jpColor(int n, const std::vector<char>& dynamic, const std::vector<int>& start, const std::vector<int>& nbr,
                           std::vector<uint32_t>& state, int cap, int maxRounds) {
  std::vector<uint32_t> A = state, Bs(n);
  auto smallestFree = [&](int b, const std::vector<uint32_t>& src, bool skipPending) -> uint32_t {
    uint32_t lo = 0, hi = 0;
    for (int e = start[b]; e < start[b + 1]; e++) {
      int j = nbr[e];
      uint32_t s = src[j];
      if (skipPending && (s & PENDING)) continue;
      uint32_t col = s & 0xff;
      if (col == NO_COLOR) continue;
      if (col < 32) lo |= 1u << col; else hi |= 1u << (col - 32);
    }
    if (~lo != 0) return __builtin_ctz(~lo);
    if (~hi != 0) return 32 + __builtin_ctz(~hi);
    return MAX_COLORS;
  };
  // compact: A -> B
  for (int b = 0; b < n; b++) {
    if (!dynamic[b]) { Bs[b] = NO_COLOR; continue; }
    uint32_t col = A[b] & 0xff;
    if (col != NO_COLOR) {
      bool isMax = true;
      for (int e = start[b]; e < start[b + 1] && isMax; e++) if (!beats(b, nbr[e])) isMax = false;
      if (isMax) col = std::min(col, smallestFree(b, A, false));
    }
    Bs[b] = col;
  }
  // mark: B -> A
  int pendingCount = 0;
  for (int b = 0; b < n; b++) {
    if (!dynamic[b]) { A[b] = NO_COLOR; continue; }
    uint32_t col = Bs[b] & 0xff;
    bool pending = col == NO_COLOR;
    for (int e = start[b]; e < start[b + 1] && !pending; e++) {
      int j = nbr[e];
      if ((Bs[j] & 0xff) == col && beats(j, b)) pending = true;
    }
    A[b] = col | (pending ? PENDING : 0);
    pendingCount += pending;
  }
  ColorResult res;
  auto round = [&](const std::vector<uint32_t>& src, std::vector<uint32_t>& dst) {
    for (int b = 0; b < n; b++) {
      uint32_t s = src[b];
      if (!(s & PENDING)) { dst[b] = s; continue; }
      bool isMax = true;
      for (int e = start[b]; e < start[b + 1] && isMax; e++) {
        int j = nbr[e];
        if ((src[j] & PENDING) && !beats(b, j)) isMax = false;
      }
      if (isMax) {
        uint32_t f = smallestFree(b, src, true);
        dst[b] = f >= uint32_t(cap) ? (uint32_t(cap - 1) | PENDING) : f;
      } else dst[b] = s;
    }
  };
  // Rounds in pairs (A -> B -> A) while anything is pending, at most maxRounds
  while (pendingCount > 0 && res.rounds < maxRounds) {
    round(A, Bs);
    round(Bs, A);
    res.rounds += 2;
    pendingCount = 0;
    for (int b = 0; b < n; b++) if (dynamic[b] && (A[b] & PENDING)) pendingCount++;
  }
  // count: NO_COLOR -> cap-1, pending kept (colorCount, wgsl-topology.ts:277-304)
  for (int b = 0; b < n; b++) {
    if (!dynamic[b]) { state[b] = A[b]; continue; }
    uint32_t s = A[b];
    uint32_t col = s & 0xff;
    if (s & PENDING) res.clashes++;
    if (col == NO_COLOR) col = cap - 1;
    state[b] = col | (s & PENDING);
    res.colors = std::max(res.colors, int(col) + 1);
  }
  return res;
}

// ---------------------------------------------------------------------------------------------
// Solver (ref/solver.ts:175-336) plus the GPU-mode step
// ---------------------------------------------------------------------------------------------
template <class T> struct Solver {
  T dt = T(1.0 / 60), gravity = -10, alpha = T(0.99), betaLin = 10000, betaAng = 100, gamma = T(0.999);
  int iterations = 10;
  // GPU-mode parameters (gpu/solver.ts:174-231; parity runs every flag off)
  uint32_t flags = 0;
  // the wind on sails (gpu/solver.ts:200-206, packed as f[32..36] at :1994-1998): velocity x, y, gust
  // fraction, pressure coefficient (0: no air, the CPU solver's world)
  T windX = 0, windY = 0, windGust = T(0.4), windPressure = 0;
  T contactMargin = T(COLLISION_MARGIN);
  bool gpuMode = false;
  std::vector<uint32_t> hulls;  // hull buffer (wgsl-hull.ts layout)
  std::vector<Body<T>> bodies;
  std::vector<std::unique_ptr<Force<T>>> forces;  // creation order
  // GPU mode: colour state, and the manifolds of the last step by pair (warm start)
  int lastColors = 0, lastClashes = 0, lastRounds = 0;
  uint32_t stepCounter = 0;  // GPU-mode steps taken (the device's step word: manifold generations, moved steps)

  void unlink(Force<T>* f) {
    for (int bi : {f->bodyA, f->bodyB}) {
      if (bi < 0) continue;
      auto& v = bodies[bi].forces;
      auto it = std::find(v.begin(), v.end(), f);
      if (it != v.end()) v.erase(it);
    }
  }
  Force<T>* addForce(std::unique_ptr<Force<T>> f) {
    Force<T>* p = f.get();
    if (p->bodyA >= 0) bodies[p->bodyA].forces.push_back(p);
    bodies[p->bodyB].forces.push_back(p);
    forces.push_back(std::move(f));
    return p;
  }
  bool constrainedTo(int a, int b) const {  // body.ts:56-61
    for (Force<T>* f : bodies[a].forces)
      if ((f->bodyA == a && f->bodyB == b) || (f->bodyA == b && f->bodyB == a)) return true;
    return false;
  }

  // Upstream step: solver.ts:249-335, in order.
  void step() {
    int n = int(bodies.size());
    for (int i = n - 1; i >= 0; i--) {
      for (int j = i - 1; j >= 0; j--) {
        V3<T> dp = sub3(bodies[i].pos, bodies[j].pos);
        T r = bodies[i].radius + bodies[j].radius;
        if (dot(dp, dp) <= r * r && !constrainedTo(i, j)) addForce(std::make_unique<Manifold<T>>(this, i, j));
      }
    }
    initializeForces();
    warmStartBodies(false);
    for (int it = 0; it < iterations; it++) {
      for (int b = n - 1; b >= 0; b--) primal(b, false, nullptr);
      for (auto& f : forces) f->updateDual(alpha);
    }
    velocities(false);
  }
  void initializeForces() {
    std::vector<std::unique_ptr<Force<T>>> kept;
    for (auto& f : forces) {
      if (f->initialize()) kept.push_back(std::move(f));
      else unlink(f.get());
    }
    forces = std::move(kept);
  }
  // The wind's acceleration of a sail (wgsl-solve.ts:262-292): pressure drag along the plate's normal,
  // linearised implicitly in its normal speed, and skin friction along it; gusts as travelling sines
  // in the wind's frame. t = step x dt; x, q, v: the step-start pose and the (damped) velocity.
  V3<T> windAccel(const Body<T>& b, T t) const {
    const V3<T> w{windX, windY, 0};
    const T speed = length(w);
    const V3<T> d = speed > T(1e-6) ? scale3(w, T(1) / speed) : V3<T>{1, 0, 0};
    const V3<T> side{-d[1], d[0], 0};
    const V3<T>& x = b.pos;
    const T a = dot(x, d), c = dot(x, side);
    const T along = T(0.5) * std::sin(T(1.1) * t - T(0.35) * a + T(0.2) * c) + T(0.3) * std::sin(T(2.9) * t - T(0.8) * a + T(0.6) * x[2]) +
                    T(0.2) * std::sin(T(6.1) * t - T(1.7) * a + T(1.3) * x[2] + T(0.9) * c);
    const T across = T(0.6) * std::sin(T(1.7) * t - T(0.6) * a + T(0.4) * x[2]) + T(0.4) * std::sin(T(4.3) * t - T(1.3) * a - T(0.7) * x[2]);
    const T lift = std::sin(T(2.3) * t - T(0.9) * a + T(1.1) * c);
    const T g = windGust;
    V3<T> u = scale3(w, T(1) + g * along);
    u = addScaled3(u, side, T(0.25) * across * g * speed);
    u[2] += T(0.1) * lift * g * speed;
    u = sub3(u, b.vel);
    const V3<T> n = rotate(b.rot, V3<T>{0, 0, 1});
    const T k = windPressure * b.size[0] * b.size[1] / b.mass;  // 1/2 rho C_d A / m
    const T un = dot(u, n);
    const V3<T> ut = addScaled3(u, n, -un);
    return addScaled3(scale3(n, k * un * std::fabs(un) / (T(1) + T(2) * dt * k * std::fabs(un))), ut, T(0.06) * k * length(ut));
  }
  void warmStartBodies(bool gpu) {  // solver.ts:273-295; GPU rules wgsl-solve.ts:294-335 (up = z)
    int n = int(bodies.size());
    for (int b = n - 1; b >= 0; b--) {
      Body<T>& body = bodies[b];
      bool dynamic = body.mass > 0;
      // GPU mode: the body's aux record (wgsl-solve.ts:9-20, 297-305) and lifecycle bits consumed
      const T g = gpu ? gravity * body.gravityScale : gravity;
      if (gpu) body.lifecycle = 0;
      if (gpu && dynamic && (body.linDamp > 0 || body.angDamp > 0)) {
        body.vel = scale3(body.vel, T(std::exp(-double(body.linDamp) * double(dt))));
        body.angVel = scale3(body.angVel, T(std::exp(-double(body.angDamp) * double(dt))));
      }
      body.inertialPos = addScaled3(body.pos, body.vel, dt);
      if (dynamic) body.inertialPos[2] += g * (dt * dt);
      if (gpu && dynamic && body.shape == SHAPE_SAIL && windPressure != 0)  // wgsl-solve.ts:310-311
        body.inertialPos = addScaled3(body.inertialPos, windAccel(body, T(stepCounter) * dt), dt * dt);
      body.inertialRot = qaddv(body.rot, scale3(body.angVel, dt));
      V3<T> accel = div3(sub3(body.vel, body.prevVel), dt);
      T accelExt = accel[2] * signv(g);
      T accelWeight = clampv(accelExt / std::fabs(g), T(0), T(1));
      if (!std::isfinite(accelWeight)) accelWeight = 0;
      bool atRest = false;
      if (gpu && (flags & FLAG_START_AT_REST)) atRest = length(body.vel) + length(body.angVel) * body.radius < T(REST_SPEED);
      body.initPos = body.pos;
      body.initRot = body.rot;
      if (dynamic && !atRest) {
        body.pos = addScaled3(body.pos, body.vel, dt);
        body.pos[2] += g * (accelWeight * dt * dt);
        body.rot = qaddv(body.rot, scale3(body.angVel, dt));
      }
      if (gpu && !dynamic && (body.vel != V3<T>{0, 0, 0} || body.angVel != V3<T>{0, 0, 0})) {
        body.pos = addScaled3(body.pos, body.vel, dt);
        body.rot = qaddv(body.rot, scale3(body.angVel, dt));
      }
    }
  }
  // One body's Newton step (solver.ts:300-321); `order` lists its forces in summation order (GPU
  // mode) or null (newest first).
  void primal(int b, bool gpu, const std::vector<Force<T>*>* order) {
    Body<T>& body = bodies[b];
    if (body.mass <= 0) return;
    BodySystem<T> sys;
    T m = body.mass;
    const V3<T>& I = body.moment;
    sys.lhsLin = diagonal(m / (dt * dt), m / (dt * dt), m / (dt * dt));
    sys.lhsAng = diagonal(I[0] / (dt * dt), I[1] / (dt * dt), I[2] / (dt * dt));
    sys.lhsCross = M3<T>{};
    sys.rhsLin = mulv(sys.lhsLin, sub3(body.pos, body.inertialPos));
    sys.rhsAng = mulv(sys.lhsAng, qsub(body.rot, body.inertialRot));
    if (order) for (Force<T>* f : *order) f->updatePrimal(b, alpha, sys);
    else for (int f = int(body.forces.size()) - 1; f >= 0; f--) body.forces[f]->updatePrimal(b, alpha, sys);
    V3<T> dxLin, dxAng;
    solve6(sys.lhsLin, sys.lhsAng, sys.lhsCross, neg3(sys.rhsLin), neg3(sys.rhsAng), dxLin, dxAng, gpu ? T(PIVOT_FLOOR) : T(0));
    body.pos = addScaled3(body.pos, dxLin, T(1));
    body.rot = qaddv(body.rot, dxAng);
  }
  void velocities(bool) {  // solver.ts:328-334
    for (auto& body : bodies) {
      body.prevVel = body.vel;
      if (body.mass > 0) {
        body.vel = div3(sub3(body.pos, body.initPos), dt);
        body.angVel = div3(qsub(body.rot, body.initRot), dt);
      }
    }
  }

  // --- GPU mode ---------------------------------------------------------------------------------
  static Body<float> toFloat(const Body<T>& b) {
    Body<float> f;
    for (int k = 0; k < 3; k++) { f.pos[k] = float(b.pos[k]); f.size[k] = float(b.size[k]); }
    for (int k = 0; k < 4; k++) f.rot[k] = float(b.rot[k]);
    f.mass = float(b.mass);
    f.radius = float(b.radius);
    f.friction = float(b.friction);
    f.shape = b.shape;
    return f;
  }
  std::vector<Rec32> records32() const {
    std::vector<Rec32> r(bodies.size());
    for (size_t i = 0; i < bodies.size(); i++) {
      const Body<T>& b = bodies[i];
      r[i].pos = {float(b.pos[0]), float(b.pos[1]), float(b.pos[2])};
      r[i].rot = {float(b.rot[0]), float(b.rot[1]), float(b.rot[2]), float(b.rot[3])};
      r[i].size = {float(b.size[0]), float(b.size[1]), float(b.size[2])};
      r[i].mass = float(b.mass);
      r[i].radius = float(b.radius);
      r[i].sphere = b.shape == SHAPE_SPHERE;
      r[i].groups = b.groups;
      r[i].mask = b.mask;
    }
    return r;
  }
  // ignored (wgsl-collision.ts:53-76): an IgnoreCollision, or a joint/spring that still acts
  bool ignoredPair(uint32_t a, uint32_t b) const {
    for (Force<T>* f : bodies[a].forces) {
      if (f->kind == K_MANIFOLD) continue;
      if (!((f->bodyA == int(a) && f->bodyB == int(b)) || (f->bodyA == int(b) && f->bodyB == int(a)))) continue;
      if (f->kind == K_JOINT && static_cast<Joint<T>*>(f)->broken) continue;
      return true;
    }
    return false;
  }
  std::vector<std::pair<uint32_t, uint32_t>> pairs() const {
    return gpuPairs(records32(), [&](uint32_t a, uint32_t b) { return ignoredPair(a, b); });
  }

  // GPU-mode step: pairs → fresh manifolds warm-started from last step's (same pair, same
  // feature) → JP colouring (or `fixedColors`) → warm starts → iterations sweeping colours →
  // velocities. Joints keep the creation order; each body sums its joints by slot, then its
  // contacts by (other body, first feature) (wgsl-topology.ts:116-153).
  // updateRefs (wgsl-collision.ts:28-43) in f32, in the device's operation order, so that both
  // decide alike: a body without a reference, or moved or turned past the tolerance since its
  // reference, takes its pose as the new reference and stamps the step.
  void updateRefs() {
    for (auto& b : bodies) {
      V3<float> p{float(b.pos[0]), float(b.pos[1]), float(b.pos[2])};
      Q4<float> q{float(b.rot[0]), float(b.rot[1]), float(b.rot[2]), float(b.rot[3])};
      const Q4<float>& r = b.refRot;
      bool moved = ((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]) + r[3] * r[3] == 0.0f || length(sub3(p, b.refPos)) > REUSE_LIN_TOL ||
                   length(qsub(q, r)) > REUSE_ANG_TOL;
      if (moved) {
        b.refPos = p;
        b.refRot = q;
        b.movedStep = stepCounter;
      }
    }
  }
  // A manifold's least normal penalty (wgsl-collision.ts contactPenaltyMin)
  T contactPenaltyMin(const Body<T>& A, const Body<T>& B) const {
    if (!(flags & FLAG_MASS_PENALTY)) return T(PENALTY_MIN);
    T mA = A.mass <= 0 ? T(3.4e38) : A.mass, mB = B.mass <= 0 ? T(3.4e38) : B.mass;
    return clampv(tmin(mA, mB) / (dt * dt), T(PENALTY_MIN), T(PENALTY_MAX));
  }
  // copyContacts (wgsl-collision.ts:721-753): last step's manifold of a pair kept, its points'
  // C(x-) evaluated at the current poses and their multipliers and penalties warm-started
  std::unique_ptr<Manifold<T>> copyContacts(int a, int b, const Manifold<T>& prev) {
    Body<T>& A = bodies[a];
    Body<T>& B = bodies[b];
    auto m = std::make_unique<Manifold<T>>(this, a, b);
    m->basis = prev.basis;
    m->friction = prev.friction;
    m->generated = prev.generated;
    const T penaltyMin = contactPenaltyMin(A, B);
    for (const Contact<T>& o : prev.contacts) {
      Contact<T> c = o;
      V3<T> d = sub3(add3(rotate(A.rot, c.rA), A.pos), add3(rotate(B.rot, c.rB), B.pos));
      c.C0 = V3<T>{dot(V3<T>{m->basis[0], m->basis[1], m->basis[2]}, d) + contactMargin, dot(V3<T>{m->basis[3], m->basis[4], m->basis[5]}, d),
                   dot(V3<T>{m->basis[6], m->basis[7], m->basis[8]}, d)};
      for (int k = 0; k < 3; k++) {
        c.lambda[k] = c.lambda[k] * alpha * gamma;
        c.penalty[k] = clampv(c.penalty[k] * gamma, T(PENALTY_MIN), T(PENALTY_MAX));
      }
      c.penalty[0] = tmax(c.penalty[0], penaltyMin);
      m->contacts.push_back(c);
    }
    return m;
  }

  // reuseManifolds: every manifold of last step is kept (copyContacts) and no pair is detected
  // (the substep option of GpuSolver3D.step, gpu/solver.ts:2121-2188).
  void stepGpu(const uint32_t* fixedColors, bool reuseManifolds = false) {
    gpuMode = true;
    stepCounter++;
    if (flags & FLAG_REUSE_CONTACTS) updateRefs();
    int n = int(bodies.size());
    // Last step's manifolds by pair
    std::map<std::pair<int, int>, std::vector<Contact<T>>> prev;
    std::map<std::pair<int, int>, std::unique_ptr<Force<T>>> prevMan;
    std::vector<std::unique_ptr<Force<T>>> keep;
    for (auto& f : forces) {
      if (f->kind == K_MANIFOLD) {
        auto* m = static_cast<Manifold<T>*>(f.get());
        prev[{m->bodyA, m->bodyB}] = m->contacts;
        unlink(m);
        prevMan[{m->bodyA, m->bodyB}] = std::move(f);
      } else keep.push_back(std::move(f));
    }
    forces = std::move(keep);
    // Joints warm start before the new manifolds (both read poses at x-)
    {
      std::vector<std::unique_ptr<Force<T>>> kept;
      for (auto& f : forces) {
        if (f->initialize()) kept.push_back(std::move(f));
        else unlink(f.get());
      }
      forces = std::move(kept);
    }
    std::vector<std::pair<uint32_t, uint32_t>> pr;
    if (reuseManifolds)
      for (auto& kv : prevMan) pr.push_back({uint32_t(kv.first.first), uint32_t(kv.first.second)});
    else
      pr = pairs();
    std::vector<std::unique_ptr<Manifold<T>>> made(pr.size());
#pragma omp parallel for schedule(dynamic, 64)
    for (long pi = 0; pi < long(pr.size()); pi++) {
      auto& p = pr[pi];
      int a = int(p.first), b = int(p.second);
      Body<T>& A = bodies[a];
      Body<T>& B = bodies[b];
      {
        // reuseContacts (wgsl-collision.ts:706-717): last step's points of a pair generated no
        // earlier than either body's last move; every manifold under reuseManifolds
        auto pm = prevMan.find({a, b});
        if (pm != prevMan.end()) {
          const auto& old = *static_cast<const Manifold<T>*>(pm->second.get());
          if (reuseManifolds || ((flags & FLAG_REUSE_CONTACTS) && !old.contacts.empty() && old.generated >= std::max(A.movedStep, B.movedStep))) {
            made[pi] = copyContacts(a, b, old);
            continue;
          }
        }
      }
      // The GPU's own arithmetic (f32) finds the contacts, so both sides solve one contact set
      Body<float> fA = toFloat(A), fB = toFloat(B);
      V3<float> nf;
      Found<float> ff = narrowphase(fA, fB, (flags & FLAG_FACE_BIAS) != 0, nf, hulls.empty() ? nullptr : hulls.data());
      if (ff.count == 0) continue;
      V3<T> normal{T(nf[0]), T(nf[1]), T(nf[2])};
      auto m = std::make_unique<Manifold<T>>(this, a, b);
      m->friction = std::sqrt(A.friction * B.friction);
      m->basis = orthonormal(normal);
      m->generated = stepCounter;
      auto it = prev.find({a, b});
      const std::vector<Contact<T>>* old = it == prev.end() ? nullptr : &it->second;
      bool anySphere = A.shape == SHAPE_SPHERE || B.shape == SHAPE_SPHERE;
      T minSide = tmin(tmin(tmin(A.size[0], A.size[1]), A.size[2]) * T(0.5), tmin(tmin(B.size[0], B.size[1]), B.size[2]) * T(0.5)) * 2;
      T penaltyMin = T(PENALTY_MIN);
      if (flags & FLAG_MASS_PENALTY) {
        T mA = A.mass <= 0 ? T(3.4e38) : A.mass, mB = B.mass <= 0 ? T(3.4e38) : B.mass;
        penaltyMin = clampv(tmin(mA, mB) / (dt * dt), T(PENALTY_MIN), T(PENALTY_MAX));
      }
      for (int i = 0; i < ff.count; i++) {
        Contact<T> c;
        c.feature = ff.feature[i];
        V3<float> ra = rotate(conjugate(fA.rot), sub3(ff.xA[i], fA.pos)), rb = rotate(conjugate(fB.rot), sub3(ff.xB[i], fB.pos));
        c.rA = V3<T>{T(ra[0]), T(ra[1]), T(ra[2])};
        c.rB = V3<T>{T(rb[0]), T(rb[1]), T(rb[2])};
        const Contact<T>* pc = nullptr;
        if (old) {
          for (auto& o : *old) if (o.feature == c.feature) { pc = &o; break; }
          if (!pc && (flags & FLAG_MATCH_NEAREST)) {
            T bestDist = T(NEAREST_FRACTION) * minSide;
            for (auto& o : *old) {
              T dist = length(sub3(o.rA, c.rA));
              if (dist <= bestDist) { bestDist = dist; pc = &o; }
            }
          }
        }
        if (pc) {
          c.penalty = pc->penalty;
          c.lambda = pc->lambda;
          c.stick = pc->stick;
          if (c.stick && !anySphere) { c.rA = pc->rA; c.rB = pc->rB; }
        }
        V3<T> d = sub3(add3(rotate(A.rot, c.rA), A.pos), add3(rotate(B.rot, c.rB), B.pos));
        c.C0 = V3<T>{dot(V3<T>{m->basis[0], m->basis[1], m->basis[2]}, d) + contactMargin,
                     dot(V3<T>{m->basis[3], m->basis[4], m->basis[5]}, d), dot(V3<T>{m->basis[6], m->basis[7], m->basis[8]}, d)};
        for (int k = 0; k < 3; k++) {
          c.lambda[k] = c.lambda[k] * alpha * gamma;
          c.penalty[k] = clampv(c.penalty[k] * gamma, T(PENALTY_MIN), T(PENALTY_MAX));
        }
        c.penalty[0] = tmax(c.penalty[0], penaltyMin);
        m->contacts.push_back(c);
      }
      made[pi] = std::move(m);
    }
    for (auto& m : made)
      if (m) addForce(std::move(m));
    // Per-body summation order
    std::vector<std::vector<Force<T>*>> order(n);
    for (auto& up : forces) {
      Force<T>* f = up.get();
      if (f->kind == K_IGNORE) continue;
      for (int e : {f->bodyA, f->bodyB}) if (e >= 0 && bodies[e].mass > 0) order[e].push_back(f);
    }
    std::vector<int> slot(forces.size());
    {
      std::unordered_map<Force<T>*, int> idx;
      int s = 0;
      for (auto& up : forces) idx[up.get()] = s++;
#pragma omp parallel for schedule(dynamic, 256)
      for (int b = 0; b < n; b++) {
        std::stable_sort(order[b].begin(), order[b].end(), [&](Force<T>* x, Force<T>* y) {
          auto key = [&](Force<T>* f) -> std::pair<uint64_t, uint64_t> {
            if (f->kind != K_MANIFOLD) return {0, uint64_t(idx.at(f))};
            int other = f->bodyA == b ? f->bodyB : f->bodyA;
            auto* m = static_cast<Manifold<T>*>(f);
            return {uint64_t(other + 2), uint64_t(m->contacts.empty() ? 0 : m->contacts[0].feature & ~STICK_BIT)};
          };
          return key(x) < key(y);
        });
      }
    }
    // Colouring
    std::vector<char> dynamic(n);
    for (int b = 0; b < n; b++) dynamic[b] = bodies[b].mass > 0;
    std::vector<uint32_t> state(n);
    if (fixedColors) {
      for (int b = 0; b < n; b++) state[b] = dynamic[b] ? fixedColors[b] : NO_COLOR;
      lastColors = 0;
      for (int b = 0; b < n; b++) if (dynamic[b]) lastColors = std::max(lastColors, int(state[b] & 0xff) + 1);
      lastClashes = 0;
      lastRounds = 0;
    } else {
      std::vector<int> start(n + 1, 0), nbr;
      for (int b = 0; b < n; b++) {
        start[b] = int(nbr.size());
        if (dynamic[b])
          for (Force<T>* f : order[b]) {
            int o = f->bodyA == b ? f->bodyB : f->bodyA;
            if (o >= 0 && dynamic[o]) nbr.push_back(o);
          }
      }
      start[n] = int(nbr.size());
      for (int b = 0; b < n; b++) state[b] = bodies[b].color;
      ColorResult r = jpColor(n, dynamic, start, nbr, state, MAX_COLORS, 32);
      lastColors = r.colors;
      lastClashes = r.clashes;
      lastRounds = r.rounds;
    }
    for (int b = 0; b < n; b++) bodies[b].color = state[b];
    int ncol = 0;
    for (int b = 0; b < n; b++) if (dynamic[b]) ncol = std::max(ncol, int(state[b] & 0xff) + 1);
    std::vector<std::vector<int>> buckets(ncol);
    for (int b = 0; b < n; b++) if (dynamic[b]) buckets[state[b] & 0xff].push_back(b);

    warmStartBodies(true);
    for (int it = 0; it < iterations; it++) {
      for (int c = 0; c < ncol; c++) {
        const std::vector<int>& bucket = buckets[c];
#pragma omp parallel for schedule(dynamic, 64)
        for (long k = 0; k < long(bucket.size()); k++) primal(bucket[k], true, &order[bucket[k]]);
      }
#pragma omp parallel for schedule(dynamic, 256)
      for (long f = 0; f < long(forces.size()); f++) forces[f]->updateDual(alpha);
    }
    velocities(true);
  }
};

}  // namespace orc

// ---------------------------------------------------------------------------------------------
// FP64 adjoint of the GPU-mode step with the contact structure frozen (test infrastructure).
// A forward rollout of the oracle records, per step, its contact structure: the pairs, each pair's
// normal (its basis), each point's body-frame anchors and the last-step point it warm-starts from,
// and the colouring. The replay steps that structure again from any parameters (initial linear and
// angular velocities, masses with moments in proportion, friction coefficients): C(x-) from the
// poses, warm starts, the coloured primal sweeps, the duals (penalty ramps, friction cone) and the
// velocities, as stepGpu does. Its gradient comes from the AD tape, one step at a time, from the
// step-start states the replay keeps. Only boxes on static bodies and on each other (no joints).
// ---------------------------------------------------------------------------------------------
namespace orc {
struct AdjPoint { double rA[3], rB[3]; int man, prev; };
struct AdjMan { int a, b; double basis[9]; };
struct AdjStep { std::vector<AdjMan> mans; std::vector<AdjPoint> pts; std::vector<int> color; int ncol = 0; };
struct AdjProblem {
  int n = 0;
  std::vector<char> dynamic;
  std::vector<double> pos, rot, prevVel, unitMoment, friction, mass, vel, angVel;  // initial state and nominal params
  double dt, gravity, alpha, gamma, betaLin, margin;
  int iterations;
  std::vector<AdjStep> steps;
  std::vector<double> target;  // 7 per body
};
template <class S> struct AdjState {
  std::vector<V3<S>> pos, vel, angVel, initPos;
  std::vector<Q4<S>> rot, initRot, inRot;
  std::vector<V3<S>> inPos;
  std::vector<S> prevVz;
  std::vector<V3<S>> lam, pen;  // per point of the last step replayed
};

// One replayed step (stepGpu with the recorded structure; manifold.ts / wgsl-solve.ts maths)
template <class S>
void adjStep(const AdjProblem& P, const AdjStep& st, AdjState<S>& X, const std::vector<S>& mass, const std::vector<S>& mu) {
  const int n = P.n;
  const S dt(P.dt), g(P.gravity), alpha(P.alpha), gamma(P.gamma), beta(P.betaLin);
  const size_t np = st.pts.size();
  std::vector<V3<S>> lam(np), pen(np), C0(np);
  std::vector<S> fr(st.mans.size());
  for (size_t m = 0; m < st.mans.size(); m++) fr[m] = std::sqrt(mu[st.mans[m].a] * mu[st.mans[m].b]);
  // points: warm starts from the recorded last-step point, C(x-) at the step-start poses
  for (size_t k = 0; k < np; k++) {
    const AdjPoint& q = st.pts[k];
    const AdjMan& m = st.mans[q.man];
    V3<S> l{S(0), S(0), S(0)}, pe{S(0), S(0), S(0)};
    if (q.prev >= 0) { l = X.lam[q.prev]; pe = X.pen[q.prev]; }
    for (int c = 0; c < 3; c++) {
      lam[k][c] = l[c] * alpha * gamma;
      pen[k][c] = clampv(pe[c] * gamma, S(PENALTY_MIN), S(PENALTY_MAX));
    }
    V3<S> rA{S(q.rA[0]), S(q.rA[1]), S(q.rA[2])}, rB{S(q.rB[0]), S(q.rB[1]), S(q.rB[2])};
    V3<S> d = sub3(add3(rotate(X.rot[m.a], rA), X.pos[m.a]), add3(rotate(X.rot[m.b], rB), X.pos[m.b]));
    for (int c = 0; c < 3; c++) C0[k][c] = S(m.basis[3 * c]) * d[0] + S(m.basis[3 * c + 1]) * d[1] + S(m.basis[3 * c + 2]) * d[2];
    C0[k][0] = C0[k][0] + S(P.margin);
  }
  // warm start bodies (solver.ts:273-295, up = z)
  for (int b = 0; b < n; b++) {
    X.initPos[b] = X.pos[b];
    X.initRot[b] = X.rot[b];
    if (!P.dynamic[b]) continue;
    X.inPos[b] = addScaled3(X.pos[b], X.vel[b], dt);
    X.inPos[b][2] = X.inPos[b][2] + g * (dt * dt);
    X.inRot[b] = qaddv(X.rot[b], scale3(X.angVel[b], dt));
    S accelExt = (X.vel[b][2] - X.prevVz[b]) / dt * S(signv(P.gravity));
    S wgt = clampv(accelExt / S(std::fabs(P.gravity)), S(0), S(1));
    X.pos[b] = addScaled3(X.pos[b], X.vel[b], dt);
    X.pos[b][2] = X.pos[b][2] + g * (wgt * dt * dt);
    X.rot[b] = qaddv(X.rot[b], scale3(X.angVel[b], dt));
  }
  std::vector<std::vector<int>> touch(n);
  for (size_t k = 0; k < np; k++) {
    const AdjMan& m = st.mans[st.pts[k].man];
    touch[m.a].push_back(int(k));
    touch[m.b].push_back(int(k));
  }
  // C, F of point k at the current poses (manifold.ts:139-168)
  auto evalPoint = [&](size_t k, V3<S>& C, V3<S>& F, S& fs, S& bd, V3<S>& rAW, V3<S>& rBW) {
    const AdjPoint& q = st.pts[k];
    const AdjMan& m = st.mans[q.man];
    V3<S> rA{S(q.rA[0]), S(q.rA[1]), S(q.rA[2])}, rB{S(q.rB[0]), S(q.rB[1]), S(q.rB[2])};
    rAW = rotate(X.rot[m.a], rA);
    rBW = rotate(X.rot[m.b], rB);
    V3<S> dAL = sub3(X.pos[m.a], X.initPos[m.a]), dAA = qsub(X.rot[m.a], X.initRot[m.a]);
    V3<S> dBL = sub3(X.pos[m.b], X.initPos[m.b]), dBA = qsub(X.rot[m.b], X.initRot[m.b]);
    for (int c = 0; c < 3; c++) {
      V3<S> bk{S(m.basis[3 * c]), S(m.basis[3 * c + 1]), S(m.basis[3 * c + 2])};
      S v = C0[k][c] * (S(1) - alpha);
      v = v + dot(bk, dAL) - dot(bk, dBL) + dot(cross(rAW, bk), dAA) + dot(cross(rBW, neg3(bk)), dBA);
      C[c] = v;
      F[c] = pen[k][c] * v + lam[k][c];
    }
    F[0] = tmin(F[0], S(0));
    bd = std::fabs(F[0]) * fr[q.man];
    fs = std::sqrt(F[1] * F[1] + F[2] * F[2]);
    if (fs > bd && fs > S(0)) {
      F[1] = F[1] * (bd / fs);
      F[2] = F[2] * (bd / fs);
    }
  };
  std::vector<std::vector<int>> buckets(st.ncol);
  for (int b = 0; b < n; b++)
    if (P.dynamic[b] && st.color[b] >= 0 && st.color[b] < st.ncol) buckets[st.color[b]].push_back(b);
  for (int it = 0; it < P.iterations; it++) {
    for (int c = 0; c < st.ncol; c++) {
      for (int b : buckets[c]) {
        S mdt = mass[b] / (dt * dt);
        V3<S> I{mass[b] * S(P.unitMoment[3 * b]) / (dt * dt), mass[b] * S(P.unitMoment[3 * b + 1]) / (dt * dt), mass[b] * S(P.unitMoment[3 * b + 2]) / (dt * dt)};
        M3<S> hL = diagonal(mdt, mdt, mdt), hA = diagonal(I[0], I[1], I[2]), hC{};
        for (auto& e : hC) e = S(0);
        V3<S> gL = scale3(sub3(X.pos[b], X.inPos[b]), mdt);
        V3<S> qd = qsub(X.rot[b], X.inRot[b]);
        V3<S> gA{I[0] * qd[0], I[1] * qd[1], I[2] * qd[2]};
        for (int k : touch[b]) {
          const AdjMan& m = st.mans[st.pts[k].man];
          V3<S> C, F, rAW, rBW;
          S fs, bd;
          evalPoint(size_t(k), C, F, fs, bd, rAW, rBW);
          bool isA = b == m.a;
          S sg = isA ? S(1) : S(-1);
          V3<S> r = isA ? rAW : rBW;
          for (int cc = 0; cc < 3; cc++) {
            V3<S> l{S(m.basis[3 * cc]) * sg, S(m.basis[3 * cc + 1]) * sg, S(m.basis[3 * cc + 2]) * sg};
            V3<S> a = cross(r, l);
            S kk = pen[k][cc];
            for (int i = 0; i < 3; i++)
              for (int j = 0; j < 3; j++) {
                hL[3 * i + j] = hL[3 * i + j] + kk * l[i] * l[j];
                hA[3 * i + j] = hA[3 * i + j] + kk * a[i] * a[j];
                hC[3 * i + j] = hC[3 * i + j] + kk * a[i] * l[j];
              }
            gL = addScaled3(gL, l, F[cc]);
            gA = addScaled3(gA, a, F[cc]);
          }
        }
        V3<S> dxL, dxA;
        solve6(hL, hA, hC, neg3(gL), neg3(gA), dxL, dxA, S(PIVOT_FLOOR));
        X.pos[b] = add3(X.pos[b], dxL);
        X.rot[b] = qaddv(X.rot[b], dxA);
      }
    }
    for (size_t k = 0; k < np; k++) {  // duals (manifold.ts:202-217)
      V3<S> C, F, rAW, rBW;
      S fs, bd;
      evalPoint(k, C, F, fs, bd, rAW, rBW);
      lam[k] = F;
      if (F[0] < S(0)) pen[k][0] = tmin(pen[k][0] + beta * std::fabs(C[0]), S(PENALTY_MAX));
      if (fs <= bd) {
        pen[k][1] = tmin(pen[k][1] + beta * std::fabs(C[1]), S(PENALTY_MAX));
        pen[k][2] = tmin(pen[k][2] + beta * std::fabs(C[2]), S(PENALTY_MAX));
      }
    }
  }
  for (int b = 0; b < n; b++) {  // velocities (solver.ts:328-334)
    X.prevVz[b] = X.vel[b][2];
    if (!P.dynamic[b]) continue;
    X.vel[b] = div3(sub3(X.pos[b], X.initPos[b]), dt);
    X.angVel[b] = div3(qsub(X.rot[b], X.initRot[b]), dt);
  }
  X.lam = lam;
  X.pen = pen;
}

template <class S> void adjInit(const AdjProblem& P, const double* params, AdjState<S>& X, std::vector<S>& mass, std::vector<S>& mu, bool inputs) {
  const int n = P.n;
  auto in = [&](double v) { return inputs ? S(v) : S(v); };
  X.pos.resize(n); X.vel.resize(n); X.angVel.resize(n); X.initPos.resize(n); X.inPos.resize(n);
  X.rot.resize(n); X.initRot.resize(n); X.inRot.resize(n); X.prevVz.resize(n);
  mass.resize(n); mu.resize(n);
  for (int b = 0; b < n; b++) {
    for (int k = 0; k < 3; k++) X.pos[b][k] = S(P.pos[3 * b + k]);
    for (int k = 0; k < 4; k++) X.rot[b][k] = S(P.rot[4 * b + k]);
    const double* q = params + 8 * b;
    for (int k = 0; k < 3; k++) { X.vel[b][k] = in(q[k]); X.angVel[b][k] = in(q[3 + k]); }
    mass[b] = in(q[6]);
    mu[b] = in(q[7]);
    X.prevVz[b] = S(P.prevVel[3 * b + 2]);
  }
  X.lam.clear();
  X.pen.clear();
}

template <class S> S adjLoss(const AdjProblem& P, const AdjState<S>& X) {
  S L(0);
  for (int b = 0; b < P.n; b++) {
    if (!P.dynamic[b]) continue;
    for (int k = 0; k < 3; k++) { S d = X.pos[b][k] - S(P.target[7 * b + k]); L = L + d * d; }
    for (int k = 0; k < 4; k++) { S d = X.rot[b][k] - S(P.target[7 * b + 3 + k]); L = L + d * d; }
  }
  return L;
}

// The gradient of the loss with respect to params (8 per body): forward replay keeping every step's
// start state, then per step (last first) the step taped from its start state and swept backwards.
inline double adjGradient(const AdjProblem& P, const double* params, double* grad) {
  const int n = P.n, K = int(P.steps.size());
  AdjState<double> X;
  std::vector<double> mass, mu;
  adjInit(P, params, X, mass, mu, false);
  std::vector<AdjState<double>> starts;
  starts.reserve(K);
  for (int k = 0; k < K; k++) {
    starts.push_back(X);
    adjStep(P, P.steps[k], X, mass, mu);
  }
  double loss = adjLoss(P, X);
  // cotangents of the state after step k (bodies; this step's points)
  std::vector<V3<double>> gPos(n), gVel(n), gAng(n), gLam, gPen;
  std::vector<Q4<double>> gRot(n);
  std::vector<double> gPrevVz(n, 0.0);
  for (int b = 0; b < n; b++) {
    gPos[b] = {0, 0, 0}; gVel[b] = {0, 0, 0}; gAng[b] = {0, 0, 0}; gRot[b] = {0, 0, 0, 0};
    if (!P.dynamic[b]) continue;
    for (int c = 0; c < 3; c++) gPos[b][c] = 2 * (X.pos[b][c] - P.target[7 * b + c]);
    for (int c = 0; c < 4; c++) gRot[b][c] = 2 * (X.rot[b][c] - P.target[7 * b + 3 + c]);
  }
  gLam.assign(X.lam.size(), V3<double>{0, 0, 0});
  gPen.assign(X.pen.size(), V3<double>{0, 0, 0});
  std::vector<double> gMass(n, 0.0), gMu(n, 0.0);
  auto& tape = adTape();
  for (int k = K - 1; k >= 0; k--) {
    tape.clear();
    const AdjState<double>& S0 = starts[k];
    AdjState<AD> A;
    auto V = [](const V3<double>& v) { return V3<AD>{AD::input(v[0]), AD::input(v[1]), AD::input(v[2])}; };
    auto Q = [](const Q4<double>& q) { return Q4<AD>{AD::input(q[0]), AD::input(q[1]), AD::input(q[2]), AD::input(q[3])}; };
    A.pos.resize(n); A.vel.resize(n); A.angVel.resize(n); A.rot.resize(n); A.prevVz.resize(n);
    A.initPos.resize(n); A.initRot.resize(n); A.inPos.resize(n); A.inRot.resize(n);
    for (int b = 0; b < n; b++) {
      A.pos[b] = V(S0.pos[b]); A.vel[b] = V(S0.vel[b]); A.angVel[b] = V(S0.angVel[b]); A.rot[b] = Q(S0.rot[b]);
      A.prevVz[b] = AD::input(S0.prevVz[b]);
    }
    for (auto& l : S0.lam) A.lam.push_back(V(l));
    for (auto& p : S0.pen) A.pen.push_back(V(p));
    std::vector<AD> am(n), au(n);
    for (int b = 0; b < n; b++) { am[b] = AD::input(mass[b]); au[b] = AD::input(mu[b]); }
    // input node ids, before the step replaces them
    AdjState<AD> In = A;
    adjStep(P, P.steps[k], A, am, au);
    std::vector<double> adj(tape.size(), 0.0);
    auto seedV = [&](const V3<AD>& v, const V3<double>& g) { for (int c = 0; c < 3; c++) if (v[c].i >= 0) adj[v[c].i] += g[c]; };
    auto seedQ = [&](const Q4<AD>& v, const Q4<double>& g) { for (int c = 0; c < 4; c++) if (v[c].i >= 0) adj[v[c].i] += g[c]; };
    for (int b = 0; b < n; b++) {
      seedV(A.pos[b], gPos[b]); seedQ(A.rot[b], gRot[b]); seedV(A.vel[b], gVel[b]); seedV(A.angVel[b], gAng[b]);
      if (A.prevVz[b].i >= 0) adj[A.prevVz[b].i] += gPrevVz[b];
    }
    for (size_t p = 0; p < A.lam.size(); p++) { seedV(A.lam[p], gLam[p]); seedV(A.pen[p], gPen[p]); }
    for (int i = int(tape.size()) - 1; i >= 0; i--) {
      const ADNode& nd = tape[i];
      if (adj[i] == 0.0) continue;
      if (nd.a >= 0) adj[nd.a] += nd.da * adj[i];
      if (nd.b >= 0) adj[nd.b] += nd.db * adj[i];
    }
    auto getV = [&](const V3<AD>& v) { return V3<double>{v[0].i >= 0 ? adj[v[0].i] : 0, v[1].i >= 0 ? adj[v[1].i] : 0, v[2].i >= 0 ? adj[v[2].i] : 0}; };
    auto getQ = [&](const Q4<AD>& v) { Q4<double> o; for (int c = 0; c < 4; c++) o[c] = v[c].i >= 0 ? adj[v[c].i] : 0; return o; };
    for (int b = 0; b < n; b++) {
      gPos[b] = getV(In.pos[b]); gVel[b] = getV(In.vel[b]); gAng[b] = getV(In.angVel[b]); gRot[b] = getQ(In.rot[b]);
      gPrevVz[b] = In.prevVz[b].i >= 0 ? adj[In.prevVz[b].i] : 0;
      gMass[b] += am[b].i >= 0 ? adj[am[b].i] : 0;
      gMu[b] += au[b].i >= 0 ? adj[au[b].i] : 0;
    }
    gLam.resize(In.lam.size());
    gPen.resize(In.pen.size());
    for (size_t p = 0; p < In.lam.size(); p++) { gLam[p] = getV(In.lam[p]); gPen[p] = getV(In.pen[p]); }
  }
  tape.clear();
  tape.shrink_to_fit();
  for (int b = 0; b < n; b++) {
    double* o = grad + 8 * b;
    for (int c = 0; c < 3; c++) { o[c] = gVel[b][c]; o[3 + c] = gAng[b][c]; }
    o[6] = gMass[b];
    o[7] = gMu[b];
  }
  return loss;
}
}  // namespace orc

// ---------------------------------------------------------------------------------------------
// C interface for ctypes (tests, smoke, bench cpu_baseline)
// ---------------------------------------------------------------------------------------------
using namespace orc;

struct OrcHandle {
  int fp32;
  std::unique_ptr<Solver<double>> d;
  std::unique_ptr<Solver<float>> f;
};

template <class F> static auto with(void* h, F fn) {
  OrcHandle* o = static_cast<OrcHandle*>(h);
  if (o->fp32) return fn(*o->f);
  return fn(*o->d);
}

// Body record for orc_add_body / orc_get_body (doubles):
//  0 pos3 | 3 rot4 | 7 vel3 | 10 angVel3 | 13 prevVel3 | 16 size3 | 19 mass | 20 moment3 |
//  23 friction | 24 radius | 25 shape | 26 initPos3 | 29 initRot4 | 33 inertialPos3 |
//  36 inertialRot4 | 40 groups | 41 mask | 42 colour state
static const int BODY_REC = 43;
template <class T> static void putBody(Body<T>& b, const double* r) {
  for (int k = 0; k < 3; k++) { b.pos[k] = T(r[k]); b.vel[k] = T(r[7 + k]); b.angVel[k] = T(r[10 + k]); b.prevVel[k] = T(r[13 + k]); b.size[k] = T(r[16 + k]); b.moment[k] = T(r[20 + k]); b.initPos[k] = T(r[26 + k]); b.inertialPos[k] = T(r[33 + k]); }
  for (int k = 0; k < 4; k++) { b.rot[k] = T(r[3 + k]); b.initRot[k] = T(r[29 + k]); b.inertialRot[k] = T(r[36 + k]); }
  b.mass = T(r[19]); b.friction = T(r[23]); b.radius = T(r[24]); b.shape = int(r[25]);
  b.groups = uint32_t(r[40]); b.mask = uint32_t(r[41]); b.color = uint32_t(r[42]);
}
template <class T> static void getBody(const Body<T>& b, double* r) {
  for (int k = 0; k < 3; k++) { r[k] = b.pos[k]; r[7 + k] = b.vel[k]; r[10 + k] = b.angVel[k]; r[13 + k] = b.prevVel[k]; r[16 + k] = b.size[k]; r[20 + k] = b.moment[k]; r[26 + k] = b.initPos[k]; r[33 + k] = b.inertialPos[k]; }
  for (int k = 0; k < 4; k++) { r[3 + k] = b.rot[k]; r[29 + k] = b.initRot[k]; r[36 + k] = b.inertialRot[k]; }
  r[19] = b.mass; r[23] = b.friction; r[24] = b.radius; r[25] = b.shape; r[40] = b.groups; r[41] = b.mask; r[42] = b.color;
}

// Joint record (orc_get_force / orc_set_joint), doubles:
//  0 kind | 1 a | 2 b | 3 penLin3 | 6 penAng3 | 9 lamLin3 | 12 lamAng3 | 15 C0Lin3 | 18 C0Ang3 |
//  21 stiffLin | 22 stiffAng | 23 fracture | 24 fractureLinear | 25 torqueArm | 26 broken |
//  27 yield | 28 breakBend | 29 rest4 | 33 hasRest | 34 restStart4 | 38 hasRestStart | 39 rA3 |
//  42 rB3 | 45 springStiffness | 46 springRest
static const int FORCE_REC = 47;

extern "C" {

int orc_body_record_size() { return BODY_REC; }
int orc_force_record_size() { return FORCE_REC; }

void* orc_create(int fp32) {
  auto* h = new OrcHandle();
  h->fp32 = fp32;
  if (fp32) h->f = std::make_unique<Solver<float>>();
  else h->d = std::make_unique<Solver<double>>();
  return h;
}
void orc_destroy(void* h) { delete static_cast<OrcHandle*>(h); }

// params: dt, gravity, iterations, alpha, betaLin, betaAng, gamma, contactMargin
void orc_set_params(void* h, const double* p, unsigned flags) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    s.dt = T(p[0]); s.gravity = T(p[1]); s.iterations = int(p[2]); s.alpha = T(p[3]);
    s.betaLin = T(p[4]); s.betaAng = T(p[5]); s.gamma = T(p[6]); s.contactMargin = T(p[7]);
    s.flags = flags;
    return 0;
  });
}

// the wind on sails: velocity x, y (m/s), gust fraction, pressure coefficient 1/2 rho C_d
void orc_set_wind(void* h, const double* w) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    s.windX = T(w[0]); s.windY = T(w[1]); s.windGust = T(w[2]); s.windPressure = T(w[3]);
    return 0;
  });
}

int orc_add_body(void* h, const double* rec) {
  return with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    Body<T> b;
    putBody(b, rec);
    s.bodies.push_back(b);
    return int(s.bodies.size()) - 1;
  });
}
int orc_body_count(void* h) { return with(h, [&](auto& s) { return int(s.bodies.size()); }); }
void orc_get_body(void* h, int i, double* rec) { with(h, [&](auto& s) { getBody(s.bodies[i], rec); return 0; }); }
// Overwrites state, keeps the body's force list
void orc_set_body(void* h, int i, const double* rec) {
  with(h, [&](auto& s) {
    auto forces = s.bodies[i].forces;
    putBody(s.bodies[i], rec);
    s.bodies[i].forces = forces;
    return 0;
  });
}

// Returns the force index (creation order)
int orc_add_joint(void* h, int a, int b, const double* rA, const double* rB, double stiffLin, double stiffAng, double fracture) {
  return with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    s.addForce(std::make_unique<Joint<T>>(&s, a, b, V3<T>{T(rA[0]), T(rA[1]), T(rA[2])}, V3<T>{T(rB[0]), T(rB[1]), T(rB[2])}, T(stiffLin), T(stiffAng), T(fracture)));
    return int(s.forces.size()) - 1;
  });
}
int orc_add_spring(void* h, int a, int b, const double* rA, const double* rB, double stiffness, double rest) {
  return with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    s.addForce(std::make_unique<Spring<T>>(&s, a, b, V3<T>{T(rA[0]), T(rA[1]), T(rA[2])}, V3<T>{T(rB[0]), T(rB[1]), T(rB[2])}, T(stiffness), T(rest)));
    return int(s.forces.size()) - 1;
  });
}
int orc_add_ignore(void* h, int a, int b) {
  return with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    s.addForce(std::make_unique<Ignore<T>>(&s, a, b));
    return int(s.forces.size()) - 1;
  });
}
int orc_force_count(void* h) { return with(h, [&](auto& s) { return int(s.forces.size()); }); }

void orc_get_force(void* h, int i, double* r) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    for (int k = 0; k < FORCE_REC; k++) r[k] = 0;
    Force<T>* f = s.forces[i].get();
    r[0] = f->kind; r[1] = f->bodyA; r[2] = f->bodyB;
    if (f->kind == K_JOINT) {
      auto* j = static_cast<Joint<T>*>(f);
      for (int k = 0; k < 3; k++) {
        r[3 + k] = j->penaltyLin[k]; r[6 + k] = j->penaltyAng[k]; r[9 + k] = j->lambdaLin[k]; r[12 + k] = j->lambdaAng[k];
        r[15 + k] = j->C0Lin[k]; r[18 + k] = j->C0Ang[k]; r[39 + k] = j->rA[k]; r[42 + k] = j->rB[k];
      }
      r[21] = j->stiffnessLin; r[22] = j->stiffnessAng; r[23] = j->fracture; r[24] = j->fractureLinear; r[25] = j->torqueArm;
      r[26] = j->broken; r[27] = j->yield; r[28] = j->breakBend;
      for (int k = 0; k < 4; k++) { r[29 + k] = j->rest[k]; r[34 + k] = j->restStart[k]; }
      r[33] = j->hasRest; r[38] = j->hasRestStart;
    } else if (f->kind == K_SPRING) {
      auto* sp = static_cast<Spring<T>*>(f);
      for (int k = 0; k < 3; k++) { r[39 + k] = sp->rA[k]; r[42 + k] = sp->rB[k]; }
      r[45] = sp->stiffness; r[46] = sp->rest;
    }
    return 0;
  });
}
// Sets a joint's mutable state and options from a record (kind/a/b/rA/rB/torqueArm ignored)
void orc_set_joint(void* h, int i, const double* r) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    auto* j = static_cast<Joint<T>*>(s.forces[i].get());
    for (int k = 0; k < 3; k++) {
      j->penaltyLin[k] = T(r[3 + k]); j->penaltyAng[k] = T(r[6 + k]); j->lambdaLin[k] = T(r[9 + k]); j->lambdaAng[k] = T(r[12 + k]);
      j->C0Lin[k] = T(r[15 + k]); j->C0Ang[k] = T(r[18 + k]);
    }
    j->stiffnessLin = T(r[21]); j->stiffnessAng = T(r[22]); j->fracture = T(r[23]); j->fractureLinear = r[24] != 0;
    j->broken = r[26] != 0; j->yield = T(r[27]); j->breakBend = T(r[28]);
    for (int k = 0; k < 4; k++) { j->rest[k] = T(r[29 + k]); j->restStart[k] = T(r[34 + k]); }
    j->hasRest = r[33] != 0; j->hasRestStart = r[38] != 0;
    return 0;
  });
}

// setWorldAnchor (gpu/solver.ts:1937-1939): joint i's rA (the world point of a joint with no body A)
void orc_set_joint_anchor(void* h, int i, const double* p) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    auto* j = static_cast<Joint<T>*>(s.forces[i].get());
    for (int k = 0; k < 3; k++) j->rA[k] = T(p[k]);
    return 0;
  });
}

// Manifolds in force order. Manifold record (8 doubles): force index, a, b, count, normal3,
// friction. Contact record (17): feature, stick, rA3, rB3, C0 3, pen3, lam3.
int orc_manifold_count(void* h) {
  return with(h, [&](auto& s) { int n = 0; for (auto& f : s.forces) n += f->kind == K_MANIFOLD; return n; });
}
int orc_contact_count(void* h) {
  return with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    int n = 0;
    for (auto& f : s.forces) if (f->kind == K_MANIFOLD) n += int(static_cast<Manifold<T>*>(f.get())->contacts.size());
    return n;
  });
}
void orc_get_manifolds(void* h, double* mrec, double* crec) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    int mi = 0, ci = 0, fi = 0;
    for (auto& f : s.forces) {
      if (f->kind == K_MANIFOLD) {
        auto* m = static_cast<Manifold<T>*>(f.get());
        double* r = mrec + 8 * mi++;
        r[0] = fi; r[1] = m->bodyA; r[2] = m->bodyB; r[3] = double(m->contacts.size());
        r[4] = m->basis[0]; r[5] = m->basis[1]; r[6] = m->basis[2]; r[7] = m->friction;
        for (auto& c : m->contacts) {
          double* q = crec + 17 * ci++;
          q[0] = c.feature; q[1] = c.stick;
          for (int k = 0; k < 3; k++) { q[2 + k] = c.rA[k]; q[5 + k] = c.rB[k]; q[8 + k] = c.C0[k]; q[11 + k] = c.penalty[k]; q[14 + k] = c.lambda[k]; }
        }
      }
      fi++;
    }
    return 0;
  });
}
// Overwrites every contact's penalty (the pivot-floor test's saturated contacts)
void orc_set_contact_penalty(void* h, double pen) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    for (auto& f : s.forces)
      if (f->kind == K_MANIFOLD)
        for (auto& c : static_cast<Manifold<T>*>(f.get())->contacts) c.penalty = V3<T>{T(pen), T(pen), T(pen)};
    return 0;
  });
}

void orc_step(void* h) { with(h, [&](auto& s) { s.step(); return 0; }); }
// fixed_colors: one colour per body (NULL: Jones-Plassmann). stats: colours, clashes, rounds.
void orc_step_gpu(void* h, const unsigned* fixed_colors, int* stats) {
  with(h, [&](auto& s) {
    s.stepGpu(fixed_colors);
    if (stats) { stats[0] = s.lastColors; stats[1] = s.lastClashes; stats[2] = s.lastRounds; }
    return 0;
  });
}

// The GPU-mode step with manifold reuse (the step option reuseManifolds): last step's manifolds are
// all kept and no pair is detected.
void orc_step_gpu_reuse(void* h, const unsigned* fixed_colors, int* stats) {
  with(h, [&](auto& s) {
    s.stepGpu(fixed_colors, true);
    if (stats) { stats[0] = s.lastColors; stats[1] = s.lastClashes; stats[2] = s.lastRounds; }
    return 0;
  });
}

// Contact-reuse state (GPU mode): the step counter, per body its reference pose (8 floats: pos,
// 0, rot) and the step it last moved, per manifold (force order, as orc_get_manifolds) the step
// that generated its points. Any pointer may be NULL.
void orc_get_reuse(void* h, unsigned* step, float* refs, unsigned* moved, unsigned* generated) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    if (step) *step = s.stepCounter;
    for (size_t i = 0; i < s.bodies.size(); i++) {
      const auto& b = s.bodies[i];
      if (refs) {
        for (int k = 0; k < 3; k++) refs[8 * i + k] = b.refPos[k];
        refs[8 * i + 3] = 0.0f;
        for (int k = 0; k < 4; k++) refs[8 * i + 4 + k] = b.refRot[k];
      }
      if (moved) moved[i] = b.movedStep;
    }
    int mi = 0;
    for (auto& f : s.forces)
      if (f->kind == K_MANIFOLD) {
        if (generated) generated[mi] = static_cast<Manifold<T>*>(f.get())->generated;
        mi++;
      }
    return 0;
  });
}
void orc_set_reuse(void* h, unsigned step, const float* refs, const unsigned* moved, const unsigned* generated) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    s.stepCounter = step;
    for (size_t i = 0; i < s.bodies.size(); i++) {
      auto& b = s.bodies[i];
      if (refs) {
        for (int k = 0; k < 3; k++) b.refPos[k] = refs[8 * i + k];
        for (int k = 0; k < 4; k++) b.refRot[k] = refs[8 * i + 4 + k];
      }
      if (moved) b.movedStep = moved[i];
    }
    int mi = 0;
    for (auto& f : s.forces)
      if (f->kind == K_MANIFOLD) {
        if (generated) static_cast<Manifold<T>*>(f.get())->generated = generated[mi];
        mi++;
      }
    return 0;
  });
}

// The GPU broadphase's pair set for the solver's current bodies (f32 records), sorted (hi, lo).
int orc_pairs(void* h, unsigned* out, int cap) {
  return with(h, [&](auto& s) {
    auto p = s.pairs();
    int n = int(p.size());
    for (int i = 0; i < n && i < cap; i++) { out[2 * i] = p[i].first; out[2 * i + 1] = p[i].second; }
    return n;
  });
}

// Narrowphase of bodies a, b of the solver, in its precision (f32 handle: the GPU's arithmetic).
// out: per contact 7 values: feature, rA3, rB3 (body-local); normal3 (B to A). Returns the count.
int orc_narrowphase(void* h, int a, int b, int faceBias, double* out, double* normal) {
  return with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    const Body<T>& A = s.bodies[a];
    const Body<T>& B = s.bodies[b];
    V3<T> nrm;
    Found<T> f = narrowphase(A, B, faceBias != 0, nrm, s.hulls.empty() ? nullptr : s.hulls.data());
    for (int i = 0; i < f.count; i++) {
      V3<T> rA = rotate(conjugate(A.rot), sub3(f.xA[i], A.pos));
      V3<T> rB = rotate(conjugate(B.rot), sub3(f.xB[i], B.pos));
      out[7 * i] = f.feature[i];
      for (int k = 0; k < 3; k++) { out[7 * i + 1 + k] = rA[k]; out[7 * i + 4 + k] = rB[k]; }
    }
    for (int k = 0; k < 3; k++) normal[k] = nrm[k];
    return f.count;
  });
}

// Jones-Plassmann on an explicit graph: n bodies, dynamic flags, CSR neighbours (dynamic ones),
// state in/out (colour | PENDING). stats: colours, clashes, rounds.
void orc_color_graph(int n, const unsigned char* dynamic, const int* start, const int* nbr, unsigned* state, int cap, int maxRounds, int* stats) {
  std::vector<char> dyn(dynamic, dynamic + n);
  std::vector<int> st(start, start + n + 1), nb(nbr, nbr + start[n]);
  std::vector<uint32_t> s(state, state + n);
  ColorResult r = jpColor(n, dyn, st, nb, s, cap, maxRounds);
  for (int i = 0; i < n; i++) state[i] = s[i];
  if (stats) { stats[0] = r.colors; stats[1] = r.clashes; stats[2] = r.rounds; }
}

unsigned orc_hash32(unsigned x) { return hash32(x); }

// Adjoint problems (FP64 handle): record `steps` GPU-mode steps of the solver's scene (boxes and
// static bodies, no joints) from its current state; null if the scene has joints or is FP32.
void* orc_adj_record(void* h, int steps) {
  OrcHandle* o = static_cast<OrcHandle*>(h);
  if (o->fp32) return nullptr;
  Solver<double>& s = *o->d;
  for (auto& f : s.forces)
    if (f->kind == K_JOINT || f->kind == K_SPRING) return nullptr;
  auto* P = new AdjProblem();
  const int n = int(s.bodies.size());
  P->n = n;
  P->dt = s.dt; P->gravity = s.gravity; P->alpha = s.alpha; P->gamma = s.gamma; P->betaLin = s.betaLin; P->margin = s.contactMargin;
  P->iterations = s.iterations;
  for (auto& b : s.bodies) {
    P->dynamic.push_back(b.mass > 0);
    for (int k = 0; k < 3; k++) {
      P->pos.push_back(b.pos[k]); P->prevVel.push_back(b.prevVel[k]); P->vel.push_back(b.vel[k]); P->angVel.push_back(b.angVel[k]);
      P->unitMoment.push_back(b.mass > 0 ? b.moment[k] / b.mass : 0.0);
    }
    for (int k = 0; k < 4; k++) P->rot.push_back(b.rot[k]);
    P->friction.push_back(b.friction);
    P->mass.push_back(b.mass);
  }
  std::map<std::tuple<int, int, uint32_t>, int> prevIndex;
  for (int k = 0; k < steps; k++) {
    s.stepGpu(nullptr);
    AdjStep st;
    std::map<std::tuple<int, int, uint32_t>, int> index;
    for (auto& f : s.forces) {
      if (f->kind != K_MANIFOLD) continue;
      auto* m = static_cast<Manifold<double>*>(f.get());
      AdjMan am;
      am.a = m->bodyA;
      am.b = m->bodyB;
      for (int c = 0; c < 9; c++) am.basis[c] = m->basis[c];
      int mi = int(st.mans.size());
      st.mans.push_back(am);
      for (auto& c : m->contacts) {
        AdjPoint p;
        for (int q = 0; q < 3; q++) { p.rA[q] = c.rA[q]; p.rB[q] = c.rB[q]; }
        p.man = mi;
        uint32_t feature = c.feature & ~STICK_BIT;
        auto it = prevIndex.find({am.a, am.b, feature});
        p.prev = it == prevIndex.end() ? -1 : it->second;
        index[{am.a, am.b, feature}] = int(st.pts.size());
        st.pts.push_back(p);
      }
    }
    for (auto& b : s.bodies) st.color.push_back(b.mass > 0 ? int(b.color & 0xffu) : -1);
    st.ncol = s.lastColors;
    P->steps.push_back(std::move(st));
    prevIndex = std::move(index);
  }
  P->target.assign(size_t(7) * n, 0.0);
  return P;
}
void orc_adj_destroy(void* a) { delete static_cast<AdjProblem*>(a); }
int orc_adj_bodies(void* a) { return static_cast<AdjProblem*>(a)->n; }
int orc_adj_points(void* a, int step) { return int(static_cast<AdjProblem*>(a)->steps[step].pts.size()); }
// The recorded parameters: per body v0 (3), omega0 (3), mass, friction
void orc_adj_nominal(void* a, double* params) {
  auto* P = static_cast<AdjProblem*>(a);
  for (int b = 0; b < P->n; b++) {
    for (int k = 0; k < 3; k++) { params[8 * b + k] = P->vel[3 * b + k]; params[8 * b + 3 + k] = P->angVel[3 * b + k]; }
    params[8 * b + 6] = P->mass[b];
    params[8 * b + 7] = P->friction[b];
  }
}
void orc_adj_set_target(void* a, const double* target) {
  auto* P = static_cast<AdjProblem*>(a);
  P->target.assign(target, target + size_t(7) * P->n);
}
// Replay with `params`; the loss, and the final poses (7 per body) into `final_state` if not null
double orc_adj_loss(void* a, const double* params, double* final_state) {
  auto* P = static_cast<AdjProblem*>(a);
  AdjState<double> X;
  std::vector<double> mass, mu;
  adjInit(*P, params, X, mass, mu, false);
  for (auto& st : P->steps) adjStep(*P, st, X, mass, mu);
  if (final_state)
    for (int b = 0; b < P->n; b++) {
      for (int k = 0; k < 3; k++) final_state[7 * b + k] = X.pos[b][k];
      for (int k = 0; k < 4; k++) final_state[7 * b + 3 + k] = X.rot[b][k];
    }
  return adjLoss(*P, X);
}
double orc_adj_gradient(void* a, const double* params, double* grad) { return adjGradient(*static_cast<AdjProblem*>(a), params, grad); }
// The recorded structure as flat arrays (one world): totals first (out[0] manifolds, out[1] points)
void orc_adj_sizes(void* a, int* out) {
  auto* P = static_cast<AdjProblem*>(a);
  int m = 0, p = 0;
  for (auto& st : P->steps) { m += int(st.mans.size()); p += int(st.pts.size()); }
  out[0] = m;
  out[1] = p;
}
// bodies: 13 per body (pos3 rot4 prevVz unitMoment3 dynamic friction); stepMan/stepPt: steps + 1
// firsts; manBodies 2, basis 9 per manifold; anchors 6, man, prev per point (indices over all steps);
// colors: steps x bodies (-1 static); ncol: per step
void orc_adj_export(void* a, double* bodies, int* stepMan, int* stepPt, int* manBodies, double* basis, double* anchors, int* ptMan, int* ptPrev,
                    int* colors, int* ncol) {
  auto* P = static_cast<AdjProblem*>(a);
  for (int b = 0; b < P->n; b++) {
    double* r = bodies + 13 * b;
    for (int k = 0; k < 3; k++) { r[k] = P->pos[3 * b + k]; r[8 + k] = P->unitMoment[3 * b + k]; }
    for (int k = 0; k < 4; k++) r[3 + k] = P->rot[4 * b + k];
    r[7] = P->prevVel[3 * b + 2];
    r[11] = P->dynamic[b] ? 1.0 : 0.0;
    r[12] = P->friction[b];
  }
  int m = 0, p = 0, prevFirst = 0;
  for (size_t s = 0; s < P->steps.size(); s++) {
    const AdjStep& st = P->steps[s];
    stepMan[s] = m;
    stepPt[s] = p;
    for (auto& am : st.mans) {
      manBodies[2 * m] = am.a;
      manBodies[2 * m + 1] = am.b;
      for (int c = 0; c < 9; c++) basis[9 * m + c] = am.basis[c];
      m++;
    }
    for (auto& q : st.pts) {
      for (int k = 0; k < 3; k++) { anchors[6 * p + k] = q.rA[k]; anchors[6 * p + 3 + k] = q.rB[k]; }
      ptMan[p] = stepMan[s] + q.man;
      ptPrev[p] = q.prev < 0 ? -1 : prevFirst + q.prev;
      p++;
    }
    prevFirst = stepPt[s];
    for (int b = 0; b < P->n; b++) colors[s * P->n + b] = st.color[b];
    ncol[s] = st.ncol;
  }
  stepMan[P->steps.size()] = m;
  stepPt[P->steps.size()] = p;
}
// The inverse of orc_adj_export: a problem from one world's recorded structure (indices over its
// own steps) and nominal parameters (8 per body); params7: dt gravity alpha gamma betaLin margin iterations
void* orc_adj_import(const double* params7, int n, int steps, const double* bodies, const double* nominal, const int* stepMan, const int* stepPt,
                     const int* manBodies, const double* basis, const double* anchors, const int* ptMan, const int* ptPrev, const int* colors,
                     const int* ncol) {
  auto* P = new AdjProblem();
  P->n = n;
  P->dt = params7[0]; P->gravity = params7[1]; P->alpha = params7[2]; P->gamma = params7[3]; P->betaLin = params7[4]; P->margin = params7[5];
  P->iterations = int(params7[6]);
  for (int b = 0; b < n; b++) {
    const double* r = bodies + 13 * b;
    const double* q = nominal + 8 * b;
    P->dynamic.push_back(r[11] != 0.0);
    for (int k = 0; k < 3; k++) {
      P->pos.push_back(r[k]);
      P->prevVel.push_back(k == 2 ? r[7] : 0.0);
      P->unitMoment.push_back(r[8 + k]);
      P->vel.push_back(q[k]);
      P->angVel.push_back(q[3 + k]);
    }
    for (int k = 0; k < 4; k++) P->rot.push_back(r[3 + k]);
    P->mass.push_back(q[6]);
    P->friction.push_back(r[11] != 0.0 ? q[7] : r[12]);
  }
  for (int s = 0; s < steps; s++) {
    AdjStep st;
    for (int m = stepMan[s]; m < stepMan[s + 1]; m++) {
      AdjMan am;
      am.a = manBodies[2 * m];
      am.b = manBodies[2 * m + 1];
      for (int c = 0; c < 9; c++) am.basis[c] = basis[9 * m + c];
      st.mans.push_back(am);
    }
    for (int k = stepPt[s]; k < stepPt[s + 1]; k++) {
      AdjPoint q;
      for (int c = 0; c < 3; c++) { q.rA[c] = anchors[6 * k + c]; q.rB[c] = anchors[6 * k + 3 + c]; }
      q.man = ptMan[k] - stepMan[s];
      q.prev = ptPrev[k] < 0 ? -1 : ptPrev[k] - stepPt[s - 1];
      st.pts.push_back(q);
    }
    st.color.assign(colors + size_t(s) * n, colors + size_t(s + 1) * n);
    st.ncol = ncol[s];
    P->steps.push_back(std::move(st));
  }
  P->target.assign(size_t(7) * n, 0.0);
  return P;
}
double orc_adj_param(void* a, int which) {  // 0 dt 1 gravity 2 alpha 3 gamma 4 betaLin 5 margin 6 iterations
  auto* P = static_cast<AdjProblem*>(a);
  double v[7] = {P->dt, P->gravity, P->alpha, P->gamma, P->betaLin, P->margin, double(P->iterations)};
  return v[which];
}

// GPU-mode body aux (gravity scale, damping rates) and lifecycle bits of body i
void orc_set_body_aux(void* h, int i, double scale, double lin, double ang) {
  with(h, [&](auto& s) {
    s.bodies[i].gravityScale = scale;
    s.bodies[i].linDamp = lin;
    s.bodies[i].angDamp = ang;
    return 0;
  });
}
void orc_set_lifecycle(void* h, int i, unsigned bits) {
  with(h, [&](auto& s) {
    s.bodies[i].lifecycle = bits;
    return 0;
  });
}

// The hull buffer (gpu/solver.ts:313-338 layout, absolute offsets) the bodies' shape codes name
void orc_set_hulls(void* h, const unsigned* words, int n) {
  with(h, [&](auto& s) {
    s.hulls.assign(words, words + n);
    return 0;
  });
}

// Rounds the whole state to f32 in place (bodies, aux records, joints, springs, manifolds and their
// contacts), so that a double solver and an f32 copy of its state (the CUDA world's records) start
// a step from the same numbers.
void orc_round_f32(void* h) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    auto r = [](T& x) { x = T(float(x)); };
    auto r3 = [&](V3<T>& v) { for (auto& x : v) r(x); };
    auto r4 = [&](Q4<T>& q) { for (auto& x : q) r(x); };
    for (auto& b : s.bodies) {
      r3(b.pos); r3(b.initPos); r3(b.inertialPos); r3(b.vel); r3(b.angVel); r3(b.prevVel); r3(b.size); r3(b.moment);
      r4(b.rot); r4(b.initRot); r4(b.inertialRot);
      r(b.mass); r(b.friction); r(b.radius); r(b.gravityScale); r(b.linDamp); r(b.angDamp);
    }
    for (auto& f : s.forces) {
      if (f->kind == K_JOINT) {
        auto* j = static_cast<Joint<T>*>(f.get());
        r3(j->rA); r3(j->rB); r3(j->C0Lin); r3(j->C0Ang); r3(j->penaltyLin); r3(j->penaltyAng); r3(j->lambdaLin); r3(j->lambdaAng);
        r(j->stiffnessLin); r(j->stiffnessAng); r(j->fracture); r(j->torqueArm); r(j->yield); r(j->breakBend);
        r4(j->rest); r4(j->restStart);
      } else if (f->kind == K_SPRING) {
        auto* sp = static_cast<Spring<T>*>(f.get());
        r3(sp->rA); r3(sp->rB); r(sp->rest); r(sp->stiffness);
      } else if (f->kind == K_MANIFOLD) {
        auto* m = static_cast<Manifold<T>*>(f.get());
        for (auto& x : m->basis) r(x);
        r(m->friction);
        for (auto& c : m->contacts) { r3(c.rA); r3(c.rB); r3(c.C0); r3(c.penalty); r3(c.lambda); }
      }
    }
    return 0;
  });
}

// Replaces last step's manifolds (the GPU-mode step's warm-start source) with the given records, in
// orc_get_manifolds' layout: manifold (8): ignored, a, b, count, normal3, friction; contact (17):
// feature, stick, rA3, rB3, C0 3, pen3, lam3. A manifold's contacts follow the previous manifold's.
// Manifolds are appended after the joints, springs and ignore pairs, as a step leaves them.
void orc_set_manifolds(void* h, int nm, const double* mrec, int nc, const double* crec) {
  with(h, [&](auto& s) {
    using T = std::decay_t<decltype(s.dt)>;
    std::vector<std::unique_ptr<Force<T>>> keep;
    for (auto& f : s.forces) {
      if (f->kind == K_MANIFOLD) s.unlink(f.get());
      else keep.push_back(std::move(f));
    }
    s.forces = std::move(keep);
    int ci = 0;
    for (int i = 0; i < nm; i++) {
      const double* r = mrec + 8 * i;
      auto m = std::make_unique<Manifold<T>>(&s, int(r[1]), int(r[2]));
      m->basis = orthonormal(V3<T>{T(r[4]), T(r[5]), T(r[6])});
      m->friction = T(r[7]);
      for (int k = 0; k < int(r[3]) && ci < nc; k++, ci++) {
        const double* q = crec + 17 * ci;
        Contact<T> c;
        c.feature = uint32_t(q[0]);
        c.stick = q[1] != 0;
        for (int e = 0; e < 3; e++) {
          c.rA[e] = T(q[2 + e]); c.rB[e] = T(q[5 + e]); c.C0[e] = T(q[8 + e]); c.penalty[e] = T(q[11 + e]); c.lambda[e] = T(q[14 + e]);
        }
        m->contacts.push_back(c);
      }
      s.addForce(std::move(m));
    }
    return 0;
  });
}

// Host threads for the GPU-mode step (OpenMP); returns the count in use.
int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

}  // extern "C"
