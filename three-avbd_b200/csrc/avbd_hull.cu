// Convex hull builder (host): the hull shape a body collides as, built once from a point set.
//
// A restatement of the reference's procedure in src/avbd3d/hull.ts (convexHull, buildHull, foldOf,
// mergeTriangles, eigenSymmetric, quatFromBasis, spreadVertices) in C++, in double: the same
// quickhull with coplanar faces merged, farthest-point simplification to AVBD_MAX_HULL_VERTICES, and
// principal frame, so that the same points give the same hull (vertex set, faces, mass properties)
// as the reference's hull tests pin them (tests/hull.test.ts, tests/hull-degenerate.test.ts). The
// face and edge numbering is not pinned (the reference holds no built hull to compare with); it
// only has to be consistent within one record, whose feature keys this backend both writes and
// warm-starts from. The output is the reference's hull record (gpu/solver.ts:313-338 packHull with
// the header at 0) plus the mass properties.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <unordered_map>
#include <vector>

#include "avbd.h"

namespace {

using V3 = std::array<double, 3>;
V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
V3 cross(const V3& a, const V3& b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
double len(const V3& a) { return std::sqrt(dot(a, a)); }

struct Tri {
  int id;
  std::array<int, 3> v;
  V3 n;
  double d;
};

struct Face {
  V3 normal;
  double d;
  std::vector<int> verts;
};

struct Shape {
  std::vector<V3> local;  // principal frame, double
  std::vector<Face> faces;
  std::vector<std::array<int, 4>> edges;
  double volume;
  V3 moments, size, center;
  double radius;
  std::array<double, 4> rotation;
};

uint64_t edgeKey(int a, int b) { return (uint64_t(uint32_t(a)) << 32) | uint32_t(b); }

// hull.ts:449-491 (Jacobi rotations; columns right-handed)
void eigenSymmetric(const double m[3][3], V3& values, double vectors[3][3]) {
  double a[3][3];
  std::memcpy(a, m, sizeof(a));
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 50; sweep++) {
    double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    if (off < 1e-30 * (a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2] + 1e-300)) break;
    for (int p = 0; p < 3; p++) {
      for (int q = p + 1; q < 3; q++) {
        if (std::fabs(a[p][q]) < 1e-300) continue;
        double theta = (a[q][q] - a[p][p]) / (2 * a[p][q]);
        double sg = theta > 0 ? 1.0 : theta < 0 ? -1.0 : 1.0;  // Math.sign(theta || 1)
        double t = sg / (std::fabs(theta) + std::sqrt(theta * theta + 1));
        double c = 1 / std::sqrt(t * t + 1);
        double s = t * c;
        for (int k = 0; k < 3; k++) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; k++) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; k++) {
          double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq;
          v[k][q] = s * vkp + c * vkq;
        }
      }
    }
  }
  V3 x{v[0][0], v[1][0], v[2][0]}, y{v[0][1], v[1][1], v[2][1]};
  V3 z = cross(x, y);
  double out[3][3] = {{x[0], y[0], z[0]}, {x[1], y[1], z[1]}, {x[2], y[2], z[2]}};
  std::memcpy(vectors, out, sizeof(out));
  values = {a[0][0], a[1][1], a[2][2]};
}

// hull.ts:494-512
std::array<double, 4> quatFromBasis(const double m[3][3]) {
  double tr = m[0][0] + m[1][1] + m[2][2];
  double x, y, z, w;
  if (tr > 0) {
    double s = 0.5 / std::sqrt(tr + 1);
    w = 0.25 / s;
    x = (m[2][1] - m[1][2]) * s;
    y = (m[0][2] - m[2][0]) * s;
    z = (m[1][0] - m[0][1]) * s;
  } else if (m[0][0] > m[1][1] && m[0][0] > m[2][2]) {
    double s = 2 * std::sqrt(1 + m[0][0] - m[1][1] - m[2][2]);
    w = (m[2][1] - m[1][2]) / s;
    x = 0.25 * s;
    y = (m[0][1] + m[1][0]) / s;
    z = (m[0][2] + m[2][0]) / s;
  } else if (m[1][1] > m[2][2]) {
    double s = 2 * std::sqrt(1 + m[1][1] - m[0][0] - m[2][2]);
    w = (m[0][2] - m[2][0]) / s;
    x = (m[0][1] + m[1][0]) / s;
    y = 0.25 * s;
    z = (m[1][2] + m[2][1]) / s;
  } else {
    double s = 2 * std::sqrt(1 + m[2][2] - m[0][0] - m[1][1]);
    w = (m[1][0] - m[0][1]) / s;
    x = (m[0][2] + m[2][0]) / s;
    y = (m[1][2] + m[2][1]) / s;
    z = 0.25 * s;
  }
  double l = std::sqrt(x * x + y * y + z * z + w * w);
  return {x / l, y / l, z / l, w / l};
}

// hull.ts:326-446: coplanar triangles merged into faces, edges, mass properties, principal frame
bool mergeTriangles(const std::vector<V3>& p, const std::vector<std::array<int, 3>>& indices, Shape& out) {
  double scale = 0;
  for (const V3& v : p) scale = std::max({scale, std::fabs(v[0]), std::fabs(v[1]), std::fabs(v[2])});
  const double planeTol = std::max(scale, 1e-9) * 1e-5;
  struct T3 {
    std::array<int, 3> v;
    V3 n;
    double d;
  };
  std::vector<T3> tris;
  for (const auto& v : indices) {
    V3 c = cross(sub(p[v[1]], p[v[0]]), sub(p[v[2]], p[v[0]]));
    double l = len(c);
    if (!(l > 0)) continue;
    V3 n{c[0] / l, c[1] / l, c[2] / l};
    tris.push_back({v, n, dot(n, p[v[0]])});
  }
  std::unordered_map<uint64_t, int> edgeTri;
  for (int k = 0; k < (int)tris.size(); k++)
    for (int j = 0; j < 3; j++) edgeTri[edgeKey(tris[k].v[j], tris[k].v[(j + 1) % 3])] = k;
  std::vector<int> groupOf(tris.size(), -1);
  std::vector<std::vector<int>> groups;
  for (int k = 0; k < (int)tris.size(); k++) {
    if (groupOf[k] >= 0) continue;
    const T3& seed = tris[k];
    std::vector<int> members{k};
    groupOf[k] = (int)groups.size();
    for (size_t m = 0; m < members.size(); m++) {
      const T3& t = tris[members[m]];
      for (int j = 0; j < 3; j++) {
        auto it = edgeTri.find(edgeKey(t.v[(j + 1) % 3], t.v[j]));
        if (it == edgeTri.end() || groupOf[it->second] >= 0) continue;
        const T3& u = tris[it->second];
        bool flat = dot(seed.n, u.n) > 1 - 1e-5;
        for (int q = 0; q < 3 && flat; q++) flat = std::fabs(dot(seed.n, p[u.v[q]]) - seed.d) <= planeTol;
        if (flat) {
          groupOf[it->second] = (int)groups.size();
          members.push_back(it->second);
        }
      }
    }
    groups.push_back(members);
  }
  struct Poly {
    V3 n;
    std::vector<int> verts;
  };
  std::vector<Poly> polys;
  for (const auto& members : groups) {
    std::set<uint64_t> inGroup;
    for (int k : members)
      for (int j = 0; j < 3; j++) inGroup.insert(edgeKey(tris[k].v[j], tris[k].v[(j + 1) % 3]));
    std::vector<std::pair<int, int>> nextOrder;  // insertion order of the boundary's directed edges
    std::unordered_map<int, int> next;
    for (int k : members) {
      for (int j = 0; j < 3; j++) {
        int a = tris[k].v[j], b = tris[k].v[(j + 1) % 3];
        if (!inGroup.count(edgeKey(b, a))) {
          if (next.count(a)) return false;  // the region's boundary isn't one loop
          next[a] = b;
          nextOrder.push_back({a, b});
        }
      }
    }
    V3 n{0, 0, 0};
    for (int k : members) {
      const T3& t = tris[k];
      V3 c = cross(sub(p[t.v[1]], p[t.v[0]]), sub(p[t.v[2]], p[t.v[0]]));
      n[0] += c[0];
      n[1] += c[1];
      n[2] += c[2];
    }
    double l = len(n);
    if (l == 0) l = 1;
    if (nextOrder.empty()) return false;
    int start = nextOrder[0].first;
    std::vector<int> loop{start};
    for (int v = next[start]; v != start && loop.size() <= next.size(); v = next.count(v) ? next[v] : start) loop.push_back(v);
    if (loop.size() != next.size()) return false;
    polys.push_back({{n[0] / l, n[1] / l, n[2] / l}, loop});
  }
  std::unordered_map<int, int> index;
  std::vector<V3> verts;
  for (auto& poly : polys)
    for (int v : poly.verts)
      if (!index.count(v)) {
        index[v] = (int)verts.size();
        verts.push_back(p[v]);
      }
  for (auto& poly : polys)
    for (int& v : poly.verts) v = index[v];
  // A closed surface: every edge on two faces in opposite directions, V - E + F = 2
  std::set<uint64_t> directed;
  size_t sides = 0;
  for (auto& poly : polys)
    for (size_t k = 0; k < poly.verts.size(); k++) {
      directed.insert(edgeKey(poly.verts[k], poly.verts[(k + 1) % poly.verts.size()]));
      sides++;
    }
  if (directed.size() != sides) return false;
  for (uint64_t e : directed)
    if (!directed.count(edgeKey(int(uint32_t(e)), int(e >> 32)))) return false;
  if ((long)verts.size() - (long)directed.size() / 2 + (long)polys.size() != 2) return false;
  // Mass properties: signed tetrahedra over fan-triangulated faces
  double volume = 0;
  V3 com{0, 0, 0};
  double C[6] = {0, 0, 0, 0, 0, 0};
  for (auto& poly : polys) {
    const V3& a = verts[poly.verts[0]];
    for (size_t k = 1; k + 1 < poly.verts.size(); k++) {
      const V3& b = verts[poly.verts[k]];
      const V3& c = verts[poly.verts[k + 1]];
      double det = dot(a, cross(b, c));
      volume += det / 6;
      for (int j = 0; j < 3; j++) com[j] += (det / 24) * (a[j] + b[j] + c[j]);
      auto s = [&](int i, int j) { return (det / 120) * (a[i] * a[j] + b[i] * b[j] + c[i] * c[j] + (a[i] + b[i] + c[i]) * (a[j] + b[j] + c[j])); };
      C[0] += s(0, 0);
      C[1] += s(1, 1);
      C[2] += s(2, 2);
      C[3] += s(0, 1);
      C[4] += s(0, 2);
      C[5] += s(1, 2);
    }
  }
  if (!(volume > 0)) return false;
  for (int j = 0; j < 3; j++) com[j] /= volume;
  C[0] -= volume * com[0] * com[0];
  C[1] -= volume * com[1] * com[1];
  C[2] -= volume * com[2] * com[2];
  C[3] -= volume * com[0] * com[1];
  C[4] -= volume * com[0] * com[2];
  C[5] -= volume * com[1] * com[2];
  double tr = C[0] + C[1] + C[2];
  double I[3][3] = {{tr - C[0], -C[3], -C[4]}, {-C[3], tr - C[1], -C[5]}, {-C[4], -C[5], tr - C[2]}};
  V3 values;
  double R[3][3];
  eigenSymmetric(I, values, R);
  auto toLocal = [&](const V3& v) -> V3 {
    V3 d = sub(v, com);
    return {R[0][0] * d[0] + R[1][0] * d[1] + R[2][0] * d[2], R[0][1] * d[0] + R[1][1] * d[1] + R[2][1] * d[2],
            R[0][2] * d[0] + R[1][2] * d[1] + R[2][2] * d[2]};
  };
  out.local.clear();
  for (const V3& v : verts) out.local.push_back(toLocal(v));
  out.faces.clear();
  for (auto& poly : polys) {
    const V3& n = poly.n;
    V3 nl{R[0][0] * n[0] + R[1][0] * n[1] + R[2][0] * n[2], R[0][1] * n[0] + R[1][1] * n[1] + R[2][1] * n[2],
          R[0][2] * n[0] + R[1][2] * n[1] + R[2][2] * n[2]};
    double d = -INFINITY;
    for (int v : poly.verts) d = std::max(d, dot(nl, out.local[v]));
    out.faces.push_back({nl, d, poly.verts});
  }
  std::unordered_map<uint64_t, int> faceOf;
  for (int k = 0; k < (int)out.faces.size(); k++) {
    const auto& f = out.faces[k].verts;
    for (size_t j = 0; j < f.size(); j++) faceOf[edgeKey(f[j], f[(j + 1) % f.size()])] = k;
  }
  out.edges.clear();
  for (int k = 0; k < (int)out.faces.size(); k++) {
    const auto& f = out.faces[k].verts;
    for (size_t j = 0; j < f.size(); j++) {
      int a = f[j], b = f[(j + 1) % f.size()];
      auto it = faceOf.find(edgeKey(b, a));
      if (a < b && it != faceOf.end()) out.edges.push_back({a, b, k, it->second});
    }
  }
  out.size = {0, 0, 0};
  out.radius = 0;
  for (const V3& v : out.local) {
    for (int j = 0; j < 3; j++) out.size[j] = std::max(out.size[j], 2 * std::fabs(v[j]));
    out.radius = std::max(out.radius, len(v));
  }
  out.volume = volume;
  out.moments = values;
  out.center = com;
  out.rotation = quatFromBasis(R);
  return true;
}

// hull.ts:248-275
int foldOf(const std::vector<std::pair<int, int>>& horizon, const std::vector<Tri>& fan, const std::vector<const Tri*>& kept,
           const std::vector<V3>& p, double tol) {
  const int H = (int)horizon.size();
  std::unordered_map<int, int> next;
  for (auto& e : horizon) {
    if (next.count(e.first)) return H;
    next[e.first] = e.second;
  }
  if (!H) return H;
  int start = horizon[0].first;
  int steps = 0;
  for (int v = start; steps == 0 || v != start; steps++) {
    auto it = next.find(v);
    if (it == next.end() || steps >= H) return H;
    v = it->second;
  }
  if (steps != H) return H;
  std::vector<int> verts;
  std::set<int> seen;
  for (const Tri* t : kept)
    for (int v : t->v)
      if (seen.insert(v).second) verts.push_back(v);
  for (int k = 0; k < (int)fan.size(); k++) {
    const Tri& t = fan[k];
    if (!(len(cross(sub(p[t.v[1]], p[t.v[0]]), sub(p[t.v[2]], p[t.v[0]]))) > 0)) return k;
    for (int v : verts)
      if (dot(t.n, p[v]) - t.d > tol) return k;
  }
  return -1;
}

// hull.ts:100-240
bool buildHull(const std::vector<V3>& points, Shape& out) {
  V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
  double magnitude = 0;
  for (const V3& q : points)
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], q[k]);
      hi[k] = std::max(hi[k], q[k]);
      magnitude = std::max(magnitude, std::fabs(q[k]));
    }
  double extent = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]});
  if (!(extent > 0 && extent < INFINITY)) return false;
  const double tol = std::max(extent, magnitude) * 1e-7;
  const double weld = 100 * tol;
  std::map<std::array<long long, 3>, std::vector<V3>> cells;
  std::vector<V3> p;
  for (const V3& v : points) {
    std::array<long long, 3> c{(long long)std::floor(v[0] / weld), (long long)std::floor(v[1] / weld), (long long)std::floor(v[2] / weld)};
    bool near = false;
    for (int dx = -1; dx <= 1 && !near; dx++)
      for (int dy = -1; dy <= 1 && !near; dy++)
        for (int dz = -1; dz <= 1 && !near; dz++) {
          auto it = cells.find({c[0] + dx, c[1] + dy, c[2] + dz});
          if (it != cells.end())
            for (const V3& u : it->second)
              if (len(sub(u, v)) <= weld) near = true;
        }
    if (near) continue;
    cells[c].push_back(v);
    p.push_back(v);
  }
  const int np = (int)p.size();
  if (np < 4) return false;
  int i0 = 0;
  for (int i = 1; i < np; i++)
    if (p[i][0] < p[i0][0]) i0 = i;
  int i1 = -1;
  double best = 0;
  for (int i = 0; i < np; i++) {
    double d = len(sub(p[i], p[i0]));
    if (d > best) {
      best = d;
      i1 = i;
    }
  }
  if (i1 < 0 || best < tol) return false;
  int i2 = -1;
  best = 0;
  V3 e01 = sub(p[i1], p[i0]);
  for (int i = 0; i < np; i++) {
    double d = len(cross(e01, sub(p[i], p[i0])));
    if (d > best) {
      best = d;
      i2 = i;
    }
  }
  if (i2 < 0 || best < tol * len(e01)) return false;
  V3 n012 = cross(e01, sub(p[i2], p[i0]));
  int i3 = -1;
  best = 0;
  for (int i = 0; i < np; i++) {
    double d = std::fabs(dot(n012, sub(p[i], p[i0])));
    if (d > best) {
      best = d;
      i3 = i;
    }
  }
  if (i3 < 0 || best < tol * len(n012)) return false;

  int nextId = 0;
  auto make = [&](int a, int b, int c) -> Tri {
    V3 n = cross(sub(p[b], p[a]), sub(p[c], p[a]));
    double l = len(n);
    if (l == 0) l = 1;
    V3 u{n[0] / l, n[1] / l, n[2] / l};
    return Tri{nextId++, {a, b, c}, u, dot(u, p[a])};
  };
  std::vector<Tri> tris;
  bool flip = dot(n012, sub(p[i3], p[i0])) > 0;
  std::array<int, 3> base = flip ? std::array<int, 3>{i0, i2, i1} : std::array<int, 3>{i0, i1, i2};
  tris.push_back(make(base[0], base[1], base[2]));
  tris.push_back(make(base[0], i3, base[1]));
  tris.push_back(make(base[1], i3, base[2]));
  tris.push_back(make(base[2], i3, base[0]));

  // `outside`: insertion-ordered (point, the face it is farthest in front of, that distance)
  struct Out {
    int j;
    int face;  // triangle id
    double d;
    bool alive;
  };
  std::vector<Out> outside;
  std::unordered_map<int, int> outAt;
  auto assign = [&](int j) {
    int face = -1;
    double d = tol;
    for (const Tri& t : tris) {
      double e = dot(t.n, p[j]) - t.d;
      if (e > d) {
        face = t.id;
        d = e;
      }
    }
    auto it = outAt.find(j);
    if (face >= 0) {
      if (it != outAt.end() && outside[it->second].alive) {
        outside[it->second].face = face;
        outside[it->second].d = d;
      } else {
        outAt[j] = (int)outside.size();
        outside.push_back({j, face, d, true});
      }
    } else if (it != outAt.end()) {
      outside[it->second].alive = false;
    }
  };
  for (int j = 0; j < np; j++)
    if (j != i0 && j != i1 && j != i2 && j != i3) assign(j);
  auto anyOutside = [&]() {
    for (const Out& o : outside)
      if (o.alive) return true;
    return false;
  };
  while (anyOutside()) {
    int i = -1;
    double farthest = -INFINITY;
    for (const Out& o : outside)
      if (o.alive && o.d > farthest) {
        farthest = o.d;
        i = o.j;
      }
    outside[outAt[i]].alive = false;
    std::vector<int> region;  // triangle ids, insertion order
    std::set<int> inRegion;
    std::unordered_map<uint64_t, int> byEdge;  // directed edge -> index into tris
    for (int k = 0; k < (int)tris.size(); k++)
      for (int q = 0; q < 3; q++) byEdge[edgeKey(tris[k].v[q], tris[k].v[(q + 1) % 3])] = k;
    std::unordered_map<int, int> atOf;  // triangle id -> index into tris
    for (int k = 0; k < (int)tris.size(); k++) atOf[tris[k].id] = k;
    std::vector<int> queue;
    for (const Tri& t : tris)
      if (dot(t.n, p[i]) - t.d > tol) {
        region.push_back(t.id);
        inRegion.insert(t.id);
        queue.push_back(t.id);
      }
    while (!queue.empty()) {
      const Tri& t = tris[atOf[queue.back()]];
      queue.pop_back();
      for (int q = 0; q < 3; q++) {
        auto it = byEdge.find(edgeKey(t.v[(q + 1) % 3], t.v[q]));
        if (it == byEdge.end()) continue;
        const Tri& u = tris[it->second];
        if (!inRegion.count(u.id) && dot(u.n, p[i]) - u.d > -tol) {
          region.push_back(u.id);
          inRegion.insert(u.id);
          queue.push_back(u.id);
        }
      }
    }
    auto horizonOf = [&]() {
      std::set<uint64_t> onVisible;
      for (int id : region) {
        const Tri& t = tris[atOf[id]];
        for (int q = 0; q < 3; q++) onVisible.insert(edgeKey(t.v[q], t.v[(q + 1) % 3]));
      }
      std::vector<std::pair<int, int>> horizon;
      for (int id : region) {
        const Tri& t = tris[atOf[id]];
        for (int q = 0; q < 3; q++) {
          int a = t.v[q], b = t.v[(q + 1) % 3];
          if (!onVisible.count(edgeKey(b, a))) horizon.push_back({a, b});
        }
      }
      return horizon;
    };
    std::vector<Tri> fan;
    bool ok = false;
    const int firstFanId = nextId;
    for (int tries = 0; tries <= (int)tris.size() && !ok; tries++) {
      auto horizon = horizonOf();
      nextId = firstFanId;
      fan.clear();
      for (auto& e : horizon) fan.push_back(make(e.first, e.second, i));
      std::vector<const Tri*> kept;
      for (const Tri& t : tris)
        if (!inRegion.count(t.id)) kept.push_back(&t);
      int bad = foldOf(horizon, fan, kept, p, 10 * tol);
      ok = bad < 0;
      if (!ok) {
        const Tri* u = nullptr;
        if (bad < (int)horizon.size()) {
          auto it = byEdge.find(edgeKey(horizon[bad].second, horizon[bad].first));
          if (it != byEdge.end()) u = &tris[it->second];
        }
        if (!u || inRegion.count(u->id) || dot(u->n, p[i]) - u->d < -10 * tol) break;
        region.push_back(u->id);
        inRegion.insert(u->id);
      }
    }
    if (!ok) {
      nextId = firstFanId;
      continue;
    }
    std::vector<Tri> keptTris;
    for (const Tri& t : tris)
      if (!inRegion.count(t.id)) keptTris.push_back(t);
    for (const Tri& t : fan) keptTris.push_back(t);
    tris.swap(keptTris);
    if ((long)tris.size() > 2L * np) return false;
    for (Out& o : outside)
      if (o.alive && inRegion.count(o.face)) assign(o.j);
  }
  std::vector<std::array<int, 3>> idx;
  for (const Tri& t : tris) idx.push_back(t.v);
  return mergeTriangles(p, idx, out);
}

// hull.ts:78-98: `count` of a hull's vertices, spread out, in the input points' frame
std::vector<V3> spreadVertices(const Shape& h, int count) {
  double x = h.rotation[0], y = h.rotation[1], z = h.rotation[2], w = h.rotation[3];
  auto back = [&](const V3& v) -> V3 {
    V3 t{2 * (y * v[2] - z * v[1]), 2 * (z * v[0] - x * v[2]), 2 * (x * v[1] - y * v[0])};
    return {v[0] + w * t[0] + (y * t[2] - z * t[1]) + h.center[0], v[1] + w * t[1] + (z * t[0] - x * t[2]) + h.center[1],
            v[2] + w * t[2] + (x * t[1] - y * t[0]) + h.center[2]};
  };
  std::vector<V3> verts;
  for (const V3& v : h.local) {
    V3 f{double(float(v[0])), double(float(v[1])), double(float(v[2]))};  // the stored (f32) vertices
    verts.push_back(back(f));
  }
  int first = 0;
  for (int i = 0; i < (int)verts.size(); i++)
    if (len(sub(verts[i], h.center)) > len(sub(verts[first], h.center))) first = i;
  std::vector<int> chosen{first};
  std::vector<double> dist;
  for (const V3& v : verts) dist.push_back(len(sub(v, verts[first])));
  while ((int)chosen.size() < count) {
    int far = 0;
    for (int i = 0; i < (int)dist.size(); i++)
      if (dist[i] > dist[far]) far = i;
    chosen.push_back(far);
    for (int i = 0; i < (int)verts.size(); i++) dist[i] = std::min(dist[i], len(sub(verts[i], verts[far])));
  }
  std::vector<V3> out;
  for (int i : chosen) out.push_back(verts[i]);
  return out;
}

// gpu/solver.ts:313-338 (packHull at header 0): header, vertices, faces, indices, edges as vec4s
uint32_t packedSize(const Shape& s) {
  uint32_t indices = 0;
  for (const Face& f : s.faces) indices += (uint32_t)f.verts.size();
  return 2 + (uint32_t)s.local.size() + 2 * (uint32_t)s.faces.size() + (indices + 3) / 4 + (uint32_t)s.edges.size();
}
void pack(const Shape& s, uint32_t* u) {
  const uint32_t V = (uint32_t)s.local.size(), F = (uint32_t)s.faces.size(), E = (uint32_t)s.edges.size();
  uint32_t indexCount = 0;
  for (const Face& f : s.faces) indexCount += (uint32_t)f.verts.size();
  const uint32_t I = (indexCount + 3) / 4;
  std::memset(u, 0, size_t(packedSize(s)) * 16);
  const uint32_t vs = 2, fs = vs + V, is = fs + 2 * F, es = is + I;
  const uint32_t head[8] = {vs, V, fs, F, es, E, is, 0};
  std::memcpy(u, head, sizeof(head));
  auto putf = [&](uint32_t word, double v) {
    float f = float(v);
    std::memcpy(&u[word], &f, 4);
  };
  for (uint32_t v = 0; v < V; v++)
    for (int k = 0; k < 3; k++) putf((vs + v) * 4 + k, s.local[v][k]);
  uint32_t index = 0;
  for (uint32_t k = 0; k < F; k++) {
    const Face& f = s.faces[k];
    uint32_t o = (fs + 2 * k) * 4;
    for (int j = 0; j < 3; j++) putf(o + j, f.normal[j]);
    putf(o + 3, f.d);
    u[o + 4] = index;
    u[o + 5] = (uint32_t)f.verts.size();
    for (int v : f.verts) u[is * 4 + index++] = (uint32_t)v;
  }
  for (uint32_t k = 0; k < E; k++)
    for (int j = 0; j < 4; j++) u[(es + k) * 4 + j] = (uint32_t)s.edges[k][j];
}

}  // namespace

extern "C" int avbd_hull_build(const float* points, uint32_t n, uint32_t* packed, uint32_t cap_vec4s, uint32_t* vec4s, avbd_hull_props* props) {
  if ((n && !points) || !vec4s) return AVBD_ERR_INVALID;
  *vec4s = 0;
  std::vector<V3> pts(n);
  for (uint32_t i = 0; i < n; i++) pts[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};
  Shape s;
  if (!buildHull(pts, s)) return AVBD_ERR_INVALID;  // no volume (too few points, flat, or degenerate)
  if ((int)s.local.size() > AVBD_MAX_HULL_VERTICES) {
    Shape full = s;
    if (!buildHull(spreadVertices(full, AVBD_MAX_HULL_VERTICES), s)) return AVBD_ERR_INVALID;
  }
  if (s.faces.size() > 255 || s.edges.size() > 255) return AVBD_ERR_INVALID;
  const uint32_t size = packedSize(s);
  *vec4s = size;
  if (props) {
    props->volume = s.volume;
    for (int k = 0; k < 3; k++) {
      props->moments[k] = s.moments[k];
      props->size[k] = s.size[k];
      props->center[k] = s.center[k];
    }
    for (int k = 0; k < 4; k++) props->rotation[k] = s.rotation[k];
    props->radius = s.radius;
    props->vertices = (uint32_t)s.local.size();
    props->faces = (uint32_t)s.faces.size();
    props->edges = (uint32_t)s.edges.size();
  }
  if (!packed) return AVBD_OK;
  if (cap_vec4s < size) return AVBD_ERR_CAPACITY;
  pack(s, packed);
  return AVBD_OK;
}
