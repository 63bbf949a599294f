// scene_gen.cpp - seeded synthetic packings of capsules (host C++).
//
// Random sequential addition with overlap rejection, following the
// reference's "nonoverlap" populate (src/app/main.cpp:1857-2140): centres
// uniform in the periodic box, axes uniform on S^2 (cosθ ~ U[-1,1],
// φ ~ U[0,2π), main.cpp:1918-1923), the quaternion that turns +Y onto the
// axis (:1924-1932), and rejection when the closest segment distance to any
// placed rod (nearest periodic image) is below one diameter (:1933-1995).
// Velocities: v, ω ~ N(0, σ²) per component.  A splitmix64 / xoshiro256**
// generator makes the packings identical on every platform.
//
// Mass properties follow RigidBody::makeCapsule (src/physics/rigid_body.cpp:
// 11-47): m = max(1e-6, ρ π r² 2h), Ixx = Izz = m (3r² + (2h)²)/12,
// Iyy = m r²/2.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed) {
    for (int i = 0; i < 4; ++i) s[i] = splitmix(seed);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * 0x1.0p-53; }
  double normal() {  // Box-Muller
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct P3 { double x, y, z; };
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double dot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

double seg_dist2(P3 p0, P3 p1, P3 q0, P3 q1) {
  P3 e1 = sub(p1, p0), e2 = sub(q1, q0), e12 = sub(q0, p0);
  double D1 = dot(e1, e1), D2 = dot(e2, e2), S1 = dot(e1, e12), S2 = dot(e2, e12), R = dot(e1, e2);
  double den = D1 * D2 - R * R, s, t, uf;
  auto fix = [](double& u) { if (u > 1) u = 1; else if (u < 0) u = 0; };
  if (den == 0.0) {
    s = 0; t = D2 > 0 ? -S2 / D2 : 0; uf = t; fix(uf);
    if (uf != t) { s = D1 > 0 ? (uf * R + S1) / D1 : 0; fix(s); t = uf; }
  } else {
    s = (S1 * D2 - S2 * R) / den; fix(s);
    t = (s * R - S2) / D2; uf = t; fix(uf);
    if (uf != t) { s = (uf * R + S1) / D1; fix(s); t = uf; }
  }
  P3 pa{p0.x + e1.x * s, p0.y + e1.y * s, p0.z + e1.z * s};
  P3 pb{q0.x + e2.x * t, q0.y + e2.y * t, q0.z + e2.z * t};
  P3 d = sub(pb, pa);
  return dot(d, d);
}

}  // namespace

extern "C" {

// Capsule mass properties of RigidBody::makeCapsule.
void rg_capsule_mass(int n, const double* radius, const double* half_height, const double* density,
                     double* mass, double* inertia) {
  for (int i = 0; i < n; ++i) {
    double r = radius[i], h = half_height[i], L = 2.0 * h;
    double m = std::max(1e-6, density[i] * (M_PI * r * r * L));
    double Ixx = m * (3.0 * r * r + L * L) / 12.0, Iyy = m * (r * r) / 2.0;
    mass[i] = m;
    inertia[3 * i] = Ixx;
    inertia[3 * i + 1] = Iyy;
    inertia[3 * i + 2] = Ixx;
  }
}

// Places up to n rods of length L and diameter d in the periodic cube
// [lo, lo+side)^3.  Returns the number placed (stops at the first rod that
// cannot be placed within max_attempts draws).  x[3n], q[4n] (w,x,y,z).
int rg_scene_rsa(int n, double L, double d, double lo, double side, uint64_t seed, int max_attempts,
                 double* x, double* q) {
  Rng rng(seed);
  const double h = 0.5 * L;
  const double cut = L + d;  // centres farther than this cannot overlap
  int nc = std::max(1, (int)std::floor(side / cut));
  if (nc > 512) nc = 512;
  const double cs = side / nc;
  std::vector<std::vector<int>> cells((size_t)nc * nc * nc);
  std::vector<P3> C, U;
  C.reserve(n);
  U.reserve(n);
  const double d2 = d * d;
  auto cidx = [&](double v) {
    int c = (int)std::floor((v - lo) / cs);
    c %= nc;
    if (c < 0) c += nc;
    return c;
  };
  auto wrapd = [&](double v) { return v - side * std::floor(v / side + 0.5); };
  int placed = 0;
  for (int i = 0; i < n; ++i) {
    bool ok = false;
    P3 c{}, u{};
    for (int att = 0; att < max_attempts && !ok; ++att) {
      c = {lo + side * rng.uniform(), lo + side * rng.uniform(), lo + side * rng.uniform()};
      double cz = 2.0 * rng.uniform() - 1.0, ph = 6.283185307179586 * rng.uniform();
      double sn = std::sqrt(std::max(0.0, 1.0 - cz * cz));
      u = {sn * std::cos(ph), cz, sn * std::sin(ph)};
      int cx = cidx(c.x), cy = cidx(c.y), czc = cidx(c.z);
      ok = true;
      for (int dz = -1; dz <= 1 && ok && nc >= 3; ++dz)
        for (int dy = -1; dy <= 1 && ok; ++dy)
          for (int dx = -1; dx <= 1 && ok; ++dx) {
            int X = (cx + dx + nc) % nc, Y = (cy + dy + nc) % nc, Z = (czc + dz + nc) % nc;
            for (int j : cells[((size_t)Z * nc + Y) * nc + X]) {
              P3 dd{wrapd(C[j].x - c.x), wrapd(C[j].y - c.y), wrapd(C[j].z - c.z)};
              if (dot(dd, dd) > cut * cut) continue;
              P3 p0{c.x - u.x * h, c.y - u.y * h, c.z - u.z * h};
              P3 p1{c.x + u.x * h, c.y + u.y * h, c.z + u.z * h};
              P3 cj{c.x + dd.x, c.y + dd.y, c.z + dd.z};
              P3 q0{cj.x - U[j].x * h, cj.y - U[j].y * h, cj.z - U[j].z * h};
              P3 q1{cj.x + U[j].x * h, cj.y + U[j].y * h, cj.z + U[j].z * h};
              if (seg_dist2(p0, p1, q0, q1) < d2) { ok = false; break; }
            }
          }
      if (ok && nc < 3) {  // tiny box: test every placed rod
        for (int j = 0; j < placed && ok; ++j) {
          P3 dd{wrapd(C[j].x - c.x), wrapd(C[j].y - c.y), wrapd(C[j].z - c.z)};
          P3 p0{c.x - u.x * h, c.y - u.y * h, c.z - u.z * h};
          P3 p1{c.x + u.x * h, c.y + u.y * h, c.z + u.z * h};
          P3 cj{c.x + dd.x, c.y + dd.y, c.z + dd.z};
          P3 q0{cj.x - U[j].x * h, cj.y - U[j].y * h, cj.z - U[j].z * h};
          P3 q1{cj.x + U[j].x * h, cj.y + U[j].y * h, cj.z + U[j].z * h};
          if (seg_dist2(p0, p1, q0, q1) < d2) ok = false;
        }
      }
    }
    if (!ok) break;
    C.push_back(c);
    U.push_back(u);
    cells[((size_t)cidx(c.z) * nc + cidx(c.y)) * nc + cidx(c.x)].push_back(i);
    // quaternion turning +Y onto u
    double dd = std::max(-1.0, std::min(1.0, u.y));
    double ang = std::acos(dd);
    double qw = 1, qx = 0, qy = 0, qz = 0;
    if (ang >= 1e-6) {
      P3 ax{u.z, 0.0, -u.x};  // cross(+Y, u)
      double l = std::sqrt(dot(ax, ax));
      if (l > 0) {
        ax = {ax.x / l, ax.y / l, ax.z / l};
        qw = std::cos(0.5 * ang);
        double s = std::sin(0.5 * ang);
        qx = ax.x * s; qy = ax.y * s; qz = ax.z * s;
      }
    }
    x[3 * i] = c.x; x[3 * i + 1] = c.y; x[3 * i + 2] = c.z;
    q[4 * i] = qw; q[4 * i + 1] = qx; q[4 * i + 2] = qy; q[4 * i + 3] = qz;
    ++placed;
  }
  return placed;
}

// v, ω ~ N(0, sigma^2) per component.
void rg_scene_velocities(int n, double sigma_v, double sigma_w, uint64_t seed, double* v, double* w) {
  Rng rng(seed ^ 0x5DEECE66Dull);
  for (int i = 0; i < 3 * n; ++i) v[i] = sigma_v * rng.normal();
  for (int i = 0; i < 3 * n; ++i) w[i] = sigma_w * rng.normal();
}

}  // extern "C"
