// rod_oracle.cpp - FP64 CPU restatement of rod-dynamics-3d's contact hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
// only as the checker or the timed CPU baseline.  The product (librodgpu.so)
// never links or calls it.
//
// It restates, single-threaded and in double precision, the reference
// functions named in each comment (paths relative to the reference repo).
// Where the reference computes in float, this file computes the same formula
// in double.  Two documented extensions follow the reference's own law:
//   * Hertz-Mindlin is applied to capsule contacts from the capsule narrow
//     phase (the reference's HertzMindlinSolver is sphere-only,
//     src/physics/hertz_mindlin.cpp:101-144), with the minimum-image shift of
//     ContactDetector and r x F torques of the total contact force.
//   * PSOR can run in the device's graph-coloured order: the sequential
//     Gauss-Seidel of nsc_contact.cpp:385-552 applied to the manifolds
//     permuted colour-major.  Contacts of one colour share no dynamic body,
//     so this equals the parallel sweep bit for bit.
//
// Pinning: checked against the reference's own sources compiled here
// (oracle/ref_harness.cpp, FP32) and against the reference's smoke-test
// known answers (tests/smoke_test.py:165-233) in tests/test_oracle_pin.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "../include/rodgpu.h"

namespace {

struct V3 {
  double x, y, z;
};
inline V3 v3(double x, double y, double z) { return {x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
inline V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double length(V3 a) { return std::sqrt(dot(a, a)); }
inline double comp(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
inline void setcomp(V3& a, int k, double v) { (k == 0 ? a.x : (k == 1 ? a.y : a.z)) = v; }

struct Q {
  double w, x, y, z;
};
// Hamilton product a*b.
inline Q qmul(Q a, Q b) {
  return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
          a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
          a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
          a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
inline Q qnormalize(Q q) {
  double len = std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  if (len <= 0.0) return {1, 0, 0, 0};
  double inv = 1.0 / len;
  return {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
}
// Rotation of `angle` about unit `axis` (glm::angleAxis semantics).
inline Q angle_axis(double angle, V3 axis) {
  double h = 0.5 * angle;
  double s = std::sin(h);
  return {std::cos(h), axis.x * s, axis.y * s, axis.z * s};
}
// Columns of the rotation matrix of q (glm::mat3_cast; rigid_body.cpp:112-114).
// col1 is RigidBody::axisY (rigid_body.cpp:137-139).
inline void rot_cols(Q q, V3& c0, V3& c1, V3& c2) {
  double qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
  double qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
  double qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
  c0 = {1.0 - 2.0 * (qyy + qzz), 2.0 * (qxy + qwz), 2.0 * (qxz - qwy)};
  c1 = {2.0 * (qxy - qwz), 1.0 - 2.0 * (qxx + qzz), 2.0 * (qyz + qwx)};
  c2 = {2.0 * (qxz + qwy), 2.0 * (qyz - qwx), 1.0 - 2.0 * (qxx + qyy)};
}
inline V3 axis_y(Q q) {
  double qxx = q.x * q.x, qzz = q.z * q.z;
  double qxy = q.x * q.y, qyz = q.y * q.z;
  double qwx = q.w * q.x, qwz = q.w * q.z;
  return {2.0 * (qxy - qwz), 1.0 - 2.0 * (qxx + qzz), 2.0 * (qyz + qwx)};
}
// R * diag(d) * R^T * v, evaluated as R (d .* (R^T v)).  Used for
// IworldInv (rigid_body.cpp:116-121) and the world inertia Iw
// (integrator.cpp:39-54).
inline V3 rot_diag_apply(Q q, V3 d, V3 v) {
  V3 c0, c1, c2;
  rot_cols(q, c0, c1, c2);
  double b0 = dot(c0, v) * d.x, b1 = dot(c1, v) * d.y, b2 = dot(c2, v) * d.z;
  return c0 * b0 + c1 * b1 + c2 * b2;
}

struct Body {
  double r = 0.05, h = 0.5, mass = 1, inv_mass = 1, restitution = 0.2;
  V3 I{1, 1, 1}, Iinv{1, 1, 1};
};

struct Contact {
  int a, b, type;
  V3 pa, pb, n, shift;
  double distance, surface_limit;
  double s, t;
};

struct Manifold {  // NscManifold (include/physics/nsc_contact.hpp:37-63)
  int a, b;
  V3 n, t1, t2, ra, rb;
  double phi;
  V3 v_rel_pre;
  double v_n_pre, restitution;
  double g_n, g_t1, g_t2;
  V3 IA_n, IA_t1, IA_t2, IB_n, IB_t1, IB_t2;
  double invMA, invMB;
  double ln = 0, lt1 = 0, lt2 = 0;
  int color = 0;
  bool wall = false;  // cylinder wall contact of body a (b == a), isWall
};

inline uint64_t pair_key(int a, int b) {
  if (a > b) std::swap(a, b);
  return (uint64_t(uint32_t(a)) << 32) | uint64_t(uint32_t(b));
}

struct HistEntry {
  V3 value{0, 0, 0};
  int64_t last_frame = 0;
};

// Deterministic contact priority for the Jones-Plassmann colouring; the
// device computes the same function.
inline uint64_t jp_priority(uint32_t c) {
  uint32_t h = c * 0x9E3779B1u;
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return (uint64_t(h) << 32) | uint64_t(c);
}

}  // namespace

struct orc_system {
  rg_config cfg;
  int n = 0;
  std::vector<Body> body;
  std::vector<V3> x, v, w, f, tau;
  std::vector<Q> q;
  V3 pbc_min{0, 0, 0}, pbc_max{0, 0, 0}, pbc_size{0, 0, 0};
  bool pbc = false;

  // Soft (Cundall) history: never pruned (soft_contact.hpp:96-102; the
  // declared pruneContactHistory at :83 has no definition).
  std::map<uint64_t, HistEntry> soft_hist;
  int64_t soft_frame = 0;
  // HM history with 4-frame retention (hertz_mindlin.hpp:143, .cpp:385-393).
  std::map<uint64_t, HistEntry> hm_hist;
  int64_t hm_frame = 0;
  // NSC warm cache (nsc_contact.hpp:178-188).
  std::map<uint64_t, V3> warm;

  std::vector<Manifold> manifolds;  // last velocity solve, sorted (a,b) order
  double last_residual = 0, last_pe = 0;
  int last_sweeps = 0, last_colors = 0;
  int64_t last_contacts = 0, last_collisions = 0;
  double jn_sum = 0, jt_sum = 0;
};

namespace {

// ---------------------------------------------------------------------------
// Narrow phase: ContactDetector::detectCapsuleCapsule (contact_detector.cpp:
// 811-910) with closestPointsSegmentSegment (:978-1035), in double.
// ---------------------------------------------------------------------------
void lumelsky(V3 a1, V3 a2, V3 b1, V3 b2, double& s, double& t) {
  V3 e1 = a2 - a1, e2 = b2 - b1, e12 = b1 - a1;
  double D1 = dot(e1, e1), D2 = dot(e2, e2);
  double S1 = dot(e1, e12), S2 = dot(e2, e12), R = dot(e1, e2);
  double den = D1 * D2 - R * R;
  auto fix = [](double& u) -> bool {
    if (u > 1.0) { u = 1.0; return true; }
    if (u < 0.0) { u = 0.0; return true; }
    return false;
  };
  double uf;
  if (den == 0.0) {
    s = 0.0;
    t = -S2 / D2;
    uf = t;
    fix(uf);
    if (uf != t) { s = (uf * R + S1) / D1; fix(s); t = uf; }
  } else {
    s = (S1 * D2 - S2 * R) / den;
    fix(s);
    t = (s * R - S2) / D2;
    uf = t;
    fix(uf);
    if (uf != t) { s = (uf * R + S1) / D1; fix(s); t = uf; }
  }
}

V3 min_image_shift(const orc_system& S, V3 xa, V3 xb) {
  V3 sh{0, 0, 0};
  if (!S.pbc) return sh;
  V3 d = xb - xa;
  for (int k = 0; k < 3; ++k) {
    double L = comp(S.pbc_size, k);
    if (L > 0.0) {
      double m = std::floor(comp(d, k) / L + 0.5);
      setcomp(sh, k, -(m * L));
    }
  }
  return sh;
}

bool narrow(const orc_system& S, int ia, int ib, double delta, Contact& c) {
  const Body& A = S.body[ia];
  const Body& B = S.body[ib];
  V3 ua = axis_y(S.q[ia]), ub = axis_y(S.q[ib]);
  V3 a1 = S.x[ia] - ua * A.h, a2 = S.x[ia] + ua * A.h;
  V3 b1 = S.x[ib] - ub * B.h, b2 = S.x[ib] + ub * B.h;
  V3 sh = min_image_shift(S, S.x[ia], S.x[ib]);
  b1 = b1 + sh;
  b2 = b2 + sh;
  double hsum = A.r + B.r;
  double s, t;
  lumelsky(a1, a2, b1, b2, s, t);
  V3 pa = a1 + (a2 - a1) * s;
  V3 pb = b1 + (b2 - b1) * t;
  V3 diff = pb - pa;
  double d2 = dot(diff, diff);
  double act = hsum + delta;
  if (!(d2 < act * act)) return false;
  double dist = std::sqrt(d2);
  const double eps = 1e-6;
  int type;
  if (s < eps && t < eps) type = 0;
  else if (s > 1.0 - eps && t > 1.0 - eps) type = 0;
  else if (s < eps || s > 1.0 - eps) type = 1;
  else if (t < eps || t > 1.0 - eps) type = 1;
  else type = 2;
  c.a = ia; c.b = ib; c.type = type;
  c.pa = pa; c.pb = pb; c.shift = sh;
  c.distance = dist; c.surface_limit = hsum;
  c.s = s; c.t = t;
  c.n = dist > 1e-10 ? diff / dist : v3(1, 0, 0);
  return true;
}

// Contact set of ContactDetector::detectContacts (contact_detector.cpp:71-
// 211): every pair a < b, not both static, whose narrow phase fires, sorted by
// (a,b) as sortedContactOrder does (nsc_contact.cpp:91-102).  Candidate pairs
// come from a centre grid whose cell is at least the largest possible
// contacting centre distance, so the set equals the all-pairs loop of
// detectContactsNaive (:213-281).
std::vector<Contact> detect(const orc_system& S, double delta) {
  std::vector<Contact> out;
  const int n = S.n;
  if (n < 2) return out;
  double maxext = 0;
  for (int i = 0; i < n; ++i) maxext = std::max(maxext, S.body[i].h + S.body[i].r);
  double cut = 2.0 * maxext + delta;
  cut = cut * (1.0 + 1e-12) + 1e-12;
  // Two conservative prefilters skip the narrow phase of pairs that cannot
  // touch; neither changes the set.  (1) Centre distance: the segment
  // distance is at least |dc| - h_a - h_b.  (2) Axis-line distance: the
  // distance of the two infinite lines is a lower bound of the segment
  // distance.  Both reject only beyond the activation distance plus a
  // relative 1e-9 and absolute 1e-12 margin, far above their rounding error.
  std::vector<V3> axis(n);
  for (int i = 0; i < n; ++i) axis[i] = axis_y(S.q[i]);
  auto test = [&](int i, int j) {
    if (S.body[i].inv_mass <= 0.0 && S.body[j].inv_mass <= 0.0) return;
    const Body& A = S.body[i];
    const Body& B = S.body[j];
    V3 dc = (S.x[j] + min_image_shift(S, S.x[i], S.x[j])) - S.x[i];
    const double act = A.r + B.r + delta;
    const double cc = A.h + B.h + act;
    if (dot(dc, dc) > cc * cc * (1.0 + 1e-9) + 1e-12) return;
    V3 cr = cross(axis[i], axis[j]);
    double c2 = dot(cr, cr);
    if (c2 > 1e-6) {
      double proj = dot(dc, cr);
      if (proj * proj > (act * act * (1.0 + 1e-9) + 1e-12) * c2) return;
    }
    Contact c;
    if (narrow(S, i, j, delta, c)) out.push_back(c);
  };
  bool brute = (n <= 1500);
  int dims[3] = {1, 1, 1};
  V3 lo{0, 0, 0};
  double cell[3] = {1, 1, 1};
  if (!brute) {
    V3 hi;
    if (S.pbc) {
      lo = S.pbc_min; hi = S.pbc_max;
    } else {
      lo = S.x[0]; hi = S.x[0];
      for (int i = 1; i < n; ++i) {
        lo = v3(std::min(lo.x, S.x[i].x), std::min(lo.y, S.x[i].y), std::min(lo.z, S.x[i].z));
        hi = v3(std::max(hi.x, S.x[i].x), std::max(hi.y, S.x[i].y), std::max(hi.z, S.x[i].z));
      }
    }
    for (int k = 0; k < 3; ++k) {
      double span = comp(hi, k) - comp(lo, k);
      int d = (int)std::floor(span / cut);
      d = std::max(1, std::min(d, 256));
      dims[k] = d;
      cell[k] = span > 0 ? span / d : 1.0;
    }
    if (S.pbc) {
      for (int k = 0; k < 3; ++k)
        if (dims[k] < 3) brute = true;  // tiny box: all pairs
    }
  }
  if (brute) {
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) test(i, j);
  } else {
    auto cidx = [&](V3 p, int k) {
      int c = (int)std::floor((comp(p, k) - comp(lo, k)) / cell[k]);
      if (S.pbc) {
        c %= dims[k];
        if (c < 0) c += dims[k];
      } else {
        c = std::max(0, std::min(c, dims[k] - 1));
      }
      return c;
    };
    std::vector<std::vector<int>> cells((size_t)dims[0] * dims[1] * dims[2]);
    std::vector<int> ci(n);
    for (int i = 0; i < n; ++i) {
      int cx = cidx(S.x[i], 0), cy = cidx(S.x[i], 1), cz = cidx(S.x[i], 2);
      ci[i] = (cz * dims[1] + cy) * dims[0] + cx;
      cells[ci[i]].push_back(i);
    }
    std::vector<int> cand;
    for (int i = 0; i < n; ++i) {
      int cx = ci[i] % dims[0], cy = (ci[i] / dims[0]) % dims[1], cz = ci[i] / (dims[0] * dims[1]);
      cand.clear();
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int X = cx + dx, Y = cy + dy, Z = cz + dz;
            if (S.pbc) {
              X = (X + dims[0]) % dims[0]; Y = (Y + dims[1]) % dims[1]; Z = (Z + dims[2]) % dims[2];
            } else if (X < 0 || Y < 0 || Z < 0 || X >= dims[0] || Y >= dims[1] || Z >= dims[2]) {
              continue;
            }
            for (int j : cells[(Z * dims[1] + Y) * dims[0] + X])
              if (j > i) cand.push_back(j);
          }
      // the 27 cells are distinct (every dimension has at least 3 cells
      // here), so no candidate repeats; the contacts are sorted below
      for (int j : cand) test(i, j);
    }
  }
  std::sort(out.begin(), out.end(), [](const Contact& p, const Contact& r) {
    return p.a != r.a ? p.a < r.a : p.b < r.b;
  });
  return out;
}

// ---------------------------------------------------------------------------
// Soft penalty contact: SoftContactSolver::computeForces (soft_contact.cpp:
// 80-213), potentialGradient / potentialEnergy (:215-253), computeFriction
// (:288-486).
// ---------------------------------------------------------------------------
double soft_grad(const rg_config& c, double d, double h) {
  double K1 = 15.0 / c.soft_delta;
  if (d > h - c.soft_delta) {
    double arg = K1 * (h - d);
    double e = std::exp(arg);
    double lt = std::log(1.0 + e);
    return -2.0 / (K1 * K1) * lt * e / (1.0 + e);
  }
  return -2.0 * (h - d);
}
double soft_energy(const rg_config& c, double d, double h) {
  double K1 = 15.0 / c.soft_delta;
  if (d > h - c.soft_delta) {
    double arg = K1 * (h - d);
    double lt = std::log(1.0 + std::exp(arg));
    double base = lt / K1;
    return base * base;
  }
  double pen = h - d;
  return pen * pen;
}

void soft_forces(orc_system& S, const std::vector<Contact>& cs) {
  const rg_config& c = S.cfg;
  const double dt = c.dt;
  double pe = 0;
  S.soft_frame++;
  for (const Contact& ct : cs) {
    double grad = soft_grad(c, ct.distance, ct.surface_limit);
    double fm = -c.soft_k_scaler * grad;
    V3 fa = ct.n * (-fm);
    V3 fb = ct.n * fm;
    V3 ra = ct.pa - S.x[ct.a];
    V3 rb = ct.pb - (S.x[ct.b] + ct.shift);
    V3 va = S.v[ct.a] + cross(S.w[ct.a], ra);
    V3 vb = S.v[ct.b] + cross(S.w[ct.b], rb);
    V3 vrel = va - vb;
    if (c.soft_damping > 1e-9) {
      double vn = dot(vrel, ct.n);
      V3 fd = ct.n * (-c.soft_damping * vn);
      fa += fd;
      fb -= fd;
    }
    V3 fra{0, 0, 0};
    if (c.soft_enable_friction) {
      double fn_mag = length(fa);
      V3 vt = vrel - ct.n * dot(vrel, ct.n);
      double vt_mag = length(vt);
      if (!(vt_mag < 1e-10)) {
        if (c.soft_friction_mode == RG_FRICTION_CUNDALL) {
          HistEntry& e = S.soft_hist[pair_key(ct.a, ct.b)];
          V3 ft = e.value - vt * (c.soft_kt * dt);
          double nc = dot(ft, ct.n);
          ft = ft - ct.n * nc;
          double ftm = length(ft);
          double lim = c.soft_mu * fn_mag;
          if (ftm > lim) {
            if (ftm > 1e-8) ft = ft * (lim / ftm);
            else ft = v3(0, 0, 0);
          }
          e.value = ft;
          e.last_frame = S.soft_frame;
          fra = ft;
        } else if (c.soft_friction_mode == RG_FRICTION_KARNOPP) {
          const Body& A = S.body[ct.a];
          const Body& B = S.body[ct.b];
          if (vt_mag < c.soft_vel_deadband) {
            double ma = A.inv_mass > 0 ? A.mass : 0.0;
            double mb = B.inv_mass > 0 ? B.mass : 0.0;
            double meff = 0;
            if (ma > 0 && mb > 0) meff = (ma * mb) / (ma + mb);
            else if (ma > 0) meff = ma;
            else if (mb > 0) meff = mb;
            V3 fstop = vt * (-(meff / dt));
            V3 g = v3(c.gravity[0], c.gravity[1], c.gravity[2]);
            V3 gt = g - ct.n * dot(g, ct.n);
            V3 fdrive = gt * meff;
            V3 freq = fstop - fdrive;
            double frm = length(freq);
            double maxs = c.soft_mu_static * fn_mag;
            if (frm <= maxs) fra = freq;
            else if (frm > 1e-12) fra = freq * (maxs / frm);
          } else {
            fra = (vt * -1.0 / vt_mag) * (c.soft_mu * fn_mag);
          }
        } else {
          double K2 = 15.0 / c.soft_nu;
          double gamma = vt_mag > c.soft_nu ? 1.0 : 2.0 / (1.0 + std::exp(-K2 * vt_mag)) - 1.0;
          double mu_eff = c.soft_mu;
          if (c.soft_mu_static > c.soft_mu)
            mu_eff = c.soft_mu + (c.soft_mu_static - c.soft_mu) * std::exp(-vt_mag / c.soft_nu);
          V3 dir = (-vt) / vt_mag;
          fra = dir * (mu_eff * gamma * fn_mag);
        }
      }
    }
    V3 ta = fa + fra, tb = fb - fra;
    S.f[ct.a] += ta;
    S.f[ct.b] += tb;
    S.tau[ct.a] += cross(ra, ta);
    S.tau[ct.b] += cross(rb, tb);
    pe += c.soft_k_scaler * soft_energy(c, ct.distance, ct.surface_limit);
  }
  S.last_pe = pe;
}

// ---------------------------------------------------------------------------
// Hertz-Mindlin on capsule contacts: computeForces (hertz_mindlin.cpp:183-
// 247), computeHertzForce (:249-287), computeMindlinForce (:289-354),
// computeRollingFriction (:356-383), pruneContactHistory (:385-393); damping
// from restitution (include/config/config.hpp:54-63).
// ---------------------------------------------------------------------------
double hm_gamma(double e) {
  if (e >= 1.0) return 0.0;
  double l = std::log(e);
  return -l / std::sqrt(M_PI * M_PI + l * l);
}

void hm_forces(orc_system& S, const std::vector<Contact>& cs) {
  const rg_config& c = S.cfg;
  const double dt = c.dt;
  const double nu = c.hm_poisson_ratio;
  const double Es = c.hm_youngs_modulus / (2.0 * (1.0 - nu * nu));
  const double Gs = c.hm_youngs_modulus / (2.0 * (1.0 + nu));
  const double gam = hm_gamma(c.hm_restitution);
  double pe = 0;
  for (const Contact& ct : cs) {
    const Body& A = S.body[ct.a];
    const Body& B = S.body[ct.b];
    HistEntry& st = S.hm_hist[pair_key(ct.a, ct.b)];
    double delta = ct.surface_limit - ct.distance;
    double Rs = (A.r * B.r) / (A.r + B.r);
    double ms = (A.mass * B.mass) / (A.mass + B.mass);
    double sd = std::max(delta, 0.0);
    double sqd = std::sqrt(sd);
    double sqR = std::sqrt(std::max(Rs, 0.0));
    double kn = (4.0 / 3.0) * Es * sqR * sqd;
    double Fel = kn * sd * sqd;
    V3 ra = ct.pa - S.x[ct.a];
    V3 rb = ct.pb - (S.x[ct.b] + ct.shift);
    V3 va = S.v[ct.a] + cross(S.w[ct.a], ra);
    V3 vb = S.v[ct.b] + cross(S.w[ct.b], rb);
    V3 vrel = vb - va;
    double vn = dot(vrel, ct.n);
    double Cn = gam * 2.0 * std::sqrt(ms * kn);
    double Fn = std::max(0.0, Fel + (-Cn * vn));
    V3 fn = ct.n * Fn;
    V3 ft{0, 0, 0};
    if (c.hm_enable_tangential) {
      double kt = 8.0 * Gs * sqR * sqd;
      V3 vt = vrel - ct.n * vn;
      st.value = st.value + vt * dt;
      V3 fel = st.value * (-kt);
      double Ct = gam * 2.0 * std::sqrt(ms * kt);
      ft = fel - vt * Ct;
      double vtm = length(vt);
      double mu_eff = c.hm_friction;
      if (c.hm_friction_static > c.hm_friction && c.hm_friction_transition_vel > 0.0)
        mu_eff += (c.hm_friction_static - c.hm_friction) * std::exp(-vtm / c.hm_friction_transition_vel);
      double fnm = length(fn);
      double ftm = length(ft);
      double ftmax = mu_eff * fnm;
      if (ftm > ftmax && ftm > 1e-10) {
        ft = ft * (ftmax / ftm);
        if (kt > 1e-10) st.value = ft / (-kt);
      }
    }
    V3 tra{0, 0, 0}, trb{0, 0, 0};
    if (c.hm_enable_rolling) {
      V3 wr = S.w[ct.a] - S.w[ct.b];
      double wm = length(wr);
      if (!(wm < 1e-10)) {
        V3 wh = wr / wm;
        double trm = c.hm_rolling_friction * Rs * length(fn);
        V3 tr = wh * (-trm);
        tra = tr * 0.5;
        trb = tr * -0.5;
      }
    }
    V3 F = fn + ft;
    S.f[ct.a] -= F;
    S.f[ct.b] += F;
    S.tau[ct.a] += cross(ra, -F) + tra;
    S.tau[ct.b] += cross(rb, F) + trb;
    pe += (8.0 / 15.0) * Es * std::sqrt(Rs) * std::pow(delta, 2.5);
    st.last_frame = S.hm_frame;
  }
  // pruneContactHistory: drop entries untouched for more than 4 frames.
  for (auto it = S.hm_hist.begin(); it != S.hm_hist.end();) {
    if (S.hm_frame - it->second.last_frame > 4 || it->second.last_frame == 0) it = S.hm_hist.erase(it);
    else ++it;
  }
  S.last_pe = pe;
}

// One force evaluation at the current state: detect + computeForces.
// Cylinder wall of the soft model: penalty spring on the centre's radial
// overshoot plus smooth Coulomb friction, forces only (main.cpp:4661-4690 at
// phase t, :4756-4787 at phase t + dt).
void soft_wall_forces(orc_system& S) {
  const rg_config& c = S.cfg;
  if (!c.cylinder_enabled) return;
  V3 ax = v3(c.cylinder_axis[0], c.cylinder_axis[1], c.cylinder_axis[2]);
  ax = ax / length(ax);
  const double k = c.soft_k_scaler, cd = c.soft_damping, mu = c.soft_mu;
  const double nu = std::max(c.soft_nu, 1e-10);
  for (int i = 0; i < S.n; ++i) {
    const Body& B = S.body[i];
    if (!(B.inv_mass > 0.0)) continue;
    const double maxd = c.cylinder_radius - B.r;
    V3 pp = S.x[i] - ax * dot(S.x[i], ax);
    double d = length(pp);
    double pen = d - maxd;
    if (pen <= 0.0) continue;
    V3 n;
    if (d > 1e-8) {
      n = pp / d;
    } else {
      V3 cr = cross(ax, std::fabs(ax.x) < 0.9 ? v3(1, 0, 0) : v3(0, 1, 0));
      n = cr / length(cr);
    }
    double vn = dot(S.v[i], n);
    double fn = k * pen + cd * std::max(vn, 0.0);
    S.f[i] -= n * fn;
    V3 vt = S.v[i] - n * vn;
    double vtl = length(vt);
    if (vtl > 1e-12) S.f[i] -= vt * (mu * fn * std::tanh(vtl / nu) / vtl);
  }
}

void force_eval(orc_system& S) {
  if (S.cfg.model == RG_MODEL_HARMONIC) {
    auto cs = detect(S, S.cfg.soft_delta);
    S.last_contacts = (int64_t)cs.size();
    soft_forces(S, cs);
    soft_wall_forces(S);
  } else if (S.cfg.model == RG_MODEL_HERTZ_MINDLIN) {
    S.hm_frame++;  // frame_counter_ advances per detectContacts (:31)
    auto cs = detect(S, 0.0);
    S.last_contacts = (int64_t)cs.size();
    hm_forces(S, cs);
  }
}

// ---------------------------------------------------------------------------
// Integrators: integrateHalfPos / integrateSecondHalf (integrator.cpp:113-
// 159), angularAccelGyro (:39-54), wrap_position (:23-35).
// ---------------------------------------------------------------------------
void wrap(const orc_system& S, V3& p) {
  for (int k = 0; k < 3; ++k) {
    double L = comp(S.pbc_size, k);
    if (L <= 0.0) continue;
    double lo = comp(S.pbc_min, k), hi = comp(S.pbc_max, k);
    double x = comp(p, k);
    while (x < lo) x += L;
    while (x >= hi) x -= L;
    setcomp(p, k, x);
  }
}

V3 ang_accel(const orc_system& S, int i) {
  const Body& B = S.body[i];
  if (B.inv_mass <= 0.0) return {0, 0, 0};
  V3 Iw_w = rot_diag_apply(S.q[i], B.I, S.w[i]);
  V3 gyro = cross(S.w[i], Iw_w);
  return rot_diag_apply(S.q[i], B.Iinv, S.tau[i] - gyro);
}

void rotate_by_omega(Q& q, V3 w, double dt) {
  double wl = length(w);
  if (wl > 1e-8) {
    double ang = wl * dt;
    V3 ax = w / wl;
    q = qnormalize(qmul(angle_axis(ang, ax), q));
  }
}

void half_pos(orc_system& S) {
  const rg_config& c = S.cfg;
  V3 g = v3(c.gravity[0], c.gravity[1], c.gravity[2]);
  double hdt = 0.5 * c.dt;
  for (int i = 0; i < S.n; ++i) {
    const Body& B = S.body[i];
    if (B.inv_mass <= 0.0) continue;
    V3 al = S.f[i] / B.mass + g;
    V3 aa = ang_accel(S, i);
    S.v[i] += al * hdt;
    S.w[i] += aa * hdt;
    S.x[i] += S.v[i] * c.dt;
    if (S.pbc) wrap(S, S.x[i]);
    rotate_by_omega(S.q[i], S.w[i], c.dt);
  }
}

void second_half(orc_system& S) {
  const rg_config& c = S.cfg;
  V3 g = v3(c.gravity[0], c.gravity[1], c.gravity[2]);
  double hdt = 0.5 * c.dt;
  double el = std::exp(-c.lin_damp * c.dt), ea = std::exp(-c.ang_damp * c.dt);
  for (int i = 0; i < S.n; ++i) {
    const Body& B = S.body[i];
    if (B.inv_mass <= 0.0) continue;
    V3 al = S.f[i] / B.mass + g;
    V3 aa = ang_accel(S, i);
    S.v[i] += al * hdt;
    S.w[i] += aa * hdt;
    if (c.lin_damp > 0.0) S.v[i] = S.v[i] * el;
    if (c.ang_damp > 0.0) S.w[i] = S.w[i] * ea;
    double wl = length(S.w[i]);
    if (wl > c.w_max) S.w[i] = S.w[i] * (c.w_max / wl);
  }
}

// Velocity-Verlet step of App::physicsStep for the soft and HM branches
// (main.cpp:4529-4609 and :4610-4810) with random forces and sleep disabled.
// Both evaluations start from zero forces: integrateSecondHalf clears them
// for the next frame (integrator.cpp:156-158) and the step clears them
// before the second evaluation.  The forces at t + dt are left in f and tau
// (the library's state after a step reports them).
void verlet_step(orc_system& S) {
  for (int i = 0; i < S.n; ++i) { S.f[i] = v3(0, 0, 0); S.tau[i] = v3(0, 0, 0); }
  force_eval(S);
  half_pos(S);
  for (int i = 0; i < S.n; ++i) { S.f[i] = v3(0, 0, 0); S.tau[i] = v3(0, 0, 0); }
  force_eval(S);
  second_half(S);
}

// ---------------------------------------------------------------------------
// NSC: colouring, manifold build, PSOR, position projection and the
// semi-implicit step (main.cpp:4383-4528).
// ---------------------------------------------------------------------------

// Jones-Plassmann first-fit colouring of contacts; contacts conflict when
// they share a dynamic body.  Round by round: an uncoloured contact whose
// priority beats every uncoloured neighbour takes the smallest colour no
// coloured neighbour uses.  Returns the colour count (-1 if > 64 colours).
int jp_color(const orc_system& S, const std::vector<int>& ca, const std::vector<int>& cb,
             std::vector<int>& color) {
  const int C = (int)ca.size();
  color.assign(C, -1);
  if (C == 0) return 0;
  std::vector<std::vector<int>> inc(S.n);
  for (int c = 0; c < C; ++c) {
    if (S.body[ca[c]].inv_mass > 0.0) inc[ca[c]].push_back(c);
    if (S.body[cb[c]].inv_mass > 0.0) inc[cb[c]].push_back(c);
  }
  int left = C, ncol = 0;
  std::vector<int> sel;
  while (left > 0) {
    sel.clear();
    for (int c = 0; c < C; ++c) {
      if (color[c] >= 0) continue;
      uint64_t pc = jp_priority((uint32_t)c);
      bool best = true;
      for (int side = 0; side < 2 && best; ++side) {
        int bd = side ? cb[c] : ca[c];
        if (S.body[bd].inv_mass <= 0.0) continue;
        for (int o : inc[bd]) {
          if (o == c || color[o] >= 0) continue;
          if (jp_priority((uint32_t)o) > pc) { best = false; break; }
        }
      }
      if (best) sel.push_back(c);
    }
    for (int c : sel) {
      uint64_t used = 0;
      for (int side = 0; side < 2; ++side) {
        int bd = side ? cb[c] : ca[c];
        if (S.body[bd].inv_mass <= 0.0) continue;
        for (int o : inc[bd])
          if (o != c && color[o] >= 0 && color[o] < 64) used |= (1ull << color[o]);
      }
      int k = 0;
      while (k < 64 && (used >> k) & 1ull) ++k;
      if (k >= 64) return -1;
      color[c] = k;
      ncol = std::max(ncol, k + 1);
    }
    left -= (int)sel.size();
  }
  return ncol;
}

// Order in which PSOR visits contacts: sorted (a,b) order of the reference,
// or colour-major with the sorted order inside a colour.
std::vector<int> visit_order(int C, const std::vector<int>& color, bool colored) {
  std::vector<int> ord(C);
  for (int i = 0; i < C; ++i) ord[i] = i;
  if (colored)
    std::stable_sort(ord.begin(), ord.end(), [&](int p, int r) { return color[p] < color[r]; });
  return ord;
}

V3 iinv_apply(const orc_system& S, int i, V3 v) {
  const Body& B = S.body[i];
  if (B.inv_mass <= 0.0) return {0, 0, 0};
  return rot_diag_apply(S.q[i], B.Iinv, v);
}

// computeDiag (nsc_contact.cpp:106-117).
double diag(const orc_system& S, int a, int b, V3 ra, V3 rb, V3 d, double cfm) {
  V3 rad = cross(ra, d), rbd = cross(rb, d);
  double g = S.body[a].inv_mass + S.body[b].inv_mass + dot(rad, iinv_apply(S, a, rad)) +
             dot(rbd, iinv_apply(S, b, rbd)) + cfm;
  return std::max(g, 1e-12);
}

// buildTangentBasis (nsc_contact.cpp:78-85).
void tangent_basis(V3 n, V3& t1, V3& t2) {
  V3 ref = std::fabs(n.x) < 0.9 ? v3(1, 0, 0) : v3(0, 1, 0);
  V3 c = cross(n, ref);
  t1 = c / length(c);
  t2 = cross(n, t1);
}

// detectAndBuildManifolds (nsc_contact.cpp:239-321).
void build_manifolds(orc_system& S, const std::vector<Contact>& cs) {
  const rg_config& c = S.cfg;
  S.manifolds.clear();
  S.manifolds.reserve(cs.size());
  for (const Contact& ct : cs) {
    Manifold m;
    m.a = ct.a; m.b = ct.b;
    m.n = ct.n;
    m.phi = ct.distance - ct.surface_limit;
    tangent_basis(m.n, m.t1, m.t2);
    m.ra = ct.pa - S.x[ct.a];
    m.rb = ct.pb - (S.x[ct.b] + ct.shift);
    m.g_n = diag(S, m.a, m.b, m.ra, m.rb, m.n, c.nsc_cfm);
    m.g_t1 = diag(S, m.a, m.b, m.ra, m.rb, m.t1, c.nsc_cfm);
    m.g_t2 = diag(S, m.a, m.b, m.ra, m.rb, m.t2, c.nsc_cfm);
    m.invMA = S.body[m.a].inv_mass;
    m.invMB = S.body[m.b].inv_mass;
    m.IA_n = iinv_apply(S, m.a, cross(m.ra, m.n));
    m.IA_t1 = iinv_apply(S, m.a, cross(m.ra, m.t1));
    m.IA_t2 = iinv_apply(S, m.a, cross(m.ra, m.t2));
    m.IB_n = iinv_apply(S, m.b, cross(m.rb, m.n));
    m.IB_t1 = iinv_apply(S, m.b, cross(m.rb, m.t1));
    m.IB_t2 = iinv_apply(S, m.b, cross(m.rb, m.t2));
    m.v_rel_pre = (S.v[m.b] + cross(S.w[m.b], m.rb)) - (S.v[m.a] + cross(S.w[m.a], m.ra));
    m.v_n_pre = dot(m.n, m.v_rel_pre);
    m.restitution = std::min(S.body[m.a].restitution, S.body[m.b].restitution);
    m.ln = m.lt1 = m.lt2 = 0;
    if (c.nsc_warm_start == RG_WARM_CACHE) {
      auto it = S.warm.find(pair_key(m.a, m.b));
      if (it != S.warm.end()) {
        m.ln = std::max(0.0, it->second.x);
        m.lt1 = it->second.y;
        m.lt2 = it->second.z;
      }
    }
    S.manifolds.push_back(m);
  }
}

// Wall manifolds of the cylindrical tube (collideCapsuleInsideCylinder,
// collision.cpp:197-241, for each dynamic capsule, main.cpp:4431-4447;
// NscContactSolver::addWallContact, nsc_contact.cpp:190-235): for the two
// end points and the centre of the axis, a contact where the capsule surface
// passes the tube wall; appended after the pair manifolds, in body order.
void add_wall_manifolds(orc_system& S) {
  const rg_config& c = S.cfg;
  if (!c.cylinder_enabled) return;
  V3 ax = v3(c.cylinder_axis[0], c.cylinder_axis[1], c.cylinder_axis[2]);
  ax = ax / length(ax);
  const double R = c.cylinder_radius;
  for (int i = 0; i < S.n; ++i) {
    const Body& B = S.body[i];
    if (!(B.inv_mass > 0.0)) continue;
    V3 u = axis_y(S.q[i]);
    u = u / length(u);
    const V3 pts[3] = {S.x[i] - u * B.h, S.x[i], S.x[i] + u * B.h};
    for (const V3& p : pts) {
      V3 pp = p - ax * dot(p, ax);
      double d = length(pp);
      double pen = d + B.r - R;
      if (pen <= 0.0) continue;
      Manifold m;
      m.a = m.b = i;
      m.wall = true;
      if (d > 1e-8) {
        m.n = pp / d;
      } else {
        V3 arb = std::fabs(ax.x) < 0.9 ? v3(1, 0, 0) : v3(0, 1, 0);
        V3 cr = cross(ax, arb);
        m.n = cr / length(cr);
      }
      V3 point = p + m.n * (R - d);
      m.phi = -pen;
      tangent_basis(m.n, m.t1, m.t2);
      m.ra = point - S.x[i];
      m.rb = v3(0, 0, 0);
      // computeDiagWall (nsc_contact.cpp:144-150)
      auto gw = [&](V3 dir) {
        V3 rd = cross(m.ra, dir);
        return std::max(B.inv_mass + dot(rd, iinv_apply(S, i, rd)) + c.nsc_cfm, 1e-12);
      };
      m.g_n = gw(m.n);
      m.g_t1 = gw(m.t1);
      m.g_t2 = gw(m.t2);
      m.invMA = B.inv_mass;
      m.invMB = 0.0;
      m.IA_n = iinv_apply(S, i, cross(m.ra, m.n));
      m.IA_t1 = iinv_apply(S, i, cross(m.ra, m.t1));
      m.IA_t2 = iinv_apply(S, i, cross(m.ra, m.t2));
      m.IB_n = m.IB_t1 = m.IB_t2 = v3(0, 0, 0);
      m.v_rel_pre = -(S.v[i] + cross(S.w[i], m.ra));
      m.v_n_pre = dot(m.n, m.v_rel_pre);
      m.restitution = B.restitution;
      S.manifolds.push_back(m);
    }
  }
}

// Relative contact velocity v_B - v_A; the wall is at rest (b unused).
inline V3 rel_vel(const orc_system& S, const Manifold& m) {
  V3 va = S.v[m.a] + cross(S.w[m.a], m.ra);
  if (m.wall) return -va;
  return (S.v[m.b] + cross(S.w[m.b], m.rb)) - va;
}

void apply_impulse(orc_system& S, const Manifold& m, V3 d, V3 IA, V3 IB, double l) {
  S.v[m.a] -= d * (l * m.invMA);
  S.w[m.a] -= IA * l;
  if (m.wall) return;
  S.v[m.b] += d * (l * m.invMB);
  S.w[m.b] += IB * l;
}

// solveVelocities (nsc_contact.cpp:325-655) over manifolds visited in `ord`.
void solve_velocities(orc_system& S, const std::vector<int>& ord) {
  const rg_config& c = S.cfg;
  S.last_residual = 0;
  S.last_sweeps = 0;
  if (S.manifolds.empty()) return;
  const double omega = c.nsc_omega, cfm = c.nsc_cfm, mu = c.nsc_mu, dt = c.dt;
  const double beta = c.nsc_position_stabilization ? c.nsc_beta * 0.01 : c.nsc_beta;
  if (c.nsc_warm_start != RG_WARM_NONE) {
    for (int idx : ord) {
      const Manifold& m = S.manifolds[idx];
      if (m.ln != 0.0) apply_impulse(S, m, m.n, m.IA_n, m.IB_n, m.ln);
      if (m.lt1 != 0.0) apply_impulse(S, m, m.t1, m.IA_t1, m.IB_t1, m.lt1);
      if (m.lt2 != 0.0) apply_impulse(S, m, m.t2, m.IA_t2, m.IB_t2, m.lt2);
    }
  }
  double maxres = 0;
  int sweeps = 0;
  for (int it = 0; it < c.nsc_velocity_iters; ++it) {
    double res = 0;
    for (int idx : ord) {
      Manifold& m = S.manifolds[idx];
      V3 vrel = rel_vel(S, m);
      double bn = m.phi < 0.0 ? beta * m.phi / dt : 0.0;
      double brest = m.v_n_pre < 0.0 ? m.restitution * m.v_n_pre : 0.0;
      double wn = dot(m.n, vrel) + bn + brest + cfm * m.ln;
      double dn_ = -(omega / m.g_n) * wn;
      double old = m.ln;
      m.ln = std::max(0.0, old + dn_);
      double dn = m.ln - old;
      if (dn != 0.0) {
        V3 dvA = m.n * (dn * m.invMA);
        S.v[m.a] -= dvA;
        S.w[m.a] -= m.IA_n * dn;
        vrel += dvA + cross(m.IA_n * dn, m.ra);
        if (!m.wall) {
          V3 dvB = m.n * (dn * m.invMB);
          S.v[m.b] += dvB;
          S.w[m.b] += m.IB_n * dn;
          vrel += dvB + cross(m.IB_n * dn, m.rb);
        }
      }
      double mf = mu * m.ln;
      double lim1 = std::sqrt(std::max(0.0, mf * mf - m.lt2 * m.lt2));
      double w1 = dot(m.t1, vrel) + cfm * m.lt1;
      double d1_ = -(omega / m.g_t1) * w1;
      double o1 = m.lt1;
      m.lt1 = std::min(std::max(o1 + d1_, -lim1), lim1);
      double d1 = m.lt1 - o1;
      if (d1 != 0.0) {
        V3 dvA = m.t1 * (d1 * m.invMA);
        S.v[m.a] -= dvA;
        S.w[m.a] -= m.IA_t1 * d1;
        vrel += dvA + cross(m.IA_t1 * d1, m.ra);
        if (!m.wall) {
          V3 dvB = m.t1 * (d1 * m.invMB);
          S.v[m.b] += dvB;
          S.w[m.b] += m.IB_t1 * d1;
          vrel += dvB + cross(m.IB_t1 * d1, m.rb);
        }
      }
      double lim2 = std::sqrt(std::max(0.0, mf * mf - m.lt1 * m.lt1));
      double w2 = dot(m.t2, vrel) + cfm * m.lt2;
      double d2_ = -(omega / m.g_t2) * w2;
      double o2 = m.lt2;
      m.lt2 = std::min(std::max(o2 + d2_, -lim2), lim2);
      double d2 = m.lt2 - o2;
      if (d2 != 0.0) {
        S.v[m.a] -= m.t2 * (d2 * m.invMA);
        S.w[m.a] -= m.IA_t2 * d2;
        if (!m.wall) {
          S.v[m.b] += m.t2 * (d2 * m.invMB);
          S.w[m.b] += m.IB_t2 * d2;
        }
      }
      res = std::max(res, std::fabs(dn) + std::fabs(d1) + std::fabs(d2));
    }
    maxres = res;
    sweeps = it + 1;
    if (res < c.nsc_tol) break;
  }
  S.last_residual = maxres;
  S.last_sweeps = sweeps;
  S.warm.clear();
  if (c.nsc_warm_start == RG_WARM_CACHE) {
    // wall manifolds start cold every step (addWallContact, nsc_contact.cpp:
    // 226-228): their (a, a) entries would never be read, so none is kept
    for (const Manifold& m : S.manifolds)
      if (!m.wall) S.warm[pair_key(m.a, m.b)] = v3(m.ln, m.lt1, m.lt2);
  }
}

struct PosRow {
  int a, b, color;
  V3 n, ra, rb;
  double phi, g, l;
};

// projectPositions, multi-body path (nsc_contact.cpp:698-879).
void project_positions(orc_system& S, bool colored) {
  const rg_config& c = S.cfg;
  if (!c.nsc_position_stabilization) return;
  const double omega = c.nsc_omega, cfm = c.nsc_cfm, slop = c.nsc_slop;
  struct Cached { int a, b; double surf; int color; };
  std::vector<Cached> cached;
  std::vector<PosRow> pm;
  std::vector<V3> dx(S.n), dth(S.n);
  for (int outer = 0; outer < c.nsc_position_iters; ++outer) {
    pm.clear();
    if (outer == 0) {
      auto cs = detect(S, 0.0);
      std::vector<int> ca(cs.size()), cb(cs.size()), col;
      for (size_t i = 0; i < cs.size(); ++i) { ca[i] = cs[i].a; cb[i] = cs[i].b; }
      jp_color(S, ca, cb, col);
      cached.clear();
      for (size_t i = 0; i < cs.size(); ++i) cached.push_back({cs[i].a, cs[i].b, cs[i].surface_limit, col[i]});
      for (size_t i = 0; i < cs.size(); ++i) {
        const Contact& ct = cs[i];
        double phi = ct.distance - ct.surface_limit;
        if (phi >= -slop) continue;
        PosRow p;
        p.a = ct.a; p.b = ct.b; p.color = col[i];
        p.n = ct.n;
        p.phi = phi + slop;
        p.ra = ct.pa - S.x[ct.a];
        p.rb = ct.pb - (S.x[ct.b] + ct.shift);
        p.g = diag(S, p.a, p.b, p.ra, p.rb, p.n, cfm);
        p.l = 0;
        pm.push_back(p);
      }
    } else {
      for (const Cached& cp : cached) {
        int a = cp.a, b = cp.b;
        V3 ua = axis_y(S.q[a]), ub = axis_y(S.q[b]);
        V3 a1 = S.x[a] - ua * S.body[a].h, a2 = S.x[a] + ua * S.body[a].h;
        V3 b1 = S.x[b] - ub * S.body[b].h, b2 = S.x[b] + ub * S.body[b].h;
        V3 sh = min_image_shift(S, S.x[a], S.x[b]);
        b1 = b1 + sh;
        b2 = b2 + sh;
        double s, t;
        lumelsky(a1, a2, b1, b2, s, t);
        V3 pA = a1 + (a2 - a1) * s;
        V3 pB = b1 + (b2 - b1) * t;
        V3 diff = pB - pA;
        double dist = length(diff);
        double phi = dist - cp.surf;
        if (phi >= -slop) continue;
        PosRow p;
        p.a = a; p.b = b; p.color = cp.color;
        p.n = dist > 1e-10 ? diff / dist : v3(1, 0, 0);
        p.phi = phi + slop;
        p.ra = pA - S.x[a];
        p.rb = pB - (S.x[b] + sh);
        p.g = diag(S, a, b, p.ra, p.rb, p.n, cfm);
        p.l = 0;
        pm.push_back(p);
      }
    }
    if (pm.empty()) return;
    std::fill(dx.begin(), dx.end(), v3(0, 0, 0));
    std::fill(dth.begin(), dth.end(), v3(0, 0, 0));
    std::vector<int> ord(pm.size());
    for (size_t i = 0; i < pm.size(); ++i) ord[i] = (int)i;
    if (colored)
      std::stable_sort(ord.begin(), ord.end(), [&](int p, int r) { return pm[p].color < pm[r].color; });
    for (int inner = 0; inner < c.nsc_position_psor_iters; ++inner) {
      double res = 0;
      for (int idx : ord) {
        PosRow& p = pm[idx];
        double corr = dot(p.n, ((dx[p.b] + cross(dth[p.b], p.rb)) - dx[p.a]) - cross(dth[p.a], p.ra));
        double r = corr + p.phi + cfm * p.l;
        double d = -(omega / p.g) * r;
        double old = p.l;
        p.l = std::max(0.0, old + d);
        double dl = p.l - old;
        if (dl != 0.0) {
          V3 rAxn = cross(p.ra, p.n);
          dx[p.a] -= p.n * (dl * S.body[p.a].inv_mass);
          dth[p.a] -= iinv_apply(S, p.a, rAxn) * dl;
          V3 rBxn = cross(p.rb, p.n);
          dx[p.b] += p.n * (dl * S.body[p.b].inv_mass);
          dth[p.b] += iinv_apply(S, p.b, rBxn) * dl;
        }
        res = std::max(res, std::fabs(dl));
      }
      if (res < 1e-8) break;
    }
    for (int i = 0; i < S.n; ++i) {
      if (S.body[i].inv_mass <= 0.0) continue;
      S.x[i] += dx[i];
      double ang = length(dth[i]);
      if (ang > 1e-8) {
        V3 ax = dth[i] / ang;
        S.q[i] = qnormalize(qmul(angle_axis(ang, ax), S.q[i]));
      }
    }
  }
}

void nsc_step(orc_system& S) {
  const rg_config& c = S.cfg;
  V3 g = v3(c.gravity[0], c.gravity[1], c.gravity[2]);
  const double dt = c.dt;
  const bool colored = c.psor_order == RG_ORDER_COLORED;
  // 1) free flight (main.cpp:4397-4408)
  for (int i = 0; i < S.n; ++i) {
    const Body& B = S.body[i];
    if (!(B.inv_mass > 0)) continue;
    S.v[i] += (S.f[i] * B.inv_mass + g) * dt;
    V3 Iw_w = rot_diag_apply(S.q[i], B.I, S.w[i]);
    V3 gyro = cross(S.w[i], Iw_w);
    S.w[i] += iinv_apply(S, i, S.tau[i] - gyro) * dt;
  }
  // 2) detection + manifolds (pairs, then cylinder walls, main.cpp:4431-4447)
  auto cs = detect(S, 0.0);
  build_manifolds(S, cs);
  add_wall_manifolds(S);
  const size_t M = S.manifolds.size();
  S.last_contacts = (int64_t)M;  // getNumContacts counts the wall manifolds
  std::vector<int> ca(M), cb(M), col;
  for (size_t i = 0; i < M; ++i) { ca[i] = S.manifolds[i].a; cb[i] = S.manifolds[i].b; }
  S.last_colors = jp_color(S, ca, cb, col);
  for (size_t i = 0; i < M; ++i) S.manifolds[i].color = col[i];
  int64_t coll = 0;
  for (const Manifold& m : S.manifolds)
    if (m.v_n_pre < -1e-6) ++coll;
  S.last_collisions = coll;
  // 3) velocity PSOR
  solve_velocities(S, visit_order((int)M, col, colored));
  // impulse sums of the profile CSV (main.cpp:3339-3343); collisions above
  // are NscContactSolver::countImpacts (nsc_contact.hpp:112-117)
  S.jn_sum = 0; S.jt_sum = 0;
  for (const Manifold& m : S.manifolds) {
    S.jn_sum += std::abs(m.ln);
    S.jt_sum += std::abs(m.lt1) + std::abs(m.lt2);
  }
  // 4) position + orientation update with linear damping (main.cpp:4469-4483)
  for (int i = 0; i < S.n; ++i) {
    S.x[i] += S.v[i] * dt;
    V3 hw = S.w[i] * (0.5 * dt);
    Q wq{0.0, hw.x, hw.y, hw.z};
    Q dq = qmul(wq, S.q[i]);
    Q qn{S.q[i].w + dq.w, S.q[i].x + dq.x, S.q[i].y + dq.y, S.q[i].z + dq.z};
    S.q[i] = qnormalize(qn);
    S.v[i] = S.v[i] * (1.0 - c.lin_damp * dt);
    S.w[i] = S.w[i] * (1.0 - c.ang_damp * dt);
    double wl = length(S.w[i]);
    if (wl > c.w_max) S.w[i] = S.w[i] * (c.w_max / wl);
  }
  // 4b) inside the tube, spin about the rod axis is projected out
  // (main.cpp:4486-4494)
  if (c.cylinder_enabled)
    for (int i = 0; i < S.n; ++i) {
      V3 u = axis_y(S.q[i]);
      u = u / length(u);
      S.w[i] = S.w[i] - u * dot(S.w[i], u);
    }
  // 5) position projection
  project_positions(S, colored);
  // 6) PBC wrap (main.cpp:4508-4517)
  if (S.pbc)
    for (int i = 0; i < S.n; ++i) wrap(S, S.x[i]);
  // 7) clear forces
  for (int i = 0; i < S.n; ++i) { S.f[i] = v3(0, 0, 0); S.tau[i] = v3(0, 0, 0); }
}

double kinetic_energy(const orc_system& S) {
  double ke = 0;
  for (int i = 0; i < S.n; ++i) {
    ke += 0.5 * S.body[i].mass * dot(S.v[i], S.v[i]);
    ke += 0.5 * dot(S.w[i], rot_diag_apply(S.q[i], S.body[i].I, S.w[i]));
  }
  return ke;
}

}  // namespace

extern "C" {

int orc_create(const rg_config* cfg, orc_system** out) {
  if (!cfg || !out || cfg->n_bodies <= 0) return RG_ERR_ARG;
  orc_system* S = new orc_system();
  S->cfg = *cfg;
  S->n = cfg->n_bodies;
  S->body.resize(S->n);
  S->x.assign(S->n, v3(0, 0, 0));
  S->v = S->w = S->f = S->tau = S->x;
  S->q.assign(S->n, Q{1, 0, 0, 0});
  S->pbc = cfg->pbc_enabled != 0;
  S->pbc_min = v3(cfg->pbc_min[0], cfg->pbc_min[1], cfg->pbc_min[2]);
  S->pbc_max = v3(cfg->pbc_max[0], cfg->pbc_max[1], cfg->pbc_max[2]);
  S->pbc_size = S->pbc_max - S->pbc_min;
  *out = S;
  return RG_OK;
}

int orc_destroy(orc_system* S) {
  delete S;
  return RG_OK;
}

int orc_set_bodies(orc_system* S, const double* radius, const double* half_height,
                   const double* mass, const double* inertia, const double* restitution) {
  if (!S || !radius || !half_height || !mass || !inertia) return RG_ERR_ARG;
  for (int i = 0; i < S->n; ++i) {
    Body& B = S->body[i];
    B.r = radius[i];
    B.h = half_height[i];
    B.mass = mass[i] > 0 ? mass[i] : 0.0;
    B.inv_mass = mass[i] > 0 ? 1.0 / mass[i] : 0.0;
    B.I = v3(inertia[3 * i], inertia[3 * i + 1], inertia[3 * i + 2]);
    if (B.inv_mass > 0) {
      B.Iinv = v3(B.I.x > 0 ? 1.0 / B.I.x : 0.0, B.I.y > 0 ? 1.0 / B.I.y : 0.0,
                  B.I.z > 0 ? 1.0 / B.I.z : 0.0);
    } else {
      B.I = v3(0, 0, 0);
      B.Iinv = v3(0, 0, 0);
    }
    B.restitution = restitution ? restitution[i] : 0.2;
  }
  return RG_OK;
}

int orc_set_state(orc_system* S, const double* x, const double* q, const double* v,
                  const double* w, const double* f, const double* tau) {
  if (!S || !x || !q || !v || !w) return RG_ERR_ARG;
  for (int i = 0; i < S->n; ++i) {
    S->x[i] = v3(x[3 * i], x[3 * i + 1], x[3 * i + 2]);
    S->q[i] = Q{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
    S->v[i] = v3(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    S->w[i] = v3(w[3 * i], w[3 * i + 1], w[3 * i + 2]);
    S->f[i] = f ? v3(f[3 * i], f[3 * i + 1], f[3 * i + 2]) : v3(0, 0, 0);
    S->tau[i] = tau ? v3(tau[3 * i], tau[3 * i + 1], tau[3 * i + 2]) : v3(0, 0, 0);
  }
  return RG_OK;
}

int orc_get_state(const orc_system* S, double* x, double* q, double* v, double* w,
                  double* f, double* tau) {
  if (!S) return RG_ERR_ARG;
  for (int i = 0; i < S->n; ++i) {
    if (x) { x[3 * i] = S->x[i].x; x[3 * i + 1] = S->x[i].y; x[3 * i + 2] = S->x[i].z; }
    if (q) { q[4 * i] = S->q[i].w; q[4 * i + 1] = S->q[i].x; q[4 * i + 2] = S->q[i].y; q[4 * i + 3] = S->q[i].z; }
    if (v) { v[3 * i] = S->v[i].x; v[3 * i + 1] = S->v[i].y; v[3 * i + 2] = S->v[i].z; }
    if (w) { w[3 * i] = S->w[i].x; w[3 * i + 1] = S->w[i].y; w[3 * i + 2] = S->w[i].z; }
    if (f) { f[3 * i] = S->f[i].x; f[3 * i + 1] = S->f[i].y; f[3 * i + 2] = S->f[i].z; }
    if (tau) { tau[3 * i] = S->tau[i].x; tau[3 * i + 1] = S->tau[i].y; tau[3 * i + 2] = S->tau[i].z; }
  }
  return RG_OK;
}

int orc_step(orc_system* S, int nsteps, rg_step_stats* st) {
  if (!S || nsteps < 0) return RG_ERR_ARG;
  rg_step_stats loc;
  std::memset(&loc, 0, sizeof(loc));
  for (int k = 0; k < nsteps; ++k) {
    if (S->cfg.model == RG_MODEL_NSC) {
      nsc_step(*S);
      loc.psor_sweeps += S->last_sweeps;
      loc.max_residual = std::max(loc.max_residual, S->last_residual);
      if (S->last_residual >= S->cfg.nsc_tol && !S->manifolds.empty()) loc.not_converged++;
    } else if (S->cfg.model == RG_MODEL_HARMONIC || S->cfg.model == RG_MODEL_HERTZ_MINDLIN) {
      verlet_step(*S);
    }
    loc.steps++;
  }
  loc.contacts = S->last_contacts;
  loc.collisions = S->last_collisions;
  loc.psor_sweeps_last = S->last_sweeps;
  loc.colors = S->last_colors;
  loc.residual = S->last_residual;
  loc.jn_sum = S->jn_sum;
  loc.jt_sum = S->jt_sum;
  loc.potential_energy = S->last_pe;
  loc.kinetic_energy = kinetic_energy(*S);
  loc.history_size = (int64_t)(S->cfg.model == RG_MODEL_HERTZ_MINDLIN ? S->hm_hist.size() : S->soft_hist.size());
  if (st) *st = loc;
  return RG_OK;
}

int orc_detect(orc_system* S, double delta, int32_t* pairs, double* geom, double* shift,
               size_t cap, size_t* n) {
  if (!S || !n) return RG_ERR_ARG;
  auto cs = detect(*S, delta);
  *n = cs.size();
  size_t m = std::min(cap, cs.size());
  for (size_t i = 0; i < m; ++i) {
    const Contact& c = cs[i];
    if (pairs) { pairs[2 * i] = c.a; pairs[2 * i + 1] = c.b; }
    if (geom) {
      double* g = geom + 12 * i;
      g[0] = c.pa.x; g[1] = c.pa.y; g[2] = c.pa.z;
      g[3] = c.pb.x; g[4] = c.pb.y; g[5] = c.pb.z;
      g[6] = c.n.x; g[7] = c.n.y; g[8] = c.n.z;
      g[9] = c.distance; g[10] = c.surface_limit; g[11] = (double)c.type;
    }
    if (shift) { shift[3 * i] = c.shift.x; shift[3 * i + 1] = c.shift.y; shift[3 * i + 2] = c.shift.z; }
  }
  return cs.size() > cap ? RG_ERR_CAPACITY : RG_OK;
}

// Pair manifolds of the last velocity solve (the wall manifolds follow them
// and are left out, as from the warm cache).
static size_t pair_manifolds(const orc_system* S) {
  size_t k = 0;
  while (k < S->manifolds.size() && !S->manifolds[k].wall) ++k;
  return k;
}

int orc_get_impulses(const orc_system* S, int32_t* pairs, double* lambda, int32_t* color,
                     size_t cap, size_t* n) {
  if (!S || !n) return RG_ERR_ARG;
  const size_t P = pair_manifolds(S);
  *n = P;
  size_t m = std::min(cap, P);
  for (size_t i = 0; i < m; ++i) {
    const Manifold& mf = S->manifolds[i];
    if (pairs) { pairs[2 * i] = mf.a; pairs[2 * i + 1] = mf.b; }
    if (lambda) { lambda[3 * i] = mf.ln; lambda[3 * i + 1] = mf.lt1; lambda[3 * i + 2] = mf.lt2; }
    if (color) color[i] = mf.color;
  }
  return P > cap ? RG_ERR_CAPACITY : RG_OK;
}

// The wall manifolds of the last velocity solve: body, contact point
// x_a + r_a, normal, phi, impulses, colour.
int orc_get_wall_contacts(const orc_system* S, int32_t* body, double* rows, int32_t* color, size_t cap,
                          size_t* n) {
  if (!S || !n) return RG_ERR_ARG;
  const size_t P = pair_manifolds(S), W = S->manifolds.size() - P;
  *n = W;
  for (size_t i = 0; i < W && i < cap; ++i) {
    const Manifold& m = S->manifolds[P + i];
    if (body) body[i] = m.a;
    if (rows) {
      double* o = rows + 10 * i;
      V3 pt = S->x[m.a] + m.ra;
      o[0] = pt.x; o[1] = pt.y; o[2] = pt.z;
      o[3] = m.n.x; o[4] = m.n.y; o[5] = m.n.z;
      o[6] = m.phi; o[7] = m.ln; o[8] = m.lt1; o[9] = m.lt2;
    }
    if (color) color[i] = m.color;
  }
  return W > cap ? RG_ERR_CAPACITY : RG_OK;
}

// Network rows of the last velocity solve (App::logNetworkFrame NSC branch,
// main.cpp:3664-3690): point x_a + r_a and v_n after the solve from the
// current state; phi, impulses and v_n_pre from the manifold.
int orc_get_contact_network(const orc_system* S, int32_t* pairs, double* rows, size_t cap, size_t* n) {
  if (!S || !n) return RG_ERR_ARG;
  const size_t m = pair_manifolds(S);  // rod-rod pairs only (walls skipped, main.cpp:3668)
  *n = m;
  for (size_t i = 0; i < m && i < cap; ++i) {
    const Manifold& M = S->manifolds[i];
    V3 va = S->v[M.a] + cross(S->w[M.a], M.ra);
    V3 vb = S->v[M.b] + cross(S->w[M.b], M.rb);
    double vn_post = dot(M.n, vb - va);
    if (pairs) { pairs[2 * i] = M.a; pairs[2 * i + 1] = M.b; }
    if (rows) {
      double* o = rows + 12 * i;
      V3 pt = S->x[M.a] + M.ra;
      o[0] = pt.x; o[1] = pt.y; o[2] = pt.z;
      o[3] = M.n.x; o[4] = M.n.y; o[5] = M.n.z;
      o[6] = M.phi; o[7] = M.ln; o[8] = M.lt1; o[9] = M.lt2;
      o[10] = M.v_n_pre; o[11] = vn_post;
    }
  }
  return m > cap ? RG_ERR_CAPACITY : RG_OK;
}

int orc_compute_forces(orc_system* S, double* f, double* tau, double* pe) {
  if (!S) return RG_ERR_ARG;
  for (int i = 0; i < S->n; ++i) { S->f[i] = v3(0, 0, 0); S->tau[i] = v3(0, 0, 0); }
  force_eval(*S);
  orc_get_state(S, nullptr, nullptr, nullptr, nullptr, f, tau);
  if (pe) *pe = S->last_pe;
  return RG_OK;
}

int orc_get_history(const orc_system* S, int32_t* pairs, double* value, int64_t* last_frame,
                    size_t cap, size_t* n) {
  if (!S || !n) return RG_ERR_ARG;
  const auto& H = S->cfg.model == RG_MODEL_HERTZ_MINDLIN ? S->hm_hist : S->soft_hist;
  *n = H.size();
  size_t i = 0;
  for (const auto& kv : H) {
    if (i >= cap) break;
    if (pairs) { pairs[2 * i] = (int32_t)(kv.first >> 32); pairs[2 * i + 1] = (int32_t)(kv.first & 0xffffffffu); }
    if (value) { value[3 * i] = kv.second.value.x; value[3 * i + 1] = kv.second.value.y; value[3 * i + 2] = kv.second.value.z; }
    if (last_frame) last_frame[i] = kv.second.last_frame;
    ++i;
  }
  return H.size() > cap ? RG_ERR_CAPACITY : RG_OK;
}

// Colouring of an arbitrary contact list (for tests of the device colouring).
int orc_color(const orc_system* S, const int32_t* pairs, size_t n, int32_t* color, int* ncolors) {
  if (!S || (!pairs && n)) return RG_ERR_ARG;
  std::vector<int> ca(n), cb(n), col;
  for (size_t i = 0; i < n; ++i) { ca[i] = pairs[2 * i]; cb[i] = pairs[2 * i + 1]; }
  int k = jp_color(*S, ca, cb, col);
  for (size_t i = 0; i < n; ++i) color[i] = col[i];
  if (ncolors) *ncolors = k;
  return k < 0 ? RG_ERR_CAPACITY : RG_OK;
}

double orc_kinetic_energy(const orc_system* S) { return S ? kinetic_energy(*S) : 0.0; }

}  // extern "C"
