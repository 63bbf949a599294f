// rg_nsc_dev.cuh - device bodies of the NSC step (manifold rows, PSOR row
// update, per-body integrators) and the view a persistent team works on.
// Reference functions: src/physics/nsc_contact.cpp (:78-117 basis and
// diagonals, :239-321 manifolds, :344-552 warm start and sweeps) and
// App::physicsStep (src/app/main.cpp:4397-4408, :4469-4483, :4508-4517).
#pragma once
#include "rg_detect_dev.cuh"
#include "rg_mlp_dev.cuh"

namespace rg {

constexpr int kMaxRounds = 512;  // colouring rounds before giving up

// Deterministic contact priority for the Jones-Plassmann colouring (the
// oracle computes the same function).
__device__ inline unsigned long long jp_priority(unsigned c) {
  unsigned h = c * 0x9E3779B1u;
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return ((unsigned long long)h << 32) | (unsigned long long)c;
}

// Manifold rows in colour-major slots (structure of arrays, ccap each).
struct RowIO {
  double* row;  // kRowComps * ccap
  double* lam;  // 3 * ccap
  int ccap;
  __device__ double& r(int k, int p) const { return row[(size_t)k * ccap + p]; }
  __device__ d3 r3(int k, int p) const { return {r(k, p), r(k + 1, p), r(k + 2, p)}; }
  __device__ void w3(int k, int p, d3 v) const { r(k, p) = v.x; r(k + 1, p) = v.y; r(k + 2, p) = v.z; }
};
enum { R_N = 0, R_T1 = 3, R_T2 = 6, R_RA = 9, R_RB = 12, R_IAN = 15, R_IAT1 = 18, R_IAT2 = 21,
       R_IBN = 24, R_IBT1 = 27, R_IBT2 = 30, R_IMA = 33, R_IMB = 34, R_GN = 35, R_GT1 = 36,
       R_GT2 = 37, R_BN = 38, R_BREST = 39, R_PHI = 40, R_VNPRE = 41 };  // R_G*: omega / g
enum { P_N = 0, P_RA = 3, P_RB = 6, P_PHI = 9, P_G = 10, P_L = 11 };

__device__ inline d3 iinv_apply(const State& st, int i, d3 v) {
  if (st.inv_mass[i] <= 0.0) return {0, 0, 0};
  return rot_diag_apply(st.q.ld(i), st.Iinv.ld(i), v);
}
// computeDiag: 1/ma + 1/mb + (ra x d).IA(ra x d) + (rb x d).IB(rb x d) + cfm.
__device__ inline double diag_of(const State& st, int a, int b, d3 ra, d3 rb, d3 d, double cfm) {
  d3 rad = cross(ra, d), rbd = cross(rb, d);
  double g = st.inv_mass[a] + st.inv_mass[b] + dot(rad, iinv_apply(st, a, rad)) +
             dot(rbd, iinv_apply(st, b, rbd)) + cfm;
  return smax(g, 1e-12);
}
__device__ inline int lower_bound_key(const unsigned long long* k, int n, unsigned long long v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (k[m] < v) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// Wall row of contact c (body a against the tube, stored with b == a): the
// manifold of NscContactSolver::addWallContact (nsc_contact.cpp:190-235):
// r_b = 0, no mass or inertia on the wall side, computeDiagWall
// (:144-150), v_rel = -(v_a + w_a x r_a), the body's own restitution, and a
// cold start (wall manifolds are never warm-started).  Returns the impact
// bit, with bit 1 set so the learned start leaves the row alone.
__device__ inline int build_wall_row(const State& st, const Contacts& con, const rg_config& cfg, int c, int p,
                                     const RowIO& R, double beta, float* feat, int fld) {
  const int a = con.a[c];
  d3 pa{con.comp(0)[c], con.comp(1)[c], con.comp(2)[c]};
  d3 n{con.comp(6)[c], con.comp(7)[c], con.comp(8)[c]};
  double phi = con.comp(12)[c] - con.comp(13)[c];
  d3 ref = fabs(n.x) < 0.9 ? mk3(1, 0, 0) : mk3(0, 1, 0);
  d3 cr = cross(n, ref);
  d3 t1 = cr / len(cr);
  d3 t2 = cross(n, t1);
  d3 ra = pa - st.x.ld(a);
  const d3 zero{0, 0, 0};
  R.w3(R_N, p, n); R.w3(R_T1, p, t1); R.w3(R_T2, p, t2);
  R.w3(R_RA, p, ra); R.w3(R_RB, p, zero);
  auto gw = [&](d3 d) {
    d3 rd = cross(ra, d);
    return smax(st.inv_mass[a] + dot(rd, iinv_apply(st, a, rd)) + cfg.nsc_cfm, 1e-12);
  };
  R.r(R_GN, p) = cfg.nsc_omega / gw(n);
  R.r(R_GT1, p) = cfg.nsc_omega / gw(t1);
  R.r(R_GT2, p) = cfg.nsc_omega / gw(t2);
  R.r(R_IMA, p) = st.inv_mass[a];
  R.r(R_IMB, p) = 0.0;
  R.w3(R_IAN, p, iinv_apply(st, a, cross(ra, n)));
  R.w3(R_IAT1, p, iinv_apply(st, a, cross(ra, t1)));
  R.w3(R_IAT2, p, iinv_apply(st, a, cross(ra, t2)));
  R.w3(R_IBN, p, zero); R.w3(R_IBT1, p, zero); R.w3(R_IBT2, p, zero);
  d3 vrel = -(st.v.ld(a) + cross(st.w.ld(a), ra));
  double vnp = dot(n, vrel);
  double e = st.rest[a];
  R.r(R_BN, p) = phi < 0.0 ? beta * phi / cfg.dt : 0.0;
  R.r(R_BREST, p) = vnp < 0.0 ? e * vnp : 0.0;
  R.r(R_PHI, p) = phi;
  R.r(R_VNPRE, p) = vnp;
  R.lam[p] = 0.0;
  R.lam[R.ccap + p] = 0.0;
  R.lam[2 * R.ccap + p] = 0.0;
  if (feat) {
    feat[p] = (float)phi;
    feat[fld + p] = (float)vnp;
    feat[2 * fld + p] = (float)dot(t1, vrel);
    feat[3 * fld + p] = (float)dot(t2, vrel);
    feat[4 * fld + p] = 0.0f;
    feat[5 * fld + p] = 0.0f;
    feat[6 * fld + p] = 0.0f;
  }
  return (vnp < -1e-6 ? 1 : 0) | 2;
}

// Manifold row of contact c into slot p; returns 1 for an impact
// (v_n_pre < -1e-6, NscContactSolver::countImpacts).  When feat is given,
// the learned warm start's features 0-6 of slot p go to feat[k * fld + p]
// (feature 7, the contact-graph degree, is filled by the caller).
__device__ inline int build_row(const State& st, const Contacts& con, const rg_config& cfg, int c, int p,
                                const RowIO& R, const unsigned long long* wkey, const double* wlam, int W,
                                int wcap, float* feat = nullptr, int fld = 0) {
  const double beta = cfg.nsc_position_stabilization ? cfg.nsc_beta * 0.01 : cfg.nsc_beta;
  const int a = con.a[c], b = con.b[c];
  if (a == b) return build_wall_row(st, con, cfg, c, p, R, beta, feat, fld);
  d3 pa{con.comp(0)[c], con.comp(1)[c], con.comp(2)[c]};
  d3 pb{con.comp(3)[c], con.comp(4)[c], con.comp(5)[c]};
  d3 n{con.comp(6)[c], con.comp(7)[c], con.comp(8)[c]};
  d3 sh{con.comp(9)[c], con.comp(10)[c], con.comp(11)[c]};
  double phi = con.comp(12)[c] - con.comp(13)[c];
  d3 ref = fabs(n.x) < 0.9 ? mk3(1, 0, 0) : mk3(0, 1, 0);
  d3 cr = cross(n, ref);
  d3 t1 = cr / len(cr);
  d3 t2 = cross(n, t1);
  d3 ra = pa - st.x.ld(a);
  d3 rb = pb - (st.x.ld(b) + sh);
  R.w3(R_N, p, n); R.w3(R_T1, p, t1); R.w3(R_T2, p, t2);
  R.w3(R_RA, p, ra); R.w3(R_RB, p, rb);
  // omega / g per direction, computed once here instead of in every sweep
  // (the same quotient the sweep would form, so results are unchanged)
  R.r(R_GN, p) = cfg.nsc_omega / diag_of(st, a, b, ra, rb, n, cfg.nsc_cfm);
  R.r(R_GT1, p) = cfg.nsc_omega / diag_of(st, a, b, ra, rb, t1, cfg.nsc_cfm);
  R.r(R_GT2, p) = cfg.nsc_omega / diag_of(st, a, b, ra, rb, t2, cfg.nsc_cfm);
  R.r(R_IMA, p) = st.inv_mass[a];
  R.r(R_IMB, p) = st.inv_mass[b];
  R.w3(R_IAN, p, iinv_apply(st, a, cross(ra, n)));
  R.w3(R_IAT1, p, iinv_apply(st, a, cross(ra, t1)));
  R.w3(R_IAT2, p, iinv_apply(st, a, cross(ra, t2)));
  R.w3(R_IBN, p, iinv_apply(st, b, cross(rb, n)));
  R.w3(R_IBT1, p, iinv_apply(st, b, cross(rb, t1)));
  R.w3(R_IBT2, p, iinv_apply(st, b, cross(rb, t2)));
  d3 vrel = (st.v.ld(b) + cross(st.w.ld(b), rb)) - (st.v.ld(a) + cross(st.w.ld(a), ra));
  double vnp = dot(n, vrel);
  double e = smin(st.rest[a], st.rest[b]);
  R.r(R_BN, p) = phi < 0.0 ? beta * phi / cfg.dt : 0.0;
  R.r(R_BREST, p) = vnp < 0.0 ? e * vnp : 0.0;
  R.r(R_PHI, p) = phi;
  R.r(R_VNPRE, p) = vnp;
  double l0 = 0, l1 = 0, l2 = 0;
  int cached = 0;
  if (cfg.nsc_warm_start != RG_WARM_NONE && W > 0) {
    unsigned long long k = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
    int q = lower_bound_key(wkey, W, k);
    if (q < W && wkey[q] == k) {
      cached = 2;
      l0 = smax(0.0, wlam[q]);
      l1 = wlam[wcap + q];
      l2 = wlam[2 * wcap + q];
    }
  }
  R.lam[p] = l0;
  R.lam[R.ccap + p] = l1;
  R.lam[2 * R.ccap + p] = l2;
  if (feat) {
    feat[p] = (float)phi;
    feat[fld + p] = (float)vnp;
    feat[2 * fld + p] = (float)dot(t1, vrel);
    feat[3 * fld + p] = (float)dot(t2, vrel);
    feat[4 * fld + p] = (float)l0;
    feat[5 * fld + p] = (float)l1;
    feat[6 * fld + p] = (float)l2;
  }
  return (vnp < -1e-6 ? 1 : 0) | cached;  // bit 0: impact, bit 1: in the warm cache
}

// Contact-network export of slot p (contact c, warm-cache order): the
// manifold's normal, r_a, r_b, phi and v_n_pre (NscManifold fields that
// App::logNetworkFrame writes, main.cpp:3670-3690).
__device__ inline void export_row(double* xrow, int wcap, int c, const RowIO& R, int p) {
  const int src[kExportComps] = {R_N, R_N + 1, R_N + 2, R_RA, R_RA + 1, R_RA + 2,
                                 R_RB, R_RB + 1, R_RB + 2, R_PHI, R_VNPRE};
#pragma unroll
  for (int k = 0; k < kExportComps; ++k) xrow[(size_t)k * wcap + c] = R.r(src[k], p);
}

// Learned warm start of slot p: previous impulse (already in R.lam) plus the
// network's predicted change, projected onto the friction cone.
__device__ inline void mlp_apply(const RowIO& R, const float* pred, int pld, int p, double mu) {
  double ln = R.lam[p] + (double)pred[p];
  double l1 = R.lam[R.ccap + p] + (double)pred[pld + p];
  double l2 = R.lam[2 * R.ccap + p] + (double)pred[2 * pld + p];
  cone_clamp(ln, l1, l2, mu);
  R.lam[p] = ln;
  R.lam[R.ccap + p] = l1;
  R.lam[2 * R.ccap + p] = l2;
}

struct Vel {
  Vec3A v, w;
};

// a == b: a wall row (the wall takes no impulse).
__device__ inline void apply_imp(const Vel& V, int a, int b, d3 d, d3 IA, d3 IB, double ima, double imb,
                                 double l) {
  V.v.st(a, V.v.ld(a) - d * (l * ima));
  V.w.st(a, V.w.ld(a) - IA * l);
  if (a == b) return;
  V.v.st(b, V.v.ld(b) + d * (l * imb));
  V.w.st(b, V.w.ld(b) + IB * l);
}

// Warm-start impulses of slot p (nsc_contact.cpp:344-380).
__device__ inline void warm_apply(const RowIO& R, const Vel& V, int p, int a, int b) {
  double ima = R.r(R_IMA, p), imb = R.r(R_IMB, p);
  double ln = R.lam[p], l1 = R.lam[R.ccap + p], l2 = R.lam[2 * R.ccap + p];
  if (ln != 0.0) apply_imp(V, a, b, R.r3(R_N, p), R.r3(R_IAN, p), R.r3(R_IBN, p), ima, imb, ln);
  if (l1 != 0.0) apply_imp(V, a, b, R.r3(R_T1, p), R.r3(R_IAT1, p), R.r3(R_IBT1, p), ima, imb, l1);
  if (l2 != 0.0) apply_imp(V, a, b, R.r3(R_T2, p), R.r3(R_IAT2, p), R.r3(R_IBT2, p), ima, imb, l2);
}

// One Gauss-Seidel row update (nsc_contact.cpp:391-548); returns
// |dλn| + |dλt1| + |dλt2|.
__device__ inline double psor_row(const RowIO& R, const Vel& V, int p, int a, int b, double omega, double cfm,
                                  double mu) {
  (void)omega;  // folded into the row (R_GN, R_GT1, R_GT2 hold omega / g)
  d3 n = R.r3(R_N, p), t1 = R.r3(R_T1, p), t2 = R.r3(R_T2, p);
  d3 ra = R.r3(R_RA, p), rb = R.r3(R_RB, p);
  d3 IAn = R.r3(R_IAN, p), IAt1 = R.r3(R_IAT1, p), IAt2 = R.r3(R_IAT2, p);
  d3 IBn = R.r3(R_IBN, p), IBt1 = R.r3(R_IBT1, p), IBt2 = R.r3(R_IBT2, p);
  double ima = R.r(R_IMA, p), imb = R.r(R_IMB, p);
  double ln = R.lam[p], lt1 = R.lam[R.ccap + p], lt2 = R.lam[2 * R.ccap + p];
  // a == b: a wall row; the wall is at rest and takes no impulse (its
  // B-side terms are zero, v_rel = -(v_a + w_a x r_a))
  const bool wall = a == b;
  const d3 zero{0, 0, 0};
  d3 vA = V.v.ld(a), wA = V.w.ld(a), vB = wall ? zero : V.v.ld(b), wB = wall ? zero : V.w.ld(b);
  d3 vrel = wall ? -(vA + cross(wA, ra)) : (vB + cross(wB, rb)) - (vA + cross(wA, ra));
  double wn = dot(n, vrel) + R.r(R_BN, p) + R.r(R_BREST, p) + cfm * ln;
  double dn_ = -R.r(R_GN, p) * wn;
  double old = ln;
  ln = smax(0.0, old + dn_);
  double dn = ln - old;
  if (dn != 0.0) {
    d3 dvA = n * (dn * ima);
    vA = vA - dvA;
    wA = wA - IAn * dn;
    vrel = vrel + (dvA + cross(IAn * dn, ra));
    d3 dvB = n * (dn * imb);
    vB = vB + dvB;
    wB = wB + IBn * dn;
    vrel = vrel + (dvB + cross(IBn * dn, rb));
  }
  double mf = mu * ln;
  double lim1 = sqrt(smax(0.0, mf * mf - lt2 * lt2));
  double w1 = dot(t1, vrel) + cfm * lt1;
  double d1_ = -R.r(R_GT1, p) * w1;
  double o1 = lt1;
  lt1 = smin(smax(o1 + d1_, -lim1), lim1);
  double d1 = lt1 - o1;
  if (d1 != 0.0) {
    d3 dvA = t1 * (d1 * ima);
    vA = vA - dvA;
    wA = wA - IAt1 * d1;
    vrel = vrel + (dvA + cross(IAt1 * d1, ra));
    d3 dvB = t1 * (d1 * imb);
    vB = vB + dvB;
    wB = wB + IBt1 * d1;
    vrel = vrel + (dvB + cross(IBt1 * d1, rb));
  }
  double lim2 = sqrt(smax(0.0, mf * mf - lt1 * lt1));
  double w2 = dot(t2, vrel) + cfm * lt2;
  double d2_ = -R.r(R_GT2, p) * w2;
  double o2 = lt2;
  lt2 = smin(smax(o2 + d2_, -lim2), lim2);
  double d2 = lt2 - o2;
  if (d2 != 0.0) {
    vA = vA - t2 * (d2 * ima);
    wA = wA - IAt2 * d2;
    vB = vB + t2 * (d2 * imb);
    wB = wB + IBt2 * d2;
  }
  if (dn != 0.0 || d1 != 0.0 || d2 != 0.0) {
    V.v.st(a, vA); V.w.st(a, wA);
    if (!wall) { V.v.st(b, vB); V.w.st(b, wB); }
    R.lam[p] = ln; R.lam[R.ccap + p] = lt1; R.lam[2 * R.ccap + p] = lt2;
  }
  return fabs(dn) + fabs(d1) + fabs(d2);
}

// ---- per-body integrator bodies ----------------------------------------------
__device__ inline void nsc_free_flight_body(const State& st, int i, d3 g, double dt) {
  double im = st.inv_mass[i];
  if (!(im > 0)) return;
  dq q = st.q.ld(i);
  d3 w = st.w.ld(i);
  d3 v = st.v.ld(i) + (st.f.ld(i) * im + g) * dt;
  d3 Iw_w = rot_diag_apply(q, st.I.ld(i), w);
  d3 gyro = cross(w, Iw_w);
  w = w + rot_diag_apply(q, st.Iinv.ld(i), st.tau.ld(i) - gyro) * dt;
  st.v.st(i, v);
  st.w.st(i, w);
}

// Returns 1 when the new state is not finite.
__device__ inline int nsc_position_update_body(const State& st, int i, const rg_config& cfg) {
  const double dt = cfg.dt;
  const double ld = 1.0 - cfg.lin_damp * dt, ad = 1.0 - cfg.ang_damp * dt;
  d3 v = st.v.ld(i), w = st.w.ld(i);
  d3 x = st.x.ld(i) + v * dt;
  dq q = st.q.ld(i);
  d3 hw = w * (0.5 * dt);
  dq wq{0.0, hw.x, hw.y, hw.z};
  dq d = qmul(wq, q);
  q = qnormalize(dq{q.w + d.w, q.x + d.x, q.y + d.y, q.z + d.z});
  v = v * ld;
  w = w * ad;
  double wl = len(w);
  if (wl > cfg.w_max) w = w * (cfg.w_max / wl);
  st.x.st(i, x);
  st.q.st(i, q);
  st.v.st(i, v);
  st.w.st(i, w);
  return (x.x == x.x && x.y == x.y && x.z == x.z && v.x == v.x) ? 0 : 1;
}

// |dx| + h|du| of a segment against reference centre/axis values already in
// registers.  The periodic image is taken with a multiplication by 1/L: it
// can differ from the division-based image only when |dx| is within rounding
// of L/2, where either image's displacement is far beyond any skin and
// triggers the rebuild all the same.
__device__ inline double disp_from(const Seg& s, const double* rf, const Box& box, const double* invL) {
  d3 dx{s.cx - rf[0], s.cy - rf[1], s.cz - rf[2]};
  if (box.pbc) {
    if (box.L[0] > 0.0) dx.x -= box.L[0] * rint(dx.x * invL[0]);
    if (box.L[1] > 0.0) dx.y -= box.L[1] * rint(dx.y * invL[1]);
    if (box.L[2] > 0.0) dx.z -= box.L[2] * rint(dx.z * invL[2]);
  }
  d3 du{s.ux - rf[3], s.uy - rf[4], s.uz - rf[5]};
  double d = len(dx) + s.h * len(du);
  return (d == d) ? d : 1e300;
}

__device__ inline Seg seg_of(d3 x, dq q, double h, double r) {
  d3 u = axis_y(q);
  Seg s;
  s.cx = x.x; s.cy = x.y; s.cz = x.z; s.h = h;
  s.ux = u.x; s.uy = u.y; s.uz = u.z; s.r = r;
  return s;
}

// Free flight of rod i alone (velocities; nsc_free_flight_body from the
// buffer bases): for rods whose segment record and displacement bounds are
// still those of the last position update.
__device__ inline void free_flight_velocity(const StateBase& S, int i, d3 g, double dt) {
  const double im = S.pc(3)[i];
  if (!(im > 0)) return;
  const dq q{S.c(3)[i], S.c(4)[i], S.c(5)[i], S.c(6)[i]};
  d3 v = S.ld3(7, i);
  d3 w = S.ld3(10, i);
  const d3 f = S.ld3(13, i), tau = S.ld3(16, i), I = S.pld3(5, i), Iinv = S.pld3(8, i);
  v = v + (f * im + g) * dt;
  d3 Iw_w = rot_diag_apply(q, I, w);
  d3 gyro = cross(w, Iw_w);
  w = w + rot_diag_apply(q, Iinv, tau - gyro) * dt;
  S.st3(7, i, v);
  S.st3(10, i, w);
}

// Free flight of rod i (nsc_free_flight_body), its segment record and the
// displacement bounds against ref (and ref2 when given), with every input
// loaded before the first store: one round trip to memory per rod instead
// of three.  Same arithmetic as the separate functions.
__device__ inline void free_flight_fused(const StateBase& S, int i, d3 g, double dt, const double* ref,
                                         const double* ref2, const Box& box, const double* invL, Seg* seg_out,
                                         double& dmax, double& dnear) {
  const int n = S.n;
  const double im = S.pc(3)[i];
  const dq q{S.c(3)[i], S.c(4)[i], S.c(5)[i], S.c(6)[i]};
  d3 v = S.ld3(7, i);
  d3 w = S.ld3(10, i);
  const d3 f = S.ld3(13, i), tau = S.ld3(16, i), I = S.pld3(5, i), Iinv = S.pld3(8, i);
  const d3 x = S.ld3(0, i);
  const double h = S.pc(1)[i], r = S.pc(0)[i];
  double rf[6], rf2[6];
  for (int k = 0; k < 6; ++k) rf[k] = ref[(size_t)k * n + i];
  if (ref2)
    for (int k = 0; k < 6; ++k) rf2[k] = ref2[(size_t)k * n + i];
  if (im > 0) {
    v = v + (f * im + g) * dt;
    d3 Iw_w = rot_diag_apply(q, I, w);
    d3 gyro = cross(w, Iw_w);
    w = w + rot_diag_apply(q, Iinv, tau - gyro) * dt;
    S.st3(7, i, v);
    S.st3(10, i, w);
  }
  const Seg s = seg_of(x, q, h, r);
  seg_out[i] = s;
  dmax = fmax(dmax, disp_from(s, rf, box, invL));
  if (ref2) dnear = fmax(dnear, disp_from(s, rf2, box, invL));
}

// Position update of rod i (nsc_position_update_body) fused the same way;
// ld, ad: the damping factors 1 - c dt.  Returns 1 when the new state is
// not finite.
__device__ inline int position_update_fused(const StateBase& S, int i, double dt, double ld, double ad,
                                            double w_max, const double* ref, const double* ref2, const Box& box,
                                            const double* invL, Seg* seg_out, double& dmax, double& dnear,
                                            unsigned char* moved, bool spin_project) {
  const int n = S.n;
  d3 v = S.ld3(7, i), w = S.ld3(10, i);
  d3 x = S.ld3(0, i);
  dq q{S.c(3)[i], S.c(4)[i], S.c(5)[i], S.c(6)[i]};
  const double h = S.pc(1)[i], r = S.pc(0)[i];
  double rf[6], rf2[6];
  for (int k = 0; k < 6; ++k) rf[k] = ref[(size_t)k * n + i];
  if (ref2)
    for (int k = 0; k < 6; ++k) rf2[k] = ref2[(size_t)k * n + i];
  x = x + v * dt;
  d3 hw = w * (0.5 * dt);
  dq wq{0.0, hw.x, hw.y, hw.z};
  dq d = qmul(wq, q);
  q = qnormalize(dq{q.w + d.w, q.x + d.x, q.y + d.y, q.z + d.z});
  v = v * ld;
  w = w * ad;
  double wl = len(w);
  if (wl > w_max) w = w * (w_max / wl);
  if (spin_project) {  // inside a tube: no spin about the rod axis (main.cpp:4486-4494)
    d3 u = axis_y(q);
    u = u / len(u);
    w = w - u * dot(w, u);
  }
  S.st3(0, i, x);
  S.c(3)[i] = q.w; S.c(4)[i] = q.x; S.c(5)[i] = q.y; S.c(6)[i] = q.z;
  S.st3(7, i, v);
  S.st3(10, i, w);
  const Seg s = seg_of(x, q, h, r);
  seg_out[i] = s;
  if (moved) moved[i] = 0;
  dmax = fmax(dmax, disp_from(s, rf, box, invL));
  if (ref2) dnear = fmax(dnear, disp_from(s, rf2, box, invL));
  return (x.x == x.x && x.y == x.y && x.z == x.z && v.x == v.x) ? 0 : 1;
}

__device__ inline void wrap_pos(const Box& box, d3& p) {
  if (!box.pbc) return;
  double* c[3] = {&p.x, &p.y, &p.z};
  for (int k = 0; k < 3; ++k) {
    double L = box.L[k];
    if (L <= 0.0) continue;
    double x = *c[k];
    for (int it = 0; x < box.lo[k] && it < 64; ++it) x += L;  // bounded
    for (int it = 0; x >= box.hi[k] && it < 64; ++it) x -= L;
    *c[k] = x;
  }
}

__device__ inline void wrap_clear_body(const State& st, const Box& box, int i, unsigned char* moved = nullptr) {
  if (box.pbc) {
    const d3 x0 = st.x.ld(i);
    d3 x = x0;
    wrap_pos(box, x);
    st.x.st(i, x);
    if (moved && (x.x != x0.x || x.y != x0.y || x.z != x0.z)) moved[i] = 1;
  }
  st.f.st(i, mk3(0, 0, 0));
  st.tau.st(i, mk3(0, 0, 0));
}
// The same from the buffer bases (persistent step).
__device__ inline void wrap_clear_body(const StateBase& S, const Box& box, int i, unsigned char* moved) {
  if (box.pbc) {
    const d3 x0 = S.ld3(0, i);
    d3 x = x0;
    wrap_pos(box, x);
    if (x.x != x0.x || x.y != x0.y || x.z != x0.z) {
      S.st3(0, i, x);
      if (moved) moved[i] = 1;
    }
  }
  S.st3(13, i, mk3(0, 0, 0));
  S.st3(16, i, mk3(0, 0, 0));
}

// Everything one team needs to step one system (device copy per system).
struct NscView {
  State st;
  Box box;
  rg_config cfg;
  Ctl* ctl;
  // detector
  Seg* seg;
  int *nbr_cnt, *nbr;
  int maxnb;
  double* ref;
  int words;
  unsigned long long* mask;
  int* hit_cnt;
  int *cell_of, *cell_cnt, *cell_start, *cell_fill, *cell_rods;
  GridDev* grid;
  unsigned long long* bounds;  // min keys [3], max keys [3]
  double skin, margin, cut_center;
  int all_pairs;
  // contacts and NSC buffers
  Contacts con;
  double *row, *lam;
  int *color, *order, *color_cnt, *color_off, *cursor, *remaining;
  unsigned long long *pmax, *cmask;
  int* owner;
  unsigned long long* wkey;
  double* wlam;
  int* wn;
  int wcap;
  double* xrow;  // contact-network export (null: off), kExportComps x wcap
  double *dx, *prow;
  int* pactive;
  int ccap;
  int* blk;      // per-block scratch of the team
  int* slot_of;  // per-body local slot of the in-block solver (-1 when unused)
  int2* near;    // near list (see Detector); null: test the whole lists
  double* ref2;
  unsigned char* moved;  // see Detector
  double near_skin;
  // learned warm start: features [8][ccap] and predictions [3][ccap] of the
  // team path, the network, and the record buffers ([n][8], [n][3])
  float *feat, *pred;
  int feat_on;   // features needed (learned warm start or recording)
  int use_mlp;   // warm start from the network
  int mlp_min_sweeps;  // ... in steps after one that needed more sweeps than this
  int mlp_all;   // ... for every contact (else only where the cache gives zero)
  MlpDev mlp;
  float *rec_x, *rec_y;
  int rec_cap;   // 0: not recording
};

// A team of blocks [b0, b0 + nb) of the persistent step and the systems it
// runs (entries first .. first + count - 1 of the member list).  A team of
// several blocks runs exactly one system.
struct TeamDesc {
  int b0, nb, first, count;
  unsigned int* bar;  // 4 words: full-team count/gen, subset count/gen
  long long* t_ns;    // optional: the team's device time for the launch
};

void nsc_set_smem();
void nsc_batch_launch(const NscView* views, const TeamDesc* teams, int nteams, const int* members, int grid,
                      int nsteps, cudaStream_t st);
int nsc_block_threads();
size_t nsc_block_smem();
NscView make_view(rg_system* s);

}  // namespace rg
