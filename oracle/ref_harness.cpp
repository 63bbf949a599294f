// ref_harness.cpp - drives the reference's OWN physics sources (compiled from
// the reference tree by oracle/Makefile into oracle/_ref/librodref.so).
//
// TEST INFRASTRUCTURE / CPU BASELINE ONLY.  It re-sequences the branches of
// App::physicsStep (src/app/main.cpp:4383-4810) around the reference solver
// classes, because main.cpp itself cannot link here (GL, lodepng and the empty
// entanglement submodule).  Random forces, walls and sleeping are off.
//
// Hertz-Mindlin on capsules has no reference code (HertzMindlinSolver is
// sphere-only, src/physics/hertz_mindlin.cpp:101-144); the HM branch here uses
// the reference ContactDetector and restates the HM law of
// hertz_mindlin.cpp:249-383 in float, labelled as such wherever it is timed.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "config/config.hpp"
#include "physics/collision.hpp"
#include "physics/contact_detector.hpp"
#include "physics/hertz_mindlin.hpp"
#include "physics/integrator.hpp"
#include "physics/nsc_contact.hpp"
#include "physics/rigid_body.hpp"
#include "physics/soft_contact.hpp"

#include "../include/rodgpu.h"

#ifdef _OPENMP
#include <omp.h>
#endif

int g_thread_limit = 0;  // main.cpp:37; 0 = OpenMP default team
extern bool gQuiet;      // runtime_flags.cpp:3; createPythonApp sets it (main.cpp:6301)

struct ref_system {
  rg_config cfg;
  std::vector<RigidBody> rods;
  glm::vec3 gravity;
  SoftContactSolver soft;
  NscContactSolver nsc;
  ContactDetector hm_detector;
  // HM-on-capsules history (restated law; the sphere solver keeps its own).
  struct HMState { glm::vec3 xi{0.0f}; uint64_t last = 0; };
  std::unordered_map<uint64_t, HMState> hm_hist;
  uint64_t hm_frame = 0;
  size_t last_contacts = 0;
};

static glm::vec3 gv(const double* p) { return glm::vec3(float(p[0]), float(p[1]), float(p[2])); }

static void hm_capsule_forces(ref_system& S) {
  const rg_config& c = S.cfg;
  const double nu = c.hm_poisson_ratio;
  const double Es = c.hm_youngs_modulus / (2.0 * (1.0 - nu * nu));
  const double Gs = c.hm_youngs_modulus / (2.0 * (1.0 + nu));
  double gam = 0.0;
  if (c.hm_restitution < 1.0) {
    double l = std::log(c.hm_restitution);
    gam = -l / std::sqrt(M_PI * M_PI + l * l);
  }
  const double dt = c.dt;
  S.hm_frame++;
  S.hm_detector.detectContacts(S.rods);
  const auto& cs = S.hm_detector.getContacts();
  S.last_contacts = cs.size();
  for (const auto& ct : cs) {
    const RigidBody& A = S.rods[ct.body_a];
    const RigidBody& B = S.rods[ct.body_b];
    uint64_t key = (uint64_t(std::min(ct.body_a, ct.body_b)) << 32) | uint64_t(std::max(ct.body_a, ct.body_b));
    auto& st = S.hm_hist[key];
    double delta = ct.surface_limit - ct.distance;
    double Rs = (double(A.cap.r) * B.cap.r) / (double(A.cap.r) + B.cap.r);
    double ms = (double(A.mass) * B.mass) / (double(A.mass) + B.mass);
    double sd = std::max(delta, 0.0), sqd = std::sqrt(sd), sqR = std::sqrt(std::max(Rs, 0.0));
    double kn = (4.0 / 3.0) * Es * sqR * sqd;
    double Fel = kn * sd * sqd;
    glm::vec3 ra = ct.point_a - A.x;
    glm::vec3 rb = ct.point_b - (B.x + ct.shift_b);
    glm::vec3 va = A.v + glm::cross(A.w, ra);
    glm::vec3 vb = B.v + glm::cross(B.w, rb);
    glm::vec3 vrel = vb - va;
    double vn = glm::dot(vrel, ct.normal);
    double Cn = gam * 2.0 * std::sqrt(ms * kn);
    double Fn = std::max(0.0, Fel - Cn * vn);
    glm::vec3 fn = ct.normal * float(Fn);
    glm::vec3 ft(0.0f);
    if (c.hm_enable_tangential) {
      double kt = 8.0 * Gs * sqR * sqd;
      glm::vec3 vt = vrel - ct.normal * float(vn);
      st.xi += vt * float(dt);
      glm::vec3 fel = -float(kt) * st.xi;
      double Ct = gam * 2.0 * std::sqrt(ms * kt);
      ft = fel - float(Ct) * vt;
      double vtm = glm::length(vt);
      double mu = c.hm_friction;
      if (c.hm_friction_static > c.hm_friction && c.hm_friction_transition_vel > 0.0)
        mu += (c.hm_friction_static - c.hm_friction) * std::exp(-vtm / c.hm_friction_transition_vel);
      double fnm = glm::length(fn), ftm = glm::length(ft), ftmax = mu * fnm;
      if (ftm > ftmax && ftm > 1e-10) {
        ft = ft * float(ftmax / ftm);
        if (kt > 1e-10) st.xi = -ft / float(kt);
      }
    }
    glm::vec3 tra(0.0f), trb(0.0f);
    if (c.hm_enable_rolling) {
      glm::vec3 wr = A.w - B.w;
      double wm = glm::length(wr);
      if (!(wm < 1e-10)) {
        glm::vec3 wh = wr / float(wm);
        glm::vec3 tr = -float(c.hm_rolling_friction * Rs * glm::length(fn)) * wh;
        tra = tr * 0.5f;
        trb = -tr * 0.5f;
      }
    }
    glm::vec3 F = fn + ft;
    S.rods[ct.body_a].f -= F;
    S.rods[ct.body_b].f += F;
    S.rods[ct.body_a].tau += glm::cross(ra, -F) + tra;
    S.rods[ct.body_b].tau += glm::cross(rb, F) + trb;
    st.last = S.hm_frame;
  }
  for (auto it = S.hm_hist.begin(); it != S.hm_hist.end();) {
    if (S.hm_frame - it->second.last > 4 || it->second.last == 0) it = S.hm_hist.erase(it);
    else ++it;
  }
}

// Cylinder wall of the soft branch, as App::physicsStep applies it after each
// computeForces (main.cpp:4661-4690, :4756-4787).
static void soft_wall(ref_system& S) {
  const rg_config& c = S.cfg;
  if (!c.cylinder_enabled) return;
  const float cylR = float(c.cylinder_radius);
  const glm::vec3 cylAxis = glm::normalize(gv(c.cylinder_axis));
  const float k_wall = float(c.soft_k_scaler), c_wall = float(c.soft_damping), mu_wall = float(c.soft_mu);
  const float nu_wall = std::max((float)c.soft_nu, 1e-10f);
  for (auto& rb : S.rods) {
    if (rb.invMass <= 0.0f) continue;
    const float maxD = cylR - rb.cap.r;
    glm::vec3 p_perp = rb.x - glm::dot(rb.x, cylAxis) * cylAxis;
    float d_perp = glm::length(p_perp);
    float pen = d_perp - maxD;
    if (pen <= 0.0f) continue;
    glm::vec3 n = (d_perp > 1e-8f) ? p_perp / d_perp
        : glm::normalize(glm::cross(cylAxis, (std::abs(cylAxis.x) < 0.9f) ? glm::vec3(1, 0, 0) : glm::vec3(0, 1, 0)));
    float v_n = glm::dot(rb.v, n);
    float Fn_mag = k_wall * pen + c_wall * std::max(v_n, 0.0f);
    rb.f -= Fn_mag * n;
    glm::vec3 v_t = rb.v - v_n * n;
    float v_t_len = glm::length(v_t);
    if (v_t_len > 1e-12f) {
      float smooth = std::tanh(v_t_len / nu_wall);
      rb.f -= (mu_wall * Fn_mag * smooth / v_t_len) * v_t;
    }
  }
}

static void force_eval(ref_system& S) {
  if (S.cfg.model == RG_MODEL_HARMONIC) {
    S.soft.detectContacts(S.rods);
    S.last_contacts = S.soft.getNumContacts();
    S.soft.computeForces(S.rods, S.cfg.dt, S.gravity);
    soft_wall(S);
  } else if (S.cfg.model == RG_MODEL_HERTZ_MINDLIN) {
    hm_capsule_forces(S);
  }
}

static void nsc_step(ref_system& S) {
  const float dt = float(S.cfg.dt);
  auto& rods = S.rods;
  // main.cpp:4397-4408
#pragma omp parallel for schedule(static) if ((int)rods.size() > 1000)
  for (int i = 0; i < (int)rods.size(); ++i) {
    auto& rb = rods[i];
    if (rb.invMass > 0) {
      rb.v += (rb.f * rb.invMass + S.gravity) * dt;
      glm::mat3 Iinv = rb.IworldInv();
      glm::mat3 Iw = rb.R() * rb.I_body * glm::transpose(rb.R());
      glm::vec3 gyro = glm::cross(rb.w, Iw * rb.w);
      rb.w += Iinv * (rb.tau - gyro) * dt;
    }
  }
  S.nsc.detectAndBuildManifolds(rods);
  // cylinder wall contacts (main.cpp:4431-4447)
  if (S.cfg.cylinder_enabled) {
    const float cylR = float(S.cfg.cylinder_radius);
    const glm::vec3 cylAxis = glm::normalize(gv(S.cfg.cylinder_axis));
    std::vector<Contact> cyl;
    for (int i = 0; i < (int)rods.size(); ++i) {
      if (rods[i].invMass <= 0.0f) continue;
      cyl.clear();
      collideCapsuleInsideCylinder(rods[i], cylR, cylAxis, cyl);
      for (const auto& c : cyl) S.nsc.addWallContact(i, c, rods, rods[i].restitution);
    }
  }
  S.last_contacts = S.nsc.getNumContacts();
  S.nsc.solveVelocities(rods, dt);
  // main.cpp:4469-4483
#pragma omp parallel for schedule(static) if ((int)rods.size() > 1000)
  for (int i = 0; i < (int)rods.size(); ++i) {
    auto& rb = rods[i];
    rb.x += rb.v * dt;
    glm::quat wq(0.0f, rb.w);
    rb.q += 0.5f * dt * wq * rb.q;
    rb.q = glm::normalize(rb.q);
    rb.v *= (1.0f - g_lin_damp * dt);
    rb.w *= (1.0f - g_ang_damp * dt);
    float wLen = glm::length(rb.w);
    if (wLen > g_w_max) rb.w *= g_w_max / wLen;
  }
  // spin about the rod axis projected out inside the tube (main.cpp:4486-4494)
  if (S.cfg.cylinder_enabled)
    for (auto& rb : rods) {
      glm::vec3 u = glm::normalize(rb.axisY());
      rb.w -= glm::dot(rb.w, u) * u;
    }
  S.nsc.projectPositions(rods);
  if (g_pbc_enabled) {
    for (auto& rb : rods) {
      for (int ax = 0; ax < 3; ++ax) {
        float span = g_pbc_max[ax] - g_pbc_min[ax];
        while (rb.x[ax] < g_pbc_min[ax]) rb.x[ax] += span;
        while (rb.x[ax] >= g_pbc_max[ax]) rb.x[ax] -= span;
      }
    }
  }
  for (auto& rb : rods) { rb.f = glm::vec3(0); rb.tau = glm::vec3(0); }
}

static void verlet_step(ref_system& S) {
  auto& rods = S.rods;
  const float dt = float(S.cfg.dt);
  force_eval(S);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < (int)rods.size(); ++i) integrateHalfPos(rods[i], S.gravity, dt);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < (int)rods.size(); ++i) { rods[i].f = glm::vec3(0); rods[i].tau = glm::vec3(0); }
  force_eval(S);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < (int)rods.size(); ++i) integrateSecondHalf(rods[i], S.gravity, dt);
}

extern "C" {

int ref_create(const rg_config* c, ref_system** out, int threads, int use_spatial_hash) {
  if (!c || !out || c->n_bodies <= 0) return RG_ERR_ARG;
  ref_system* S = new ref_system();
  S->cfg = *c;
  gQuiet = true;
  g_thread_limit = threads;
  S->gravity = gv(c->gravity);
  g_lin_damp = float(c->lin_damp);
  g_ang_damp = float(c->ang_damp);
  g_w_max = float(c->w_max);
  g_pbc_enabled = c->pbc_enabled != 0;
  g_pbc_min = gv(c->pbc_min);
  g_pbc_max = gv(c->pbc_max);
  SoftContactCfg sc;
  sc.enabled = c->model == RG_MODEL_HARMONIC;
  sc.delta = c->soft_delta;
  sc.k_scaler = float(c->soft_k_scaler);
  sc.damping = float(c->soft_damping);
  sc.mu = float(c->soft_mu);
  sc.mu_static = c->soft_mu_static;
  sc.nu = c->soft_nu;
  sc.enable_friction = c->soft_enable_friction != 0;
  sc.friction_cundall = c->soft_friction_mode == RG_FRICTION_CUNDALL;
  sc.friction_karnopp = c->soft_friction_mode == RG_FRICTION_KARNOPP;
  sc.kt = c->soft_kt;
  sc.vel_deadband = c->soft_vel_deadband;
  sc.use_spatial_hash = use_spatial_hash != 0;
  S->soft.setConfig(sc);
  S->soft.setPBC(g_pbc_enabled, g_pbc_min, g_pbc_max);
  NscContactCfg nc;
  nc.enabled = c->model == RG_MODEL_NSC;
  nc.mu = float(c->nsc_mu);
  nc.beta = float(c->nsc_beta);
  nc.cfm = float(c->nsc_cfm);
  nc.omega = float(c->nsc_omega);
  nc.velocity_iters = c->nsc_velocity_iters;
  nc.position_stabilization = c->nsc_position_stabilization != 0;
  nc.position_iters = c->nsc_position_iters;
  nc.position_psor_iters = c->nsc_position_psor_iters;
  nc.slop = float(c->nsc_slop);
  nc.use_spatial_hash = use_spatial_hash != 0;
  nc.enable_warm_start = c->nsc_warm_start == RG_WARM_CACHE;
  S->nsc.setConfig(nc);
  S->nsc.setPBC(g_pbc_enabled, g_pbc_min, g_pbc_max);
  ContactDetectionCfg dc;
  dc.delta = 0.0;
  dc.use_spatial_hash = use_spatial_hash != 0;
  S->hm_detector.setConfig(dc);
  S->hm_detector.setPBC(g_pbc_enabled, g_pbc_min, g_pbc_max);
  S->rods.resize(c->n_bodies);
  *out = S;
  return RG_OK;
}

int ref_destroy(ref_system* S) { delete S; return RG_OK; }

// Bodies are built with RigidBody::makeCapsule (rigid_body.cpp:11-47) from
// radius / half height / density; mass <= 0 marks a static body as
// App::createRod does (main.cpp:1523-1529).
int ref_set_bodies(ref_system* S, const double* radius, const double* half_height,
                   const double* density, const double* restitution, const int32_t* is_static) {
  for (size_t i = 0; i < S->rods.size(); ++i) {
    RigidBody rb = RigidBody::makeCapsule(glm::vec3(0.0f), glm::quat(1, 0, 0, 0), float(density[i]),
                                          float(radius[i]), float(half_height[i]),
                                          restitution ? float(restitution[i]) : 0.2f, 0.7f);
    if (is_static && is_static[i]) {
      rb.mass = 0.0f; rb.invMass = 0.0f;
      rb.I_body = glm::mat3(0.0f); rb.I_body_inv = glm::mat3(0.0f);
    }
    S->rods[i] = rb;
  }
  return RG_OK;
}

int ref_get_mass(const ref_system* S, double* mass, double* inertia) {
  for (size_t i = 0; i < S->rods.size(); ++i) {
    mass[i] = S->rods[i].mass;
    inertia[3 * i] = S->rods[i].I_body[0][0];
    inertia[3 * i + 1] = S->rods[i].I_body[1][1];
    inertia[3 * i + 2] = S->rods[i].I_body[2][2];
  }
  return RG_OK;
}

int ref_set_state(ref_system* S, const double* x, const double* q, const double* v, const double* w) {
  for (size_t i = 0; i < S->rods.size(); ++i) {
    auto& rb = S->rods[i];
    rb.x = gv(x + 3 * i);
    rb.q = glm::quat(float(q[4 * i]), float(q[4 * i + 1]), float(q[4 * i + 2]), float(q[4 * i + 3]));
    rb.v = gv(v + 3 * i);
    rb.w = gv(w + 3 * i);
    rb.f = glm::vec3(0.0f);
    rb.tau = glm::vec3(0.0f);
  }
  return RG_OK;
}

int ref_get_state(const ref_system* S, double* x, double* q, double* v, double* w, double* f, double* tau) {
  for (size_t i = 0; i < S->rods.size(); ++i) {
    const auto& rb = S->rods[i];
    for (int k = 0; k < 3; ++k) {
      if (x) x[3 * i + k] = rb.x[k];
      if (v) v[3 * i + k] = rb.v[k];
      if (w) w[3 * i + k] = rb.w[k];
      if (f) f[3 * i + k] = rb.f[k];
      if (tau) tau[3 * i + k] = rb.tau[k];
    }
    if (q) { q[4 * i] = rb.q.w; q[4 * i + 1] = rb.q.x; q[4 * i + 2] = rb.q.y; q[4 * i + 3] = rb.q.z; }
  }
  return RG_OK;
}

// Contact forces and torques at the current state (one force evaluation of
// the Verlet models; it advances the history as a step's evaluation does).
int ref_compute_forces(ref_system* S, double* f, double* tau) {
  for (auto& rb : S->rods) { rb.f = glm::vec3(0); rb.tau = glm::vec3(0); }
  force_eval(*S);
  for (size_t i = 0; i < S->rods.size(); ++i)
    for (int k = 0; k < 3; ++k) {
      if (f) f[3 * i + k] = S->rods[i].f[k];
      if (tau) tau[3 * i + k] = S->rods[i].tau[k];
    }
  for (auto& rb : S->rods) { rb.f = glm::vec3(0); rb.tau = glm::vec3(0); }
  return RG_OK;
}

int ref_step(ref_system* S, int nsteps, int64_t* contacts, double* residual) {
  for (int k = 0; k < nsteps; ++k) {
    if (S->cfg.model == RG_MODEL_NSC) nsc_step(*S);
    else if (S->cfg.model == RG_MODEL_HARMONIC || S->cfg.model == RG_MODEL_HERTZ_MINDLIN) verlet_step(*S);
  }
  if (contacts) *contacts = (int64_t)S->last_contacts;
  if (residual) *residual = S->cfg.model == RG_MODEL_NSC ? S->nsc.getLastResidual() : 0.0;
  return RG_OK;
}

// ContactDetector::detectContacts at the current state with margin delta.
int ref_detect(ref_system* S, double delta, int use_spatial_hash, int32_t* pairs, double* dist,
               size_t cap, size_t* n) {
  ContactDetectionCfg dc;
  dc.delta = delta;
  dc.use_spatial_hash = use_spatial_hash != 0;
  ContactDetector det(dc);
  det.setPBC(g_pbc_enabled, g_pbc_min, g_pbc_max);
  det.detectContacts(S->rods);
  std::vector<ContactPrimitive> cs = det.getContacts();
  std::sort(cs.begin(), cs.end(), [](const ContactPrimitive& a, const ContactPrimitive& b) {
    return a.body_a != b.body_a ? a.body_a < b.body_a : a.body_b < b.body_b;
  });
  *n = cs.size();
  for (size_t i = 0; i < std::min(cap, cs.size()); ++i) {
    pairs[2 * i] = cs[i].body_a;
    pairs[2 * i + 1] = cs[i].body_b;
    if (dist) dist[i] = cs[i].distance;
  }
  return cs.size() > cap ? RG_ERR_CAPACITY : RG_OK;
}

// Manifold impulses after the last NSC solve (sorted pair order).
int ref_get_impulses(const ref_system* S, int32_t* pairs, double* lambda, size_t cap, size_t* n) {
  const auto& ms = S->nsc.getManifolds();
  *n = ms.size();
  for (size_t i = 0; i < std::min(cap, ms.size()); ++i) {
    pairs[2 * i] = ms[i].body_a;
    pairs[2 * i + 1] = ms[i].body_b;
    lambda[3 * i] = ms[i].lambda_n;
    lambda[3 * i + 1] = ms[i].lambda_t1;
    lambda[3 * i + 2] = ms[i].lambda_t2;
  }
  return ms.size() > cap ? RG_ERR_CAPACITY : RG_OK;
}

int ref_threads(void) {
#ifdef _OPENMP
  return g_thread_limit > 0 ? g_thread_limit : omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
