// simulator.cpp - the reference's Python-session surface on librodgpu.
//
// Mirrors PythonSimulator (src/python/rod_dynamics_py.cpp:52-91) over
// app::createPythonApp / stepPythonSession (src/app/main.cpp:6300-6325):
// a scene JSON (and optional endpoint CSV) configures one system; step(n)
// advances it; rods() and diagnostics() read it back.  The whole contact
// step runs in librodgpu through its C ABI; this file is host-side setup
// (scene parsing, rod population, initial velocities) and result packing.
//
// Scene keys read (src/config/config.cpp, include/config/config.hpp):
//   physics: dt, gravity, lin_damp, ang_damp, w_max, contact_model,
//            soft_contact{...}, hertz_mindlin{...}, nsc{...}
//   scene:   periodic{enabled,min,max}, cylinder{enabled,axis,radius},
//            bodies[{pos, rot_quat (wxyz array,
//            or object, rot_quat_order "xyzw"), rot_axis+rot_deg, shape,
//            length, diameter|radius, density, restitution, is_static,
//            v_lin, v_ang}], populate{count, seed, length, radius, density,
//            maxAttempts}, randomInit{enabled, mode gaussian|thermal|uniform,
//            vSigma, wSigma, wSpeed, kBT, kBTTrans, kBTRot, seed,
//            projectParallelSpin}, initCsvPath
//   b200:    optional extension {warm_start "cache"|"none", tol, skin}
// Populated and randomly initialised scenes use this library's seeded
// generators (random sequential addition with overlap rejection; Gaussian /
// thermal velocities), not the reference's std::mt19937 sequences, so those
// scenes are statistically, not bitwise, the reference's.
#include "simulator.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>

#include "json_min.hpp"

extern "C" {
int rg_scene_rsa(int n, double L, double d, double lo, double side, uint64_t seed, int max_attempts, double* x,
                 double* q);
void rg_capsule_mass(int n, const double* radius, const double* half_height, const double* density,
                     double* mass, double* inertia);
}

namespace rgsim {

namespace {

using rgjson::Value;

void vec3_of(const Value& v, double out[3]) {
  if (v.is_array() && v.arr.size() >= 3)
    for (int k = 0; k < 3; ++k) out[k] = v.arr[k].number(out[k]);
}

// Quaternion (w, x, y, z) rotating +Y onto the unit vector u.
void quat_from_y(const double u[3], double q[4]) {
  const double c = u[1];
  const double ax = u[2], az = -u[0];  // (0,1,0) x u
  const double s = std::sqrt(ax * ax + az * az);
  if (s < 1e-12) {
    if (c > 0) { q[0] = 1; q[1] = q[2] = q[3] = 0; }
    else { q[0] = 0; q[1] = 1; q[2] = q[3] = 0; }  // half turn about x
    return;
  }
  const double h = 0.5 * std::atan2(s, c), sh = std::sin(h) / s;
  q[0] = std::cos(h); q[1] = ax * sh; q[2] = 0.0; q[3] = az * sh;
}

void axis_of(const double q[4], double u[3]) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  u[0] = 2 * (x * y - w * z);
  u[1] = 1 - 2 * (x * x + z * z);
  u[2] = 2 * (y * z + w * x);
}

void rotation_of(const Value& b, double q[4]) {
  q[0] = 1; q[1] = q[2] = q[3] = 0;
  if (b.has("rot_quat")) {
    const Value& r = b["rot_quat"];
    double v[4] = {1, 0, 0, 0};
    if (r.is_array() && r.arr.size() >= 4) {
      for (int k = 0; k < 4; ++k) v[k] = r.arr[k].number(v[k]);
      if (b["rot_quat_order"].string("wxyz") == "xyzw") {
        double t[4] = {v[3], v[0], v[1], v[2]};
        std::memcpy(v, t, sizeof(v));
      }
    } else if (r.is_object()) {
      v[0] = r["w"].number(1); v[1] = r["x"].number(0); v[2] = r["y"].number(0); v[3] = r["z"].number(0);
    }
    double m = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
    if (m > 0)
      for (int k = 0; k < 4; ++k) q[k] = v[k] / m;
  } else if (b.has("rot_deg")) {
    double ax[3] = {0, 1, 0};
    vec3_of(b["rot_axis"], ax);
    double m = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
    double ang = b["rot_deg"].number(0) * M_PI / 180.0;
    if (m > 0) {
      double s = std::sin(0.5 * ang) / m;
      q[0] = std::cos(0.5 * ang); q[1] = ax[0] * s; q[2] = ax[1] * s; q[3] = ax[2] * s;
    }
  }
}

std::string read_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

}  // namespace

Simulator::Simulator(const std::string& scene_path, const std::string& init_csv_path, bool quiet)
    : quiet_(quiet) {
  const Value root = rgjson::parse(read_file(scene_path));
  const Value& ph = root["physics"];
  const Value& sc = root["scene"];
  rg_config_default(&cfg_);

  // ---- physics (config.cpp:310-470) ----
  cfg_.dt = ph["dt"].number(cfg_.dt);
  vec3_of(ph["gravity"], cfg_.gravity);
  cfg_.lin_damp = ph["lin_damp"].number(cfg_.lin_damp);
  cfg_.ang_damp = ph["ang_damp"].number(cfg_.ang_damp);
  cfg_.w_max = ph["w_max"].number(cfg_.w_max);
  const Value& so = ph["soft_contact"];
  cfg_.soft_delta = so["delta"].number(cfg_.soft_delta);
  cfg_.soft_k_scaler = so["k_scaler"].number(cfg_.soft_k_scaler);
  cfg_.soft_damping = so["damping"].number(cfg_.soft_damping);
  cfg_.soft_mu = so["mu"].number(cfg_.soft_mu);
  cfg_.soft_mu_static = so["mu_static"].number(cfg_.soft_mu_static);
  cfg_.soft_nu = so["nu"].number(cfg_.soft_nu);
  cfg_.soft_kt = so["kt"].number(cfg_.soft_kt);
  cfg_.soft_vel_deadband = so["vel_deadband"].number(cfg_.soft_vel_deadband);
  cfg_.soft_enable_friction = so["enable_friction"].boolean(cfg_.soft_enable_friction != 0) ? 1 : 0;
  if (so["friction_cundall"].boolean(false)) cfg_.soft_friction_mode = RG_FRICTION_CUNDALL;
  else if (so["friction_karnopp"].boolean(false)) cfg_.soft_friction_mode = RG_FRICTION_KARNOPP;
  const Value& hm = ph["hertz_mindlin"];
  cfg_.hm_youngs_modulus = hm["youngs_modulus"].number(cfg_.hm_youngs_modulus);
  cfg_.hm_poisson_ratio = hm["poisson_ratio"].number(cfg_.hm_poisson_ratio);
  cfg_.hm_restitution = hm["restitution_coeff"].number(cfg_.hm_restitution);
  cfg_.hm_friction = hm["friction_coeff"].number(cfg_.hm_friction);
  cfg_.hm_friction_static = hm["friction_static_coeff"].number(cfg_.hm_friction_static);
  cfg_.hm_friction_transition_vel = hm["friction_transition_vel"].number(cfg_.hm_friction_transition_vel);
  cfg_.hm_rolling_friction = hm["rolling_friction_coeff"].number(cfg_.hm_rolling_friction);
  cfg_.hm_enable_tangential = hm["enable_tangential"].boolean(cfg_.hm_enable_tangential != 0) ? 1 : 0;
  cfg_.hm_enable_rolling = hm["enable_rolling"].boolean(cfg_.hm_enable_rolling != 0) ? 1 : 0;
  const Value& ns = ph["nsc"];
  cfg_.nsc_mu = ns["mu"].number(cfg_.nsc_mu);
  cfg_.nsc_beta = ns["beta"].number(cfg_.nsc_beta);
  cfg_.nsc_cfm = ns["cfm"].number(cfg_.nsc_cfm);
  cfg_.nsc_omega = ns["omega"].number(cfg_.nsc_omega);
  cfg_.nsc_velocity_iters = (int)ns["velocity_iters"].number(cfg_.nsc_velocity_iters);
  cfg_.nsc_position_stabilization =
      ns["position_stabilization"].boolean(cfg_.nsc_position_stabilization != 0) ? 1 : 0;
  cfg_.nsc_position_iters = (int)ns["position_iters"].number(cfg_.nsc_position_iters);
  cfg_.nsc_position_psor_iters = (int)ns["position_psor_iters"].number(cfg_.nsc_position_psor_iters);
  cfg_.nsc_slop = ns["slop"].number(cfg_.nsc_slop);
  if (!ns["enable_warm_start"].boolean(true)) cfg_.nsc_warm_start = RG_WARM_NONE;
  // model: contact_model overrides the enabled flags (config.cpp:160-183);
  // flags in physicsStep order: nsc, hertz-mindlin, soft (main.cpp:4383-4610)
  std::string model = ph["contact_model"].string("");
  if (model.empty()) {
    if (ns["enabled"].boolean(false)) model = "nsc";
    else if (hm["enabled"].boolean(false)) model = "hertz-mindlin";
    else if (so["enabled"].boolean(false)) model = "harmonic";
  }
  if (model == "nsc") cfg_.model = RG_MODEL_NSC;
  else if (model == "hertz-mindlin") cfg_.model = RG_MODEL_HERTZ_MINDLIN;
  else if (model == "harmonic") cfg_.model = RG_MODEL_HARMONIC;
  else if (model.empty()) cfg_.model = RG_MODEL_NONE;
  else throw std::runtime_error("contact model \"" + model + "\" is not on this library's path");
  const Value& ext = root["b200"];
  const std::string ws = ext["warm_start"].string("");
  if (ws == "none") cfg_.nsc_warm_start = RG_WARM_NONE;
  else if (ws == "cache") cfg_.nsc_warm_start = RG_WARM_CACHE;
  cfg_.nsc_tol = ext["tol"].number(cfg_.nsc_tol);
  cfg_.skin = ext["skin"].number(cfg_.skin);

  // ---- periodic box ----
  const Value& pb = sc["periodic"];
  if (pb["enabled"].boolean(false)) {
    cfg_.pbc_enabled = 1;
    double mn[3] = {-3, -1, -3}, mx[3] = {3, 3, 3};  // PeriodicCfg defaults
    vec3_of(pb["min"], mn);
    vec3_of(pb["max"], mx);
    for (int k = 0; k < 3; ++k) { cfg_.pbc_min[k] = mn[k]; cfg_.pbc_max[k] = mx[k]; }
  }

  // ---- cylindrical tube boundary (config.cpp:517-525) ----
  const Value& cy = sc["cylinder"];
  if (cy["enabled"].boolean(false)) {
    cfg_.cylinder_enabled = 1;
    cfg_.cylinder_radius = cy["radius"].number(cfg_.cylinder_radius);
    vec3_of(cy["axis"], cfg_.cylinder_axis);
    if (cfg_.model == RG_MODEL_HERTZ_MINDLIN && !quiet_)
      std::fprintf(stderr, "[rod_dynamics_py] scene.cylinder has no effect with hertz-mindlin (as in the reference)\n");
  }

  // ---- bodies: endpoint CSV, populate, or the explicit list ----
  const Value& pop = sc["populate"];
  const Value& bl = sc["bodies"];
  const Value* tmpl = (bl.is_array() && !bl.arr.empty()) ? &bl.arr[0] : nullptr;
  const std::string csv = init_csv_path.empty() ? sc["initCsvPath"].string("") : init_csv_path;
  std::vector<double> dens;
  if (!csv.empty()) {
    load_csv(csv, pop, tmpl, dens);
  } else if ((int)pop["count"].number(0) > 0) {
    populate(pop, dens);
  } else if (bl.is_array()) {
    for (const Value& b : bl.arr) add_body(&b, dens);
  }
  n_ = (int)radius_.size();
  if (n_ == 0) throw std::runtime_error("scene has no rods");
  cfg_.n_bodies = n_;

  // ---- mass properties (RigidBody::makeCapsule, rigid_body.cpp:11-55) ----
  mass_.assign(n_, 0.0);
  inertia_.assign(3 * (size_t)n_, 0.0);
  rg_capsule_mass(n_, radius_.data(), half_.data(), dens.data(), mass_.data(), inertia_.data());
  for (int i = 0; i < n_; ++i)
    if (static_[i]) {
      mass_[i] = 0.0;
      inertia_[3 * i] = inertia_[3 * i + 1] = inertia_[3 * i + 2] = 0.0;
    }

  // ---- initial velocities ----
  const Value& ri = sc["randomInit"];
  if (ri["enabled"].boolean(false)) random_init(ri);

  int rc = rg_create(&cfg_, &sys_);
  if (rc != RG_OK) {
    sys_ = nullptr;
    throw std::runtime_error(std::string("rg_create: ") + rg_status_string(rc));
  }
  check(rg_set_bodies(sys_, radius_.data(), half_.data(), mass_.data(), inertia_.data(), rest_.data()),
        "rg_set_bodies");
  check(rg_set_state(sys_, x_.data(), q_.data(), v_.data(), w_.data(), nullptr, nullptr), "rg_set_state");
  f_.assign(3 * (size_t)n_, 0.0);
  tau_.assign(3 * (size_t)n_, 0.0);
  last_ke_ = kinetic_energy();
}

Simulator::~Simulator() {
  if (sys_) rg_destroy(sys_);
}

void Simulator::check(int rc, const char* what) const {
  if (rc != RG_OK) {
    std::string msg = std::string(what) + ": " + rg_status_string(rc);
    if (sys_) msg += std::string(" (") + rg_last_error(sys_) + ")";
    throw std::runtime_error(msg);
  }
}

void Simulator::add_body(const rgjson::Value* b, std::vector<double>& dens) {
  static const Value empty;
  const Value& B = b ? *b : empty;
  const std::string shape = B["shape"].string("capsule");
  if (shape != "capsule") throw std::runtime_error("body shape \"" + shape + "\": this library steps capsules");
  const double len = B["length"].number(0.5);
  const double diam = B.has("radius") ? 2.0 * B["radius"].number(0.05) : B["diameter"].number(0.1);
  double pos[3] = {0, 0, 0}, vl[3] = {0, 0, 0}, va[3] = {0, 0, 0}, q[4];
  vec3_of(B["pos"], pos);
  vec3_of(B["v_lin"], vl);
  vec3_of(B["v_ang"], va);
  rotation_of(B, q);
  push(pos, q, vl, va, 0.5 * diam, 0.5 * len, B["density"].number(1000.0), B["restitution"].number(0.2),
       B["is_static"].boolean(false), dens);
}

void Simulator::push(const double x[3], const double q[4], const double v[3], const double w[3], double r,
                     double h, double rho, double e, bool is_static, std::vector<double>& dens) {
  for (int k = 0; k < 3; ++k) {
    x_.push_back(x[k]);
    v_.push_back(is_static ? 0.0 : v[k]);
    w_.push_back(is_static ? 0.0 : w[k]);
  }
  for (int k = 0; k < 4; ++k) q_.push_back(q[k]);
  radius_.push_back(r);
  half_.push_back(h);
  rest_.push_back(e);
  dens.push_back(rho);
  static_.push_back(is_static ? 1 : 0);
}

void Simulator::populate(const rgjson::Value& pop, std::vector<double>& dens) {
  if (!cfg_.pbc_enabled) throw std::runtime_error("scene.populate needs scene.periodic in this library");
  const int n = (int)pop["count"].number(0);
  const double L = pop["length"].number(1.0);
  const double r = pop["radius"].number(0.05);
  const double rho = pop["density"].number(2500.0);
  const double side = cfg_.pbc_max[0] - cfg_.pbc_min[0];
  for (int k = 1; k < 3; ++k)
    if (std::fabs((cfg_.pbc_max[k] - cfg_.pbc_min[k]) - side) > 1e-9 * side)
      throw std::runtime_error("scene.populate needs a cubic periodic box in this library");
  std::vector<double> x(3 * (size_t)n), q(4 * (size_t)n);
  const uint64_t seed = (uint64_t)pop["seed"].number(1);
  const int att = (int)pop["maxAttempts"].number(200000);
  const int placed = rg_scene_rsa(n, L, 2.0 * r, cfg_.pbc_min[0], side, seed, att, x.data(), q.data());
  if (placed < n && !quiet_) fprintf(stderr, "[rod_dynamics_py] populate placed %d of %d rods\n", placed, n);
  const double zero[3] = {0, 0, 0};
  for (int i = 0; i < placed; ++i) push(&x[3 * i], &q[4 * i], zero, zero, r, 0.5 * L, rho, 0.2, false, dens);
}

// Endpoint CSV (x0,y0,z0,x1,y1,z1 per row; '#' metadata lines may give
// rod_radius), as the reference's initCsvPath loader reads.
void Simulator::load_csv(const std::string& path, const rgjson::Value& pop, const rgjson::Value* tmpl,
                         std::vector<double>& dens) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("cannot open " + path);
  double r = pop.has("radius") ? pop["radius"].number(0.05) : (tmpl ? 0.5 * (*tmpl)["diameter"].number(0.1) : 0.05);
  const double rho =
      pop.has("density") ? pop["density"].number(2500.0) : (tmpl ? (*tmpl)["density"].number(1000.0) : 1000.0);
  std::string line;
  const double zero[3] = {0, 0, 0};
  while (std::getline(f, line)) {
    if (line.empty()) continue;
    if (line[0] == '#') {
      const auto pos = line.find("rod_radius");
      if (pos != std::string::npos) {
        std::string rest = line.substr(pos + 10);
        for (char& c : rest)
          if (c == ':' || c == '=' || c == ',') c = ' ';
        std::stringstream ss(rest);
        double v;
        if (ss >> v) r = v;
      }
      continue;
    }
    for (char& c : line)
      if (c == ',') c = ' ';
    std::stringstream ss(line);
    double p[6];
    int k = 0;
    while (k < 6 && (ss >> p[k])) ++k;
    if (k < 6) continue;  // header or short row
    double c[3], u[3], len = 0;
    for (int a = 0; a < 3; ++a) {
      c[a] = 0.5 * (p[a] + p[3 + a]);
      u[a] = p[3 + a] - p[a];
      len += u[a] * u[a];
    }
    len = std::sqrt(len);
    if (len > 0) {
      for (int a = 0; a < 3; ++a) u[a] /= len;
    } else {
      u[0] = 0; u[1] = 1; u[2] = 0;
    }
    double q[4];
    quat_from_y(u, q);
    push(c, q, zero, zero, r, 0.5 * len, rho, 0.2, false, dens);
  }
}

void Simulator::random_init(const rgjson::Value& ri) {
  const std::string mode = ri["mode"].string("thermal");
  std::mt19937_64 gen((uint64_t)ri["seed"].number(42));
  std::normal_distribution<double> N01(0.0, 1.0);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  const bool proj = ri["projectParallelSpin"].boolean(true);
  for (int i = 0; i < n_; ++i) {
    if (static_[i]) continue;
    double v[3], w[3];
    if (mode == "gaussian") {
      const double sv = ri["vSigma"].number(0), sw = ri["wSigma"].number(0);
      for (int k = 0; k < 3; ++k) v[k] = sv * N01(gen);
      for (int k = 0; k < 3; ++k) w[k] = sw * N01(gen);
    } else if (mode == "uniform") {
      const double sv = ri["vSigma"].number(0), wsp = ri["wSpeed"].number(0);
      for (int k = 0; k < 3; ++k) v[k] = sv * U(gen);
      double d[3] = {N01(gen), N01(gen), N01(gen)};
      const double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      for (int k = 0; k < 3; ++k) w[k] = dn > 0 ? wsp * d[k] / dn : 0.0;
    } else {  // thermal: sigma_v = sqrt(kBT/m), sigma_w = sqrt(kBT/I_perp)
      const double kbt = ri["kBT"].number(1.0);
      double kt = ri["kBTTrans"].number(-1.0), kr = ri["kBTRot"].number(-1.0);
      if (kt < 0) kt = kbt;
      if (kr < 0) kr = kbt;
      const double mi = mass_[i] > 0 ? mass_[i] : 1.0;
      const double ip = inertia_[3 * i] > 0 ? inertia_[3 * i] : 1.0;
      const double sv = std::sqrt(kt / mi), sw = std::sqrt(kr / ip);
      for (int k = 0; k < 3; ++k) v[k] = sv * N01(gen);
      for (int k = 0; k < 3; ++k) w[k] = sw * N01(gen);
    }
    if (proj) {  // remove spin about the rod axis
      double u[3];
      axis_of(&q_[4 * i], u);
      const double p = w[0] * u[0] + w[1] * u[1] + w[2] * u[2];
      for (int k = 0; k < 3; ++k) w[k] -= p * u[k];
    }
    for (int k = 0; k < 3; ++k) {
      v_[3 * i + k] = v[k];
      w_[3 * i + k] = w[k];
    }
  }
}

void Simulator::step(int steps) {
  if (steps <= 0) return;
  if (!csv_ && !net_) {
    check(rg_step(sys_, steps, &stats_), "rg_step");
    frame_ += steps;
    last_ke_ = stats_.kinetic_energy;
    last_hits_ = stats_.contacts;
    fresh_ = false;
    return;
  }
  for (int k = 0; k < steps; ++k) {  // one frame per call, each one logged
    check(rg_step(sys_, 1, &stats_), "rg_step");
    frame_ += 1;
    last_ke_ = stats_.kinetic_energy;
    last_hits_ = stats_.contacts;
    fresh_ = false;
    log_frame();
  }
}

void Simulator::enable_csv(const std::string& path) {
  csv_.reset(new std::ofstream(path.empty() ? std::string("profile.csv") : path, std::ios::out | std::ios::trunc));
  if (!*csv_) {
    csv_.reset();
    throw std::runtime_error("cannot open CSV file: " + path);
  }
  csv_header_ = false;
  rg_set_profiling(sys_, 1);  // phase / stage timers for the *_ms columns
}

void Simulator::enable_network(const std::string& path, int stride, int max_frames) {
  if (cfg_.model != RG_MODEL_NSC)
    throw std::runtime_error("the contact-network export is available for nsc scenes");
  net_.reset(new std::ofstream(path.empty() ? std::string("network.csv") : path, std::ios::out | std::ios::trunc));
  if (!*net_) {
    net_.reset();
    throw std::runtime_error("cannot open network file: " + path);
  }
  net_header_ = false;
  net_stride_ = stride < 1 ? 1 : stride;
  net_max_ = max_frames;
  net_written_ = 0;
  check(rg_set_network_export(sys_, 1), "rg_set_network_export");
}

// Centre of mass, per axis the circular mean in periodic dimensions
// (App::computeCOM, main.cpp:3500-3571).
void Simulator::com(double c[3]) const {
  const double pi = 3.14159265358979323846;
  for (int k = 0; k < 3; ++k) {
    const double L = cfg_.pbc_max[k] - cfg_.pbc_min[k];
    double m_sum = 0, s0 = 0, s1 = 0;
    for (int i = 0; i < n_; ++i) {
      const double m = mass_[i];
      m_sum += m;
      if (cfg_.pbc_enabled && L > 0) {
        const double th = 2.0 * pi * (x_[3 * i + k] - cfg_.pbc_min[k]) / L;
        s0 += m * std::cos(th);
        s1 += m * std::sin(th);
      } else {
        s0 += m * x_[3 * i + k];
      }
    }
    if (cfg_.pbc_enabled && L > 0) {
      double a = std::atan2(s1 / m_sum, s0 / m_sum);
      if (a < 0.0) a += 2.0 * pi;
      c[k] = cfg_.pbc_min[k] + a / (2.0 * pi) * L;
    } else {
      c[k] = s0 / m_sum;
    }
  }
}

namespace {
double min_image(double d, double L, bool pbc) { return pbc && L > 0 ? d - L * std::floor(d / L + 0.5) : d; }
}  // namespace

// Mean squared distance from the centre of mass (computeGyrationSq,
// main.cpp:938-960).
double Simulator::gyration_sq() const {
  if (n_ == 0) return 0.0;
  double c[3];
  com(c);
  double sum = 0;
  for (int i = 0; i < n_; ++i)
    for (int k = 0; k < 3; ++k) {
      const double d = min_image(x_[3 * i + k] - c[k], cfg_.pbc_max[k] - cfg_.pbc_min[k], cfg_.pbc_enabled);
      sum += d * d;
    }
  return sum / n_;
}

// Mean squared displacement since the last logged frame relative to the
// centre of mass motion (computeRelativeMotionSq, main.cpp:963-1022); 0 on
// the first call.
double Simulator::relative_motion_sq() {
  if (n_ == 0) return 0.0;
  double c[3];
  com(c);
  if (!has_last_pos_ || (int)last_pos_.size() != 3 * n_) {
    last_pos_ = x_;
    for (int k = 0; k < 3; ++k) last_com_[k] = c[k];
    has_last_pos_ = true;
    return 0.0;
  }
  double dc[3];
  for (int k = 0; k < 3; ++k)
    dc[k] = min_image(c[k] - last_com_[k], cfg_.pbc_max[k] - cfg_.pbc_min[k], cfg_.pbc_enabled);
  double sum = 0;
  for (int i = 0; i < n_; ++i)
    for (int k = 0; k < 3; ++k) {
      const double d = min_image(x_[3 * i + k] - last_pos_[3 * i + k], cfg_.pbc_max[k] - cfg_.pbc_min[k],
                                 cfg_.pbc_enabled) - dc[k];
      sum += d * d;
    }
  last_pos_ = x_;
  for (int k = 0; k < 3; ++k) last_com_[k] = c[k];
  return sum / n_;
}

// One frame of the profile CSV and the network CSV.  Columns this library
// has no counterpart for are written as the reference writes unavailable
// values: -1 for the per-phase kinetic energies, 0 for islands, sleeping,
// render and the entanglement observable.
void Simulator::log_frame() {
  sync();
  if (csv_) {
    std::ostream& o = *csv_;
    const bool nsc = cfg_.model == RG_MODEL_NSC;
    double ph[12] = {0}, st[RG_NSTAGES] = {0};
    rg_get_phase_times(sys_, ph, 12);
    rg_get_profile(sys_, st, nullptr);
    rg_set_profiling(sys_, 1);  // restart the accumulators: per-frame times
    if (!csv_header_) {
      if (!nsc)
        o << "frame,rods,integrate_ms,sleep_ms,broadphase_ms,bpCount_ms,bpPrefix_ms,bpFill_ms,bpPairs_ms,"
             "solve_ms,pbcWrap_ms,render_ms,contacts,collisions,KE,soft_PE,gyration_sq,reldisp_sq,"
             "ent_pairs,ent_sum,step_ms\n";
      else
        o << "frame,rods,integrate_ms,sleep_ms,broadphase_ms,bpCount_ms,bpPrefix_ms,bpFill_ms,bpPairs_ms,"
             "bpLongLong_ms,warmstart_ms,buildIslands_ms,solve_ms,floorSolve_ms,posCorrect_ms,pbcWrap_ms,"
             "render_ms,contacts,collisions,islands,KE,KE_after_integrate,KE_after_warmstart,KE_after_solve,"
             "KE_after_posCorrect,KE_after_pbcWrap,soft_PE,gyration_sq,reldisp_sq,jn_sum,jt_sum,nsc_residual,"
             "ent_pairs,ent_sum,step_ms\n";
      csv_header_ = true;
    }
    const double gyr = gyration_sq(), rel = relative_motion_sq();
    if (!nsc) {
      // stage timers: 0 integrate, 1 detect, 6 contact forces
      o << frame_ << ',' << n_ << ',' << st[0] << ",0," << st[1] << ",0,0,0,0," << st[6] << ",0,0,"
        << stats_.contacts << ",-1," << last_ke_ << ',' << stats_.potential_energy << ',' << gyr << ',' << rel
        << ",0,0," << stats_.device_ms << '\n';
    } else {
      // persistent-step phases: 0 free flight, 1 detection, 2 colouring,
      // 3 manifold rows + warm start, 4 PSOR, 5 position update + wrap,
      // 6-8 position projection
      o << frame_ << ',' << n_ << ',' << (ph[0] + ph[5]) << ",0," << ph[1] << ",0,0,0,0,0," << ph[3] << ','
        << ph[2] << ',' << ph[4] << ",0," << (ph[6] + ph[7] + ph[8]) << ",0,0," << stats_.contacts << ','
        << stats_.collisions << ",0," << last_ke_ << ",-1,-1,-1,-1,-1,0," << gyr << ',' << rel << ','
        << stats_.jn_sum << ',' << stats_.jt_sum << ',' << stats_.residual << ",0,0," << stats_.device_ms
        << '\n';
    }
    if ((frame_ & 0x3F) == 0) o.flush();
  }
  if (net_ && frame_ % net_stride_ == 0 && (net_max_ <= 0 || net_written_ < net_max_)) {
    std::ostream& o = *net_;
    if (!net_header_) {
      o << "frame,rod_i,rod_j,contact_x,contact_y,contact_z,normal_x,normal_y,normal_z,phi,lambda_n,"
           "lambda_t1,lambda_t2,vn_pre,vn_post\n";
      net_header_ = true;
    }
    size_t m = 0;
    rg_get_contact_network(sys_, nullptr, nullptr, 0, &m);
    std::vector<int32_t> pairs(2 * m + 2);
    std::vector<double> rows(12 * m + 12);
    check(rg_get_contact_network(sys_, pairs.data(), rows.data(), m, &m), "rg_get_contact_network");
    for (size_t i = 0; i < m; ++i) {
      o << frame_ << ',' << pairs[2 * i] << ',' << pairs[2 * i + 1];
      for (int k = 0; k < 12; ++k) o << ',' << rows[12 * i + k];
      o << '\n';
    }
    if ((frame_ & 0x3F) == 0) o.flush();
    ++net_written_;
  }
}

// 1/2 m |v|^2 + 1/2 w . (R I R^T) w over dynamic rods (host copy).
double Simulator::kinetic_energy() const {
  double ke = 0;
  for (int i = 0; i < n_; ++i) {
    if (static_[i]) continue;
    const double* q = &q_[4 * i];
    const double qw = q[0], qx = q[1], qy = q[2], qz = q[3];
    // body axes: rows e[a] are the columns of R
    const double e[3][3] = {{1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy + qw * qz), 2 * (qx * qz - qw * qy)},
                            {2 * (qx * qy - qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz + qw * qx)},
                            {2 * (qx * qz + qw * qy), 2 * (qy * qz - qw * qx), 1 - 2 * (qx * qx + qy * qy)}};
    double v2 = 0, rot = 0;
    for (int k = 0; k < 3; ++k) v2 += v_[3 * i + k] * v_[3 * i + k];
    for (int a = 0; a < 3; ++a) {
      const double c = e[a][0] * w_[3 * i] + e[a][1] * w_[3 * i + 1] + e[a][2] * w_[3 * i + 2];
      rot += inertia_[3 * i + a] * c * c;
    }
    ke += 0.5 * mass_[i] * v2 + 0.5 * rot;
  }
  return ke;
}

void Simulator::sync() const {
  if (fresh_) return;
  auto* self = const_cast<Simulator*>(this);
  self->check(rg_get_state(sys_, self->x_.data(), self->q_.data(), self->v_.data(), self->w_.data(),
                           self->f_.data(), self->tau_.data()),
              "rg_get_state");
  self->fresh_ = true;
}

const std::vector<double>& Simulator::x() const { sync(); return x_; }
const std::vector<double>& Simulator::q() const { sync(); return q_; }
const std::vector<double>& Simulator::v() const { sync(); return v_; }
const std::vector<double>& Simulator::w() const { sync(); return w_; }
const std::vector<double>& Simulator::f() const { sync(); return f_; }
const std::vector<double>& Simulator::tau() const { sync(); return tau_; }

void Simulator::endpoints(int i, double a[3], double b[3]) const {
  sync();
  double u[3];
  axis_of(&q_[4 * i], u);
  for (int k = 0; k < 3; ++k) {
    a[k] = x_[3 * i + k] - u[k] * half_[i];
    b[k] = x_[3 * i + k] + u[k] * half_[i];
  }
}

}  // namespace rgsim
