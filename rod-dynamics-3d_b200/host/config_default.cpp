// config_default.cpp - rg_config_default (include/rodgpu.h), host C++.
//
// The defaults follow AppCfg (include/config/config.hpp:6-110 of the
// reference): PhysicsCfg dt and gravity, damping and w_max
// (config.cpp:209-211), SoftContactCfg, HertzMindlinCfg and NscContactCfg.
// It is compiled into librodgpu.so, and also into the reference-baseline
// harness library so that both build their configurations from one source.
#include <cstring>

#include "../../include/rodgpu.h"

extern "C" void rg_config_default(rg_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->n_bodies = 0;
  c->model = RG_MODEL_NONE;
  c->dt = 1.0 / 600.0;                  // PhysicsCfg (config.hpp:91)
  c->gravity[1] = -10.0;
  c->lin_damp = 0.08; c->ang_damp = 0.12; c->w_max = 80.0;
  c->pbc_enabled = 0;
  c->pbc_min[0] = -3; c->pbc_min[1] = -1; c->pbc_min[2] = -3;
  c->pbc_max[0] = 3; c->pbc_max[1] = 3; c->pbc_max[2] = 3;
  c->soft_delta = 0.005; c->soft_k_scaler = 1000.0; c->soft_damping = 0.0; c->soft_mu = 0.5;
  c->soft_mu_static = 0.0; c->soft_nu = 1e-5; c->soft_kt = 1000.0; c->soft_vel_deadband = 1e-3;
  c->soft_enable_friction = 1; c->soft_friction_mode = RG_FRICTION_SMOOTH;
  c->hm_youngs_modulus = 7e10; c->hm_poisson_ratio = 0.25; c->hm_restitution = 0.9;
  c->hm_friction = 0.3; c->hm_friction_static = 0.5; c->hm_friction_transition_vel = 1e-3;
  c->hm_rolling_friction = 0.01; c->hm_enable_tangential = 1; c->hm_enable_rolling = 1;
  c->nsc_mu = 0.3; c->nsc_beta = 0.2; c->nsc_cfm = 0.0; c->nsc_omega = 1.0; c->nsc_slop = 1e-4;
  c->nsc_tol = 1e-6; c->nsc_velocity_iters = 40; c->nsc_position_stabilization = 1;
  c->nsc_position_iters = 5; c->nsc_position_psor_iters = 50; c->nsc_warm_start = RG_WARM_CACHE;
  c->nsc_mlp_scope = 0; c->nsc_mlp_min_sweeps = 3;
  c->psor_order = RG_ORDER_COLORED;
  c->skin = 0.0; c->max_neighbors = 0;
  c->spin_limit = 0; c->test_absent_blocks = 0;
  c->cylinder_enabled = 0; c->cylinder_radius = 0.3;  // CylinderCfg (config.hpp:150-154)
  c->cylinder_axis[0] = 0; c->cylinder_axis[1] = 1; c->cylinder_axis[2] = 0;
}
