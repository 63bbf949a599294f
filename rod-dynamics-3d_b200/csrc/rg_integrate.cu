// rg_integrate.cu - per-body update kernels (streaming, HBM-bound).
//
// integrateHalfPos / integrateSecondHalf (src/physics/integrator.cpp:113-159)
// with angularAccelGyro (:39-54) and wrap_position (:23-35); the NSC free
// flight and position update of App::physicsStep (src/app/main.cpp:4397-4408,
// :4469-4483) and its PBC wrap (:4508-4517).  State is structure-of-arrays
// FP64, so every load and store is a fully coalesced 8-byte access.
#include "rg_nsc_dev.cuh"

namespace rg {

__device__ inline d3 ang_accel(const State& st, int i, dq q, d3 w, d3 tau) {
  d3 I = st.I.ld(i), Iinv = st.Iinv.ld(i);
  d3 Iw_w = rot_diag_apply(q, I, w);
  d3 gyro = cross(w, Iw_w);
  return rot_diag_apply(q, Iinv, tau - gyro);
}

__device__ inline void rotate_by_omega(dq& q, d3 w, double dt) {
  double wl = len(w);
  if (wl > 1e-8) {
    double ang = wl * dt;
    d3 ax = w / wl;
    q = qnormalize(qmul(angle_axis(ang, ax), q));
  }
}

__global__ void k_half_pos(State st, Box box, rg_config cfg, const Ctl* ctl) {
  if (ctl->err) return;
  const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
  const double dt = cfg.dt, hdt = 0.5 * cfg.dt;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    if (st.inv_mass[i] <= 0.0) continue;
    dq q = st.q.ld(i);
    d3 v = st.v.ld(i), w = st.w.ld(i);
    d3 al = st.f.ld(i) / st.mass[i] + g;
    d3 aa = ang_accel(st, i, q, w, st.tau.ld(i));
    v = v + al * hdt;
    w = w + aa * hdt;
    d3 x = st.x.ld(i) + v * dt;
    wrap_pos(box, x);
    rotate_by_omega(q, w, dt);
    st.v.st(i, v);
    st.w.st(i, w);
    st.x.st(i, x);
    st.q.st(i, q);
  }
}

__global__ void k_second_half(State st, rg_config cfg, Ctl* ctl) {
  if (ctl->err) return;
  const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
  const double hdt = 0.5 * cfg.dt;
  const double el = exp(-cfg.lin_damp * cfg.dt), ea = exp(-cfg.ang_damp * cfg.dt);
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    if (st.inv_mass[i] <= 0.0) continue;
    dq q = st.q.ld(i);
    d3 v = st.v.ld(i), w = st.w.ld(i);
    d3 al = st.f.ld(i) / st.mass[i] + g;
    d3 aa = ang_accel(st, i, q, w, st.tau.ld(i));
    v = v + al * hdt;
    w = w + aa * hdt;
    if (cfg.lin_damp > 0.0) v = v * el;
    if (cfg.ang_damp > 0.0) w = w * ea;
    double wl = len(w);
    if (wl > cfg.w_max) w = w * (cfg.w_max / wl);
    st.v.st(i, v);
    st.w.st(i, w);
    st.f.st(i, mk3(0, 0, 0));
    st.tau.st(i, mk3(0, 0, 0));
    if (!(v.x == v.x && v.y == v.y && v.z == v.z)) bad = 1;
  }
  if (bad) atomicOr(&ctl->err, ERR_NONFINITE);
}

__global__ void k_clear_forces(State st, const Ctl* ctl) {
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    st.f.st(i, mk3(0, 0, 0));
    st.tau.st(i, mk3(0, 0, 0));
  }
}

__global__ void k_nsc_free_flight(State st, rg_config cfg, const Ctl* ctl) {
  if (ctl->err) return;
  const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    nsc_free_flight_body(st, i, g, cfg.dt);
}

__global__ void k_nsc_position_update(State st, rg_config cfg, Ctl* ctl) {
  if (ctl->err) return;
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    bad |= nsc_position_update_body(st, i, cfg);
  if (bad) atomicOr(&ctl->err, ERR_NONFINITE);
}

__global__ void k_wrap_clear(State st, Box box, const Ctl* ctl) {
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    wrap_clear_body(st, box, i);
}

static inline int body_grid(rg_system* s) { return grid_for(s->n, 256, s->sm_count * 8); }

void half_pos_launch(rg_system* s) {
  RGL k_half_pos<<<body_grid(s), 256, 0, s->stream>>>(s->st, s->box, s->cfg, s->d_ctl);
}
void second_half_launch(rg_system* s) {
  RGL k_second_half<<<body_grid(s), 256, 0, s->stream>>>(s->st, s->cfg, s->d_ctl);
}
void clear_forces_launch(rg_system* s) {
  RGL k_clear_forces<<<body_grid(s), 256, 0, s->stream>>>(s->st, s->d_ctl);
}
void nsc_free_flight_launch(rg_system* s) {
  RGL k_nsc_free_flight<<<body_grid(s), 256, 0, s->stream>>>(s->st, s->cfg, s->d_ctl);
}
void nsc_position_update_launch(rg_system* s) {
  RGL k_nsc_position_update<<<body_grid(s), 256, 0, s->stream>>>(s->st, s->cfg, s->d_ctl);
}
void wrap_launch(rg_system* s) {
  RGL k_wrap_clear<<<body_grid(s), 256, 0, s->stream>>>(s->st, s->box, s->d_ctl);
}

}  // namespace rg
