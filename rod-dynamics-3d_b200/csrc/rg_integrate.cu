// rg_integrate.cu - per-body update kernels (streaming, HBM-bound).
//
// integrateHalfPos / integrateSecondHalf (src/physics/integrator.cpp:113-159)
// with angularAccelGyro (:39-54) and wrap_position (:23-35); the NSC free
// flight and position update of App::physicsStep (src/app/main.cpp:4397-4408,
// :4469-4483) and its PBC wrap (:4508-4517).  State is structure-of-arrays
// FP64, so every load and store is a fully coalesced 8-byte access.
#include "rg_nsc_dev.cuh"

namespace rg {

// Iinv = 1/I per principal axis for a dynamic body (0 when I = 0), as the
// state's stored inverse (rg_set_bodies), recomputed here to save its load.
__device__ inline d3 ang_accel(const State& st, int i, dq q, d3 w, d3 tau) {
  const d3 I = st.I.ld(i);
  const d3 Iinv{I.x > 0.0 ? 1.0 / I.x : 0.0, I.y > 0.0 ? 1.0 / I.y : 0.0, I.z > 0.0 ? 1.0 / I.z : 0.0};
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

// Resident 256-thread blocks per SM the streaming body kernels are compiled
// for (register budget 65536 / (256 * this)); they are latency-bound at
// one rod per thread, so more resident warps hide more of each load.
#ifndef RG_BODY_MIN_BLOCKS
#define RG_BODY_MIN_BLOCKS 4
#endif

// Velocity Verlet, first half (integrateHalfPos, integrator.cpp:113-134):
// the forces at t are summed per body here from the contact addends (in
// contact order, body_sum) plus the soft cylinder wall, then the half kick,
// drift, periodic wrap and rotation.  The drifted positions' segment records
// and the displacement bound against the list reference (k_disp_check's
// check, rg_detect.cu) are written in the same pass, so the detection at
// t + dt starts at the cell/list stage.
struct DriftOut {
  Seg* seg;           // segment records of the drifted positions (n)
  const double* ref;  // list reference segments (6n), or null: no check
  const double* ref2; // near-list reference segments (6n), or null
  double skin;
};
__global__ void __launch_bounds__(256, RG_BODY_MIN_BLOCKS)
    k_reduce_drift(State st, Box box, rg_config cfg, const int* off, const int* ent, const double* cf,
                   int ccap, int wall, DriftOut o, HistFinish hf, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) hist_finish(hf, ctl);
  __shared__ double sm[32], sm2[32];
  const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
  const double dt = cfg.dt, hdt = 0.5 * cfg.dt;
  const d3 ax = wall ? soft_wall_axis(cfg) : mk3(0, 0, 0);
  const int n = st.n;
  double m = 0.0, m2 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    d3 x = st.x.ld(i);
    dq q = st.q.ld(i);
    if (st.inv_mass[i] > 0.0) {
      d3 f{0, 0, 0}, t{0, 0, 0};
      body_sum(off, ent, cf, ccap, i, f, t);
      d3 v = st.v.ld(i), w = st.w.ld(i);
      if (wall) soft_wall_apply(cfg, ax, st.r[i], x, v, f);
      d3 al = f / st.mass[i] + g;
      d3 aa = ang_accel(st, i, q, w, t);
      v = v + al * hdt;
      w = w + aa * hdt;
      x = x + v * dt;
      wrap_pos(box, x);
      rotate_by_omega(q, w, dt);
      st.v.st(i, v);
      st.w.st(i, w);
      st.x.st(i, x);
      st.q.st(i, q);
    }
    const Seg sg = seg_of(x, q, st.h[i], st.r[i]);
    o.seg[i] = sg;
    if (o.ref) {
      m = fmax(m, seg_disp(sg, o.ref, n, i, box));  // non-finite state: 1e300 forces a rebuild
      if (o.ref2) m2 = fmax(m2, seg_disp(sg, o.ref2, n, i, box));
    }
  }
  if (!o.ref) return;
  m = warp_max(m);
  m2 = warp_max(m2);
  if ((threadIdx.x & 31) == 0) {
    sm[threadIdx.x >> 5] = m;
    sm2[threadIdx.x >> 5] = m2;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    double v2 = threadIdx.x < (blockDim.x >> 5) ? sm2[threadIdx.x] : 0.0;
    v = warp_max(v);
    v2 = warp_max(v2);
    if (threadIdx.x == 0) {
      atomic_max_nonneg(&ctl->maxdisp, v);
      if (v >= 0.5 * o.skin * (1.0 - 1e-9)) atomicExch(&ctl->rebuild, 1);
      if (o.ref2) atomic_max_nonneg(&ctl->near_disp, v2);
    }
  }
}

// Velocity Verlet, second half (integrateSecondHalf, integrator.cpp:136-159):
// the forces at t + dt summed per body (contact addends + soft wall) and
// kept in f, tau; then the half kick, damping and the angular-speed clamp.
__global__ void __launch_bounds__(256, RG_BODY_MIN_BLOCKS)
    k_reduce_kick(State st, rg_config cfg, const int* off, const int* ent, const double* cf, int ccap,
                  int wall, HistFinish hf, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) hist_finish(hf, ctl);
  const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
  const double hdt = 0.5 * cfg.dt;
  const double el = exp(-cfg.lin_damp * cfg.dt), ea = exp(-cfg.ang_damp * cfg.dt);
  const d3 ax = wall ? soft_wall_axis(cfg) : mk3(0, 0, 0);
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    d3 f{0, 0, 0}, t{0, 0, 0};
    body_sum(off, ent, cf, ccap, i, f, t);
    if (st.inv_mass[i] > 0.0) {
      dq q = st.q.ld(i);
      d3 v = st.v.ld(i), w = st.w.ld(i);
      if (wall) soft_wall_apply(cfg, ax, st.r[i], st.x.ld(i), v, f);
      d3 al = f / st.mass[i] + g;
      d3 aa = ang_accel(st, i, q, w, t);
      v = v + al * hdt;
      w = w + aa * hdt;
      if (cfg.lin_damp > 0.0) v = v * el;
      if (cfg.ang_damp > 0.0) w = w * ea;
      double wl = len(w);
      if (wl > cfg.w_max) w = w * (cfg.w_max / wl);
      st.v.st(i, v);
      st.w.st(i, w);
      if (!(v.x == v.x && v.y == v.y && v.z == v.z)) bad = 1;
    }
    st.f.st(i, f);
    st.tau.st(i, t);
  }
  if (bad) atomicOr(&ctl->err, ERR_NONFINITE);
}

__global__ void k_clear_forces(State st, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    st.f.st(i, mk3(0, 0, 0));
    st.tau.st(i, mk3(0, 0, 0));
  }
}

__global__ void k_nsc_free_flight(State st, rg_config cfg, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    nsc_free_flight_body(st, i, g, cfg.dt);
}

__global__ void k_nsc_position_update(State st, rg_config cfg, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  int bad = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    bad |= nsc_position_update_body(st, i, cfg);
  if (bad) atomicOr(&ctl->err, ERR_NONFINITE);
}

__global__ void k_wrap_clear(State st, Box box, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    wrap_clear_body(st, box, i);
}

static inline int body_grid(rg_system* s) { return grid_for(s->n, 256, s->sm_count * 8); }

void reduce_drift_launch(rg_system* s, bool wall, HistFinish hf) {
  const Detector& d = s->det;
  DriftOut o;
  o.seg = d.seg;
  o.ref = d.all_pairs ? nullptr : d.ref;
  o.ref2 = (d.all_pairs || !d.near_cnt) ? nullptr : d.ref2;
  o.skin = d.skin;
  RGL launch_dep(k_reduce_drift, body_grid(s), 256, s->stream, s->st, s->box, s->cfg, s->csr.off, s->csr.ent,
                                                          s->d_cf, s->ccap, wall ? 1 : 0, o, hf, s->d_ctl);
}
void reduce_kick_launch(rg_system* s, bool wall, HistFinish hf) {
  RGL launch_dep(k_reduce_kick, body_grid(s), 256, s->stream, s->st, s->cfg, s->csr.off, s->csr.ent, s->d_cf,
                                                         s->ccap, wall ? 1 : 0, hf, s->d_ctl);
}
void clear_forces_launch(rg_system* s) {
  RGL launch_dep(k_clear_forces, body_grid(s), 256, s->stream, s->st, s->d_ctl);
}
void nsc_free_flight_launch(rg_system* s) {
  RGL launch_dep(k_nsc_free_flight, body_grid(s), 256, s->stream, s->st, s->cfg, s->d_ctl);
}
void nsc_position_update_launch(rg_system* s) {
  RGL launch_dep(k_nsc_position_update, body_grid(s), 256, s->stream, s->st, s->cfg, s->d_ctl);
}
void wrap_launch(rg_system* s) {
  RGL launch_dep(k_wrap_clear, body_grid(s), 256, s->stream, s->st, s->box, s->d_ctl);
}

}  // namespace rg
