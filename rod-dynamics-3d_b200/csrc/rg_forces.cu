// rg_forces.cu - contact forces with tangential history, per-body reduction.
//
// Soft penalty ("harmonic"): SoftContactSolver::computeForces
//   (src/physics/soft_contact.cpp:80-213), potential (:215-253), friction
//   modes smooth / Cundall-Strack / Karnopp (:288-486).
// Hertz-Mindlin: computeHertzForce / computeMindlinForce /
//   computeRollingFriction (src/physics/hertz_mindlin.cpp:249-383) applied to
//   capsule contacts, history retention of pruneContactHistory (:385-393).
//
// History tables live on the device across steps as arrays sorted by pair key
// (a<<32|b).  Each force evaluation looks every contact up by binary search,
// updates the touched entries and merges them with the retained untouched
// ones into the other buffer (a parallel merge by rank), so the table stays
// sorted without a sort.
//
// Forces are reduced per body in contact order through a body->contact CSR,
// which makes the sums deterministic and equal in order to the reference's
// sequential accumulation.
#include "rg_internal.cuh"

namespace rg {

const int* detector_n_dev(rg_system* s);

// ---------------------------------------------------------------------------
// Body CSR: cnt -> scan -> fill -> per-body insertion sort.
// ---------------------------------------------------------------------------
__global__ void k_csr_zero(int* cnt, int* fill, int n, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
    cnt[i] = 0;
    if (i < n) fill[i] = 0;
  }
}
__global__ void k_csr_count(const int* ca, const int* cb, int* cnt, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const int C = ctl->contacts;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    atomicAdd(&cnt[ca[c]], 1);
    atomicAdd(&cnt[cb[c]], 1);
  }
}
__global__ void k_csr_fill(const int* ca, const int* cb, const int* off, int* fill, int* ent,
                           const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const int C = ctl->contacts;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    int a = ca[c], b = cb[c];
    ent[off[a] + atomicAdd(&fill[a], 1)] = 2 * c;
    ent[off[b] + atomicAdd(&fill[b], 1)] = 2 * c + 1;
  }
}
__global__ void k_csr_sort(int n, const int* off, int* ent, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int s = off[i], e = off[i + 1];
    for (int k = s + 1; k < e; ++k) {
      int v = ent[k];
      int m = k;
      while (m > s && ent[m - 1] > v) {
        ent[m] = ent[m - 1];
        --m;
      }
      ent[m] = v;
    }
  }
}

void csr_launch(rg_system* s, bool counted) {
  const int bs = 256;
  cudaStream_t st = s->stream;
  if (!counted) {  // else the narrow phase zeroed and counted (detect_launch, body_csr)
    RGL launch_dep(k_csr_zero, grid_for(s->n + 1, bs), bs, st, s->csr.cnt, s->csr.fill, s->n, s->d_ctl);
    RGL launch_dep(k_csr_count, grid_for(s->ccap, bs), bs, st, s->con.a, s->con.b, s->csr.cnt, s->d_ctl);
  }
  s->scan.run(s->csr.cnt, s->csr.off, detector_n_dev(s), &s->d_ctl->err, st);
  RGL launch_dep(k_csr_fill, grid_for(s->ccap, bs), bs, st, s->con.a, s->con.b, s->csr.off, s->csr.fill,
                                                   s->csr.ent, s->d_ctl);
  RGL launch_dep(k_csr_sort, grid_for(s->n, bs), bs, st, s->n, s->csr.off, s->csr.ent, s->d_ctl);
}

// ---------------------------------------------------------------------------
// History lookup / merge.
// ---------------------------------------------------------------------------
__device__ inline unsigned long long pkey(int a, int b) {
  return ((unsigned long long)(unsigned)a << 32) | (unsigned long long)(unsigned)b;
}
__device__ inline int lower_bound_u64(const unsigned long long* k, int n, unsigned long long v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int m = (lo + hi) >> 1;
    if (k[m] < v) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// kept[e]: entries retained if untouched (HM: 4-frame retention; Cundall:
// all); the force kernel that follows clears the touched ones.  fr is the
// frame this evaluation opens (the force kernel advances ctl->frame).
__global__ void k_hist_keep_init(const long long* hframe, int* kept, int hm, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const int H = ctl->hist_n;
  const long long fr = ctl->frame + 1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < H; e += gridDim.x * blockDim.x) {
    long long lf = hframe[e];
    kept[e] = hm ? ((fr - lf > 4 || lf == 0) ? 0 : 1) : 1;
  }
}
__global__ void k_hist_merge(const int* ca, const int* cb, const int* touched, const int* toff,
                             const double* newval, const unsigned long long* okey, const double* oval,
                             const long long* oframe, const int* kept, const int* koff,
                             unsigned long long* nkey, double* nval, long long* nframe, int cap,
                             int ccap, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const int C = ctl->contacts, H = ctl->hist_n;
  const int T = toff[C], K = koff[H];
  if (T + K > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&ctl->err, ERR_HIST_CAP);
    return;
  }
  const long long fr = ctl->frame;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int c = tid; c < C; c += stride) {
    if (!touched[c]) continue;
    unsigned long long k = pkey(ca[c], cb[c]);
    int lb = lower_bound_u64(okey, H, k);  // kept entries before k
    int p = toff[c] + koff[lb];
    nkey[p] = k;
    nval[p] = newval[c];
    nval[cap + p] = newval[ccap + c];
    nval[2 * cap + p] = newval[2 * ccap + c];
    nframe[p] = fr;
  }
  for (int e = tid; e < H; e += stride) {
    if (!kept[e]) continue;
    unsigned long long k = okey[e];
    // touched contacts with key < k: contacts are sorted by key
    int lo = 0, hi = C;
    while (lo < hi) {
      int m = (lo + hi) >> 1;
      if (pkey(ca[m], cb[m]) < k) lo = m + 1;
      else hi = m;
    }
    int p = koff[e] + toff[lo];
    nkey[p] = k;
    nval[p] = oval[e];
    nval[cap + p] = oval[cap + e];
    nval[2 * cap + p] = oval[2 * cap + e];
    nframe[p] = oframe[e];
  }
}
__global__ void k_hist_finish(const int* toff, const int* koff, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  hist_finish(HistFinish{toff, koff}, ctl);
}

// ---------------------------------------------------------------------------
// Force kernels.  Outputs per contact: addends cf[0..11] = f_a, tau_a, f_b,
// tau_b; new history value (3) and a touched flag; potential energy.
// ---------------------------------------------------------------------------
struct ForceIO {
  int *ca, *cb;
  const double* g;  // contact component arrays (Contacts::comp)
  int ccap;
  const unsigned long long* hkey;  // current table keys (sorted)
  int* kept;           // per table entry: 1 = retained untouched (cleared here when touched)
  const double* hval;  // current table values (3 * hcap SoA)
  int hcap;
  double* newval;      // 3 * ccap
  int* touched;        // ccap
  double* cf;          // 12 * ccap
  double* pe;          // ccap
};

// Index of the pair (a, b) in the history table (binary search over the
// sorted keys), or -1.
__device__ inline int hist_find(const ForceIO& io, int a, int b, int H) {
  const unsigned long long k = pkey(a, b);
  const int p = lower_bound_u64(io.hkey, H, k);
  return (p < H && io.hkey[p] == k) ? p : -1;
}
// The force kernel of an evaluation advances the frame counter (the
// reference's frame_counter_ per detectContacts, hertz_mindlin.cpp:31).
__device__ inline void eval_begin(Ctl* ctl) {
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->frame += 1;
}

__device__ inline d3 ldc(const ForceIO& io, int k, int c) {
  return {io.g[(size_t)k * io.ccap + c], io.g[(size_t)(k + 1) * io.ccap + c],
          io.g[(size_t)(k + 2) * io.ccap + c]};
}
__device__ inline void st_cf(const ForceIO& io, int c, d3 fa, d3 ta, d3 fb, d3 tb) {
  const int cc = io.ccap;
  io.cf[c] = fa.x; io.cf[cc + c] = fa.y; io.cf[2 * cc + c] = fa.z;
  io.cf[3 * cc + c] = ta.x; io.cf[4 * cc + c] = ta.y; io.cf[5 * cc + c] = ta.z;
  io.cf[6 * cc + c] = fb.x; io.cf[7 * cc + c] = fb.y; io.cf[8 * cc + c] = fb.z;
  io.cf[9 * cc + c] = tb.x; io.cf[10 * cc + c] = tb.y; io.cf[11 * cc + c] = tb.z;
}

__global__ void k_soft_forces(State st, rg_config cfg, ForceIO io, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const int C = ctl->contacts, H = ctl->hist_n;
  eval_begin(ctl);
  const double dt = cfg.dt;
  const double K1 = 15.0 / cfg.soft_delta;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    const int a = io.ca[c], b = io.cb[c];
    const int hf = hist_find(io, a, b, H);
    d3 pa = ldc(io, 0, c), pb = ldc(io, 3, c), nrm = ldc(io, 6, c), sh = ldc(io, 9, c);
    double dist = io.g[(size_t)12 * io.ccap + c], hs = io.g[(size_t)13 * io.ccap + c];
    // potentialGradient / potentialEnergy
    double grad, U;
    if (dist > hs - cfg.soft_delta) {
      double arg = K1 * (hs - dist);
      double e = exp(arg);
      double lt = log(1.0 + e);
      grad = -2.0 / (K1 * K1) * lt * e / (1.0 + e);
      double base = lt / K1;
      U = base * base;
    } else {
      grad = -2.0 * (hs - dist);
      double pen = hs - dist;
      U = pen * pen;
    }
    double fm = -cfg.soft_k_scaler * grad;
    d3 fa = nrm * (-fm);
    d3 fb = nrm * fm;
    d3 xa = st.x.ld(a), xb = st.x.ld(b);
    d3 ra = pa - xa;
    d3 rb = pb - (xb + sh);
    d3 va = st.v.ld(a) + cross(st.w.ld(a), ra);
    d3 vb = st.v.ld(b) + cross(st.w.ld(b), rb);
    d3 vrel = va - vb;
    if (cfg.soft_damping > 1e-9) {
      double vn = dot(vrel, nrm);
      d3 fd = nrm * (-cfg.soft_damping * vn);
      fa = fa + fd;
      fb = fb - fd;
    }
    d3 fra{0, 0, 0};
    int touch = 0;
    d3 nv{0, 0, 0};
    if (cfg.soft_enable_friction) {
      double fn_mag = len(fa);
      d3 vt = vrel - nrm * dot(vrel, nrm);
      double vtm = len(vt);
      if (!(vtm < 1e-10)) {
        if (cfg.soft_friction_mode == RG_FRICTION_CUNDALL) {
          const int f = hf;
          d3 old{0, 0, 0};
          if (f >= 0) old = mk3(io.hval[f], io.hval[io.hcap + f], io.hval[2 * io.hcap + f]);
          d3 ft = old - vt * (cfg.soft_kt * dt);
          double ncmp = dot(ft, nrm);
          ft = ft - nrm * ncmp;
          double ftm = len(ft);
          double lim = cfg.soft_mu * fn_mag;
          if (ftm > lim) {
            if (ftm > 1e-8) ft = ft * (lim / ftm);
            else ft = mk3(0, 0, 0);
          }
          nv = ft;
          touch = 1;
          fra = ft;
        } else if (cfg.soft_friction_mode == RG_FRICTION_KARNOPP) {
          if (vtm < cfg.soft_vel_deadband) {
            double ma = st.inv_mass[a] > 0 ? st.mass[a] : 0.0;
            double mb = st.inv_mass[b] > 0 ? st.mass[b] : 0.0;
            double meff = 0;
            if (ma > 0 && mb > 0) meff = (ma * mb) / (ma + mb);
            else if (ma > 0) meff = ma;
            else if (mb > 0) meff = mb;
            d3 fstop = vt * (-(meff / dt));
            d3 gv{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
            d3 gt = gv - nrm * dot(gv, nrm);
            d3 fdrive = gt * meff;
            d3 freq = fstop - fdrive;
            double frm = len(freq);
            double maxs = cfg.soft_mu_static * fn_mag;
            if (frm <= maxs) fra = freq;
            else if (frm > 1e-12) fra = freq * (maxs / frm);
          } else {
            fra = (vt * -1.0 / vtm) * (cfg.soft_mu * fn_mag);
          }
        } else {
          double K2 = 15.0 / cfg.soft_nu;
          double gamma = vtm > cfg.soft_nu ? 1.0 : 2.0 / (1.0 + exp(-K2 * vtm)) - 1.0;
          double mu_eff = cfg.soft_mu;
          if (cfg.soft_mu_static > cfg.soft_mu)
            mu_eff = cfg.soft_mu + (cfg.soft_mu_static - cfg.soft_mu) * exp(-vtm / cfg.soft_nu);
          d3 dir = (-vt) / vtm;
          fra = dir * (mu_eff * gamma * fn_mag);
        }
      }
    }
    d3 ta = fa + fra, tb = fb - fra;
    st_cf(io, c, ta, cross(ra, ta), tb, cross(rb, tb));
    io.touched[c] = touch;
    if (touch && hf >= 0) io.kept[hf] = 0;  // the touched entry is rewritten, not retained
    io.newval[c] = nv.x; io.newval[io.ccap + c] = nv.y; io.newval[2 * io.ccap + c] = nv.z;
    io.pe[c] = cfg.soft_k_scaler * U;
  }
}

__global__ void k_hm_forces(State st, rg_config cfg, ForceIO io, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const int C = ctl->contacts, H = ctl->hist_n;
  eval_begin(ctl);
  const double dt = cfg.dt;
  const double nu = cfg.hm_poisson_ratio;
  const double Es = cfg.hm_youngs_modulus / (2.0 * (1.0 - nu * nu));
  const double Gs = cfg.hm_youngs_modulus / (2.0 * (1.0 + nu));
  double gam = 0.0;
  if (cfg.hm_restitution < 1.0) {
    double l = log(cfg.hm_restitution);
    gam = -l / sqrt(M_PI * M_PI + l * l);
  }
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < C; c += gridDim.x * blockDim.x) {
    const int a = io.ca[c], b = io.cb[c];
    const int hf = hist_find(io, a, b, H);
    d3 pa = ldc(io, 0, c), pb = ldc(io, 3, c), nrm = ldc(io, 6, c), sh = ldc(io, 9, c);
    double dist = io.g[(size_t)12 * io.ccap + c], hs = io.g[(size_t)13 * io.ccap + c];
    double ra_ = st.r[a], rb_ = st.r[b], ma = st.mass[a], mb = st.mass[b];
    double delta = hs - dist;
    double Rs = (ra_ * rb_) / (ra_ + rb_);
    double ms = (ma * mb) / (ma + mb);
    double sd = smax(delta, 0.0);
    double sqd = sqrt(sd);
    double sqR = sqrt(smax(Rs, 0.0));
    double kn = (4.0 / 3.0) * Es * sqR * sqd;
    double Fel = kn * sd * sqd;
    d3 xa = st.x.ld(a), xb = st.x.ld(b);
    d3 ra = pa - xa;
    d3 rb = pb - (xb + sh);
    d3 wa = st.w.ld(a), wb = st.w.ld(b);
    d3 va = st.v.ld(a) + cross(wa, ra);
    d3 vb = st.v.ld(b) + cross(wb, rb);
    d3 vrel = vb - va;
    double vn = dot(vrel, nrm);
    double Cn = gam * 2.0 * sqrt(ms * kn);
    double Fn = smax(0.0, Fel + (-Cn * vn));
    d3 fn = nrm * Fn;
    d3 ft{0, 0, 0};
    const int f = hf;
    d3 xi{0, 0, 0};
    if (f >= 0) xi = mk3(io.hval[f], io.hval[io.hcap + f], io.hval[2 * io.hcap + f]);
    if (cfg.hm_enable_tangential) {
      double kt = 8.0 * Gs * sqR * sqd;
      d3 vt = vrel - nrm * vn;
      xi = xi + vt * dt;
      d3 fel = xi * (-kt);
      double Ct = gam * 2.0 * sqrt(ms * kt);
      ft = fel - vt * Ct;
      double vtm = len(vt);
      double mu_eff = cfg.hm_friction;
      if (cfg.hm_friction_static > cfg.hm_friction && cfg.hm_friction_transition_vel > 0.0)
        mu_eff += (cfg.hm_friction_static - cfg.hm_friction) * exp(-vtm / cfg.hm_friction_transition_vel);
      double fnm = len(fn);
      double ftm = len(ft);
      double ftmax = mu_eff * fnm;
      if (ftm > ftmax && ftm > 1e-10) {
        ft = ft * (ftmax / ftm);
        if (kt > 1e-10) xi = ft / (-kt);
      }
    }
    d3 tra{0, 0, 0}, trb{0, 0, 0};
    if (cfg.hm_enable_rolling) {
      d3 wr = wa - wb;
      double wm = len(wr);
      if (!(wm < 1e-10)) {
        d3 wh = wr / wm;
        double trm = cfg.hm_rolling_friction * Rs * len(fn);
        d3 tr = wh * (-trm);
        tra = tr * 0.5;
        trb = tr * -0.5;
      }
    }
    d3 F = fn + ft;
    st_cf(io, c, -F, cross(ra, -F) + tra, F, cross(rb, F) + trb);
    io.touched[c] = 1;
    if (hf >= 0) io.kept[hf] = 0;  // the touched entry is rewritten, not retained
    io.newval[c] = xi.x; io.newval[io.ccap + c] = xi.y; io.newval[2 * io.ccap + c] = xi.z;
    io.pe[c] = (8.0 / 15.0) * Es * sqrt(Rs) * pow(delta, 2.5);
  }
}

// f_i += Σ addends in contact order (the reference's sequential order).
__global__ void k_body_reduce(State st, const int* off, const int* ent, const double* cf, int ccap,
                              const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    if (off[i] == off[i + 1]) continue;
    d3 f = st.f.ld(i), t = st.tau.ld(i);
    body_sum(off, ent, cf, ccap, i, f, t);
    st.f.st(i, f);
    st.tau.st(i, t);
  }
}

// Cylinder wall of the soft model on every dynamic body (soft_wall_apply).
__global__ void k_soft_wall(State st, rg_config cfg, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const d3 ax = soft_wall_axis(cfg);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    if (!(st.inv_mass[i] > 0.0)) continue;
    d3 f = st.f.ld(i);
    soft_wall_apply(cfg, ax, st.r[i], st.x.ld(i), st.v.ld(i), f);
    st.f.st(i, f);
  }
}

// Deterministic potential-energy sum: fixed-shape two-level reduction.
// Potential energy Σ pe[c] by one block in a fixed order (deterministic).
constexpr int kPeThreads = 1024;
__global__ void __launch_bounds__(kPeThreads) k_pe_sum(const double* pe, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  __shared__ double sm[32];
  const int C = ctl->contacts;
  double v = 0;
  for (int c = threadIdx.x; c < C; c += blockDim.x) v += pe[c];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double u = sm[threadIdx.x];
    u = warp_sum(u);
    if (threadIdx.x == 0) ctl->pe = u;
  }
}

// One force evaluation: detect unless the contacts are fresh (seg_ready: the
// segment records and displacement check were written by the drift kernel),
// forces and history update, then the tail:
//   kForces:     reduction into f and tau (+ soft wall) and the potential energy;
//   kHalfPos:    reduction fused with the first half kick and drift (forces
//                at t are consumed there, not stored);
//   kSecondHalf: reduction fused with the second half kick, then the
//                potential energy.
void force_eval_launch(rg_system* s, EvalTail tail, bool seg_ready) {
  const rg_config& c = s->cfg;
  const bool hm = c.model == RG_MODEL_HERTZ_MINDLIN;
  cudaStream_t st = s->stream;
  const int bs = 256;
  if (!s->contacts_fresh) {
    ProfScope p(s, ST_DETECT);
    detect_launch(s, hm ? 0.0 : c.soft_delta, true, seg_ready, true);
    csr_launch(s, true);
  }
  ProfScope prof(s, ST_FORCES);
  History& H = s->hist;
  const int cur = H.cur, nxt = 1 - H.cur;
  const int gc = grid_for(s->ccap, bs);
  RGL launch_dep(k_hist_keep_init, grid_for(H.cap, bs), bs, st, H.frame[cur], H.kept, hm ? 1 : 0, s->d_ctl);
  ForceIO io;
  io.ca = s->con.a; io.cb = s->con.b; io.g = s->con.g; io.ccap = s->ccap;
  io.hkey = H.key[cur]; io.kept = H.kept; io.hval = H.val[cur]; io.hcap = H.cap;
  io.newval = H.newval; io.touched = H.touched; io.cf = s->d_cf;
  io.pe = s->d_cf + 12 * (size_t)s->ccap;
  if (hm) {
    RGL launch_dep(k_hm_forces, gc, bs, st, s->st, c, io, s->d_ctl);
  } else {
    RGL launch_dep(k_soft_forces, gc, bs, st, s->st, c, io, s->d_ctl);
  }
  // history merge
  s->scan.run2(H.touched, H.touched_off, &s->d_ctl->contacts, H.kept, H.kept_off, &s->d_ctl->hist_n,
               &s->d_ctl->err, st);
  RGL launch_dep(k_hist_merge, gc, bs, st, s->con.a, s->con.b, H.touched, H.touched_off, H.newval, H.key[cur],
                                  H.val[cur], H.frame[cur], H.kept, H.kept_off, H.key[nxt], H.val[nxt],
                                  H.frame[nxt], H.cap, s->ccap, s->d_ctl);
  H.cur = nxt;
  const bool wall = !hm && c.cylinder_enabled;
  // the kick kernels also close the history merge (hist_finish)
  const HistFinish hf{H.touched_off, H.kept_off};
  if (tail == EvalTail::kHalfPos) {
    reduce_drift_launch(s, wall, hf);
    return;
  }
  if (tail == EvalTail::kSecondHalf) {
    reduce_kick_launch(s, wall, hf);
  } else {
    RGL launch_dep(k_hist_finish, 1, 1, st, H.touched_off, H.kept_off, s->d_ctl);
    RGL launch_dep(k_body_reduce, grid_for(s->n, bs), bs, st, s->st, s->csr.off, s->csr.ent, s->d_cf, s->ccap,
                                                     s->d_ctl);
    if (wall) {
      RGL launch_dep(k_soft_wall, grid_for(s->n, bs), bs, st, s->st, c, s->d_ctl);
    }
  }
  RGL launch_dep(k_pe_sum, 1, kPeThreads, st, static_cast<const double*>(io.pe), s->d_ctl);
}

}  // namespace rg
