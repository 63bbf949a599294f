// rg_nsc.cu - non-smooth contact: colouring, manifolds, PSOR, projection.
//
// NscContactSolver (src/physics/nsc_contact.cpp):
//   detectAndBuildManifolds :239-321, buildTangentBasis :78-85,
//   computeDiag :106-117, solveVelocities :325-655 (warm start :344-380,
//   sweeps :385-552, residual :546-551, cache :646-654),
//   projectPositions :659-880 (multi-body path :698-879).
// Step order of App::physicsStep (src/app/main.cpp:4383-4528).
//
// Gauss-Seidel runs graph-coloured: contacts are coloured (Jones-Plassmann,
// first fit) so that no two contacts of one colour share a dynamic body;
// a sweep visits the colours in order and the contacts of a colour in
// parallel.  This equals sequential Gauss-Seidel over the colour-major
// permutation of the (a,b)-sorted contacts, bit for bit.  Rows are stored in
// colour-major slots so a colour is a contiguous, coalesced range.
// The sweep loop is one persistent kernel; colour phases are separated by a
// bounded grid barrier among only as many blocks as the largest colour needs
// (a single block synchronises with __syncthreads), and the per-sweep
// residual max (warp shuffles, then one atomic per block) decides the exit on
// the device.
#include "rg_internal.cuh"

namespace rg {

const int* detector_n_dev(rg_system* s);

__device__ inline unsigned long long jp_priority(unsigned c) {
  unsigned h = c * 0x9E3779B1u;
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return ((unsigned long long)h << 32) | (unsigned long long)c;
}

__device__ inline double block_max(double v, double* sm) {
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    r = warp_max(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// ---------------------------------------------------------------------------
// Colouring + colour-major order (one persistent kernel).
// ---------------------------------------------------------------------------
struct ColorIO {
  const int *ca, *cb;
  const double* inv_mass;
  const int *off, *ent;
  int *col, *tmp, *order, *cnt, *coff;
  int* remaining;  // kMaxRounds slots
};
constexpr int kMaxRounds = 512;

__global__ void k_color(ColorIO io, Ctl* ctl, GridBar gb) {
  if (ctl->err) return;
  const int C = ctl->contacts;
  const unsigned nb = gridDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  __shared__ int s_rem;
  // init
  for (int c = tid; c < C; c += stride) io.col[c] = -1;
  if (tid < kMaxRounds) io.remaining[tid] = 0;
  if (tid <= kMaxColors) io.cnt[tid] = 0;
  if (!grid_sync(gb, nb)) return;
  int* cin = io.col;
  int* cout = io.tmp;
  int round = 0;
  int maxc = 0;
  for (; round < kMaxRounds; ++round) {
    if (threadIdx.x == 0) s_rem = 0;
    __syncthreads();
    int rem = 0;
    for (int c = tid; c < C; c += stride) {
      int cc = cin[c];
      if (cc >= 0) {
        cout[c] = cc;
        continue;
      }
      unsigned long long pc = jp_priority((unsigned)c);
      bool best = true;
      unsigned long long used = 0;
      for (int side = 0; side < 2; ++side) {
        int bd = side ? io.cb[c] : io.ca[c];
        if (!(io.inv_mass[bd] > 0.0)) continue;
        for (int k = io.off[bd]; k < io.off[bd + 1]; ++k) {
          int o = io.ent[k] >> 1;
          if (o == c) continue;
          int co = cin[o];
          if (co >= 0) used |= 1ull << co;
          else if (jp_priority((unsigned)o) > pc) best = false;
        }
      }
      if (best) {
        int k = __ffsll((long long)~used) - 1;
        if (used == ~0ull) {
          atomicOr(&ctl->err, ERR_COLOR);
          k = kMaxColors - 1;
        }
        cout[c] = k;
        maxc = k + 1 > maxc ? k + 1 : maxc;
      } else {
        cout[c] = -1;
        ++rem;
      }
    }
    rem = warp_sum_i(rem);
    if ((threadIdx.x & 31) == 0 && rem) atomicAdd(&s_rem, rem);
    __syncthreads();
    if (threadIdx.x == 0 && s_rem) atomicAdd(&io.remaining[round], s_rem);
    if (!grid_sync(gb, nb)) return;
    int* t = cin; cin = cout; cout = t;
    if (*(volatile int*)&io.remaining[round] == 0) break;
  }
  if (round >= kMaxRounds) {
    if (tid == 0) atomicOr(&ctl->err, ERR_COLOR);
    return;
  }
  // final colours are in cin; copy to io.col if needed, count per colour
  for (int c = tid; c < C; c += stride) {
    int k = cin[c];
    if (cin != io.col) io.col[c] = k;
    atomicAdd(&io.cnt[k], 1);
  }
  if (maxc) atomicMax(&ctl->colors, maxc);
  if (!grid_sync(gb, nb)) return;
  if (tid == 0) {
    int acc = 0;
    for (int k = 0; k <= kMaxColors; ++k) {
      int v = k < kMaxColors ? io.cnt[k] : 0;
      io.coff[k] = acc;
      acc += v;
      if (k < kMaxColors) io.cnt[k] = 0;
    }
  }
  if (!grid_sync(gb, nb)) return;
  for (int c = tid; c < C; c += stride) {
    int k = io.col[c];
    io.order[io.coff[k] + atomicAdd(&io.cnt[k], 1)] = c;
  }
}

__global__ void k_zero_ctl_colors(Ctl* ctl) {
  if (ctl->err) return;
  ctl->colors = 0;
  ctl->bar_count = 0;
}

static void launch_coop(const void* fn, int grid, int block, void** args, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  RGL cudaLaunchKernelExC(&cfg, fn, args);
}

static GridBar bar_of(rg_system* s) {
  GridBar g;
  g.count = &s->d_ctl->bar_count;
  g.gen = &s->d_ctl->bar_gen;
  g.err = &s->d_ctl->err;
  return g;
}

void color_launch(rg_system* s) {
  RGL k_zero_ctl_colors<<<1, 1, 0, s->stream>>>(s->d_ctl);
  ColorIO io;
  io.ca = s->con.a; io.cb = s->con.b; io.inv_mass = s->st.inv_mass;
  io.off = s->csr.off; io.ent = s->csr.ent;
  io.col = s->nsc.color; io.tmp = s->nsc.color_tmp; io.order = s->nsc.order;
  io.cnt = s->nsc.color_cnt; io.coff = s->nsc.color_off;
  io.remaining = s->nsc.color_tmp + s->ccap;  // kMaxRounds slots after tmp
  Ctl* ctl = s->d_ctl;
  GridBar gb = bar_of(s);
  void* args[] = {&io, &ctl, &gb};
  launch_coop((const void*)k_color, s->coop_blocks, 256, args, s->stream);
}

// ---------------------------------------------------------------------------
// Manifold build (rows in colour-major slots) and warm start.
// ---------------------------------------------------------------------------
struct RowIO {
  double* row;  // kRowComps * ccap
  double* lam;  // 3 * ccap (slot order)
  int ccap;
  __device__ double& r(int k, int p) const { return row[(size_t)k * ccap + p]; }
  __device__ d3 r3(int k, int p) const { return {r(k, p), r(k + 1, p), r(k + 2, p)}; }
  __device__ void w3(int k, int p, d3 v) const { r(k, p) = v.x; r(k + 1, p) = v.y; r(k + 2, p) = v.z; }
};
enum { R_N = 0, R_T1 = 3, R_T2 = 6, R_RA = 9, R_RB = 12, R_IAN = 15, R_IAT1 = 18, R_IAT2 = 21,
       R_IBN = 24, R_IBT1 = 27, R_IBT2 = 30, R_IMA = 33, R_IMB = 34, R_GN = 35, R_GT1 = 36,
       R_GT2 = 37, R_BN = 38, R_BREST = 39, R_PHI = 40, R_VNPRE = 41 };

__device__ inline d3 iinv_apply(const State& st, int i, d3 v) {
  if (st.inv_mass[i] <= 0.0) return {0, 0, 0};
  return rot_diag_apply(st.q.ld(i), st.Iinv.ld(i), v);
}
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

__global__ void k_manifolds(State st, Contacts con, rg_config cfg, const int* order, RowIO R,
                            const unsigned long long* wkey, const double* wlam, const int* wn,
                            int wcap, Ctl* ctl) {
  if (ctl->err) return;
  const int C = ctl->contacts;
  const double beta = cfg.nsc_position_stabilization ? cfg.nsc_beta * 0.01 : cfg.nsc_beta;
  const int W = *wn;
  long long coll = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < C; p += gridDim.x * blockDim.x) {
    const int c = order[p];
    const int a = con.a[c], b = con.b[c];
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
    R.r(R_GN, p) = diag_of(st, a, b, ra, rb, n, cfg.nsc_cfm);
    R.r(R_GT1, p) = diag_of(st, a, b, ra, rb, t1, cfg.nsc_cfm);
    R.r(R_GT2, p) = diag_of(st, a, b, ra, rb, t2, cfg.nsc_cfm);
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
    if (vnp < -1e-6) ++coll;
    double l0 = 0, l1 = 0, l2 = 0;
    if (cfg.nsc_warm_start == RG_WARM_CACHE && W > 0) {
      unsigned long long k = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
      int q = lower_bound_key(wkey, W, k);
      if (q < W && wkey[q] == k) {
        l0 = smax(0.0, wlam[q]);
        l1 = wlam[wcap + q];
        l2 = wlam[2 * wcap + q];
      }
    }
    R.lam[p] = l0;
    R.lam[R.ccap + p] = l1;
    R.lam[2 * R.ccap + p] = l2;
  }
  if (coll) atomicAdd((unsigned long long*)&ctl->collisions, (unsigned long long)coll);
}

// ---------------------------------------------------------------------------
// PSOR sweeps (persistent).
// ---------------------------------------------------------------------------
struct Vel {
  Vec3A v, w;
};

__device__ inline void apply_imp(const Vel& V, int a, int b, d3 d, d3 IA, d3 IB, double ima,
                                 double imb, double l) {
  V.v.st(a, V.v.ld(a) - d * (l * ima));
  V.w.st(a, V.w.ld(a) - IA * l);
  V.v.st(b, V.v.ld(b) + d * (l * imb));
  V.w.st(b, V.w.ld(b) + IB * l);
}

__device__ inline double psor_row(const RowIO& R, const Vel& V, int p, int a, int b, double omega,
                                  double cfm, double mu) {
  d3 n = R.r3(R_N, p), t1 = R.r3(R_T1, p), t2 = R.r3(R_T2, p);
  d3 ra = R.r3(R_RA, p), rb = R.r3(R_RB, p);
  d3 IAn = R.r3(R_IAN, p), IAt1 = R.r3(R_IAT1, p), IAt2 = R.r3(R_IAT2, p);
  d3 IBn = R.r3(R_IBN, p), IBt1 = R.r3(R_IBT1, p), IBt2 = R.r3(R_IBT2, p);
  double ima = R.r(R_IMA, p), imb = R.r(R_IMB, p);
  double ln = R.lam[p], lt1 = R.lam[R.ccap + p], lt2 = R.lam[2 * R.ccap + p];
  d3 vA = V.v.ld(a), wA = V.w.ld(a), vB = V.v.ld(b), wB = V.w.ld(b);
  d3 vrel = (vB + cross(wB, rb)) - (vA + cross(wA, ra));
  double wn = dot(n, vrel) + R.r(R_BN, p) + R.r(R_BREST, p) + cfm * ln;
  double dn_ = -(omega / R.r(R_GN, p)) * wn;
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
  double d1_ = -(omega / R.r(R_GT1, p)) * w1;
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
  double d2_ = -(omega / R.r(R_GT2, p)) * w2;
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
    V.v.st(b, vB); V.w.st(b, wB);
    R.lam[p] = ln; R.lam[R.ccap + p] = lt1; R.lam[2 * R.ccap + p] = lt2;
  }
  return fabs(dn) + fabs(d1) + fabs(d2);
}

__device__ inline unsigned active_blocks(const int* coff, int ncol, int bs, unsigned grid) {
  int m = 0;
  for (int k = 0; k < ncol; ++k) {
    int c = coff[k + 1] - coff[k];
    m = c > m ? c : m;
  }
  unsigned need = (unsigned)((m + bs - 1) / bs);
  if (need < 1) need = 1;
  return need < grid ? need : grid;
}

__global__ void k_psor(State st, rg_config cfg, const int* order, const int* ca, const int* cb,
                       RowIO R, const int* coff, Ctl* ctl, GridBar gb) {
  if (ctl->err) return;
  const int C = ctl->contacts;
  const int K = ctl->colors;
  __shared__ double sm[32];
  if (C == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      ctl->sweeps_last = 0;
      ctl->residual = 0.0;
    }
    return;
  }
  const unsigned nb = active_blocks(coff, K, blockDim.x, gridDim.x);
  if (blockIdx.x >= nb) return;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = nb * blockDim.x;
  Vel V{st.v, st.w};
  const double omega = cfg.nsc_omega, cfm = cfg.nsc_cfm, mu = cfg.nsc_mu;
  const int iters = cfg.nsc_velocity_iters;
  for (int i = tid; i < iters; i += stride) ctl->res_sweep[i] = 0.0;
  // warm start, colour by colour (nsc_contact.cpp:344-380)
  if (cfg.nsc_warm_start != RG_WARM_NONE) {
    for (int k = 0; k < K; ++k) {
      for (int p = coff[k] + tid; p < coff[k + 1]; p += stride) {
        int c = order[p];
        int a = ca[c], b = cb[c];
        double ima = R.r(R_IMA, p), imb = R.r(R_IMB, p);
        double ln = R.lam[p], l1 = R.lam[R.ccap + p], l2 = R.lam[2 * R.ccap + p];
        if (ln != 0.0) apply_imp(V, a, b, R.r3(R_N, p), R.r3(R_IAN, p), R.r3(R_IBN, p), ima, imb, ln);
        if (l1 != 0.0) apply_imp(V, a, b, R.r3(R_T1, p), R.r3(R_IAT1, p), R.r3(R_IBT1, p), ima, imb, l1);
        if (l2 != 0.0) apply_imp(V, a, b, R.r3(R_T2, p), R.r3(R_IAT2, p), R.r3(R_IBT2, p), ima, imb, l2);
      }
      if (!grid_sync(gb, nb)) return;
    }
  } else {
    if (!grid_sync(gb, nb)) return;
  }
  double res = 0.0;
  int sweeps = 0;
  for (int it = 0; it < iters; ++it) {
    double loc = 0.0;
    for (int k = 0; k < K; ++k) {
      for (int p = coff[k] + tid; p < coff[k + 1]; p += stride) {
        int c = order[p];
        loc = fmax(loc, psor_row(R, V, p, ca[c], cb[c], omega, cfm, mu));
      }
      if (k + 1 < K && !grid_sync(gb, nb)) return;
    }
    double bm = block_max(loc, sm);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->res_sweep[it], bm);
    if (!grid_sync(gb, nb)) return;
    res = *(volatile double*)&ctl->res_sweep[it];
    sweeps = it + 1;
    if (res < cfg.nsc_tol) break;
  }
  if (tid == 0) {
    ctl->residual = res;
    ctl->sweeps_last = sweeps;
    ctl->sweeps_sum += sweeps;
    ctl->row_sweeps += (long long)C * sweeps;
    if (res >= cfg.nsc_tol) ctl->not_conv += 1;
    if (res > ctl->max_residual) ctl->max_residual = res;
  }
}

// Warm cache for the next step (contact order, so keys stay sorted) and
// impulse statistics.
__global__ void k_warm_save(Contacts con, const int* order, const int* color, RowIO R,
                            unsigned long long* wkey, double* wlam, int* wn, int wcap, Ctl* ctl) {
  if (ctl->err) return;
  const int C = ctl->contacts;
  __shared__ double sm[32];
  double jn = 0, jt = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < C; p += gridDim.x * blockDim.x) {
    int c = order[p];
    double l0 = R.lam[p], l1 = R.lam[R.ccap + p], l2 = R.lam[2 * R.ccap + p];
    wkey[c] = ((unsigned long long)(unsigned)con.a[c] << 32) | (unsigned)con.b[c];
    wlam[c] = l0; wlam[wcap + c] = l1; wlam[2 * wcap + c] = l2;
    reinterpret_cast<int*>(wlam + 3 * (size_t)wcap)[c] = color[c];
    jn += l0;
    jt += sqrt(l1 * l1 + l2 * l2);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *wn = C;
    ctl->vel_contacts = C;
  }
  jn = warp_sum(jn);
  jt = warp_sum(jt);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&ctl->jn_sum, jn);
    atomicAdd(&ctl->jt_sum, jt);
  }
  (void)sm;
}

__global__ void k_nsc_begin(Ctl* ctl) {
  if (ctl->err) return;
  ctl->collisions = 0;
  ctl->jn_sum = 0;
  ctl->jt_sum = 0;
}

// ---------------------------------------------------------------------------
// Position projection (persistent): rows from the pass-0 detection, then
// narrow phase on the cached pairs in later passes.
// ---------------------------------------------------------------------------
enum { P_N = 0, P_RA = 3, P_RB = 6, P_PHI = 9, P_G = 10, P_L = 11 };

__global__ void k_project(State st, rg_config cfg, Box box, Contacts con, const int* order,
                          const int* coff, const int* off, const int* ent, double* prow, int* pact,
                          double* dxb, int ccap, Ctl* ctl, GridBar gb) {
  if (ctl->err) return;
  const int C = ctl->contacts;
  const int K = ctl->colors;
  if (C == 0 || !cfg.nsc_position_stabilization) return;
  const unsigned nb = active_blocks(coff, K, blockDim.x, gridDim.x);
  if (blockIdx.x >= nb) return;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = nb * blockDim.x;
  const int n = st.n;
  const double omega = cfg.nsc_omega, cfm = cfg.nsc_cfm, slop = cfg.nsc_slop;
  __shared__ double sm[32];
  __shared__ int s_cnt;
  auto P = [&](int k, int p) -> double& { return prow[(size_t)k * ccap + p]; };
  Vec3A DX{dxb, dxb + n, dxb + 2 * n}, DT{dxb + 3 * n, dxb + 4 * n, dxb + 5 * n};
  double* slots = ctl->res_sweep;  // reused: [0..iters) per-sweep max, then counters
  const int piters = cfg.nsc_position_psor_iters;
  for (int outer = 0; outer < cfg.nsc_position_iters; ++outer) {
    for (int i = tid; i < piters + 1; i += stride) slots[i] = 0.0;
    if (threadIdx.x == 0) s_cnt = 0;
    if (!grid_sync(gb, nb)) return;
    int cnt = 0;
    for (int p = tid; p < C; p += stride) {
      const int c = order[p];
      const int a = con.a[c], b = con.b[c];
      d3 xa = st.x.ld(a), xb = st.x.ld(b);
      d3 nv, ra, rb;
      double phi;
      if (outer == 0) {
        phi = con.comp(12)[c] - con.comp(13)[c];
        nv = mk3(con.comp(6)[c], con.comp(7)[c], con.comp(8)[c]);
        d3 pa{con.comp(0)[c], con.comp(1)[c], con.comp(2)[c]};
        d3 pb{con.comp(3)[c], con.comp(4)[c], con.comp(5)[c]};
        d3 sh{con.comp(9)[c], con.comp(10)[c], con.comp(11)[c]};
        ra = pa - xa;
        rb = pb - (xb + sh);
      } else {
        Seg A, B;
        d3 ua = axis_y(st.q.ld(a)), ub = axis_y(st.q.ld(b));
        A.cx = xa.x; A.cy = xa.y; A.cz = xa.z; A.h = st.h[a]; A.ux = ua.x; A.uy = ua.y; A.uz = ua.z; A.r = st.r[a];
        B.cx = xb.x; B.cy = xb.y; B.cz = xb.z; B.h = st.h[b]; B.ux = ub.x; B.uy = ub.y; B.uz = ub.z; B.r = st.r[b];
        Narrow nr = narrow_pair(A, B, box);
        d3 diff = nr.pb - nr.pa;
        double dist = len(diff);
        phi = dist - con.comp(13)[c];
        nv = dist > 1e-10 ? diff / dist : mk3(1, 0, 0);
        ra = nr.pa - xa;
        rb = nr.pb - (xb + nr.sh);
      }
      int act = phi < -slop ? 1 : 0;
      pact[p] = act;
      if (act) {
        ++cnt;
        P(P_N, p) = nv.x; P(P_N + 1, p) = nv.y; P(P_N + 2, p) = nv.z;
        P(P_RA, p) = ra.x; P(P_RA + 1, p) = ra.y; P(P_RA + 2, p) = ra.z;
        P(P_RB, p) = rb.x; P(P_RB + 1, p) = rb.y; P(P_RB + 2, p) = rb.z;
        P(P_PHI, p) = phi + slop;
        P(P_G, p) = diag_of(st, a, b, ra, rb, nv, cfm);
        P(P_L, p) = 0.0;
      }
      DX.st(a, mk3(0, 0, 0)); DT.st(a, mk3(0, 0, 0));
      DX.st(b, mk3(0, 0, 0)); DT.st(b, mk3(0, 0, 0));
    }
    cnt = warp_sum_i(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt) atomicAdd((unsigned long long*)&slots[piters], (unsigned long long)s_cnt);
    if (!grid_sync(gb, nb)) return;
    if (*(volatile unsigned long long*)&slots[piters] == 0ull) return;  // nothing penetrates
    for (int it = 0; it < piters; ++it) {
      double loc = 0.0;
      for (int k = 0; k < K; ++k) {
        for (int p = coff[k] + tid; p < coff[k + 1]; p += stride) {
          if (!pact[p]) continue;
          const int c = order[p];
          const int a = con.a[c], b = con.b[c];
          d3 nv{P(P_N, p), P(P_N + 1, p), P(P_N + 2, p)};
          d3 ra{P(P_RA, p), P(P_RA + 1, p), P(P_RA + 2, p)};
          d3 rb{P(P_RB, p), P(P_RB + 1, p), P(P_RB + 2, p)};
          double l = P(P_L, p);
          double corr = dot(nv, ((DX.ld(b) + cross(DT.ld(b), rb)) - DX.ld(a)) - cross(DT.ld(a), ra));
          double r = corr + P(P_PHI, p) + cfm * l;
          double d = -(omega / P(P_G, p)) * r;
          double nl = smax(0.0, l + d);
          double dl = nl - l;
          if (dl != 0.0) {
            P(P_L, p) = nl;
            d3 rAxn = cross(ra, nv);
            DX.st(a, DX.ld(a) - nv * (dl * st.inv_mass[a]));
            DT.st(a, DT.ld(a) - iinv_apply(st, a, rAxn) * dl);
            d3 rBxn = cross(rb, nv);
            DX.st(b, DX.ld(b) + nv * (dl * st.inv_mass[b]));
            DT.st(b, DT.ld(b) + iinv_apply(st, b, rBxn) * dl);
          }
          loc = fmax(loc, fabs(dl));
        }
        if (k + 1 < K && !grid_sync(gb, nb)) return;
      }
      double bm = block_max(loc, sm);
      if (threadIdx.x == 0) atomic_max_nonneg(&slots[it], bm);
      if (!grid_sync(gb, nb)) return;
      if (*(volatile double*)&slots[it] < 1e-8) break;
    }
    // apply corrections: each body once, by the contact owning its first
    // CSR entry
    for (int p = tid; p < C; p += stride) {
      const int c = order[p];
      for (int side = 0; side < 2; ++side) {
        int bd = side ? con.b[c] : con.a[c];
        if (ent[off[bd]] != 2 * c + side) continue;
        if (st.inv_mass[bd] <= 0.0) continue;
        st.x.st(bd, st.x.ld(bd) + DX.ld(bd));
        d3 th = DT.ld(bd);
        double ang = len(th);
        if (ang > 1e-8) {
          d3 ax = th / ang;
          st.q.st(bd, qnormalize(qmul(angle_axis(ang, ax), st.q.ld(bd))));
        }
      }
    }
    if (!grid_sync(gb, nb)) return;
  }
}

// ---------------------------------------------------------------------------
// Step.
// ---------------------------------------------------------------------------
void nsc_step_launch(rg_system* s) {
  cudaStream_t st = s->stream;
  const int bs = 256;
  const int gc = grid_for(s->ccap, bs, s->sm_count * 8);
  Ctl* ctl = s->d_ctl;
  GridBar gb = bar_of(s);
  RowIO R{s->nsc.row, s->nsc.lam, s->ccap};
  RGL k_nsc_begin<<<1, 1, 0, st>>>(ctl);
  // 1) free flight
  {
    ProfScope p(s, ST_INTEGRATE);
    nsc_free_flight_launch(s);
  }
  // 2) detection, colouring, manifolds
  {
    ProfScope p(s, ST_DETECT);
    detect_launch(s, 0.0, true);
    csr_launch(s);
  }
  {
    ProfScope p(s, ST_COLOR);
    color_launch(s);
  }
  ProfScope pm(s, ST_MANIFOLDS);
  if (s->cfg.nsc_warm_start == RG_WARM_MLP && s->mlp_ready) {
    RGL k_manifolds<<<gc, bs, 0, st>>>(s->st, s->con, s->cfg, s->nsc.order, R, s->nsc.wkey, s->nsc.wlam,
                                   s->nsc.wn, s->nsc.wcap, ctl);
    mlp_warm_launch(s);
  } else {
    RGL k_manifolds<<<gc, bs, 0, st>>>(s->st, s->con, s->cfg, s->nsc.order, R, s->nsc.wkey, s->nsc.wlam,
                                   s->nsc.wn, s->nsc.wcap, ctl);
  }
  if (s->recording) mlp_record_launch(s);  // features at the warm-start point
  pm.end();
  // 3) PSOR
  {
    ProfScope p(s, ST_PSOR);
    State stt = s->st;
    rg_config cfg = s->cfg;
    const int* order = s->nsc.order;
    const int* ca = s->con.a;
    const int* cb = s->con.b;
    const int* coff = s->nsc.color_off;
    void* args[] = {&stt, &cfg, &order, &ca, &cb, &R, &coff, &ctl, &gb};
    launch_coop((const void*)k_psor, s->coop_blocks, 256, args, st);
  }
  if (s->recording) mlp_record_launch(s);  // targets: converged impulses
  ProfScope pw(s, ST_MANIFOLDS);
  RGL k_warm_save<<<gc, bs, 0, st>>>(s->con, s->nsc.order, s->nsc.color, R, s->nsc.wkey, s->nsc.wlam, s->nsc.wn,
                                 s->nsc.wcap, ctl);
  pw.end();
  // 4) position update
  {
    ProfScope p(s, ST_INTEGRATE);
    nsc_position_update_launch(s);
  }
  // 5) projection
  if (s->cfg.nsc_position_stabilization) {
    {
      ProfScope p(s, ST_DETECT);
      detect_launch(s, 0.0, true);
      csr_launch(s);
    }
    {
      ProfScope p(s, ST_COLOR);
      color_launch(s);
    }
    ProfScope p(s, ST_PROJECT);
    State stt = s->st;
    rg_config cfg = s->cfg;
    Box box = s->box;
    Contacts con = s->con;
    const int* order = s->nsc.order;
    const int* coff = s->nsc.color_off;
    const int* off = s->csr.off;
    const int* ent = s->csr.ent;
    double* prow = s->nsc.prow;
    int* pact = s->nsc.pactive;
    double* dxb = s->nsc.dx;
    int ccap = s->ccap;
    void* args[] = {&stt, &cfg, &box, &con, &order, &coff, &off, &ent, &prow, &pact, &dxb, &ccap,
                    &ctl, &gb};
    launch_coop((const void*)k_project, s->coop_blocks, 256, args, st);
  }
  // 6) wrap + clear forces
  ProfScope p(s, ST_INTEGRATE);
  wrap_launch(s);
  s->contacts_fresh = false;
}

}  // namespace rg
