// rg_common.cuh - device-side building blocks shared by the rodgpu kernels.
//
// All arithmetic is FP64 and the library is compiled with -fmad=false, so
// every expression rounds exactly as written; the narrow-phase contact
// predicate therefore reproduces the FP64 restatement of
// ContactDetector::detectCapsuleCapsule (src/physics/contact_detector.cpp:
// 811-910) bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cuda/atomic>

#include "../../include/rodgpu.h"

namespace rg {

// ---- error bits kept in device memory (rg_system::d_err) -----------------
enum : int {
  ERR_CONTACT_CAP = 1,   // contact buffer overflow
  ERR_NBR_CAP = 2,       // neighbour list overflow
  ERR_COLOR = 4,         // more than 64 colours
  ERR_HIST_CAP = 8,      // history table overflow
  ERR_TIMEOUT = 16,      // a bounded grid barrier gave up
  ERR_CELL = 32,         // cell grid capacity
  ERR_NONFINITE = 64,    // non-finite state
  ERR_RECORD_CAP = 128   // MLP record buffer full (recording stops, not fatal)
};

constexpr int kMaxColors = 64;

struct d3 {
  double x, y, z;
};
__host__ __device__ inline d3 mk3(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 operator-(d3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ inline d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline d3 operator/(d3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline d3 cross(d3 a, d3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ inline double len(d3 a) { return sqrt(dot(a, a)); }
// std::max / std::min semantics (ties and signed zeros return the first arg).
__host__ __device__ inline double smax(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ inline double smin(double a, double b) { return (b < a) ? b : a; }

struct dq {
  double w, x, y, z;
};
__device__ inline dq qmul(dq a, dq b) {
  return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
          a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
          a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
          a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
__device__ inline dq qnormalize(dq q) {
  double l = sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
  if (l <= 0.0) return {1, 0, 0, 0};
  double inv = 1.0 / l;
  return {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
}
__device__ inline dq angle_axis(double ang, d3 ax) {
  double h = 0.5 * ang;
  double s, c;
  sincos(h, &s, &c);
  return {c, ax.x * s, ax.y * s, ax.z * s};
}
// Rotation-matrix columns of q (mat3_cast); col1 = RigidBody::axisY.
__device__ inline void rot_cols(dq q, d3& c0, d3& c1, d3& c2) {
  double qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
  double qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
  double qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
  c0 = {1.0 - 2.0 * (qyy + qzz), 2.0 * (qxy + qwz), 2.0 * (qxz - qwy)};
  c1 = {2.0 * (qxy - qwz), 1.0 - 2.0 * (qxx + qzz), 2.0 * (qyz + qwx)};
  c2 = {2.0 * (qxz + qwy), 2.0 * (qyz - qwx), 1.0 - 2.0 * (qxx + qyy)};
}
__device__ inline d3 axis_y(dq q) {
  double qxx = q.x * q.x, qzz = q.z * q.z;
  double qxy = q.x * q.y, qyz = q.y * q.z;
  double qwx = q.w * q.x, qwz = q.w * q.z;
  return {2.0 * (qxy - qwz), 1.0 - 2.0 * (qxx + qzz), 2.0 * (qyz + qwx)};
}
// R diag(d) R^T v  (IworldInv * v or Iworld * v).
__device__ inline d3 rot_diag_apply(dq q, d3 d, d3 v) {
  d3 c0, c1, c2;
  rot_cols(q, c0, c1, c2);
  double b0 = dot(c0, v) * d.x, b1 = dot(c1, v) * d.y, b2 = dot(c2, v) * d.z;
  return c0 * b0 + c1 * b1 + c2 * b2;
}

// ---- structure-of-arrays views ---------------------------------------------
struct Vec3A {  // three component arrays of length n
  double *x, *y, *z;
  __device__ d3 ld(int i) const { return {x[i], y[i], z[i]}; }
  __device__ void st(int i, d3 v) const { x[i] = v.x; y[i] = v.y; z[i] = v.z; }
};
struct QuatA {
  double *w, *x, *y, *z;
  __device__ dq ld(int i) const { return {w[i], x[i], y[i], z[i]}; }
  __device__ void st(int i, dq q) const { w[i] = q.w; x[i] = q.x; y[i] = q.y; z[i] = q.z; }
};

// Body state and static properties on the device.
struct State {
  int n;
  Vec3A x, v, w, f, tau;
  QuatA q;
  const double *r, *h, *mass, *inv_mass, *rest;
  Vec3A I, Iinv;
  // the buffers behind the component arrays: state (x 0-2, q 3-6, v 7-9,
  // w 10-12, f 13-15, tau 16-18) and properties (r 0, h 1, mass 2,
  // inv_mass 3, rest 4, I 5-7, Iinv 8-10), component k at base + k n
  double* sbase;
  const double* pbase;
};

// A system's state addressed from its two buffer bases.  Per-rod loops hold
// this in three registers instead of re-reading some thirty component
// pointers from the system's view after every store.
struct StateBase {
  double* s;
  const double* p;
  int n;
  __device__ double* c(int k) const { return s + (size_t)k * n; }
  __device__ const double* pc(int k) const { return p + (size_t)k * n; }
  __device__ d3 ld3(int k, int i) const { return {c(k)[i], c(k + 1)[i], c(k + 2)[i]}; }
  __device__ void st3(int k, int i, d3 v) const { c(k)[i] = v.x; c(k + 1)[i] = v.y; c(k + 2)[i] = v.z; }
  __device__ d3 pld3(int k, int i) const { return {pc(k)[i], pc(k + 1)[i], pc(k + 2)[i]}; }
};

// Packed per-detection segment record (two 32-byte sectors).
struct __align__(32) Seg {
  double cx, cy, cz, h;
  double ux, uy, uz, r;
};

struct Box {
  int pbc;
  double lo[3], hi[3], L[3];
};

__device__ inline d3 min_image_shift(const Box& B, d3 xa, d3 xb) {
  d3 sh{0, 0, 0};
  if (!B.pbc) return sh;
  d3 d = xb - xa;
  if (B.L[0] > 0.0) sh.x = -(floor(d.x / B.L[0] + 0.5) * B.L[0]);
  if (B.L[1] > 0.0) sh.y = -(floor(d.y / B.L[1] + 0.5) * B.L[1]);
  if (B.L[2] > 0.0) sh.z = -(floor(d.z / B.L[2] + 0.5) * B.L[2]);
  return sh;
}

// Lumelsky closest points (contact_detector.cpp:978-1035) in FP64.
__device__ inline void lumelsky(d3 a1, d3 a2, d3 b1, d3 b2, double& s, double& t) {
  d3 e1 = a2 - a1, e2 = b2 - b1, e12 = b1 - a1;
  double D1 = dot(e1, e1), D2 = dot(e2, e2);
  double S1 = dot(e1, e12), S2 = dot(e2, e12), R = dot(e1, e2);
  double den = D1 * D2 - R * R;
  double uf;
  if (den == 0.0) {
    s = 0.0;
    t = -S2 / D2;
    uf = t;
    if (uf > 1.0) uf = 1.0; else if (uf < 0.0) uf = 0.0;
    if (uf != t) {
      s = (uf * R + S1) / D1;
      if (s > 1.0) s = 1.0; else if (s < 0.0) s = 0.0;
      t = uf;
    }
  } else {
    s = (S1 * D2 - S2 * R) / den;
    if (s > 1.0) s = 1.0; else if (s < 0.0) s = 0.0;
    t = (s * R - S2) / D2;
    uf = t;
    if (uf > 1.0) uf = 1.0; else if (uf < 0.0) uf = 0.0;
    if (uf != t) {
      s = (uf * R + S1) / D1;
      if (s > 1.0) s = 1.0; else if (s < 0.0) s = 0.0;
      t = uf;
    }
  }
}

// Narrow phase of one pair from packed segment records.  Returns the squared
// closest distance and fills closest points / shift / s,t.
struct Narrow {
  d3 pa, pb, sh;
  double d2, s, t;
};
__device__ inline Narrow narrow_pair(const Seg& A, const Seg& B, const Box& box) {
  Narrow o;
  d3 xa{A.cx, A.cy, A.cz}, xb{B.cx, B.cy, B.cz};
  d3 ua{A.ux, A.uy, A.uz}, ub{B.ux, B.uy, B.uz};
  d3 a1 = xa - ua * A.h, a2 = xa + ua * A.h;
  d3 b1 = xb - ub * B.h, b2 = xb + ub * B.h;
  o.sh = min_image_shift(box, xa, xb);
  b1 = b1 + o.sh;
  b2 = b2 + o.sh;
  lumelsky(a1, a2, b1, b2, o.s, o.t);
  o.pa = a1 + (a2 - a1) * o.s;
  o.pb = b1 + (b2 - b1) * o.t;
  d3 diff = o.pb - o.pa;
  o.d2 = dot(diff, diff);
  return o;
}
__device__ inline bool contact_test(double d2, double rsum, double delta) {
  double act = rsum + delta;
  return d2 < act * act;
}
__device__ inline int contact_type(double s, double t) {
  const double eps = 1e-6;
  if (s < eps && t < eps) return 0;
  if (s > 1.0 - eps && t > 1.0 - eps) return 0;
  if (s < eps || s > 1.0 - eps) return 1;
  if (t < eps || t > 1.0 - eps) return 1;
  return 2;
}

// ---- programmatic dependent launch -------------------------------------------
// A kernel launched with programmatic stream serialization (launch_dep) may
// be scheduled while the kernel before it in the stream drains; this wait
// returns once that kernel has completed and its writes are visible.  Every
// kernel launched through launch_dep calls it before touching memory (for a
// kernel launched without the attribute it returns at once).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ---- per-body force terms of the soft / Hertz-Mindlin models ------------------
// f += Σ, tau += Σ of a body's contact addends in contact order (the
// reference's sequential accumulation, f[a] -= F; f[b] += F over the contact
// list).  off/ent: the body -> contact CSR (ent = 2c for side a, 2c + 1 for
// side b); cf: 12 addend arrays of ccap (f_a, tau_a, f_b, tau_b).
__device__ inline void body_sum(const int* off, const int* ent, const double* cf, int ccap, int i, d3& f,
                                d3& t) {
  const int s = off[i], e = off[i + 1];
  for (int k = s; k < e; ++k) {
    const int v = ent[k];
    const int c = v >> 1;
    const int base = (v & 1) ? 6 : 0;
    f.x = f.x + cf[(size_t)(base + 0) * ccap + c];
    f.y = f.y + cf[(size_t)(base + 1) * ccap + c];
    f.z = f.z + cf[(size_t)(base + 2) * ccap + c];
    t.x = t.x + cf[(size_t)(base + 3) * ccap + c];
    t.y = t.y + cf[(size_t)(base + 4) * ccap + c];
    t.z = t.z + cf[(size_t)(base + 5) * ccap + c];
  }
}

// Cylinder wall of the soft model on one dynamic body (main.cpp:4661-4690 at
// phase t, :4756-4787 at phase t + dt): a penalty spring on the centre's
// radial overshoot past R - r plus smooth Coulomb friction (tanh of |v_t| /
// nu), added to f.  ax: the unit cylinder axis (soft_wall_axis).
__device__ inline d3 soft_wall_axis(const rg_config& c) {
  const d3 ax{c.cylinder_axis[0], c.cylinder_axis[1], c.cylinder_axis[2]};
  return ax / len(ax);
}
__device__ inline void soft_wall_apply(const rg_config& cfg, d3 ax, double r, d3 x, d3 v, d3& f) {
  const double k = cfg.soft_k_scaler, cd = cfg.soft_damping, mu = cfg.soft_mu;
  const double nu = smax(cfg.soft_nu, 1e-10);
  const double maxd = cfg.cylinder_radius - r;
  const d3 pp = x - ax * dot(x, ax);
  const double d = len(pp);
  const double pen = d - maxd;
  if (pen <= 0.0) return;
  d3 n;
  if (d > 1e-8) {
    n = pp / d;
  } else {
    const d3 cr = cross(ax, fabs(ax.x) < 0.9 ? mk3(1, 0, 0) : mk3(0, 1, 0));
    n = cr / len(cr);
  }
  const double vn = dot(v, n);
  const double fn = k * pen + cd * smax(vn, 0.0);
  f = f - n * fn;
  const d3 vt = v - n * vn;
  const double vtl = len(vt);
  if (vtl > 1e-12) f = f - vt * (mu * fn * tanh(vtl / nu) / vtl);
}

// ---- reductions --------------------------------------------------------------
__device__ inline double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Non-negative doubles order like their bit patterns.
__device__ inline void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// Exclusive block-wide scan of one int per thread (blockDim multiple of 32).
__device__ inline int block_excl_scan(int v, int* sh_warp, int& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int s = lane < nw ? sh_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) sh_warp[lane] = s;
  }
  __syncthreads();
  int warp_prefix = wid > 0 ? sh_warp[wid - 1] : 0;
  total = sh_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

// ---- bounded grid barrier ----------------------------------------------------
// Sense-free generation barrier for co-resident (cooperatively launched)
// blocks.  Every wait is bounded: after `limit` polls (kSpinLimit by
// default) the block records ERR_TIMEOUT and returns false; the other
// waiters see the bit within 64 polls and return false too; callers then
// leave the kernel.  `absent` counts blocks that are expected but never
// arrive (a failure-detection test hook, 0 in normal use).
constexpr long long kSpinLimit = 20000000;  // ~1-2 s with the backoff below
struct GridBar {
  unsigned int* count;
  unsigned int* gen;
  int* err;
  long long limit = kSpinLimit;
  unsigned int absent = 0;
};

// nb = number of participating blocks (blocks 0..nb-1); nb == 1 is a plain
// __syncthreads unless blocks are marked absent.
__device__ inline bool grid_sync(const GridBar& g, unsigned int nb) {
  __syncthreads();
  nb += g.absent;
  if (nb <= 1) return !(*(volatile int*)g.err & ERR_TIMEOUT);
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    s_ok = 1;
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> gen(*g.gen);
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> cnt(*g.count);
    const unsigned int my = gen.load(cuda::memory_order_acquire);
    if (*(volatile int*)g.err & ERR_TIMEOUT) {
      s_ok = 0;
    } else if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nb - 1) {
      cnt.store(0u, cuda::memory_order_relaxed);
      gen.fetch_add(1u, cuda::memory_order_release);
    } else {
      long long it = 0;
      while (gen.load(cuda::memory_order_acquire) == my) {
        ++it;
        if ((it & 63) == 0 && (*(volatile int*)g.err & ERR_TIMEOUT)) { s_ok = 0; break; }
        if (it > g.limit) {
          atomicOr(g.err, ERR_TIMEOUT);
          s_ok = 0;
          break;
        }
        if (it > 64) __nanosleep(64);
      }
    }
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace rg
