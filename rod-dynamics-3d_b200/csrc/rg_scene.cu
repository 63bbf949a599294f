// rg_scene.cu - seeded packings of capsules generated on the device.
//
// The reference populates scenes on the host, one rod after the other
// (random sequential addition, "nonoverlap" populate, src/app/main.cpp:
// 1857-2140): centre uniform in the box, axis uniform on S^2 (cos θ ~
// U[-1,1], φ ~ U[0,2π), :1918-1923), rejected when the closest segment
// distance to a placed rod (nearest periodic image) is below one diameter
// (:1933-1995).  At 10^6 rods that serial loop dominates the set-up.
//
// Here every unplaced slot draws candidates in parallel, in rounds:
//   1. try:     each unplaced slot has D candidate draws this round
//               (counter-based random numbers of (seed, slot, draw index)),
//               each tested by its own thread against every placed rod (27
//               cells of a grid of placed rods, cell >= L + d); the first
//               clear draw (lowest index) becomes the slot's candidate;
//   2. resolve: survivors that overlap a survivor of a LOWER slot index are
//               dropped (they retry next round), so accepted rods never
//               overlap each other;
//   3. accept:  the rest are placed and inserted into the grid.
// The packing is a valid non-overlapping isotropic packing and depends only
// on the seed (no result depends on the order of atomic insertions); it is
// statistically, not bitwise, the host generator's.  A slot gives up after
// max_attempts draws; placed rods are returned in slot order.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rg_internal.cuh"

namespace rg {
namespace {

constexpr int kRsaBS = 256;

struct RsaGrid {
  int nc;            // cells per axis
  double lo, side, cs;
  int cap;           // slots per cell
  int* cnt;          // nc^3 counts
  int* slot;         // nc^3 * cap rod indices
  int* overflow;     // set when an insertion found its cell full
};

__device__ inline unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
struct Draw {
  unsigned long long s;
  __device__ double u01() {
    s += 0x9E3779B97F4A7C15ull;
    return (double)(mix64(s) >> 11) * 0x1.0p-53;
  }
};

__device__ inline int rsa_cell(double v, const RsaGrid& G) {
  int c = (int)floor((v - G.lo) / G.cs);
  c %= G.nc;
  if (c < 0) c += G.nc;
  return c;
}
__device__ inline double wrapd(double v, double side) { return v - side * floor(v / side + 0.5); }

// Candidate k of slot i: centre uniform in the box, axis uniform on S^2.
__device__ inline void rsa_draw(unsigned long long seed, int i, long long k, const RsaGrid& G, d3& c, d3& u) {
  Draw r{seed ^ mix64(0xD1B54A32D192ED03ull * (unsigned long long)(i + 1) +
                      0x9E3779B97F4A7C15ull * (unsigned long long)(k + 1))};
  c = mk3(G.lo + G.side * r.u01(), G.lo + G.side * r.u01(), G.lo + G.side * r.u01());
  const double cz = 2.0 * r.u01() - 1.0, ph = 6.283185307179586 * r.u01();
  const double sn = sqrt(smax(0.0, 1.0 - cz * cz));
  u = mk3(sn * cos(ph), cz, sn * sin(ph));
}

// Closest distance of the two segments below d (nearest periodic image).
__device__ inline bool rsa_overlap(d3 c, d3 u, d3 cj, d3 uj, double h, double d, double cut2, double side) {
  d3 dd = mk3(wrapd(cj.x - c.x, side), wrapd(cj.y - c.y, side), wrapd(cj.z - c.z, side));
  if (dot(dd, dd) > cut2) return false;
  d3 a1 = c - u * h, a2 = c + u * h;
  d3 cb = c + dd;
  d3 b1 = cb - uj * h, b2 = cb + uj * h;
  double s, t;
  lumelsky(a1, a2, b1, b2, s, t);
  d3 diff = (b1 + (b2 - b1) * t) - (a1 + (a2 - a1) * s);
  return dot(diff, diff) < d * d;
}

// Does (c, u) overlap a rod listed in grid G (other than `self`), among the
// rods with index < below when below >= 0?
__device__ inline bool rsa_hits(d3 c, d3 u, const RsaGrid& G, const double* X, const double* U, double h,
                                double d, double cut2, int self, int below) {
  const int cx = rsa_cell(c.x, G), cy = rsa_cell(c.y, G), cz = rsa_cell(c.z, G);
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int X_ = (cx + dx + G.nc) % G.nc, Y_ = (cy + dy + G.nc) % G.nc, Z_ = (cz + dz + G.nc) % G.nc;
        const size_t cell = ((size_t)Z_ * G.nc + Y_) * G.nc + X_;
        const int m = min(G.cnt[cell], G.cap);
        const int* sl = G.slot + cell * (size_t)G.cap;
        for (int q = 0; q < m; ++q) {
          const int j = sl[q];
          if (j == self || (below >= 0 && j >= below)) continue;
          if (rsa_overlap(c, u, mk3(X[3 * j], X[3 * j + 1], X[3 * j + 2]),
                          mk3(U[3 * j], U[3 * j + 1], U[3 * j + 2]), h, d, cut2, G.side))
            return true;
        }
      }
  return false;
}

__device__ inline bool rsa_insert(const RsaGrid& G, d3 c, int i) {
  const size_t cell = ((size_t)rsa_cell(c.z, G) * G.nc + rsa_cell(c.y, G)) * G.nc + rsa_cell(c.x, G);
  const int k = atomicAdd(&G.cnt[cell], 1);
  if (k < G.cap) {
    G.slot[cell * (size_t)G.cap + k] = i;
    return true;
  }
  atomicOr(G.overflow, 1);
  return false;
}

// 1. try.  a) the unplaced slots in a list (any order); every slot's
// survivor flag cleared.
__global__ void k_rsa_list(int n, const unsigned char* placed, unsigned char* surv, int* list, int* count,
                           int* best) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    surv[i] = 0;
    if (placed[i]) continue;
    best[i] = 0x7fffffff;
    list[atomicAdd(count, 1)] = i;
  }
}
// b) one thread per (listed slot, draw): a draw clear of the placed rods
// lowers the slot's best draw index.
__global__ void k_rsa_draws(unsigned long long seed, RsaGrid G, const double* X, const double* U, const int* list,
                            const int* count, const long long* draws, int D, long long max_attempts, int* best,
                            double h, double d, double cut2) {
  const long long total = (long long)*count * D;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = list[t / D];
    const long long k = draws[i] + t % D;
    if (k >= max_attempts) continue;
    d3 c, u;
    rsa_draw(seed, i, k, G, c, u);
    if (!rsa_hits(c, u, G, X, U, h, d, cut2, -1, -1)) atomicMin(&best[i], (int)k);
  }
}
// c) per listed slot: the best draw becomes its candidate (recomputed from
// its index) in the candidate grid Gc; the draw counter moves past it, or
// past the round's D draws when none was clear.
__global__ void k_rsa_pick(unsigned long long seed, RsaGrid G, RsaGrid Gc, const int* list, const int* count,
                           long long* draws, int D, long long max_attempts, const int* best, double* CX,
                           double* CU, unsigned char* surv, int* exhausted) {
  const int m = *count;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    const int i = list[j];
    const long long k0 = draws[i];
    const long long k1 = min(k0 + (long long)D, max_attempts);
    const long long kb = best[i];
    if (kb >= k1) {
      draws[i] = k1;
      if (k1 >= max_attempts) atomicOr(exhausted, 1);  // this slot cannot be placed: the packing jams
      continue;
    }
    draws[i] = kb + 1;
    d3 c, u;
    rsa_draw(seed, i, kb, G, c, u);
    CX[3 * i] = c.x; CX[3 * i + 1] = c.y; CX[3 * i + 2] = c.z;
    CU[3 * i] = u.x; CU[3 * i + 1] = u.y; CU[3 * i + 2] = u.z;
    if (rsa_insert(Gc, c, i)) surv[i] = 1;  // a full candidate cell: retry next round
  }
}

// 2.+3. resolve and accept: a survivor overlapping a lower-index survivor
// waits; the others are placed.  Reads only the candidate grid (not
// modified here) and writes the placed arrays of accepted slots.
__global__ void k_rsa_resolve(int n, RsaGrid Gc, const double* CX, const double* CU, const unsigned char* surv,
                              unsigned char* acc, double h, double d, double cut2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    acc[i] = 0;
    if (!surv[i]) continue;
    const d3 c = mk3(CX[3 * i], CX[3 * i + 1], CX[3 * i + 2]);
    const d3 u = mk3(CU[3 * i], CU[3 * i + 1], CU[3 * i + 2]);
    acc[i] = rsa_hits(c, u, Gc, CX, CU, h, d, cut2, i, i) ? 0 : 1;
  }
}

__global__ void k_rsa_accept(int n, RsaGrid G, const double* CX, const double* CU, const unsigned char* acc,
                             double* X, double* U, unsigned char* placed, int* placed_count) {
  int mine = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!acc[i]) continue;
    for (int k = 0; k < 3; ++k) { X[3 * i + k] = CX[3 * i + k]; U[3 * i + k] = CU[3 * i + k]; }
    placed[i] = 1;
    rsa_insert(G, mk3(X[3 * i], X[3 * i + 1], X[3 * i + 2]), i);
    ++mine;
  }
  mine = warp_sum_i(mine);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(placed_count, mine);
}

// Re-inserts every placed rod (after the grid grew).
__global__ void k_rsa_rebuild(int n, RsaGrid G, const double* X, const unsigned char* placed) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (placed[i]) rsa_insert(G, mk3(X[3 * i], X[3 * i + 1], X[3 * i + 2]), i);
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes); }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace
}  // namespace rg

extern "C" int rg_scene_rsa_device(int n, double L, double d, double lo, double side, uint64_t seed,
                                   int max_attempts, double* x, double* q, int* placed_out) {
  using namespace rg;
  if (n <= 0 || !(L >= 0.0) || !(d > 0.0) || !(side > 0.0) || max_attempts <= 0 || !x || !q || !placed_out)
    return RG_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  const double h = 0.5 * L, cut = L + d, cut2 = cut * cut * (1.0 + 1e-12);
  int nc = (int)std::floor(side / cut);
  if (nc < 3) return RG_ERR_ARG;  // box smaller than three rod lengths: use the host generator
  if (nc > 256) nc = 256;
  const size_t ncells = (size_t)nc * nc * nc;
  // slots per cell: well above the mean; an overflow grows the grid
  const double per_cell = (double)n / (double)ncells;
  int cap = (int)std::ceil(2.0 * per_cell + 8.0 * std::sqrt(per_cell + 1.0) + 16.0);
  DevBuf bX, bU, bCX, bCU, bPl, bSurv, bAcc, bDraw, bCnt, bCntC, bSlot, bSlotC, bFlags, bList, bBest;
  cudaError_t e;
  if ((e = bX.alloc(sizeof(double) * 3 * (size_t)n)) || (e = bU.alloc(sizeof(double) * 3 * (size_t)n)) ||
      (e = bCX.alloc(sizeof(double) * 3 * (size_t)n)) || (e = bCU.alloc(sizeof(double) * 3 * (size_t)n)) ||
      (e = bPl.alloc((size_t)n)) || (e = bSurv.alloc((size_t)n)) || (e = bAcc.alloc((size_t)n)) ||
      (e = bDraw.alloc(sizeof(long long) * (size_t)n)) || (e = bCnt.alloc(sizeof(int) * ncells)) ||
      (e = bCntC.alloc(sizeof(int) * ncells)) || (e = bFlags.alloc(sizeof(int) * 8)) ||
      (e = bList.alloc(sizeof(int) * (size_t)n)) || (e = bBest.alloc(sizeof(int) * (size_t)n))) {
    cudaGetLastError();
    return RG_ERR_CUDA;
  }
  cudaMemset(bPl.p, 0, (size_t)n);
  cudaMemset(bDraw.p, 0, sizeof(long long) * (size_t)n);
  cudaMemset(bCnt.p, 0, sizeof(int) * ncells);
  cudaMemset(bFlags.p, 0, sizeof(int) * 8);
  // [0] placed count, [1] placed-grid overflow, [2] candidate overflow,
  // [3] a slot used all its draws, [4] unplaced slots listed this round
  int* flags = bFlags.as<int>();
  auto grid_of = [&](int* cnt, int* slot, int* ovf, int capc) {
    RsaGrid G;
    G.nc = nc; G.lo = lo; G.side = side; G.cs = side / nc; G.cap = capc;
    G.cnt = cnt; G.slot = slot; G.overflow = ovf;
    return G;
  };
  int capP = cap, capC = cap;
  if ((e = bSlot.alloc(sizeof(int) * ncells * (size_t)capP)) || (e = bSlotC.alloc(sizeof(int) * ncells * (size_t)capC))) {
    cudaGetLastError();
    return RG_ERR_CUDA;
  }
  const int blocks = grid_for(n, kRsaBS, 148 * 16);
  int placed = 0, remaining = n;
  int h_flags[4] = {0, 0, 0, 0};
  for (int round = 0; remaining > 0; ++round) {
    // draws per slot this round: about 2e6 candidate draws per round, at
    // most 64 per slot, one thread per draw
    int D = (int)std::min<long long>(64, std::max<long long>(1, 2000000LL / std::max(remaining, 1)));
    RsaGrid G = grid_of(bCnt.as<int>(), bSlot.as<int>(), flags + 1, capP);
    RsaGrid Gc = grid_of(bCntC.as<int>(), bSlotC.as<int>(), flags + 2, capC);
    cudaMemsetAsync(bCntC.p, 0, sizeof(int) * ncells);
    cudaMemsetAsync(flags + 2, 0, sizeof(int));
    cudaMemsetAsync(flags + 4, 0, sizeof(int));
    RGL k_rsa_list<<<blocks, kRsaBS>>>(n, bPl.as<unsigned char>(), bSurv.as<unsigned char>(), bList.as<int>(),
                                       flags + 4, bBest.as<int>());
    RGL k_rsa_draws<<<grid_for((long long)remaining * D, kRsaBS, 148 * 32), kRsaBS>>>(
        seed, G, bX.as<double>(), bU.as<double>(), bList.as<int>(), flags + 4, bDraw.as<long long>(), D,
        (long long)max_attempts, bBest.as<int>(), h, d, cut2);
    RGL k_rsa_pick<<<blocks, kRsaBS>>>(seed, G, Gc, bList.as<int>(), flags + 4, bDraw.as<long long>(), D,
                                       (long long)max_attempts, bBest.as<int>(), bCX.as<double>(), bCU.as<double>(),
                                       bSurv.as<unsigned char>(), flags + 3);
    RGL k_rsa_resolve<<<blocks, kRsaBS>>>(n, Gc, bCX.as<double>(), bCU.as<double>(), bSurv.as<unsigned char>(),
                                          bAcc.as<unsigned char>(), h, d, cut2);
    RGL k_rsa_accept<<<blocks, kRsaBS>>>(n, G, bCX.as<double>(), bCU.as<double>(), bAcc.as<unsigned char>(),
                                         bX.as<double>(), bU.as<double>(), bPl.as<unsigned char>(), flags);
    if ((e = cudaMemcpy(h_flags, flags, sizeof(int) * 4, cudaMemcpyDeviceToHost))) return RG_ERR_CUDA;
    while (h_flags[1]) {  // a placed-grid cell overflowed: grow it and re-insert every placed rod
      capP *= 2;
      cudaFree(bSlot.p);
      bSlot.p = nullptr;
      if ((e = bSlot.alloc(sizeof(int) * ncells * (size_t)capP))) { cudaGetLastError(); return RG_ERR_CUDA; }
      cudaMemset(bCnt.p, 0, sizeof(int) * ncells);
      cudaMemset(flags + 1, 0, sizeof(int));
      G = grid_of(bCnt.as<int>(), bSlot.as<int>(), flags + 1, capP);
      RGL k_rsa_rebuild<<<blocks, kRsaBS>>>(n, G, bX.as<double>(), bPl.as<unsigned char>());
      if ((e = cudaMemcpy(h_flags, flags, sizeof(int) * 4, cudaMemcpyDeviceToHost))) return RG_ERR_CUDA;
    }
    if (h_flags[2]) {  // candidates were turned away: give the next round more room
      capC *= 2;
      cudaFree(bSlotC.p);
      bSlotC.p = nullptr;
      if ((e = bSlotC.alloc(sizeof(int) * ncells * (size_t)capC))) { cudaGetLastError(); return RG_ERR_CUDA; }
    }
    placed = h_flags[0];
    remaining = n - placed;
    // the host generator stops at the first rod it cannot place within
    // max_attempts draws; so does this one (at the end of that round)
    if (h_flags[3]) break;
  }
  if ((e = cudaGetLastError())) return RG_ERR_CUDA;
  std::vector<double> X(3 * (size_t)n), U(3 * (size_t)n);
  std::vector<unsigned char> pl(n);
  if (cudaMemcpy(X.data(), bX.p, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(U.data(), bU.p, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost) ||
      cudaMemcpy(pl.data(), bPl.p, (size_t)n, cudaMemcpyDeviceToHost))
    return RG_ERR_CUDA;
  // placed rods in slot order; quaternion turning +Y onto the axis
  int m = 0;
  for (int i = 0; i < n; ++i) {
    if (!pl[i]) continue;
    const double ux = U[3 * i], uy = U[3 * i + 1], uz = U[3 * i + 2];
    const double ang = std::acos(std::max(-1.0, std::min(1.0, uy)));
    double qw = 1, qx = 0, qy = 0, qz = 0;
    const double l = std::sqrt(uz * uz + ux * ux);  // |(+Y) x u|
    if (ang >= 1e-6 && l > 0) {
      const double s = std::sin(0.5 * ang);
      qw = std::cos(0.5 * ang);
      qx = uz / l * s;
      qz = -ux / l * s;
    }
    for (int k = 0; k < 3; ++k) x[3 * m + k] = X[3 * i + k];
    q[4 * m] = qw; q[4 * m + 1] = qx; q[4 * m + 2] = qy; q[4 * m + 3] = qz;
    ++m;
  }
  *placed_out = m;
  return RG_OK;
}
