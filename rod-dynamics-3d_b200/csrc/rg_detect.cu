// rg_detect.cu - broad phase (cell grid -> per-rod Verlet neighbour lists)
// and exact FP64 capsule narrow phase.
//
// Replaces ContactDetector::detectContacts (src/physics/contact_detector.cpp:
// 71-211) with its naive / spatial-hash broad phases (:213-281, :487-809) and
// detectCapsuleCapsule (:811-910).  The contact set is the set of pairs a < b
// (not both static) whose narrow phase fires, sorted by (a,b): exactly what
// the reference's sort+unique (:780-793) / sortedContactOrder
// (src/physics/nsc_contact.cpp:91-102) produce.
//
// Broad phase: rods are binned by centre into a box-tiling grid whose cell is
// at least the largest contacting centre distance plus a skin; each rod keeps
// the ascending list of j > i whose capsules come within margin + skin.  The
// list stays exact until some rod has moved (translation plus end-point swing)
// more than skin/2 since the build; a device-side check triggers the rebuild.
// Neighbour cells are staged through shared memory tile by tile.
#include <cstdio>

#include "rg_detect_dev.cuh"

namespace rg {

long long g_launches = 0;

// ---------------------------------------------------------------------------
// Exclusive scan in one pass: decoupled look-back (Merrill & Garland, "Single-
// pass Parallel Prefix Scan with Decoupled Look-back", 2016).  Blocks take
// tiles in increasing order from a counter; a tile publishes its aggregate,
// then one warp adds the published values of its predecessors, 32 status
// words at a time, until it meets an inclusive prefix; the tile publishes its
// own inclusive prefix and writes its outputs.  A tile only waits on tiles
// taken before it by running blocks, and every wait is bounded (ERR_TIMEOUT
// after kScanSpin polls).  n is read on the device.  The last block to leave
// clears the tile status words it used and both counters, so the next scan
// finds them zeroed without a memset (the words are zeroed once at
// allocation).  Each thread scans kScanItems consecutive values, loaded and
// stored as int4 when the arrays allow it.
// ---------------------------------------------------------------------------
constexpr int kScanBS = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBS * kScanItems;
constexpr long long kScanSpin = 1 << 24;
constexpr unsigned long long kTileAgg = 1ull << 62, kTileInc = 2ull << 62;

__device__ inline unsigned long long scan_status_load(unsigned long long* w) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*w);
  return r.load(cuda::memory_order_acquire);
}
__device__ inline void scan_status_store(unsigned long long* w, unsigned long long v) {
  cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> r(*w);
  r.store(v, cuda::memory_order_release);
}

// Exclusive prefix of tile t (t > 0) from its predecessors' status words
// (status[p] for tile p >= first, the array's first tile), by warp 0;
// valid in every lane.  Returns false when a wait ran out (ERR_TIMEOUT set).
__device__ inline bool scan_lookback(unsigned long long* status, int t, int first, int* err, int& prefix) {
  const int lane = threadIdx.x & 31;
  prefix = 0;
  for (int p = t - 1;; p -= 32) {
    const int idx = p - lane;  // lane k reads tile p - k (tiles before `first` belong to another array)
    unsigned long long w = idx >= first ? scan_status_load(&status[idx]) : kTileInc;
    long long it = 0;
    while (!__all_sync(0xffffffffu, (w >> 62) != 0)) {
      if (++it > kScanSpin) {
        if (lane == 0) atomicOr(err, ERR_TIMEOUT);
        return false;
      }
      if (it > 32) __nanosleep(32);
      if ((w >> 62) == 0) w = scan_status_load(&status[idx]);
    }
    // the nearest inclusive prefix (lowest lane) ends the walk
    const unsigned inc = __ballot_sync(0xffffffffu, (w & kTileInc) != 0);
    const int stop = inc ? __ffs(inc) - 1 : 32;
    const int v = (lane <= stop && idx >= first) ? (int)(unsigned)(w & 0xffffffffull) : 0;
    prefix += warp_sum_i(v);
    if (inc) return true;
  }
}

// words: [0] tile counter, [1] exit counter, [2 + t] status of tile t.
// One or two arrays: tiles [0, nt0) scan array 0, [nt0, nt0 + nt1) array 1.
struct ScanArrays {
  const int* in[2];
  int* out[2];
  const int* n_dev[2];
  int count;
};
__global__ void __launch_bounds__(kScanBS) k_scan_lookback(ScanArrays A, unsigned long long* words, int* err) {
  griddep_wait();
  __shared__ int shw[32];
  __shared__ int sh_tile, sh_excl, sh_ok, sh_last;
  int* tile_ctr = reinterpret_cast<int*>(&words[0]);
  int* exit_ctr = reinterpret_cast<int*>(&words[1]);
  unsigned long long* status = words + 2;
  int n_arr[2] = {0, 0}, nt[2] = {0, 0};
  for (int a = 0; a < A.count; ++a) {
    n_arr[a] = *A.n_dev[a];
    nt[a] = (n_arr[a] + kScanTile - 1) / kScanTile;
    if (nt[a] == 0 && blockIdx.x == 0 && threadIdx.x == 0) A.out[a][0] = 0;
  }
  const int ntile = nt[0] + nt[1];
  while (ntile > 0) {
    if (threadIdx.x == 0) sh_tile = atomicAdd(tile_ctr, 1);
    __syncthreads();
    const int t = sh_tile;
    if (t >= ntile) break;
    const int a = t < nt[0] ? 0 : 1;
    const int first = a ? nt[0] : 0, lt = t - first;  // the array's first tile, the tile within it
    const int n = n_arr[a];
    const int* in = A.in[a];
    int* out = A.out[a];
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15) == 0;
    const int base = lt * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    if (vec && base + kScanItems <= n) {
      const int4 x = *reinterpret_cast<const int4*>(in + base);
      const int4 y = *reinterpret_cast<const int4*>(in + base + 4);
      v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
      v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
    } else {
#pragma unroll
      for (int k = 0; k < kScanItems; ++k) v[k] = base + k < n ? in[base + k] : 0;
    }
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    int tot;
    const int ex = block_excl_scan(sum, shw, tot);
    if (threadIdx.x < 32) {
      int prefix = 0;
      bool ok = true;
      if (lt == 0) {
        if (threadIdx.x == 0) scan_status_store(&status[t], kTileInc | (unsigned)tot);
      } else {
        if (threadIdx.x == 0) scan_status_store(&status[t], kTileAgg | (unsigned)tot);
        ok = scan_lookback(status, t, first, err, prefix);
        // gave up: the call fails with ERR_TIMEOUT; later tiles see an aggregate
        if (ok && threadIdx.x == 0) scan_status_store(&status[t], kTileInc | (unsigned)(prefix + tot));
      }
      if (threadIdx.x == 0) {
        sh_excl = prefix;
        sh_ok = ok;
        if (lt == nt[a] - 1) out[n] = prefix + tot;
      }
    }
    __syncthreads();
    if (!sh_ok) break;
    int run = sh_excl + ex;
    int o[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      o[k] = run;
      run += v[k];
    }
    if (vec && base + kScanItems <= n) {
      *reinterpret_cast<int4*>(out + base) = make_int4(o[0], o[1], o[2], o[3]);
      *reinterpret_cast<int4*>(out + base + 4) = make_int4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
      for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) out[base + k] = o[k];
    }
    __syncthreads();  // sh_tile / sh_excl are reused by the next tile
  }
  // The last block out finds every tile finished and no look-back running:
  // it clears the status words and the counters for the next scan.
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    sh_last = atomicAdd(exit_ctr, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!sh_last) return;
  __threadfence();
  for (int t = threadIdx.x; t < ntile; t += blockDim.x) status[t] = 0;
  if (threadIdx.x == 0) {
    *tile_ctr = 0;
    *exit_ctr = 0;
  }
}

cudaError_t Scan::alloc(int cap_) {
  cap = cap_;
  const int tiles = (cap + kScanTile - 1) / kScanTile + 1;
  const size_t bytes = sizeof(unsigned long long) * (2 * tiles + 2);  // two arrays at most
  cudaError_t e = cudaMalloc(&d_blocks, bytes);
  if (e == cudaSuccess) e = cudaMemset(d_blocks, 0, bytes);
  return e;
}
void Scan::free_() {
  if (d_blocks) cudaFree(d_blocks);
  d_blocks = nullptr;
}
void Scan::run(const int* in, int* out, const int* n_dev, int* err, cudaStream_t s) const {
  const int tiles = (cap + kScanTile - 1) / kScanTile + 1;
  int g = tiles < 148 * 4 ? tiles : 148 * 4;
  if (g < 1) g = 1;
  ScanArrays A = {{in, nullptr}, {out, nullptr}, {n_dev, nullptr}, 1};
  RGL launch_dep(k_scan_lookback, g, kScanBS, s, A, static_cast<unsigned long long*>(d_blocks), err);
}
void Scan::run2(const int* in0, int* out0, const int* n0_dev, const int* in1, int* out1, const int* n1_dev,
                int* err, cudaStream_t s) const {
  const int tiles = 2 * ((cap + kScanTile - 1) / kScanTile + 1);
  int g = tiles < 148 * 4 ? tiles : 148 * 4;
  ScanArrays A = {{in0, in1}, {out0, out1}, {n0_dev, n1_dev}, 2};
  RGL launch_dep(k_scan_lookback, g, kScanBS, s, A, static_cast<unsigned long long*>(d_blocks), err);
}

// ---------------------------------------------------------------------------
// Segment records, displacement check, cell grid.
// ---------------------------------------------------------------------------
__global__ void k_seg(State st, Seg* seg) {
  griddep_wait();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    dq q = st.q.ld(i);
    d3 u = axis_y(q);
    Seg s;
    s.cx = st.x.x[i]; s.cy = st.x.y[i]; s.cz = st.x.z[i]; s.h = st.h[i];
    s.ux = u.x; s.uy = u.y; s.uz = u.z; s.r = st.r[i];
    seg[i] = s;
  }
}

// Largest displacement bound |Δx| + h|Δu| since the last build; sets the
// rebuild flag when it reaches skin/2.  With ref2 (near lists), the largest
// bound since the last near-list build goes to ctl->near_disp.
__global__ void k_disp_check(State st, const Seg* seg, const double* ref, const double* ref2, Box box,
                             double skin, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  __shared__ double sm[32], sm2[32];
  double m = 0.0, m2 = 0.0;
  const int n = st.n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Seg s = seg[i];
    m = fmax(m, seg_disp(s, ref, n, i, box));  // non-finite state: 1e300 forces a rebuild
    if (ref2) m2 = fmax(m2, seg_disp(s, ref2, n, i, box));
  }
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
      if (v >= 0.5 * skin * (1.0 - 1e-9)) atomicExch(&ctl->rebuild, 1);
      if (ref2) atomic_max_nonneg(&ctl->near_disp, v2);
    }
  }
}

// Near lists (multi-kernel detection): rebuilt when the lists were rebuilt
// (near_valid cleared) or some rod's bound since the near build reached
// near_skin/2.  A pair left out was, at the build, farther apart than
// r_a + r_b + margin + near_skin by seg_far's lower bound, and each of its
// rods has since moved less than near_skin/2 (the segment distance is
// 1-Lipschitz in the end points), so it cannot be within r_a + r_b + margin.
__device__ inline bool near_rebuild_due(const Ctl* ctl, double near_skin) {
  return !ctl->near_valid || ctl->near_disp >= 0.5 * near_skin * (1.0 - 1e-9);
}

__global__ void k_near_build(const Seg* seg, int n, const double* inv_mass, Box box, double extra,
                             double near_skin, const int* nbr_cnt, const int* nbr, int maxnb, int* near_cnt,
                             int* near_nbr, double* ref2, const Ctl* ctl) {
  griddep_wait();
  // a list rebuild of this detection (its flag still set: k_lists_done
  // clears it) makes the near lists due as well
  if (ctl->err || !(ctl->rebuild || near_rebuild_due(ctl, near_skin))) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Seg A = seg[i];
    const bool a_static = !(inv_mass[i] > 0.0);
    const int cnt = nbr_cnt[i];
    const int* list = nbr + (size_t)i * maxnb;
    int* out = near_nbr + (size_t)i * maxnb;
    int m = 0;
    for (int k = 0; k < cnt; ++k) {
      const int j = list[k];
      if (a_static && !(inv_mass[j] > 0.0)) continue;
      const Seg B = seg[j];
      d3 xa{A.cx, A.cy, A.cz}, xb{B.cx, B.cy, B.cz};
      if (seg_far(A, B, (xb - xa) + min_image_shift(box, xa, xb), A.r + B.r + extra)) continue;
      out[m++] = j;
    }
    near_cnt[i] = m;
    ref2[i] = A.cx; ref2[n + i] = A.cy; ref2[2 * n + i] = A.cz;
    ref2[3 * n + i] = A.ux; ref2[4 * n + i] = A.uy; ref2[5 * n + i] = A.uz;
  }
}

// Closes a detection with near lists (k_build_done and the near-list
// close-out in one): counts a list rebuild, and marks the near lists built.
__global__ void k_lists_done(double near_skin, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  const bool near_due = ctl->rebuild || near_rebuild_due(ctl, near_skin);
  if (ctl->rebuild) {
    ctl->rebuilds += 1;
    ctl->rebuild = 0;
  }
  ctl->maxdisp = 0.0;
  if (near_due) {
    ctl->near_valid = 1;
    ctl->near_disp = 0.0;
    ctl->near_rebuilds += 1;
  }
}

__global__ void k_cell_fill(int n, const int* cell_of, const int* cell_start, int* cell_fill,
                            int* cell_rods, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = cell_of[i];
    int p = atomicAdd(&cell_fill[c], 1);
    cell_rods[cell_start[c] + p] = i;
  }
}

__global__ void k_zero_cells(int* cnt, int* fill, int ncells, int* nbr_cnt, int n, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= ncells || i < n; i += gridDim.x * blockDim.x) {
    if (i <= ncells) cnt[i] = 0;
    if (i < ncells) fill[i] = 0;
    if (i < n) nbr_cnt[i] = 0;
  }
}

// One block per home cell (see build_cell).
__global__ void __launch_bounds__(kTile) k_build_lists(const Seg* seg, int n, const GridDev* gdev, Box box,
                                                       const int* cell_start, const int* cell_rods,
                                                       double margin, double skin, double cut_center,
                                                       int all_pairs, int* nbr_cnt, int* nbr,
                                                       int maxnb, Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  const GridDev g = *gdev;
  __shared__ BuildSmem sm;
  constexpr int kQ = 4 * kTile;  // candidate queues of the compacted build
  __shared__ unsigned q1[kQ], q2[kQ];
  int overflow = 0;
  double invL[3] = {1.0, 1.0, 1.0};
  for (int k = 0; k < 3; ++k)
    if (box.L[k] > 0.0) invL[k] = 1.0 / box.L[k];
  for (int cell = blockIdx.x; cell < g.ncells; cell += gridDim.x)
    build_cell_pairs(seg, g, box, invL, cell_start, cell_rods, margin, skin, all_pairs, nbr_cnt, nbr, maxnb,
                     cell, sm, q1, q2, kQ, overflow);
  if (overflow) atomicOr(&ctl->err, ERR_NBR_CAP);
  (void)n;
  (void)cut_center;
}

__global__ void k_save_ref(const Seg* seg, int n, double* ref, int* nbr, int* nbr_cnt, int maxnb, Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  int overflow = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    sort_list(nbr, nbr_cnt, maxnb, i, overflow);
    Seg s = seg[i];
    ref[i] = s.cx; ref[n + i] = s.cy; ref[2 * n + i] = s.cz;
    ref[3 * n + i] = s.ux; ref[4 * n + i] = s.uy; ref[5 * n + i] = s.uz;
  }
  if (overflow) atomicOr(&ctl->err, ERR_NBR_CAP);
}

__global__ void k_build_done(Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  if (ctl->rebuild) {
    ctl->rebuilds += 1;
    ctl->rebuild = 0;
    ctl->near_valid = 0;  // near lists are drawn from the lists
  }
  ctl->maxdisp = 0.0;
}

__global__ void k_bounds(const Seg* seg, int n, unsigned long long* mn, unsigned long long* mx,
                         const Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Seg s = seg[i];
    atomicMin(&mn[0], ord_key(s.cx)); atomicMax(&mx[0], ord_key(s.cx));
    atomicMin(&mn[1], ord_key(s.cy)); atomicMax(&mx[1], ord_key(s.cy));
    atomicMin(&mn[2], ord_key(s.cz)); atomicMax(&mx[2], ord_key(s.cz));
  }
}
__global__ void k_open_grid(const unsigned long long* mn, const unsigned long long* mx, double cut,
                            int maxdim, GridDev* g, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  open_grid(mn, mx, cut, maxdim, g);
}

// Reads the device grid descriptor into each thread (open systems).
__global__ void k_cell_count_dyn(const Seg* seg, int n, const GridDev* gd, int pbc, int* cell_of,
                                 int* cell_cnt, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  GridDev g = *gd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Seg s = seg[i];
    int cx = cell_coord(s.cx, g.lo[0], g.cell[0], g.n[0], pbc);
    int cy = cell_coord(s.cy, g.lo[1], g.cell[1], g.n[1], pbc);
    int cz = cell_coord(s.cz, g.lo[2], g.cell[2], g.n[2], pbc);
    int c = (cz * g.n[1] + cy) * g.n[0] + cx;
    cell_of[i] = c;
    atomicAdd(&cell_cnt[c], 1);
  }
}

// ---------------------------------------------------------------------------
// Narrow phase over the lists: count -> scan -> write (sorted by (a,b)).
// ---------------------------------------------------------------------------
// Resident 256-thread blocks per SM k_narrow_count is compiled for (one rod
// per thread, latency-bound on the neighbour gathers: more resident warps).
#ifndef RG_NARROW_MIN_BLOCKS
#define RG_NARROW_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(256, RG_NARROW_MIN_BLOCKS) k_narrow_count(const Seg* seg, State st, Box box, double delta, const int* nbr_cnt,
                               const int* nbr, int maxnb, int words, unsigned long long* mask,
                               int* hit_cnt, BodyCSR csr, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    hit_cnt[i] = narrow_count_rod(i, seg, st.inv_mass, box, delta, nbr_cnt, nbr, maxnb, words, mask);
    if (csr.cnt) {  // body CSR counts start from zero (counted by k_narrow_write)
      csr.cnt[i] = 0;
      csr.fill[i] = 0;
      if (i == 0) csr.cnt[st.n] = 0;
    }
  }
}

__global__ void k_narrow_write(const Seg* seg, int n, Box box, const int* nbr_cnt, const int* nbr,
                               int maxnb, int words, const unsigned long long* mask, const int* hit_off,
                               Contacts con, BodyCSR csr, Ctl* ctl) {
  griddep_wait();
  if (ctl->err) return;
  int total = hit_off[n];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->contacts = total < con.cap ? total : con.cap;
    if (total > con.cap) atomicOr(&ctl->err, ERR_CONTACT_CAP);
  }
  if (total > con.cap) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int o0 = hit_off[i], o1 = hit_off[i + 1];
    if (o1 == o0) continue;
    narrow_write_rod(i, o0, seg, box, nbr_cnt, nbr, maxnb, words, mask, con);
    if (csr.cnt) {  // contacts per body for the body CSR (both sides)
      atomicAdd(&csr.cnt[i], o1 - o0);
      for (int o = o0; o < o1; ++o) atomicAdd(&csr.cnt[con.b[o]], 1);
    }
  }
}

cudaError_t Contacts::alloc(int cap_) {
  cap = cap_;
  cudaError_t e;
  if ((e = cudaMalloc(&a, sizeof(int) * cap))) return e;
  if ((e = cudaMalloc(&b, sizeof(int) * cap))) return e;
  if ((e = cudaMalloc(&type, sizeof(int) * cap))) return e;
  return cudaMalloc(&g, sizeof(double) * 14 * (size_t)cap);
}
void Contacts::free_() {
  cudaFree(a); cudaFree(b); cudaFree(type); cudaFree(g);
  a = b = type = nullptr;
  g = nullptr;
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
struct DetDev {  // device-resident grid descriptor and scratch
  GridDev grid;
  unsigned long long mn[3], mx[3];  // contiguous: bounds[0..2] min, [3..5] max
  int n;       // body count (scan length for per-rod arrays)
  int ncells;  // cell count (scan length for cell arrays)
};
static DetDev* det_dev(rg_system* s) {
  return reinterpret_cast<DetDev*>(s->det.ref + 6 * (size_t)s->n);
}
const int* detector_n_dev(rg_system* s) { return &det_dev(s)->n; }
GridDev* detector_grid(rg_system* s) { return &det_dev(s)->grid; }
unsigned long long* detector_bounds(rg_system* s) { return det_dev(s)->mn; }

__global__ void k_grid_ncells(DetDev* dd, const Ctl* ctl) {
  griddep_wait();
  if (ctl->err || !ctl->rebuild) return;
  dd->ncells = dd->grid.ncells;
}

// Near lists are on unless near_skin_pct is negative (full lists).
static bool check_near_lists(const rg_config& c) { return c.near_skin_pct >= 0; }

cudaError_t detector_alloc(rg_system* s) {
  ++s->buf_gen;
  Detector& d = s->det;
  const int n = s->n;
  const rg_config& c = s->cfg;
  double rmax = 0, hmax = 0, dsum = 0, lsum = 0;
  std::vector<double> r(n), h(n);
  cudaMemcpy(r.data(), s->st.r, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(h.data(), s->st.h, sizeof(double) * n, cudaMemcpyDeviceToHost);
  for (int i = 0; i < n; ++i) {
    rmax = r[i] > rmax ? r[i] : rmax;
    hmax = h[i] > hmax ? h[i] : hmax;
    dsum += 2 * r[i];
    lsum += 2 * h[i];
  }
  d.margin = c.model == RG_MODEL_HARMONIC ? c.soft_delta : 0.0;
  // Default skin: half a diameter, but at least a tenth of the rod length,
  // so thin rods (whose lists stay short, and whose per-step narrow phase
  // runs over the near list only) rebuild rarely.
  d.skin = c.skin > 0 ? c.skin : fmax(0.5 * (dsum / n), 0.1 * (lsum / n)) + 1e-6;
  d.cut_center = 2.0 * (hmax + rmax) + d.margin + d.skin;
  d.all_pairs = false;
  GridDev gd{};
  if (s->box.pbc) {
    for (int k = 0; k < 3; ++k) {
      double L = s->box.L[k];
      int nc = (int)floor(L / d.cut_center);
      if (nc < 1) nc = 1;
      if (nc > 256) nc = 256;
      d.ncell[k] = nc;
      d.cell[k] = L / nc;
      // Minimum-image shifts of a listed pair must stay on the same image
      // while the list is valid: needs L/2 > cut_center + skin.
      if (0.5 * L <= d.cut_center + d.skin) d.all_pairs = true;
      gd.lo[k] = s->box.lo[k];
      gd.cell[k] = d.cell[k];
      gd.n[k] = nc;
    }
    d.ncells = d.ncell[0] * d.ncell[1] * d.ncell[2];
    gd.ncells = d.ncells;
  } else {
    d.ncells = 64 * 64 * 64;
  }
  if (d.all_pairs && n > 4096) return cudaErrorInvalidValue;
  if (d.maxnb <= 0) {
    if (d.all_pairs) d.maxnb = n;
    else d.maxnb = c.max_neighbors > 0 ? c.max_neighbors : 64;
  }
  d.mask_words = (d.maxnb + 63) / 64;
  cudaError_t e;
  if ((e = cudaMalloc(&d.nbr_cnt, sizeof(int) * n))) return e;
  if ((e = cudaMalloc(&d.nbr, sizeof(int) * (size_t)n * d.maxnb))) return e;
  if ((e = cudaMalloc(&d.ref, sizeof(double) * 6 * (size_t)n + sizeof(DetDev)))) return e;
  if ((e = cudaMalloc(&d.seg, sizeof(Seg) * (size_t)n))) return e;
  if ((e = cudaMalloc(&d.cell_of, sizeof(int) * n))) return e;
  if ((e = cudaMalloc(&d.cell_cnt, sizeof(int) * (d.ncells + 1)))) return e;
  if ((e = cudaMalloc(&d.cell_start, sizeof(int) * (d.ncells + 1)))) return e;
  if ((e = cudaMalloc(&d.cell_fill, sizeof(int) * (d.ncells + 1)))) return e;
  if ((e = cudaMalloc(&d.cell_rods, sizeof(int) * n))) return e;
  if ((e = cudaMalloc(&d.hit_cnt, sizeof(int) * (n + 1)))) return e;
  if ((e = cudaMalloc(&d.hit_off, sizeof(int) * (n + 1)))) return e;
  if ((e = cudaMalloc(&d.hit_mask, sizeof(unsigned long long) * (size_t)n * d.mask_words))) return e;
  if ((e = cudaMemset(d.nbr_cnt, 0, sizeof(int) * n))) return e;
  if (c.model != RG_MODEL_NSC && !d.all_pairs && check_near_lists(c)) {
    // near lists of the multi-kernel detection (the soft / HM step)
    d.near_skin = (c.near_skin_pct > 0 ? 0.01 * c.near_skin_pct : 0.05) * d.skin;
    if ((e = cudaMalloc(&d.near_cnt, sizeof(int) * n))) return e;
    if ((e = cudaMalloc(&d.near_nbr, sizeof(int) * (size_t)n * d.maxnb))) return e;
    if ((e = cudaMalloc(&d.ref2, sizeof(double) * 6 * (size_t)n))) return e;
  }
  if (c.model == RG_MODEL_NSC) {
    // all-pairs boxes rebuild the near list from every pair: a wider near
    // skin makes those rebuilds rare
    d.near_skin = (c.near_skin_pct > 0 ? 0.01 * c.near_skin_pct : (d.all_pairs ? 0.5 : 0.05)) * d.skin;
    if ((e = cudaMalloc(&d.near, sizeof(int2) * (size_t)n * d.maxnb))) return e;
    if ((e = cudaMalloc(&d.ref2, sizeof(double) * 6 * (size_t)n))) return e;
    if ((e = cudaMalloc(&d.moved, (size_t)n))) return e;
    if ((e = cudaMemset(d.moved, 1, (size_t)n))) return e;
  }
  DetDev hd{};
  hd.grid = gd;
  hd.n = n;
  hd.ncells = s->box.pbc ? d.ncells : 1;
  return cudaMemcpy(det_dev(s), &hd, sizeof(DetDev), cudaMemcpyHostToDevice);
}

void detector_free(rg_system* s) {
  Detector& d = s->det;
  cudaFree(d.nbr_cnt); cudaFree(d.nbr); cudaFree(d.ref); cudaFree(d.seg);
  cudaFree(d.cell_of); cudaFree(d.cell_cnt); cudaFree(d.cell_start); cudaFree(d.cell_fill);
  cudaFree(d.cell_rods); cudaFree(d.hit_cnt); cudaFree(d.hit_off); cudaFree(d.hit_mask);
  cudaFree(d.near); cudaFree(d.ref2); cudaFree(d.moved);
  cudaFree(d.near_cnt); cudaFree(d.near_nbr);
  d = Detector();
}

void force_rebuild(rg_system* s) {
  int one = 1;
  cudaMemcpyAsync(&s->d_ctl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, s->stream);
}

// Full detection at the current state with activation margin `delta`:
// segment records, (optional) displacement check and list rebuild, narrow
// phase.  Result: s->con sorted by (a,b) and ctl->contacts.
void detect_launch(rg_system* s, double delta, bool check_rebuild, bool seg_ready, bool body_csr) {
  Detector& d = s->det;
  const int n = s->n;
  cudaStream_t st = s->stream;
  Ctl* ctl = s->d_ctl;
  DetDev* dd = det_dev(s);
  const int bs = 256;
  const int g = grid_for(n, bs);
  const bool near = d.near_cnt != nullptr;
  if (!seg_ready) {
    RGL launch_dep(k_seg, g, bs, st, s->st, d.seg);
    if (check_rebuild && !d.all_pairs) {
      RGL launch_dep(k_disp_check, g, bs, st, s->st, d.seg, d.ref, near ? d.ref2 : nullptr, s->box, d.skin, ctl);
    }
  }
  // --- rebuild: every kernel below returns at once unless ctl->rebuild ---
  if (!s->box.pbc) {
    cudaMemsetAsync(dd->mn, 0xff, sizeof(dd->mn), st);
    cudaMemsetAsync(dd->mx, 0x00, sizeof(dd->mx), st);
    RGL launch_dep(k_bounds, g, bs, st, d.seg, n, dd->mn, dd->mx, ctl);
    RGL launch_dep(k_open_grid, 1, 1, st, dd->mn, dd->mx, d.cut_center, 64, &dd->grid, ctl);
    RGL launch_dep(k_grid_ncells, 1, 1, st, dd, ctl);
  }
  RGL launch_dep(k_zero_cells, grid_for((d.ncells + 1 > n ? d.ncells + 1 : n), bs), bs, st, d.cell_cnt, d.cell_fill, d.ncells,
                                                                                     d.nbr_cnt, n, ctl);
  RGL launch_dep(k_cell_count_dyn, g, bs, st, d.seg, n, &dd->grid, s->box.pbc, d.cell_of, d.cell_cnt, ctl);
  s->scan.run(d.cell_cnt, d.cell_start, &dd->ncells, &ctl->err, st);
  RGL launch_dep(k_cell_fill, g, bs, st, n, d.cell_of, d.cell_start, d.cell_fill, d.cell_rods, ctl);
  int gb = d.ncells < s->sm_count * 8 ? d.ncells : s->sm_count * 8;
  RGL launch_dep(k_build_lists, gb, kTile, st, d.seg, n, &dd->grid, s->box, d.cell_start, d.cell_rods,
                                       d.margin, d.skin, d.cut_center, d.all_pairs ? 1 : 0,
                                       d.nbr_cnt, d.nbr, d.maxnb, ctl);
  RGL launch_dep(k_save_ref, g, bs, st, d.seg, n, d.ref, d.nbr, d.nbr_cnt, d.maxnb, ctl);
  // --- near lists (every kernel below returns at once unless they are due) ---
  const int* lcnt = d.nbr_cnt;
  const int* lnbr = d.nbr;
  if (near) {
    RGL launch_dep(k_near_build, g, bs, st, d.seg, n, s->st.inv_mass, s->box, d.margin + d.near_skin, d.near_skin,
                                       d.nbr_cnt, d.nbr, d.maxnb, d.near_cnt, d.near_nbr, d.ref2, ctl);
    RGL launch_dep(k_lists_done, 1, 1, st, d.near_skin, ctl);
    lcnt = d.near_cnt;
    lnbr = d.near_nbr;
  } else {
    RGL launch_dep(k_build_done, 1, 1, st, ctl);
  }
  // --- narrow phase ---
  const BodyCSR csr = body_csr ? s->csr : BodyCSR{};
  RGL launch_dep(k_narrow_count, g, bs, st, d.seg, s->st, s->box, delta, lcnt, lnbr, d.maxnb,
                                   d.mask_words, d.hit_mask, d.hit_cnt, csr, ctl);
  s->scan.run(d.hit_cnt, d.hit_off, &dd->n, &ctl->err, st);
  RGL launch_dep(k_narrow_write, g, bs, st, d.seg, n, s->box, lcnt, lnbr, d.maxnb, d.mask_words,
                                   d.hit_mask, d.hit_off, s->con, csr, ctl);
}

}  // namespace rg
