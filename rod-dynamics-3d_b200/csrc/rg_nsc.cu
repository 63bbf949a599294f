// rg_nsc.cu - the non-smooth-contact (PSOR) step as one persistent kernel.
//
// NscContactSolver (src/physics/nsc_contact.cpp):
//   detectAndBuildManifolds :239-321, buildTangentBasis :78-85,
//   computeDiag :106-117, solveVelocities :325-655 (warm start :344-380,
//   sweeps :385-552, residual :546-551, cache :646-654),
//   projectPositions :659-880 (multi-body path :698-879);
// step order of App::physicsStep (src/app/main.cpp:4383-4528).
//
// Execution model.  A "team" of co-resident blocks (cooperative launch) runs
// every phase of one system's step - free flight, detection, colouring,
// manifold rows, PSOR sweeps, position update, projection, wrap - for
// nsteps steps in ONE launch.  Phases are separated by a bounded team
// barrier instead of kernel boundaries.  Independent systems run as separate
// teams of one launch (batching).
//
// Gauss-Seidel is graph-coloured: Jones-Plassmann first-fit colouring of the
// contacts (no two contacts of a colour share a dynamic body), computed with
// per-body atomic maxima of contact priorities and per-body colour masks
// instead of adjacency lists.  A sweep visits colours in order and the
// contacts of a colour in parallel; this is sequential Gauss-Seidel over the
// colour-major permutation of the (a,b)-sorted contacts, bit for bit.  Rows
// live in colour-major slots so each colour is a contiguous, coalesced range;
// the per-sweep residual max is a warp-shuffle reduction plus one atomic per
// block, and the exit test runs on the device.
#include <cstring>

#include "rg_nsc_dev.cuh"

namespace rg {

#ifndef RG_NARROW_LANES
#define RG_NARROW_LANES 2  // lanes per rod in the narrow phase over the lists
#endif

GridDev* detector_grid(rg_system* s);
unsigned long long* detector_bounds(rg_system* s);
MlpDev mlp_dev(rg_system* s);

// ---------------------------------------------------------------------------
// Teams and team barriers.
// ---------------------------------------------------------------------------
struct Team {
  int b0, nb;
  unsigned int* bar;
  int* err;
  long long spin_limit;   // polls per barrier wait before ERR_TIMEOUT
  unsigned int absent;    // test hook: blocks the barriers wait for in vain
  __device__ int rank() const { return (int)blockIdx.x - b0; }
  __device__ int tid() const { return rank() * (int)blockDim.x + (int)threadIdx.x; }
  __device__ int size() const { return nb * (int)blockDim.x; }
};

__device__ inline bool team_sync(const Team& T) {
  GridBar g{T.bar, T.bar + 1, T.err, T.spin_limit, T.absent};
  return grid_sync(g, (unsigned)T.nb);
}
// Barrier among the first nsub blocks of the team (the others must not call it).
__device__ inline bool team_sync_sub(const Team& T, int nsub) {
  GridBar g{T.bar + 2, T.bar + 3, T.err, T.spin_limit, T.absent};
  return grid_sync(g, (unsigned)nsub);
}

__device__ inline double block_reduce_max(double v, double* sm) {
  v = warp_max(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
  if (threadIdx.x < 32) r = warp_max(r);
  return r;  // valid in thread 0
}
__device__ inline int block_reduce_sum_i(int v, int* sm) {
  v = warp_sum_i(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  int r = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0;
  if (threadIdx.x < 32) r = warp_sum_i(r);
  return r;  // valid in thread 0
}

// Phase timers (team rank 0, thread 0; %globaltimer in ns) when enabled.
// ---------------------------------------------------------------------------
__device__ inline unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
struct PhaseClock {
  Ctl* ctl;
  bool on;
  unsigned long long t;
  __device__ PhaseClock(Ctl* c, bool enabled) : ctl(c), on(enabled), t(enabled ? gtimer() : 0) {}
  __device__ void mark(int k) {
    if (!on) return;
    unsigned long long u = gtimer();
    ctl->phase_ns[k] += (long long)(u - t);
    t = u;
  }
};

// Dynamic shared memory of the persistent step: the small-solve arrays, or
// the list-build tiles while a rebuild runs (phases never overlap).
extern __shared__ __align__(16) unsigned char nsc_dyn_smem[];
// list-build candidate queues, after the tiles
constexpr int kBuildQ = 4096;
constexpr size_t kBuildQOff = (sizeof(BuildSmem) + 15) & ~(size_t)15;

struct SmemNsc {
  double red_d[32];
  int red_i[32];
  int scan_w[32];
  int pre[32];
  int coff[kMaxColors + 1];
  int bcast;
};

// Every block computes Σ blk[0..rank) and Σ blk[0..nb).
__device__ inline void block_prefix(const int* blk, int nb, int rank, int& prefix, int& total, SmemNsc& sm) {
  int a = 0, b = 0;
  for (int r = threadIdx.x; r < nb; r += blockDim.x) {
    int v = *(volatile const int*)&blk[r];
    b += v;
    if (r < rank) a += v;
  }
  int pa = warp_sum_i(a), pb = warp_sum_i(b);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    sm.pre[threadIdx.x >> 5] = pa;
    sm.red_i[threadIdx.x >> 5] = pb;
  }
  __syncthreads();
  int x = 0, y = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    x += sm.pre[w];
    y += sm.red_i[w];
  }
  prefix = x;
  total = y;
  __syncthreads();
}

// Exclusive scan of in[0..m) into out[0..m], out[m] = total (team, blocked).
__device__ inline bool team_excl_scan(const Team& T, const int* in, int* out, int m, int* blk, SmemNsc& sm) {
  const int rank = T.rank();
  const int seg = (m + T.nb - 1) / T.nb;
  const int lo = rank * seg < m ? rank * seg : m;
  const int hi = lo + seg < m ? lo + seg : m;
  int s = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) s += in[i];
  int bsum = block_reduce_sum_i(s, sm.red_i);
  if (threadIdx.x == 0) blk[rank] = bsum;
  if (!team_sync(T)) return false;
  int prefix, total;
  block_prefix(blk, T.nb, rank, prefix, total, sm);
  int run = prefix;
  for (int base = lo; base < hi; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < hi ? in[i] : 0;
    int tot;
    int ex = block_excl_scan(v, sm.scan_w, tot);
    if (i < hi) out[i] = run + ex;
    run += tot;
  }
  if (rank == 0 && threadIdx.x == 0) out[m] = total;
  return team_sync(T);
}

// ---------------------------------------------------------------------------
// Detection inside the persistent kernel.
// ---------------------------------------------------------------------------
__device__ __noinline__ bool rebuild_phase(const Team& T, const NscView& V, SmemNsc& sm) {
  Ctl* ctl = V.ctl;
  const int n = V.st.n;
  const int tid = T.tid(), TS = T.size(), rank = T.rank();
  if (!V.box.pbc) {
    if (rank == 0 && threadIdx.x < 3) {
      V.bounds[threadIdx.x] = ~0ull;
      V.bounds[3 + threadIdx.x] = 0ull;
    }
    if (!team_sync(T)) return false;
    for (int i = tid; i < n; i += TS) {
      Seg s = V.seg[i];
      atomicMin(&V.bounds[0], ord_key(s.cx)); atomicMax(&V.bounds[3], ord_key(s.cx));
      atomicMin(&V.bounds[1], ord_key(s.cy)); atomicMax(&V.bounds[4], ord_key(s.cy));
      atomicMin(&V.bounds[2], ord_key(s.cz)); atomicMax(&V.bounds[5], ord_key(s.cz));
    }
    if (!team_sync(T)) return false;
    if (rank == 0 && threadIdx.x == 0) open_grid(V.bounds, V.bounds + 3, V.cut_center, 64, V.grid);
    if (!team_sync(T)) return false;
  }
  GridDev g;
  {
    const volatile GridDev* vg = V.grid;
    for (int k = 0; k < 3; ++k) {
      g.lo[k] = vg->lo[k];
      g.cell[k] = vg->cell[k];
      g.n[k] = vg->n[k];
    }
    g.ncells = vg->ncells;
  }
  unsigned long long t_start = (ctl->prof_phases && rank == 0 && threadIdx.x == 0) ? gtimer() : 0;
  for (int c = tid; c <= g.ncells; c += TS) {
    V.cell_cnt[c] = 0;
    V.cell_fill[c] = 0;
  }
  for (int i = tid; i < n; i += TS) V.nbr_cnt[i] = 0;
  if (!team_sync(T)) return false;
  for (int i = tid; i < n; i += TS) {
    Seg s = V.seg[i];
    int cx = cell_coord(s.cx, g.lo[0], g.cell[0], g.n[0], V.box.pbc);
    int cy = cell_coord(s.cy, g.lo[1], g.cell[1], g.n[1], V.box.pbc);
    int cz = cell_coord(s.cz, g.lo[2], g.cell[2], g.n[2], V.box.pbc);
    int c = (cz * g.n[1] + cy) * g.n[0] + cx;
    V.cell_of[i] = c;
    atomicAdd(&V.cell_cnt[c], 1);
  }
  if (!team_sync(T)) return false;
  if (!team_excl_scan(T, V.cell_cnt, V.cell_start, g.ncells, V.blk, sm)) return false;
  for (int i = tid; i < n; i += TS) {
    int c = V.cell_of[i];
    V.cell_rods[V.cell_start[c] + atomicAdd(&V.cell_fill[c], 1)] = i;
  }
  if (!team_sync(T)) return false;
  int overflow = 0;
  double invL[3] = {1.0, 1.0, 1.0};
  for (int k = 0; k < 3; ++k)
    if (V.box.L[k] > 0.0) invL[k] = 1.0 / V.box.L[k];
  if (n < 48 * g.ncells) {
    // sparse cells: one thread per home rod
    for (int i = tid; i < n; i += TS)
      build_rod_list(i, V.seg, g, V.box, invL, V.cell_of, V.cell_start, V.cell_rods, V.margin, V.skin,
                     V.all_pairs, V.nbr_cnt, V.nbr, V.maxnb, overflow);
  } else {
    // crowded cells: the block splits the pairs of one home cell at a time
    for (int cell = rank; cell < g.ncells; cell += T.nb)
      build_cell_pairs(V.seg, g, V.box, invL, V.cell_start, V.cell_rods, V.margin, V.skin, V.all_pairs,
                       V.nbr_cnt, V.nbr, V.maxnb, cell, *reinterpret_cast<BuildSmem*>(nsc_dyn_smem),
                       reinterpret_cast<unsigned*>(nsc_dyn_smem + kBuildQOff),
                       reinterpret_cast<unsigned*>(nsc_dyn_smem + kBuildQOff) + kBuildQ, kBuildQ, overflow);
  }
  if (!team_sync(T)) return false;
  for (int i = tid; i < n; i += TS) {
    sort_list(V.nbr, V.nbr_cnt, V.maxnb, i, overflow);
    Seg s = V.seg[i];
    V.ref[i] = s.cx; V.ref[n + i] = s.cy; V.ref[2 * n + i] = s.cz;
    V.ref[3 * n + i] = s.ux; V.ref[4 * n + i] = s.uy; V.ref[5 * n + i] = s.uz;
  }
  if (overflow) atomicOr(&ctl->err, ERR_NBR_CAP);
  if (!team_sync(T)) return false;
  if (*(volatile int*)&ctl->err) return false;
  if (rank == 0 && threadIdx.x == 0) {
    ctl->rebuild = 0;
    ctl->rebuilds += 1;
    if (t_start) ctl->phase_ns[9] += (long long)(gtimer() - t_start);
  }
  return true;
}

// Contacts at the current segment records (V.seg current, ctl->maxdisp
// accumulated by the caller, all blocks past a team barrier).  Returns the
// contact count, or -1 on error.
// Two-level lists: the near list holds the list entries within the contact
// reach (r_a + r_b + margin) plus near_skin, rebuilt from the lists when a
// rod has moved near_skin/2 since its build (or the lists were rebuilt).  A
// pair outside it was at least near_skin beyond contact at the build, and
// each rod has since moved less than near_skin/2 (|dx| + h|du| bounds every
// point of a segment), so it cannot touch: the contact set found from the
// near list is the exact one.  Contacts come out in near-list order, which
// is (a, b) order.
__device__ __noinline__ int detect_near(const Team& T, const NscView& V, double delta, SmemNsc& sm,
                                        bool lists_rebuilt, bool position_level) {
  Ctl* ctl = V.ctl;
  const int n = V.st.n;
  const int rank = T.rank();
  const int mode = V.all_pairs ? 2 : 1;
  double invL[3] = {1.0, 1.0, 1.0};
  for (int k = 0; k < 3; ++k)
    if (V.box.L[k] > 0.0) invL[k] = 1.0 / V.box.L[k];
  const bool rebuild_near = lists_rebuilt || !*(volatile int*)&ctl->near_valid ||
                            *(volatile double*)&ctl->near_disp >= 0.5 * V.near_skin * (1.0 - 1e-9);
  int prefix, total;
  if (rebuild_near) {
    const int seg = (n + T.nb - 1) / T.nb;
    const int lo = rank * seg < n ? rank * seg : n;
    const int hi = lo + seg < n ? lo + seg : n;
    constexpr int G = RG_NARROW_LANES;
    int mine = 0;
    for (int base = lo; base < hi; base += blockDim.x / G) {
      const int i = base + threadIdx.x / G;
      const bool valid = i < hi;
      const int c = near_count_lanes<G>(i, valid, V.seg, V.st.inv_mass, V.box, invL, mode, V.margin + V.near_skin,
                                        V.nbr_cnt, V.nbr, V.maxnb, V.words, V.mask);
      if (valid && (threadIdx.x & (G - 1)) == 0) {
        V.hit_cnt[i] = c;
        mine += c;
      }
    }
    const int bsum = block_reduce_sum_i(mine, sm.red_i);
    if (threadIdx.x == 0) V.blk[rank] = bsum;
    if (!team_sync(T)) return -1;
    if (rank == 0 && threadIdx.x == 0) {
      ctl->near_disp = 0.0;  // every block has read it
      ctl->near_rebuilds += 1;
    }
    block_prefix(V.blk, T.nb, rank, prefix, total, sm);
    int run = prefix;
    for (int base = lo; base < hi; base += blockDim.x) {
      const int i = base + threadIdx.x;
      const int c = i < hi ? V.hit_cnt[i] : 0;
      int tot;
      const int ex = block_excl_scan(c, sm.scan_w, tot);
      if (i < hi) {
        if (c) near_write_rod(i, run + ex, V.nbr_cnt, V.nbr, V.maxnb, V.words, V.mask, V.near);
        const Seg s = V.seg[i];
        V.ref2[i] = s.cx; V.ref2[n + i] = s.cy; V.ref2[2 * n + i] = s.cz;
        V.ref2[3 * n + i] = s.ux; V.ref2[4 * n + i] = s.uy; V.ref2[5 * n + i] = s.uz;
      }
      run += tot;
    }
    if (rank == 0 && threadIdx.x == 0) {
      ctl->near_n = total;
      ctl->near_valid = 1;
    }
    if (!team_sync(T)) return -1;
  }
  // exact narrow phase over the near list: each block a 64-aligned range
  const int P = *(volatile int*)&ctl->near_n;
  const int segp = (((P + T.nb - 1) / T.nb) + 63) & ~63;
  const int plo = rank * segp < P ? rank * segp : P;
  const int phi = plo + segp < P ? plo + segp : P;
  unsigned long long* bits = V.mask;  // one bit per near pair
  const double* im = V.st.inv_mass;
  // the block's words (none for an empty range: plo is then P, whose word
  // may belong to the block before)
  const int wlo = plo >> 6, whi = plo < phi ? (phi + 63) >> 6 : wlo;
  // The velocity-level detection follows the previous step's position-level
  // one over the same near list; only the position projection and the
  // periodic wrap moved rods in between.  A pair of two unmoved rods has
  // bit-identical segments, so its hit bit carries over; the other pairs
  // are tested again.
  const bool carry = !position_level && !rebuild_near && V.moved && *(volatile int*)&ctl->det_valid;
  if (carry) {
    constexpr int U = 4;  // pairs per thread and round: independent loads in flight
    for (int p0 = plo + threadIdx.x; p0 < phi; p0 += U * blockDim.x) {
      int2 pr[U];
      bool mv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int p = p0 + u * blockDim.x;
        pr[u] = p < phi ? V.near[p] : make_int2(0, 0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) mv[u] = p0 + u * (int)blockDim.x < phi && (V.moved[pr[u].x] | V.moved[pr[u].y]);
#pragma unroll 1
      for (int u = 0; u < U; ++u) {
        if (!mv[u]) continue;
        const int p = p0 + u * blockDim.x;
        const bool was = (__ldcg(&bits[p >> 6]) >> (p & 63)) & 1ull;
        bool hit = false;
        if (im[pr[u].x] > 0.0 || im[pr[u].y] > 0.0) {
          const Seg A = V.seg[pr[u].x], B = V.seg[pr[u].y];
          if (!seg_far(A, B, prefilter_offset(A, B, V.box, invL, mode), A.r + B.r + delta)) {
            const Narrow nr = narrow_pair(A, B, V.box);
            hit = contact_test(nr.d2, A.r + B.r, delta);
          }
        }
        if (hit != was) atomicXor(&bits[p >> 6], 1ull << (p & 63));
      }
    }
  } else {
    for (int w = wlo + threadIdx.x; w < whi; w += blockDim.x) bits[w] = 0ull;
    __syncthreads();
    for (int p = plo + threadIdx.x; p < phi; p += blockDim.x) {
      const int2 pr = V.near[p];
      if (!(im[pr.x] > 0.0) && !(im[pr.y] > 0.0)) continue;
      const Seg A = V.seg[pr.x], B = V.seg[pr.y];
      if (seg_far(A, B, prefilter_offset(A, B, V.box, invL, mode), A.r + B.r + delta)) continue;
      const Narrow nr = narrow_pair(A, B, V.box);
      if (contact_test(nr.d2, A.r + B.r, delta)) atomicOr(&bits[p >> 6], 1ull << (p & 63));
    }
  }
  __syncthreads();
  int mine = 0;
  for (int w = wlo + threadIdx.x; w < whi; w += blockDim.x) mine += __popcll(__ldcg(&bits[w]));
  const int bsum = block_reduce_sum_i(mine, sm.red_i);
  if (threadIdx.x == 0) V.blk[rank] = bsum;
  if (!team_sync(T)) return -1;
  // every block has read maxdisp.  After a position-level pass it stays:
  // the next free flight refreshes only the rods moved since, and the
  // unmoved rods' bounds are the ones it holds (unless the lists were just
  // rebuilt, when every bound restarts at zero).
  if (rank == 0 && threadIdx.x == 0 && (!position_level || lists_rebuilt)) ctl->maxdisp = 0.0;
  block_prefix(V.blk, T.nb, rank, prefix, total, sm);
  if (total > V.ccap) {
    if (rank == 0 && threadIdx.x == 0) atomicOr(&ctl->err, ERR_CONTACT_CAP);
    return -1;
  }
  // contacts in pair order: one word (64 pairs) per thread, scanned by
  // population count, places each hit's pair in its slot; then one thread
  // per slot runs the exact narrow phase (a word may hold several hits,
  // which one thread would otherwise evaluate one after the other)
  int run = prefix;
  for (int wb = wlo; wb < whi; wb += blockDim.x) {
    const int w = wb + threadIdx.x;
    const unsigned long long m = w < whi ? __ldcg(&bits[w]) : 0ull;
    int tot;
    int slot = run + block_excl_scan(__popcll(m), sm.scan_w, tot);
    for (unsigned long long r = m; r; r &= r - 1) {
      const int2 pr = V.near[(w << 6) + __ffsll((long long)r) - 1];
      V.con.a[slot] = pr.x;
      V.con.b[slot] = pr.y;
      ++slot;
    }
    run += tot;
  }
  __syncthreads();
  for (int c = prefix + (int)threadIdx.x; c < run; c += blockDim.x) {
    const int a = V.con.a[c], b = V.con.b[c];
    const Seg A = V.seg[a], B = V.seg[b];
    const Narrow nr = narrow_pair(A, B, V.box);
    write_contact(V.con, c, a, b, A.r + B.r, nr);
  }
  if (rank == 0 && threadIdx.x == 0) {
    ctl->contacts = total;
    ctl->det_valid = position_level ? 1 : 0;
  }
  if (!team_sync(T)) return -1;
  return total;
}

__device__ __noinline__ int detect_phase(const Team& T, const NscView& V, double delta, SmemNsc& sm,
                                         bool position_level) {
  Ctl* ctl = V.ctl;
  const int n = V.st.n;
  const int rank = T.rank();
  const bool need = *(volatile int*)&ctl->rebuild ||
                    (!V.all_pairs && *(volatile double*)&ctl->maxdisp >= 0.5 * V.skin * (1.0 - 1e-9));
  if (need && !rebuild_phase(T, V, sm)) return -1;
  if (V.near) return detect_near(T, V, delta, sm, need, position_level);
  const int seg = (n + T.nb - 1) / T.nb;
  const int lo = rank * seg < n ? rank * seg : n;
  const int hi = lo + seg < n ? lo + seg : n;
  constexpr int G = RG_NARROW_LANES;  // lanes per rod
  int mine = 0;
  for (int base = lo; base < hi; base += blockDim.x / G) {
    int i = base + threadIdx.x / G;
    bool valid = i < hi;
    int c = narrow_count_lanes<G>(i, valid, V.seg, V.st.inv_mass, V.box, delta, V.nbr_cnt, V.nbr, V.maxnb,
                                  V.words, V.mask, V.all_pairs ? 2 : 1);
    if (valid && (threadIdx.x & (G - 1)) == 0) {
      V.hit_cnt[i] = c;
      mine += c;
    }
  }
  int run = block_reduce_sum_i(mine, sm.red_i);
  if (threadIdx.x == 0) V.blk[rank] = run;
  if (!team_sync(T)) return -1;
  // every block has read maxdisp (kept after a position-level pass, as above)
  if (rank == 0 && threadIdx.x == 0 && (!position_level || need)) ctl->maxdisp = 0.0;
  int prefix, total;
  block_prefix(V.blk, T.nb, rank, prefix, total, sm);
  if (total > V.ccap) {
    if (rank == 0 && threadIdx.x == 0) atomicOr(&ctl->err, ERR_CONTACT_CAP);
    return -1;
  }
  run = prefix;
  for (int base = lo; base < hi; base += blockDim.x) {
    int i = base + threadIdx.x;
    int c = i < hi ? V.hit_cnt[i] : 0;
    int tot;
    int ex = block_excl_scan(c, sm.scan_w, tot);
    if (c) narrow_write_rod(i, run + ex, V.seg, V.box, V.nbr_cnt, V.nbr, V.maxnb, V.words, V.mask, V.con);
    run += tot;
  }
  if (rank == 0 && threadIdx.x == 0) ctl->contacts = total;
  if (!team_sync(T)) return -1;
  return total;
}

// ---------------------------------------------------------------------------
// Colouring: Jones-Plassmann first fit with per-body priority maxima.
// ---------------------------------------------------------------------------
__device__ __noinline__ bool color_phase(const Team& T, const NscView& V, int C, SmemNsc& sm) {
  Ctl* ctl = V.ctl;
  const int n = V.st.n;
  const int tid = T.tid(), TS = T.size(), rank = T.rank();
  const double* im = V.st.inv_mass;
  for (int c = tid; c < C; c += TS) {
    int x[2] = {V.con.a[c], V.con.b[c]};
    for (int k = 0; k < 2; ++k) {
      if (!(im[x[k]] > 0.0)) continue;
      V.pmax[x[k]] = 0;
      V.pmax[n + x[k]] = 0;
      V.cmask[x[k]] = 0;
      V.owner[x[k]] = 0x7fffffff;
    }
    V.color[c] = -1;
  }
  if (rank == 0) {
    for (int k = threadIdx.x; k <= kMaxColors; k += blockDim.x) {
      V.color_cnt[k] = 0;
      V.cursor[k] = 0;
    }
    for (int r = threadIdx.x; r < kMaxRounds; r += blockDim.x) V.remaining[r] = 0;
    if (threadIdx.x == 0) ctl->colors = 0;
  }
  if (!team_sync(T)) return false;
  int round = 0;
  for (; round < kMaxRounds; ++round) {
    unsigned long long* pm = V.pmax + (size_t)(round & 1) * n;
    unsigned long long* pn = V.pmax + (size_t)((round + 1) & 1) * n;
    for (int c = tid; c < C; c += TS) {
      if (V.color[c] >= 0) continue;
      int x[2] = {V.con.a[c], V.con.b[c]};
      unsigned long long p = jp_priority((unsigned)c);
      for (int k = 0; k < 2; ++k) {
        if (!(im[x[k]] > 0.0)) continue;
        atomicMax(&pm[x[k]], p);
        if (round == 0) atomicMin(&V.owner[x[k]], c);
      }
    }
    if (!team_sync(T)) return false;
    int rem = 0, maxc = 0;
    for (int c = tid; c < C; c += TS) {
      if (V.color[c] >= 0) continue;
      int x[2] = {V.con.a[c], V.con.b[c]};
      unsigned long long p = jp_priority((unsigned)c);
      bool win = true;
      unsigned long long used = 0;
      for (int k = 0; k < 2; ++k) {
        if (!(im[x[k]] > 0.0)) continue;
        if (*(volatile unsigned long long*)&pm[x[k]] != p) win = false;
        used |= *(volatile unsigned long long*)&V.cmask[x[k]];
        pn[x[k]] = 0;
      }
      if (win) {
        int col = __ffsll((long long)~used) - 1;
        if (used == ~0ull) {
          atomicOr(&ctl->err, ERR_COLOR);
          col = kMaxColors - 1;
        }
        V.color[c] = col;
        for (int k = 0; k < 2; ++k)
          if (im[x[k]] > 0.0) atomicOr(&V.cmask[x[k]], 1ull << col);
        atomicAdd(&V.color_cnt[col], 1);
        maxc = col + 1 > maxc ? col + 1 : maxc;
      } else {
        ++rem;
      }
    }
    int br = block_reduce_sum_i(rem, sm.red_i);
    if (threadIdx.x == 0 && br) atomicAdd(&V.remaining[round], br);
    if (maxc) atomicMax(&ctl->colors, maxc);
    if (!team_sync(T)) return false;
    if (*(volatile int*)&V.remaining[round] == 0) break;
  }
  if (round >= kMaxRounds) {
    if (rank == 0 && threadIdx.x == 0) atomicOr(&ctl->err, ERR_COLOR);
    return false;
  }
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int k = 0; k <= kMaxColors; ++k) {
      sm.coff[k] = acc;
      if (k < kMaxColors) acc += *(volatile int*)&V.color_cnt[k];
    }
  }
  __syncthreads();
  if (rank == 0)
    for (int k = threadIdx.x; k <= kMaxColors; k += blockDim.x) V.color_off[k] = sm.coff[k];
  for (int c = tid; c < C; c += TS) {
    int k = V.color[c];
    V.order[sm.coff[k] + atomicAdd(&V.cursor[k], 1)] = c;
  }
  return team_sync(T);
}

// ---------------------------------------------------------------------------
// PSOR sweeps.
// ---------------------------------------------------------------------------
__device__ inline int active_blocks(const int* coff, int ncol, int bs, int nb) {
  int m = 0;
  for (int k = 0; k < ncol; ++k) {
    int c = coff[k + 1] - coff[k];
    m = c > m ? c : m;
  }
  int need = (m + bs - 1) / bs;
  if (need < 1) need = 1;
  return need < nb ? need : nb;
}

__device__ __noinline__ bool psor_phase(const Team& T, const NscView& V, int C, SmemNsc& sm) {
  Ctl* ctl = V.ctl;
  const int K = *(volatile int*)&ctl->colors;
  const int rank = T.rank();
  const rg_config& cfg = V.cfg;
  if (C > 0) {
    const int na = active_blocks(V.color_off, K, blockDim.x, T.nb);
    if (rank < na) {
      const int tid = rank * blockDim.x + threadIdx.x, stride = na * blockDim.x;
      RowIO R{V.row, V.lam, V.ccap};
      Vel Vv{V.st.v, V.st.w};
      const double omega = cfg.nsc_omega, cfm = cfg.nsc_cfm, mu = cfg.nsc_mu;
      const int iters = cfg.nsc_velocity_iters;
      const int* coff = V.color_off;
      for (int i = tid; i < iters; i += stride) ctl->res_sweep[i] = 0.0;
      if (cfg.nsc_warm_start != RG_WARM_NONE) {
        for (int k = 0; k < K; ++k) {
          for (int p = coff[k] + tid; p < coff[k + 1]; p += stride) {
            int c = V.order[p];
            warm_apply(R, Vv, p, V.con.a[c], V.con.b[c]);
          }
          if (!team_sync_sub(T, na)) return false;
        }
      } else if (!team_sync_sub(T, na)) {
        return false;
      }
      double res = 0.0;
      int sweeps = 0;
      for (int it = 0; it < iters; ++it) {
        double loc = 0.0;
        for (int k = 0; k < K; ++k) {
          for (int p = coff[k] + tid; p < coff[k + 1]; p += stride) {
            int c = V.order[p];
            loc = fmax(loc, psor_row(R, Vv, p, V.con.a[c], V.con.b[c], omega, cfm, mu));
          }
          if (k + 1 < K && !team_sync_sub(T, na)) return false;
        }
        double bm = block_reduce_max(loc, sm.red_d);
        if (threadIdx.x == 0) atomic_max_nonneg(&ctl->res_sweep[it], bm);
        if (!team_sync_sub(T, na)) return false;
        res = *(volatile double*)&ctl->res_sweep[it];
        sweeps = it + 1;
        if (res < cfg.nsc_tol) break;
      }
      if (tid == 0) {
        ctl->residual = res;
        ctl->sweeps_last = sweeps;
        ctl->sweeps_sum += sweeps;
        ctl->row_sweeps += (long long)C * sweeps;
        ctl->contact_steps += C;
        if (res >= cfg.nsc_tol) ctl->not_conv += 1;
        if (res > ctl->max_residual) ctl->max_residual = res;
      }
    }
  } else if (rank == 0 && threadIdx.x == 0) {
    ctl->residual = 0.0;
    ctl->sweeps_last = 0;
  }
  return team_sync(T);
}

// ---------------------------------------------------------------------------
// Position projection (rows from the pass-0 detection, then narrow phase on
// the cached pairs in later passes).  Runs on the na active blocks.
// ---------------------------------------------------------------------------
__device__ __noinline__ bool project_rows(const NscView& V, int C, int K, int na, int rank, const Team& T, SmemNsc& sm) {
  Ctl* ctl = V.ctl;
  const rg_config& cfg = V.cfg;
  const State& st = V.st;
  const int n = st.n;
  const int tid = rank * blockDim.x + threadIdx.x, stride = na * blockDim.x;
  const double omega = cfg.nsc_omega, cfm = cfg.nsc_cfm, slop = cfg.nsc_slop;
  const int* coff = V.color_off;
  const size_t ccap = (size_t)V.ccap;
  double* PR = V.prow;
  Vec3A DX{V.dx, V.dx + n, V.dx + 2 * n}, DT{V.dx + 3 * n, V.dx + 4 * n, V.dx + 5 * n};
  double* slots = ctl->res_sweep;
  const int piters = cfg.nsc_position_psor_iters;
  for (int outer = 0; outer < cfg.nsc_position_iters; ++outer) {
    for (int i = tid; i < piters + 1; i += stride) slots[i] = 0.0;
    if (!team_sync_sub(T, na)) return false;
    int cnt = 0;
    for (int p = tid; p < C; p += stride) {
      const int c = V.order[p];
      const int a = V.con.a[c], b = V.con.b[c];
      d3 xa = st.x.ld(a), xb = st.x.ld(b);
      d3 nv, ra, rb;
      double phi;
      if (outer == 0) {
        phi = V.con.comp(12)[c] - V.con.comp(13)[c];
        nv = mk3(V.con.comp(6)[c], V.con.comp(7)[c], V.con.comp(8)[c]);
        d3 pa{V.con.comp(0)[c], V.con.comp(1)[c], V.con.comp(2)[c]};
        d3 pb{V.con.comp(3)[c], V.con.comp(4)[c], V.con.comp(5)[c]};
        d3 sh{V.con.comp(9)[c], V.con.comp(10)[c], V.con.comp(11)[c]};
        ra = pa - xa;
        rb = pb - (xb + sh);
      } else {
        Seg A = make_seg(st, a), B = make_seg(st, b);
        Narrow nr = narrow_pair(A, B, V.box);
        d3 diff = nr.pb - nr.pa;
        double dist = len(diff);
        phi = dist - V.con.comp(13)[c];
        nv = dist > 1e-10 ? diff / dist : mk3(1, 0, 0);
        ra = nr.pa - xa;
        rb = nr.pb - (xb + nr.sh);
      }
      int act = phi < -slop ? 1 : 0;
      V.pactive[p] = act;
      if (act) {
        ++cnt;
        PR[P_N * ccap + p] = nv.x; PR[(P_N + 1) * ccap + p] = nv.y; PR[(P_N + 2) * ccap + p] = nv.z;
        PR[P_RA * ccap + p] = ra.x; PR[(P_RA + 1) * ccap + p] = ra.y; PR[(P_RA + 2) * ccap + p] = ra.z;
        PR[P_RB * ccap + p] = rb.x; PR[(P_RB + 1) * ccap + p] = rb.y; PR[(P_RB + 2) * ccap + p] = rb.z;
        PR[P_PHI * ccap + p] = phi + slop;
        PR[P_G * ccap + p] = diag_of(st, a, b, ra, rb, nv, cfm);
        PR[P_L * ccap + p] = 0.0;
      }
      DX.st(a, mk3(0, 0, 0)); DT.st(a, mk3(0, 0, 0));
      DX.st(b, mk3(0, 0, 0)); DT.st(b, mk3(0, 0, 0));
    }
    int bc = block_reduce_sum_i(cnt, sm.red_i);
    if (threadIdx.x == 0 && bc)
      atomicAdd(reinterpret_cast<unsigned long long*>(&slots[piters]), (unsigned long long)bc);
    if (!team_sync_sub(T, na)) return false;
    if (*(volatile unsigned long long*)&slots[piters] == 0ull) return true;  // nothing penetrates
    for (int it = 0; it < piters; ++it) {
      double loc = 0.0;
      for (int k = 0; k < K; ++k) {
        for (int p = coff[k] + tid; p < coff[k + 1]; p += stride) {
          if (!V.pactive[p]) continue;
          const int c = V.order[p];
          const int a = V.con.a[c], b = V.con.b[c];
          d3 nv{PR[P_N * ccap + p], PR[(P_N + 1) * ccap + p], PR[(P_N + 2) * ccap + p]};
          d3 ra{PR[P_RA * ccap + p], PR[(P_RA + 1) * ccap + p], PR[(P_RA + 2) * ccap + p]};
          d3 rb{PR[P_RB * ccap + p], PR[(P_RB + 1) * ccap + p], PR[(P_RB + 2) * ccap + p]};
          double l = PR[P_L * ccap + p];
          double corr = dot(nv, ((DX.ld(b) + cross(DT.ld(b), rb)) - DX.ld(a)) - cross(DT.ld(a), ra));
          double r = corr + PR[P_PHI * ccap + p] + cfm * l;
          double d = -(omega / PR[P_G * ccap + p]) * r;
          double nl = smax(0.0, l + d);
          double dl = nl - l;
          if (dl != 0.0) {
            PR[P_L * ccap + p] = nl;
            d3 rAxn = cross(ra, nv);
            DX.st(a, DX.ld(a) - nv * (dl * st.inv_mass[a]));
            DT.st(a, DT.ld(a) - iinv_apply(st, a, rAxn) * dl);
            d3 rBxn = cross(rb, nv);
            DX.st(b, DX.ld(b) + nv * (dl * st.inv_mass[b]));
            DT.st(b, DT.ld(b) + iinv_apply(st, b, rBxn) * dl);
          }
          loc = fmax(loc, fabs(dl));
        }
        if (k + 1 < K && !team_sync_sub(T, na)) return false;
      }
      double bm = block_reduce_max(loc, sm.red_d);
      if (threadIdx.x == 0) atomic_max_nonneg(&slots[it], bm);
      if (!team_sync_sub(T, na)) return false;
      if (*(volatile double*)&slots[it] < 1e-8) break;
    }
    // apply: each body once, by the lowest-index contact touching it
    for (int p = tid; p < C; p += stride) {
      const int c = V.order[p];
      for (int side = 0; side < 2; ++side) {
        int bd = side ? V.con.b[c] : V.con.a[c];
        if (st.inv_mass[bd] <= 0.0 || V.owner[bd] != c) continue;
        if (V.moved) V.moved[bd] = 1;
        st.x.st(bd, st.x.ld(bd) + DX.ld(bd));
        d3 th = DT.ld(bd);
        double ang = len(th);
        if (ang > 1e-8) {
          d3 ax = th / ang;
          st.q.st(bd, qnormalize(qmul(angle_axis(ang, ax), st.q.ld(bd))));
        }
      }
    }
    if (!team_sync_sub(T, na)) return false;
  }
  return true;
}

__device__ __noinline__ bool project_phase(const Team& T, const NscView& V, int C, SmemNsc& sm) {
  const int rank = T.rank();
  const int K = *(volatile int*)&V.ctl->colors;
  if (C > 0 && V.cfg.nsc_position_stabilization) {
    const int na = active_blocks(V.color_off, K, blockDim.x, T.nb);
    if (rank < na && !project_rows(V, C, K, na, rank, T, sm)) return false;
  }
  return team_sync(T);
}


// ---------------------------------------------------------------------------
// Small contact sets (C <= kSmallC): one block solves everything in shared
// memory.  Contact c is owned by thread c; its bodies get compact local slots
// (a per-body slot map in global memory, reset afterwards), so colouring
// scratch, body velocities, manifold rows and impulses all live on chip and
// phases synchronise with __syncthreads.  Same arithmetic, same order as the
// team path and the oracle.
// ---------------------------------------------------------------------------
#ifndef RG_SMALL_C
#define RG_SMALL_C kTile
#endif
constexpr int kSmallC = RG_SMALL_C;      // one contact per thread
constexpr int kSmallB = 2 * kSmallC;     // local body slots

struct SmallSmem {
  double row[kRowComps * kSmallC];   // manifold rows (or projection rows)
  double lam[3 * kSmallC];
  double vel[6 * kSmallB];           // v, w (or dx, dθ) per local slot
  unsigned long long pmax[2 * kSmallB];
  unsigned long long cmask[kSmallB];
  int body[kSmallB];                 // body of a slot (-1: unused)
  int dyn[kSmallB];                  // 1: dynamic body
  int la[kSmallC], lb[kSmallC];      // local slots of contact c
  int color[kSmallC], order[kSmallC];
  int cnt[kMaxColors + 1], coff[kMaxColors + 1], cur[kMaxColors + 1];
  int nloc, rem, ncol, act;
  double red[32];
  float feat[kMlpIn * kSmallC];      // learned warm start features [8][kSmallC]
  float pred[kMlpOut * kSmallC];     // predicted impulse changes [3][kSmallC]
  int mtile[kSmallC / 16];           // 16-contact tiles that need the network
  unsigned char cached[kSmallC];     // 1: the slot's contact is in the warm cache
  // one hidden layer of the network (the rest is staged in pmax/cmask)
#ifndef RG_NO_MLP_STAGE
  alignas(16) __nv_bfloat16 wh[kStageWh];
#else
  alignas(16) __nv_bfloat16 wh[8];  // build without in-step inference staging
#endif
};
#ifndef RG_NO_MLP_STAGE
static_assert(sizeof(unsigned long long) * 3 * kSmallB >= kStageSmallBytes, "MLP staging space");
#endif
static_assert(sizeof(SmallSmem) >= kBuildQOff + 2 * sizeof(unsigned) * kBuildQ,
              "list-build tiles and queues share the small-solve memory");

__device__ inline double small_block_max(double v, SmallSmem& S) {
  v = warp_max(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = v;
  __syncthreads();
  // every warp combines the per-warp maxima itself (one load per lane)
  const int lane = threadIdx.x & 31;
  return warp_max(lane < (int)(blockDim.x >> 5) ? S.red[lane] : 0.0);  // every thread
}

// True when contact c has an entry in the warm cache of the previous step
// (W entries): the learned start by default serves only the others.
__device__ inline bool warm_cached(const NscView& V, int c, int W) {
  if (W <= 0) return false;
  const unsigned long long k = ((unsigned long long)(unsigned)V.con.a[c] << 32) | (unsigned)V.con.b[c];
  const int q = lower_bound_key(V.wkey, W, k);
  return q < W && V.wkey[q] == k;
}

// Local slots for the bodies of contacts 0..C-1 (C <= blockDim).
__device__ __noinline__ void small_map(const NscView& V, int C, SmallSmem& S) {
  const int t = threadIdx.x;
  if (t == 0) S.nloc = 0;
  __syncthreads();
  if (t < C) {
    int x[2] = {V.con.a[t], V.con.b[t]};
    int sl[2];
    for (int k = 0; k < 2; ++k) {
      int idx = atomicAdd(&S.nloc, 1);
      int old = atomicCAS(&V.slot_of[x[k]], -1, idx);
      S.body[idx] = old == -1 ? x[k] : -1;
      sl[k] = old == -1 ? idx : old;
    }
    S.la[t] = sl[0];
    S.lb[t] = sl[1];
  }
  __syncthreads();
  for (int s = t; s < S.nloc; s += blockDim.x) {
    int x = S.body[s];
    S.dyn[s] = (x >= 0 && V.st.inv_mass[x] > 0.0) ? 1 : 0;
  }
  __syncthreads();
}
__device__ void small_unmap(const NscView& V, SmallSmem& S) {
  for (int s = threadIdx.x; s < S.nloc; s += blockDim.x)
    if (S.body[s] >= 0) V.slot_of[S.body[s]] = -1;
}

// Jones-Plassmann first fit on local slots; fills S.color / S.order /
// S.coff and the global colour arrays.  Returns the colour count or -1.
__device__ __noinline__ int small_color(const NscView& V, int C, SmallSmem& S) {
  const int t = threadIdx.x;
  for (int s = t; s < S.nloc; s += blockDim.x) {
    S.pmax[s] = 0; S.pmax[kSmallB + s] = 0; S.cmask[s] = 0;
  }
  for (int k = t; k <= kMaxColors; k += blockDim.x) { S.cnt[k] = 0; S.cur[k] = 0; }
  if (t < C) S.color[t] = -1;
  if (t == 0) S.ncol = 0;
  __syncthreads();
  int round = 0;
  for (; round < kMaxRounds; ++round) {
    unsigned long long* pm = S.pmax + (round & 1) * kSmallB;
    unsigned long long* pn = S.pmax + ((round + 1) & 1) * kSmallB;
    if (t == 0) S.rem = 0;
    if (t < C && S.color[t] < 0) {
      unsigned long long p = jp_priority((unsigned)t);
      if (S.dyn[S.la[t]]) atomicMax(&pm[S.la[t]], p);
      if (S.dyn[S.lb[t]]) atomicMax(&pm[S.lb[t]], p);
    }
    __syncthreads();
    if (t < C && S.color[t] < 0) {
      unsigned long long p = jp_priority((unsigned)t);
      int sl[2] = {S.la[t], S.lb[t]};
      bool win = true;
      unsigned long long used = 0;
      for (int k = 0; k < 2; ++k) {
        if (!S.dyn[sl[k]]) continue;
        if (pm[sl[k]] != p) win = false;
        used |= S.cmask[sl[k]];
        pn[sl[k]] = 0;
      }
      if (win) {
        int col = __ffsll((long long)~used) - 1;
        if (used == ~0ull) {
          atomicOr(&V.ctl->err, ERR_COLOR);
          col = kMaxColors - 1;
        }
        S.color[t] = col;
        for (int k = 0; k < 2; ++k)
          if (S.dyn[sl[k]]) atomicOr(&S.cmask[sl[k]], 1ull << col);
        atomicAdd(&S.cnt[col], 1);
        atomicMax(&S.ncol, col + 1);
      } else {
        atomicAdd(&S.rem, 1);
      }
    }
    __syncthreads();
    int rem = S.rem;
    __syncthreads();
    if (rem == 0) break;
  }
  if (round >= kMaxRounds) {
    if (t == 0) atomicOr(&V.ctl->err, ERR_COLOR);
    return -1;
  }
  if (t == 0) {
    int acc = 0;
    for (int k = 0; k <= kMaxColors; ++k) {
      S.coff[k] = acc;
      if (k < kMaxColors) acc += S.cnt[k];
    }
    V.ctl->colors = S.ncol;
  }
  __syncthreads();
  if (t < C) {
    int k = S.color[t];
    int p = S.coff[k] + atomicAdd(&S.cur[k], 1);
    S.order[p] = t;
    V.order[p] = t;
    V.color[t] = k;
  }
  for (int k = t; k <= kMaxColors; k += blockDim.x) V.color_off[k] = S.coff[k];
  __syncthreads();
  return S.ncol;
}

// Colouring, manifold rows, PSOR and the warm cache for C <= kSmallC.
__device__ __noinline__ bool small_solve(const NscView& V, int C, int Cp, SmallSmem& S, PhaseClock& pc) {
  Ctl* ctl = V.ctl;
  const rg_config& cfg = V.cfg;
  const int t = threadIdx.x;
  // the learned start's gate is known now: its first hidden layer travels to
  // shared memory while the colouring and the rows are built
  const bool mlp_gate = V.use_mlp && (*(volatile int*)V.wn == 0 ||
                                      *(volatile int*)&ctl->sweeps_last > V.mlp_min_sweeps);
  if (mlp_gate) stage_bf16(S.wh, kWhLd, V.mlp.w2, kMlpH, kMlpH);
  small_map(V, C, S);
  pc.mark(10);
  int K = small_color(V, C, S);
  if (K < 0) {
    if (mlp_gate) stage_wait();
    return false;
  }
  pc.mark(2);
  // body velocities on chip
  for (int s = t; s < S.nloc; s += blockDim.x) {
    int x = S.body[s];
    if (x < 0) continue;
    d3 v = V.st.v.ld(x), w = V.st.w.ld(x);
    S.vel[s] = v.x; S.vel[kSmallB + s] = v.y; S.vel[2 * kSmallB + s] = v.z;
    S.vel[3 * kSmallB + s] = w.x; S.vel[4 * kSmallB + s] = w.y; S.vel[5 * kSmallB + s] = w.z;
  }
  RowIO R{S.row, S.lam, kSmallC};
  const int W = *(volatile int*)V.wn;
  int* deg = reinterpret_cast<int*>(S.pmax);  // free after colouring
  if (V.feat_on) {
    for (int s = t; s < S.nloc; s += blockDim.x) deg[s] = 0;
    __syncthreads();
  }
  int coll = 0;
  if (t < C) {
    const int c = S.order[t];
    const int br = build_row(V.st, V.con, cfg, c, t, R, V.wkey, V.wlam, W, V.wcap, V.feat_on ? S.feat : nullptr,
                             kSmallC);
    coll = br & 1;
    S.cached[t] = (unsigned char)(br >> 1);
    if (V.feat_on && c < Cp) {  // wall rows (after the pairs) have no graph degree
      if (S.dyn[S.la[c]]) atomicAdd(&deg[S.la[c]], 1);
      if (S.dyn[S.lb[c]]) atomicAdd(&deg[S.lb[c]], 1);
    }
  }
  int bcoll = __syncthreads_count(coll);
  if (t == 0 && bcoll) atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->collisions), (unsigned long long)bcoll);
  if (V.feat_on) {
    if (t < C) {
      const int c = S.order[t], sa = S.la[c], sb = S.lb[c];
      S.feat[7 * kSmallC + t] = (float)((S.dyn[sa] ? deg[sa] - 1 : 0) + (S.dyn[sb] ? deg[sb] - 1 : 0));
    }
    __syncthreads();
    if (mlp_gate) {
      // the contacts the learned start is for (every contact, or those new
      // since the last step); the network runs only on tiles that hold one
      const bool want = t < C && S.order[t] < Cp && (V.mlp_all || !S.cached[t]);  // never a wall row
      if (t < kSmallC / 16) S.mtile[t] = 0;
      __syncthreads();
      if (want) S.mtile[t >> 4] = 1;
      if (__syncthreads_or(want)) {
        // one warp per 16 contacts on the tensor cores, then the cone.  The
        // weights come from shared memory: W1, W4 and the small parameters
        // in pmax/cmask (free after colouring and degrees), the hidden
        // layers one after the other in wh.
        const MlpStage ms = mlp_stage_at(S.pmax);
        stage_small(ms, V.mlp);  // W2 is already on its way (start of the solve)
        stage_wait();
        __syncthreads();
        const int row0 = (t >> 5) * 16, lane = t & 31;
        const bool mine = row0 < C && S.mtile[t >> 5];
        const MlpSmall q = ms.small();
        unsigned a[8][4];
        if (mine) {
          mlp_layer1(ms.w1, kW1Ld, q, S.feat, kSmallC, row0, C, lane, a);
          hidden_layer(a, S.wh, kWhLd, q.b2, lane);
        }
        __syncthreads();
        stage_bf16(S.wh, kWhLd, V.mlp.w3, kMlpH, kMlpH);
        stage_wait();
        __syncthreads();
        if (mine) {
          hidden_layer(a, S.wh, kWhLd, q.b3, lane);
          mlp_layer4(a, ms.w4, kWhLd, q, S.pred, kSmallC, row0, C, lane);
        }
        __syncthreads();
        if (want) mlp_apply(R, S.pred, kSmallC, t, cfg.nsc_mu);
        __syncthreads();
      }
    }
  }
  if (mlp_gate) stage_wait();  // no copy outlives the solve
  pc.mark(3);
  Vel Vv{Vec3A{S.vel, S.vel + kSmallB, S.vel + 2 * kSmallB},
         Vec3A{S.vel + 3 * kSmallB, S.vel + 4 * kSmallB, S.vel + 5 * kSmallB}};
  const double omega = cfg.nsc_omega, cfm = cfg.nsc_cfm, mu = cfg.nsc_mu;
  const int p = t;
  const int c = p < C ? S.order[p] : 0;
  int my_color = -1;
  if (p < C)
    for (int k = 0; k < K; ++k)
      if (p >= S.coff[k] && p < S.coff[k + 1]) my_color = k;
  if (cfg.nsc_warm_start != RG_WARM_NONE) {
    for (int k = 0; k < K; ++k) {
      if (my_color == k) warm_apply(R, Vv, p, S.la[c], S.lb[c]);
      __syncthreads();
    }
  }
  double res = 0.0;
  int sweeps = 0;
  for (int it = 0; C > 0 && it < cfg.nsc_velocity_iters; ++it) {
    double loc = 0.0;
    for (int k = 0; k < K; ++k) {
      if (my_color == k) loc = psor_row(R, Vv, p, S.la[c], S.lb[c], omega, cfm, mu);
      __syncthreads();
    }
    res = small_block_max(loc, S);
    sweeps = it + 1;
    if (res < cfg.nsc_tol) break;
  }
  __syncthreads();
  pc.mark(4);
  // velocities back; warm cache and impulse sums (contact order)
  for (int s = t; s < S.nloc; s += blockDim.x) {
    int x = S.body[s];
    if (x < 0) continue;
    V.st.v.st(x, mk3(S.vel[s], S.vel[kSmallB + s], S.vel[2 * kSmallB + s]));
    V.st.w.st(x, mk3(S.vel[3 * kSmallB + s], S.vel[4 * kSmallB + s], S.vel[5 * kSmallB + s]));
  }
  small_unmap(V, S);
  if (V.rec_cap > 0 && C > 0) {
    // records (features, converged impulses) in slot order
    const int base = *(volatile int*)&ctl->rec_n;
    if (p < C && base + p < V.rec_cap) {
      const size_t r = (size_t)(base + p);
      for (int k = 0; k < kMlpIn; ++k) V.rec_x[r * kMlpIn + k] = S.feat[k * kSmallC + p];
      for (int k = 0; k < kMlpOut; ++k) V.rec_y[r * kMlpOut + k] = (float)S.lam[k * kSmallC + p];
    }
    __syncthreads();
    if (t == 0) ctl->rec_n = base + C;
  }
  double jn = 0, jt = 0;
  if (p < C) {
    double l0 = S.lam[p], l1 = S.lam[kSmallC + p], l2 = S.lam[2 * kSmallC + p];
    if (c < Cp) {  // wall rows start cold every step: they stay out of the cache
      V.wkey[c] = ((unsigned long long)(unsigned)V.con.a[c] << 32) | (unsigned)V.con.b[c];
      V.wlam[c] = l0;
      V.wlam[V.wcap + c] = l1;
      V.wlam[2 * V.wcap + c] = l2;
      reinterpret_cast<int*>(V.wlam + 3 * (size_t)V.wcap)[c] = S.color[c];
      if (V.xrow) export_row(V.xrow, V.wcap, c, R, p);
    }
    jn = fabs(l0);  // profile-CSV sums of main.cpp:3339-3343
    jt = fabs(l1) + fabs(l2);
  }
  jn = warp_sum(jn);
  jt = warp_sum(jt);
  if ((t & 31) == 0 && (jn != 0.0 || jt != 0.0)) {
    atomicAdd(&ctl->jn_sum, jn);
    atomicAdd(&ctl->jt_sum, jt);
  }
  if (t == 0) {
    *V.wn = Cp;
    ctl->vel_contacts = C;
    ctl->residual = res;
    ctl->sweeps_last = sweeps;
    if (C > 0) {
      ctl->sweeps_sum += sweeps;
      ctl->row_sweeps += (long long)C * sweeps;
      ctl->contact_steps += C;
      if (res >= cfg.nsc_tol) ctl->not_conv += 1;
      if (res > ctl->max_residual) ctl->max_residual = res;
    }
  }
  return true;
}

// Position projection for C <= kSmallC (nsc_contact.cpp:698-879).
__device__ __noinline__ bool small_project(const NscView& V, int C, SmallSmem& S) {
  const rg_config& cfg = V.cfg;
  const State& st = V.st;
  const int t = threadIdx.x;
  small_map(V, C, S);
  int K = small_color(V, C, S);
  if (K < 0) return false;
  const double omega = cfg.nsc_omega, cfm = cfg.nsc_cfm, slop = cfg.nsc_slop;
  double* PR = S.row;  // kPosComps x kSmallC
  double* DX = S.vel;  // 6 x kSmallB: dx, dθ per local slot
  const int p = t;
  const int c = p < C ? S.order[p] : 0;
  int my_color = -1;
  if (p < C)
    for (int k = 0; k < K; ++k)
      if (p >= S.coff[k] && p < S.coff[k + 1]) my_color = k;
  const int sa = p < C ? S.la[c] : 0, sb = p < C ? S.lb[c] : 0;
  const int a = p < C ? V.con.a[c] : 0, b = p < C ? V.con.b[c] : 0;
  for (int outer = 0; outer < cfg.nsc_position_iters; ++outer) {
    int act = 0;
    if (p < C) {
      d3 xa = st.x.ld(a), xb = st.x.ld(b);
      d3 nv, ra, rb;
      double phi;
      if (outer == 0) {
        phi = V.con.comp(12)[c] - V.con.comp(13)[c];
        nv = mk3(V.con.comp(6)[c], V.con.comp(7)[c], V.con.comp(8)[c]);
        d3 pa{V.con.comp(0)[c], V.con.comp(1)[c], V.con.comp(2)[c]};
        d3 pb{V.con.comp(3)[c], V.con.comp(4)[c], V.con.comp(5)[c]};
        d3 sh{V.con.comp(9)[c], V.con.comp(10)[c], V.con.comp(11)[c]};
        ra = pa - xa;
        rb = pb - (xb + sh);
      } else {
        Seg A = make_seg(st, a), B = make_seg(st, b);
        Narrow nr = narrow_pair(A, B, V.box);
        d3 diff = nr.pb - nr.pa;
        double dist = len(diff);
        phi = dist - V.con.comp(13)[c];
        nv = dist > 1e-10 ? diff / dist : mk3(1, 0, 0);
        ra = nr.pa - xa;
        rb = nr.pb - (xb + nr.sh);
      }
      act = phi < -slop ? 1 : 0;
      if (act) {
        PR[P_N * kSmallC + p] = nv.x; PR[(P_N + 1) * kSmallC + p] = nv.y; PR[(P_N + 2) * kSmallC + p] = nv.z;
        PR[P_RA * kSmallC + p] = ra.x; PR[(P_RA + 1) * kSmallC + p] = ra.y; PR[(P_RA + 2) * kSmallC + p] = ra.z;
        PR[P_RB * kSmallC + p] = rb.x; PR[(P_RB + 1) * kSmallC + p] = rb.y; PR[(P_RB + 2) * kSmallC + p] = rb.z;
        PR[P_PHI * kSmallC + p] = phi + slop;
        PR[P_G * kSmallC + p] = diag_of(st, a, b, ra, rb, nv, cfm);
        PR[P_L * kSmallC + p] = 0.0;
      }
    }
    for (int s = t; s < S.nloc; s += blockDim.x)
      for (int k = 0; k < 6; ++k) DX[k * kSmallB + s] = 0.0;
    int nact = __syncthreads_count(act);
    if (nact == 0) break;  // nothing penetrates
    for (int it = 0; it < cfg.nsc_position_psor_iters; ++it) {
      double loc = 0.0;
      for (int k = 0; k < K; ++k) {
        if (my_color == k && act) {
          d3 nv{PR[P_N * kSmallC + p], PR[(P_N + 1) * kSmallC + p], PR[(P_N + 2) * kSmallC + p]};
          d3 ra{PR[P_RA * kSmallC + p], PR[(P_RA + 1) * kSmallC + p], PR[(P_RA + 2) * kSmallC + p]};
          d3 rb{PR[P_RB * kSmallC + p], PR[(P_RB + 1) * kSmallC + p], PR[(P_RB + 2) * kSmallC + p]};
          d3 dxa{DX[sa], DX[kSmallB + sa], DX[2 * kSmallB + sa]};
          d3 dta{DX[3 * kSmallB + sa], DX[4 * kSmallB + sa], DX[5 * kSmallB + sa]};
          d3 dxb{DX[sb], DX[kSmallB + sb], DX[2 * kSmallB + sb]};
          d3 dtb{DX[3 * kSmallB + sb], DX[4 * kSmallB + sb], DX[5 * kSmallB + sb]};
          double l = PR[P_L * kSmallC + p];
          double corr = dot(nv, ((dxb + cross(dtb, rb)) - dxa) - cross(dta, ra));
          double r = corr + PR[P_PHI * kSmallC + p] + cfm * l;
          double d = -(omega / PR[P_G * kSmallC + p]) * r;
          double nl = smax(0.0, l + d);
          double dl = nl - l;
          if (dl != 0.0) {
            PR[P_L * kSmallC + p] = nl;
            d3 rAxn = cross(ra, nv);
            dxa = dxa - nv * (dl * st.inv_mass[a]);
            dta = dta - iinv_apply(st, a, rAxn) * dl;
            d3 rBxn = cross(rb, nv);
            dxb = dxb + nv * (dl * st.inv_mass[b]);
            dtb = dtb + iinv_apply(st, b, rBxn) * dl;
            DX[sa] = dxa.x; DX[kSmallB + sa] = dxa.y; DX[2 * kSmallB + sa] = dxa.z;
            DX[3 * kSmallB + sa] = dta.x; DX[4 * kSmallB + sa] = dta.y; DX[5 * kSmallB + sa] = dta.z;
            DX[sb] = dxb.x; DX[kSmallB + sb] = dxb.y; DX[2 * kSmallB + sb] = dxb.z;
            DX[3 * kSmallB + sb] = dtb.x; DX[4 * kSmallB + sb] = dtb.y; DX[5 * kSmallB + sb] = dtb.z;
          }
          loc = fabs(dl);
        }
        __syncthreads();
      }
      double res = small_block_max(loc, S);
      if (res < 1e-8) break;
    }
    __syncthreads();
    for (int s = t; s < S.nloc; s += blockDim.x) {
      int x = S.body[s];
      if (x < 0 || !S.dyn[s]) continue;
      if (V.moved) V.moved[x] = 1;
      st.x.st(x, st.x.ld(x) + mk3(DX[s], DX[kSmallB + s], DX[2 * kSmallB + s]));
      d3 th{DX[3 * kSmallB + s], DX[4 * kSmallB + s], DX[5 * kSmallB + s]};
      double ang = len(th);
      if (ang > 1e-8) {
        d3 ax = th / ang;
        st.q.st(x, qnormalize(qmul(angle_axis(ang, ax), st.q.ld(x))));
      }
    }
    __syncthreads();
  }
  small_unmap(V, S);
  return true;
}

// ---------------------------------------------------------------------------
// Cylinder walls of the velocity solve: for every dynamic capsule, contacts
// where its surface passes the tube wall at the two end points or the centre
// of its axis (collideCapsuleInsideCylinder, collision.cpp:197-241), in body
// order then sample order, appended after the Cp pair contacts as rows with
// b == a (main.cpp:4431-4447).  The team's first block lists them (block
// scan per round of rods); returns the total contact count.
// ---------------------------------------------------------------------------
__device__ inline int wall_hits(const NscView& V, int i, d3 ax, double R, d3* pt, d3* nrm, double* pen) {
  const State& st = V.st;
  if (!(st.inv_mass[i] > 0.0)) return 0;
  const double h = st.h[i], r = st.r[i];
  const d3 x = st.x.ld(i);
  d3 u = axis_y(st.q.ld(i));
  u = u / len(u);
  const d3 smp[3] = {x - u * h, x, x + u * h};
  int k = 0;
  for (int j = 0; j < 3; ++j) {
    const d3 p = smp[j];
    const d3 pp = p - ax * dot(p, ax);
    const double d = len(pp);
    const double pe = d + r - R;
    if (pe <= 0.0) continue;
    d3 nv;
    if (d > 1e-8) {
      nv = pp / d;
    } else {
      const d3 cr = cross(ax, fabs(ax.x) < 0.9 ? mk3(1, 0, 0) : mk3(0, 1, 0));
      nv = cr / len(cr);
    }
    if (pt) {
      pt[k] = p + nv * (R - d);
      nrm[k] = nv;
      pen[k] = pe;
    }
    ++k;
  }
  return k;
}

__device__ __noinline__ int wall_phase(const Team& T, const NscView& V, int Cp, SmemNsc& sm) {
  Ctl* ctl = V.ctl;
  const int n = V.st.n;
  const rg_config& cfg = V.cfg;
  if (T.rank() == 0) {
    d3 ax{cfg.cylinder_axis[0], cfg.cylinder_axis[1], cfg.cylinder_axis[2]};
    ax = ax / len(ax);
    const double R = cfg.cylinder_radius;
    int run = Cp;
    for (int base = 0; base < n; base += blockDim.x) {
      const int i = base + threadIdx.x;
      d3 pt[3], nv[3];
      double pe[3];
      const int k = i < n ? wall_hits(V, i, ax, R, pt, nv, pe) : 0;
      int tot;
      const int ex = block_excl_scan(k, sm.scan_w, tot);
      for (int j = 0; j < k; ++j) {
        const int c = run + ex + j;
        if (c >= V.ccap) break;
        V.con.a[c] = i;
        V.con.b[c] = i;
        V.con.type[c] = 3;  // wall
        V.con.comp(0)[c] = pt[j].x; V.con.comp(1)[c] = pt[j].y; V.con.comp(2)[c] = pt[j].z;
        V.con.comp(3)[c] = pt[j].x; V.con.comp(4)[c] = pt[j].y; V.con.comp(5)[c] = pt[j].z;
        V.con.comp(6)[c] = nv[j].x; V.con.comp(7)[c] = nv[j].y; V.con.comp(8)[c] = nv[j].z;
        V.con.comp(9)[c] = 0.0; V.con.comp(10)[c] = 0.0; V.con.comp(11)[c] = 0.0;
        V.con.comp(12)[c] = -pe[j];  // phi = comp12 - comp13 = -penetration
        V.con.comp(13)[c] = 0.0;
      }
      run += tot;
    }
    if (threadIdx.x == 0) {
      if (run > V.ccap) atomicOr(&ctl->err, ERR_CONTACT_CAP);
      ctl->contacts = run;
    }
  }
  if (!team_sync(T)) return -1;
  const int C = *(volatile int*)&ctl->contacts;
  return C > V.ccap ? -1 : C;
}

// ---------------------------------------------------------------------------
// One NSC step of one system by one team.
// ---------------------------------------------------------------------------
__device__ bool nsc_step(const Team& T, const NscView& V, SmemNsc& sm, SmallSmem& S, bool first) {
  Ctl* ctl = V.ctl;
  const State& st = V.st;
  const rg_config& cfg = V.cfg;
  const int n = st.n;
  const int tid = T.tid(), TS = T.size(), rank = T.rank();
  if (*(volatile int*)&ctl->err) return false;
  PhaseClock pc(ctl, rank == 0 && threadIdx.x == 0 && ctl->prof_phases);
  if (rank == 0 && threadIdx.x == 0) {
    ctl->collisions = 0;
    ctl->jn_sum = 0;
    ctl->jt_sum = 0;
  }
  // 1) free flight (main.cpp:4397-4408) + segment records + displacement
  {
    const d3 g{cfg.gravity[0], cfg.gravity[1], cfg.gravity[2]};
    double dmax = 0.0, dnear = 0.0;
    const double* ref2 = V.near ? V.ref2 : nullptr;
    double invL[3] = {1.0, 1.0, 1.0};
    for (int k = 0; k < 3; ++k)
      if (V.box.L[k] > 0.0) invL[k] = 1.0 / V.box.L[k];
    const StateBase SB{st.sbase, st.pbase, n};
    const double dt = cfg.dt;
    const double* ref = V.ref;
    Seg* seg = V.seg;
    const Box box = V.box;
    // Only the position update, the projection and the wrap move rods, and
    // the last two flag what they move: other rods keep the segment record
    // and displacement bounds of the position update (still folded into
    // ctl->maxdisp / near_disp), and need their velocities only.  The first
    // step of a launch refreshes every rod (the state may have been set
    // from the host).
    const unsigned char* moved = first ? nullptr : V.moved;
    for (int i = tid; i < n; i += TS) {
      if (moved && !moved[i]) free_flight_velocity(SB, i, g, dt);
      else free_flight_fused(SB, i, g, dt, ref, ref2, box, invL, seg, dmax, dnear);
    }
    double bm = block_reduce_max(dmax, sm.red_d);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxdisp, bm);
    if (V.near) {
      double bn = block_reduce_max(dnear, sm.red_d);
      if (threadIdx.x == 0) atomic_max_nonneg(&ctl->near_disp, bn);
    }
    if (!team_sync(T)) return false;
  }
  pc.mark(0);
  // 2) detection (pairs, then cylinder walls), colouring, manifold rows
  const int Cp = detect_phase(T, V, 0.0, sm, false);
  if (Cp < 0) return false;
  const int C = cfg.cylinder_enabled ? wall_phase(T, V, Cp, sm) : Cp;
  if (C < 0) return false;
  pc.mark(1);
  const bool small = C <= kSmallC;
  if (small) {
    // colouring, rows, PSOR and warm cache in one block, on chip
    bool ok = true;
    const unsigned long long ts = (rank == 0 && threadIdx.x == 0) ? gtimer() : 0ull;
    if (rank == 0) ok = small_solve(V, C, Cp, S, pc);
    if (rank == 0 && threadIdx.x == 0) ctl->serial_ns += (long long)(gtimer() - ts);
    if (!ok) atomicOr(&ctl->err, ERR_COLOR);
    pc.mark(10);
    if (!team_sync(T)) return false;
    pc.mark(11);
  } else {
  if (!color_phase(T, V, C, sm)) return false;
  pc.mark(2);
  {
    RowIO R{V.row, V.lam, V.ccap};
    const int W = *(volatile int*)V.wn;
    const double* im = st.inv_mass;
    int* deg = V.owner;  // free between colouring and the next colouring
    if (V.feat_on) {
      for (int c = tid; c < C; c += TS) {
        deg[V.con.a[c]] = 0;
        deg[V.con.b[c]] = 0;
      }
      if (!team_sync(T)) return false;
    }
    int coll = 0;
    for (int p = tid; p < C; p += TS) {
      const int c = V.order[p];
      coll += build_row(st, V.con, cfg, c, p, R, V.wkey, V.wlam, W, V.wcap, V.feat_on ? V.feat : nullptr, V.ccap) & 1;
      if (V.feat_on && c < Cp) {  // wall rows have no graph degree
        if (im[V.con.a[c]] > 0.0) atomicAdd(&deg[V.con.a[c]], 1);
        if (im[V.con.b[c]] > 0.0) atomicAdd(&deg[V.con.b[c]], 1);
      }
    }
    int bcoll = block_reduce_sum_i(coll, sm.red_i);
    if (threadIdx.x == 0 && bcoll)
      atomicAdd(reinterpret_cast<unsigned long long*>(&ctl->collisions), (unsigned long long)bcoll);
    if (!team_sync(T)) return false;
    if (V.feat_on) {
      for (int p = tid; p < C; p += TS) {
        const int c = V.order[p], a = V.con.a[c], b = V.con.b[c];
        V.feat[7 * (size_t)V.ccap + p] = (float)((im[a] > 0.0 ? deg[a] - 1 : 0) + (im[b] > 0.0 ? deg[b] - 1 : 0));
      }
      if (V.use_mlp && (W == 0 || *(volatile int*)&ctl->sweeps_last > V.mlp_min_sweeps)) {
        // each warp of the team evaluates tiles of 16 slots on the tensor
        // cores; its own lanes then apply the tile's predictions.  Every
        // block stages the whole network in its (here unused) small-solve
        // shared memory: W1, W4 and the small parameters in pmax/cmask, W2
        // in wh, W3 over the rows.
        const MlpStage ms = mlp_stage_at(S.pmax);
        __nv_bfloat16* w3s = reinterpret_cast<__nv_bfloat16*>(S.row);
        stage_small(ms, V.mlp);
        stage_bf16(S.wh, kWhLd, V.mlp.w2, kMlpH, kMlpH);
        stage_bf16(w3s, kWhLd, V.mlp.w3, kMlpH, kMlpH);
        stage_wait();
        __syncthreads();
        if (!team_sync(T)) return false;
        const MlpSmall q = ms.small();
        const int lane = threadIdx.x & 31, gw = tid >> 5, nw = TS >> 5;
        for (int row0 = gw * 16; row0 < C; row0 += nw * 16) {
          const int p = row0 + (lane & 15);
          const bool want = lane < 16 && p < C && V.order[p] < Cp &&  // never a wall row
                            (V.mlp_all || !warm_cached(V, V.order[p], W));
          if (!__ballot_sync(0xffffffffu, want)) continue;  // no row of this tile needs the network
          unsigned a[8][4];
          mlp_layer1(ms.w1, kW1Ld, q, V.feat, V.ccap, row0, C, lane, a);
          hidden_layer(a, S.wh, kWhLd, q.b2, lane);
          hidden_layer(a, w3s, kWhLd, q.b3, lane);
          mlp_layer4(a, ms.w4, kWhLd, q, V.pred, V.ccap, row0, C, lane);
          __syncwarp();
          if (want) mlp_apply(R, V.pred, V.ccap, p, cfg.nsc_mu);
          __syncwarp();
        }
      }
      if (!team_sync(T)) return false;
    }
  }
  pc.mark(3);
  // 3) PSOR
  if (!psor_phase(T, V, C, sm)) return false;
  pc.mark(4);
  }
  // 4) warm cache and impulse sums (large path); position update + segments
  {
    RowIO R{V.row, V.lam, V.ccap};
    double jn = 0, jt = 0;
    for (int p = tid; !small && p < C; p += TS) {
      int c = V.order[p];
      double l0 = R.lam[p], l1 = R.lam[R.ccap + p], l2 = R.lam[2 * R.ccap + p];
      if (c < Cp) {  // wall rows start cold every step: they stay out of the cache
        V.wkey[c] = ((unsigned long long)(unsigned)V.con.a[c] << 32) | (unsigned)V.con.b[c];
        V.wlam[c] = l0;
        V.wlam[V.wcap + c] = l1;
        V.wlam[2 * V.wcap + c] = l2;
        reinterpret_cast<int*>(V.wlam + 3 * (size_t)V.wcap)[c] = V.color[c];
        if (V.xrow) export_row(V.xrow, V.wcap, c, R, p);
      }
      jn += fabs(l0);  // profile-CSV sums of main.cpp:3339-3343
      jt += fabs(l1) + fabs(l2);
    }
    jn = warp_sum(jn);
    jt = warp_sum(jt);
    if ((threadIdx.x & 31) == 0 && (jn != 0.0 || jt != 0.0)) {
      atomicAdd(&ctl->jn_sum, jn);
      atomicAdd(&ctl->jt_sum, jt);
    }
    if (tid == 0 && !small) {
      *V.wn = Cp;
      ctl->vel_contacts = C;
    }
    int rec_base = 0;
    if (V.rec_cap > 0 && !small && C > 0) {
      // records (features, converged impulses) in slot order
      rec_base = *(volatile int*)&ctl->rec_n;
      for (int p = tid; p < C && rec_base + p < V.rec_cap; p += TS) {
        const size_t r = (size_t)(rec_base + p);
        for (int k = 0; k < kMlpIn; ++k) V.rec_x[r * kMlpIn + k] = V.feat[(size_t)k * V.ccap + p];
        for (int k = 0; k < kMlpOut; ++k) V.rec_y[r * kMlpOut + k] = (float)R.lam[(size_t)k * R.ccap + p];
      }
    }
    int bad = 0;
    double dmax = 0.0, dnear = 0.0;
    const double* ref2 = V.near ? V.ref2 : nullptr;
    double invL[3] = {1.0, 1.0, 1.0};
    for (int k = 0; k < 3; ++k)
      if (V.box.L[k] > 0.0) invL[k] = 1.0 / V.box.L[k];
    {
      const StateBase SB{st.sbase, st.pbase, n};
      const double dt = cfg.dt, w_max = cfg.w_max;
      const double ld = 1.0 - cfg.lin_damp * dt, ad = 1.0 - cfg.ang_damp * dt;
      const double* ref = V.ref;
      Seg* seg = V.seg;
      unsigned char* moved = V.moved;
      const bool spin = cfg.cylinder_enabled != 0;
      const Box box = V.box;
      for (int i = tid; i < n; i += TS)
        bad |= position_update_fused(SB, i, dt, ld, ad, w_max, ref, ref2, box, invL, seg, dmax, dnear, moved,
                                     spin);
    }
    if (bad) atomicOr(&ctl->err, ERR_NONFINITE);
    double bm = block_reduce_max(dmax, sm.red_d);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctl->maxdisp, bm);
    if (V.near) {
      double bn = block_reduce_max(dnear, sm.red_d);
      if (threadIdx.x == 0) atomic_max_nonneg(&ctl->near_disp, bn);
    }
    if (!team_sync(T)) return false;
    // every block has read rec_n before the barrier
    if (V.rec_cap > 0 && !small && C > 0 && tid == 0) ctl->rec_n = rec_base + C;
  }
  pc.mark(5);
  // 5) position projection (nsc_contact.cpp:659-880)
  if (cfg.nsc_position_stabilization) {
    int C2 = detect_phase(T, V, 0.0, sm, true);
    if (C2 < 0) return false;
    pc.mark(6);
    if (C2 <= kSmallC) {
      bool ok = true;
      const unsigned long long ts = (rank == 0 && threadIdx.x == 0) ? gtimer() : 0ull;
      if (rank == 0) ok = small_project(V, C2, S);
      if (rank == 0 && threadIdx.x == 0) ctl->serial_ns += (long long)(gtimer() - ts);
      if (!ok) atomicOr(&ctl->err, ERR_COLOR);
      if (!team_sync(T)) return false;
    } else {
      if (!color_phase(T, V, C2, sm)) return false;
      pc.mark(7);
      if (!project_phase(T, V, C2, sm)) return false;
    }
    pc.mark(8);
  }
  // 6) PBC wrap + clear forces (main.cpp:4508-4527); the next step touches
  // rod i from this same thread, so no barrier is needed here.
  {
    const StateBase SB{st.sbase, st.pbase, n};
    const Box box = V.box;
    unsigned char* moved = V.moved;
    for (int i = tid; i < n; i += TS) wrap_clear_body(SB, box, i, moved);
  }
  return true;
}

#ifndef RG_NSC_BLOCK
#define RG_NSC_BLOCK (2 * kTile)
#endif
constexpr int kBlock = RG_NSC_BLOCK;  // threads per block of the persistent step

// Each block finds its team (teams are sorted by b0), then runs nsteps steps
// of the team's systems, one system after the other within a step.  A
// system whose step failed (error bits set) returns at once from its later
// steps; the others carry on.
#ifndef RG_NSC_MIN_BLOCKS
#define RG_NSC_MIN_BLOCKS 1
#endif
__global__ void __launch_bounds__(kBlock, RG_NSC_MIN_BLOCKS) k_nsc_run(const NscView* views, const TeamDesc* teams, int nteams,
                                                   const int* members, int nsteps) {
  __shared__ SmemNsc sm;
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  SmallSmem& S = *reinterpret_cast<SmallSmem*>(dyn_smem);
  int lo = 0, hi = nteams;  // last team with b0 <= blockIdx.x
  while (hi - lo > 1) {
    int m = (lo + hi) >> 1;
    if (teams[m].b0 <= (int)blockIdx.x) lo = m;
    else hi = m;
  }
  const TeamDesc td = teams[lo];
  if ((int)blockIdx.x < td.b0 || (int)blockIdx.x >= td.b0 + td.nb) return;
  const bool team_timer = td.t_ns && threadIdx.x == 0 && (int)blockIdx.x == td.b0;
  const unsigned long long t_start = team_timer ? gtimer() : 0ull;
  for (int s = 0; s < nsteps; ++s) {
    bool any = false;
    for (int m = td.first; m < td.first + td.count; ++m) {
      const NscView& V = views[members ? members[m] : m];
      Team T{td.b0, td.nb, td.bar, &V.ctl->err,
             V.cfg.spin_limit > 0 ? (long long)V.cfg.spin_limit : kSpinLimit,
             V.cfg.test_absent_blocks > 0 ? (unsigned)V.cfg.test_absent_blocks : 0u};
      const bool timer = threadIdx.x == 0 && (int)blockIdx.x == td.b0;
      const unsigned long long t0 = timer ? gtimer() : 0ull;
      any |= nsc_step(T, V, sm, S, s == 0);
      if (timer) V.ctl->member_ns += (long long)(gtimer() - t0);  // one writer per system
    }
    if (!any) break;
  }
  if (team_timer) *td.t_ns = (long long)(gtimer() - t_start);
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
NscView make_view(rg_system* s) {
  NscView V;
  std::memset(&V, 0, sizeof(V));
  V.st = s->st;
  V.box = s->box;
  V.cfg = s->cfg;
  V.ctl = s->d_ctl;
  const Detector& d = s->det;
  V.seg = d.seg; V.nbr_cnt = d.nbr_cnt; V.nbr = d.nbr; V.maxnb = d.maxnb; V.ref = d.ref;
  V.words = d.mask_words; V.mask = d.hit_mask; V.hit_cnt = d.hit_cnt;
  V.cell_of = d.cell_of; V.cell_cnt = d.cell_cnt; V.cell_start = d.cell_start;
  V.cell_fill = d.cell_fill; V.cell_rods = d.cell_rods;
  V.grid = detector_grid(s);
  V.bounds = detector_bounds(s);
  V.skin = d.skin; V.margin = d.margin; V.cut_center = d.cut_center; V.all_pairs = d.all_pairs ? 1 : 0;
  V.con = s->con;
  const Nsc& N = s->nsc;
  V.row = N.row; V.lam = N.lam; V.color = N.color; V.order = N.order;
  V.color_cnt = N.color_cnt; V.color_off = N.color_off; V.cursor = N.cursor; V.remaining = N.remaining;
  V.pmax = N.pmax; V.cmask = N.cmask; V.owner = N.owner;
  V.wkey = N.wkey; V.wlam = N.wlam; V.wn = N.wn; V.wcap = N.wcap;
  V.xrow = s->export_on ? N.xrow : nullptr;
  V.dx = N.dx; V.prow = N.prow; V.pactive = N.pactive;
  V.ccap = s->ccap;
  V.blk = N.blk;
  V.slot_of = N.slot_of;
  V.near = d.near;
  V.ref2 = d.ref2;
  V.moved = d.moved;
  V.near_skin = d.near_skin;
  V.feat = s->d_feat;
  V.pred = s->d_pred;
  V.use_mlp = (s->cfg.nsc_warm_start == RG_WARM_MLP && s->mlp_ready) ? 1 : 0;
  V.mlp_all = s->cfg.nsc_mlp_scope == 1 ? 1 : 0;
  V.mlp_min_sweeps = s->cfg.nsc_mlp_min_sweeps;
  V.rec_cap = s->recording ? s->rec_cap : 0;
  V.rec_x = s->d_rec_x;
  V.rec_y = s->d_rec_y;
  V.feat_on = (V.use_mlp || V.rec_cap > 0) ? 1 : 0;
  if (V.use_mlp) V.mlp = mlp_dev(s);
  return V;
}

int nsc_team_blocks(const rg_system* s) {
  int nb = s->team_blocks;  // explicit team size (tests, sweeps)
  if (nb <= 0) nb = (s->n + 127) / 128;  // about one block per 128 rods, up to every SM
  if (nb < 1) nb = 1;
  if (nb > s->coop_blocks) nb = s->coop_blocks;
  return nb;
}

static void launch_coop(const void* fn, int grid, int block, void** args, cudaStream_t st,
                        size_t smem = 0) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  RGL cudaLaunchKernelExC(&cfg, fn, args);
}

// nsteps NSC steps of one system as one persistent cooperative launch.
void nsc_run_launch(rg_system* s, int nsteps) {
  NscView V = make_view(s);
  const int nb = nsc_team_blocks(s);
  TeamDesc td{0, nb, 0, 1, s->nsc.bar};
  cudaMemcpyAsync(s->nsc.view_dev, &V, sizeof(NscView), cudaMemcpyHostToDevice, s->stream);
  cudaMemcpyAsync(s->nsc.team_dev, &td, sizeof(TeamDesc), cudaMemcpyHostToDevice, s->stream);
  cudaMemsetAsync(s->nsc.bar, 0, 4 * sizeof(unsigned int), s->stream);
  const NscView* views = reinterpret_cast<const NscView*>(s->nsc.view_dev);
  const TeamDesc* teams = reinterpret_cast<const TeamDesc*>(s->nsc.team_dev);
  int nteams = 1;
  const int* members = nullptr;
  void* args[] = {&views, &teams, &nteams, &members, &nsteps};
  nsc_set_smem();
  ProfScope p(s, ST_OTHER);
  launch_coop((const void*)k_nsc_run, nb, kBlock, args, s->stream, sizeof(SmallSmem));
  s->contacts_fresh = false;
}

void nsc_set_smem() {
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute((const void*)k_nsc_run, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(SmallSmem));
    attr_set = true;
  }
}

// nsteps steps of many systems as one persistent cooperative launch: teams
// (device array, sorted by b0) cover blocks [0, grid); team k runs the
// systems members[first_k .. first_k + count_k) of views.
void nsc_batch_launch(const NscView* views, const TeamDesc* teams, int nteams, const int* members, int grid,
                      int nsteps, cudaStream_t st) {
  nsc_set_smem();
  void* args[] = {&views, &teams, &nteams, &members, &nsteps};
  launch_coop((const void*)k_nsc_run, grid, kBlock, args, st, sizeof(SmallSmem));
}

int nsc_block_threads() { return kBlock; }

// Co-resident blocks of the persistent kernel per SM (its registers and
// shared memory decide; the cooperative launch needs them all resident).
int nsc_blocks_per_sm() {
  static int per_sm = -1;
  if (per_sm < 0) {
    nsc_set_smem();
    int k = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, k_nsc_run, kBlock, sizeof(SmallSmem)) != cudaSuccess ||
        k < 1) {
      cudaGetLastError();
      k = 1;
    }
    per_sm = k;
  }
  return per_sm;
}
size_t nsc_block_smem() { return sizeof(SmallSmem) + sizeof(SmemNsc); }

size_t nsc_view_bytes() { return sizeof(NscView); }
size_t nsc_team_bytes() { return sizeof(TeamDesc); }

}  // namespace rg
