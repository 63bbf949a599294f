// rg_detect_dev.cuh - device bodies of the broad and narrow phase, shared
// by the multi-kernel detection (rg_detect.cu) and the persistent NSC step
// kernel (rg_nsc.cu).  See rg_detect.cu for the algorithm and its reference.
#pragma once
#include "rg_internal.cuh"

namespace rg {

constexpr int kTile = 256;  // threads per block; segment records per shared-memory tile

__device__ inline int cell_coord(double x, double lo, double cell, int nc, int pbc) {
  int c = (int)floor((x - lo) / cell);
  if (pbc) {
    c %= nc;
    if (c < 0) c += nc;
  } else {
    c = c < 0 ? 0 : (c >= nc ? nc - 1 : c);
  }
  return c;
}

struct GridDev {
  double lo[3], cell[3];
  int n[3], ncells;
};


// Bounding box of the centres for open (non-periodic) systems.
__device__ inline unsigned long long ord_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ inline double ord_val(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}
// Cell grid over the bounding box of the centres (open systems).
__device__ inline void open_grid(const unsigned long long* mn, const unsigned long long* mx, double cut,
                                 int maxdim, GridDev* g) {
  int total = 1;
  for (int k = 0; k < 3; ++k) {
    double lo = ord_val(mn[k]), hi = ord_val(mx[k]);
    double span = hi - lo;
    int d = (int)floor(span / cut);
    d = d < 1 ? 1 : (d > maxdim ? maxdim : d);
    g->lo[k] = lo;
    g->cell[k] = span > 0 ? span / d : 1.0;
    if (g->cell[k] < cut) g->cell[k] = cut;
    g->n[k] = d;
    total *= d;
  }
  g->ncells = total;
}

// Staged segment records in structure-of-arrays form: consecutive threads
// read consecutive 8-byte words (no shared-memory bank conflicts; a 64-byte
// Seg stride would serialise 16 ways).
struct SegTile {
  double cx[kTile], cy[kTile], cz[kTile], h[kTile], ux[kTile], uy[kTile], uz[kTile], r[kTile];
  __device__ void put(int k, const Seg& s) {
    cx[k] = s.cx; cy[k] = s.cy; cz[k] = s.cz; h[k] = s.h;
    ux[k] = s.ux; uy[k] = s.uy; uz[k] = s.uz; r[k] = s.r;
  }
  __device__ Seg get(int k) const {
    Seg s;
    s.cx = cx[k]; s.cy = cy[k]; s.cz = cz[k]; s.h = h[k];
    s.ux = ux[k]; s.uy = uy[k]; s.uz = uz[k]; s.r = r[k];
    return s;
  }
};

struct BuildSmem {
  SegTile tile;
  int tidx[kTile];
  SegTile home;
  int hidx[kTile];
  int ncl[27];
  int nstart[27];  // first entry of each neighbour cell in cell_rods
  int npre[28];    // prefix of the neighbour cells' rod counts
  int nn;
  int qn[2];       // queue fills (see build_cell_pairs)
};

__device__ inline int list_insert(int* list, int cnt, int cap, int j, int& overflow) {
  if (cnt >= cap) {
    overflow = 1;
    return cnt;
  }
  int k = cnt;
  while (k > 0 && list[k - 1] > j) {
    list[k] = list[k - 1];
    --k;
  }
  list[k] = j;
  return cnt + 1;
}

// Conservative minimum-image centre offset B - A without divisions (for list
// building only; the exact narrow phase uses min_image_shift).
__device__ inline d3 centre_offset(const Seg& A, const Seg& B, const Box& box, const double* invL) {
  d3 d{B.cx - A.cx, B.cy - A.cy, B.cz - A.cz};
  if (box.pbc) {
    if (box.L[0] > 0.0) d.x -= box.L[0] * rint(d.x * invL[0]);
    if (box.L[1] > 0.0) d.y -= box.L[1] * rint(d.y * invL[1]);
    if (box.L[2] > 0.0) d.z -= box.L[2] * rint(d.z * invL[2]);
  }
  return d;
}

// True when segments A and B (B displaced by the centre offset d) are
// certainly farther apart than lim: two axial slabs and the axis-line
// distance bound the segment distance from below (|q - p| >= |(q - p).u|
// for a unit u, and (q - p).c = d.c for c = uA x uB).  FP64 with the same
// relative slack as the centre test; the line bound is used only when the
// axes are not near parallel, where c carries full relative precision.
// Callers still decide with the exact narrow phase: this only skips pairs
// whose exact distance is >= lim, so lists and contacts do not change.
__device__ inline bool seg_far(const Seg& A, const Seg& B, d3 d, double lim) {
  const double L = lim * (1.0 + 1e-9) + 1e-12;
  const d3 ua{A.ux, A.uy, A.uz}, ub{B.ux, B.uy, B.uz};
  const double cab = fabs(dot(ua, ub));
  if (fabs(dot(d, ua)) - cab * B.h - A.h > L) return true;
  if (fabs(dot(d, ub)) - cab * A.h - B.h > L) return true;
  const d3 c = cross(ua, ub);
  const double c2 = dot(c, c);
  if (c2 > 1e-6) {
    const double dc = dot(d, c);
    if (dc * dc > L * L * c2) return true;
  }
  return false;
}

// Pair-parallel list build for one home cell (all block threads call it):
// home rods and each neighbour cell are staged in shared memory and the
// block's threads split the (home rod, neighbour rod) pairs.  Accepted j > i
// are appended with an atomic per-rod counter (nbr_cnt zeroed beforehand);
// sort_lists() orders every list afterwards.  Acceptance is the same
// conservative test as build_cell.
__device__ inline void build_cell_pairs(const Seg* seg, const GridDev& g, const Box& box, const double* invL,
                                        const int* cell_start, const int* cell_rods, double margin,
                                        double skin, int all_pairs, int* nbr_cnt, int* nbr, int maxnb,
                                        int cell, BuildSmem& sm, unsigned* q1, unsigned* q2, int qcap,
                                        int& overflow) {
  int cx = cell % g.n[0], cy = (cell / g.n[0]) % g.n[1], cz = cell / (g.n[0] * g.n[1]);
  // Half shell: the home cell (pairs j > i) and the 13 cells ahead of it
  // (every pair), each unordered pair met once and listed under its lower
  // index.  Needs distinct neighbour cells: three or more cells along every
  // periodic axis, and not the all-pairs scan.
  const bool half = !all_pairs && !(box.pbc && (g.n[0] < 3 || g.n[1] < 3 || g.n[2] < 3));
  if (threadIdx.x == 0 && half) {
    int cnt = 0;
    const int c3[3] = {cx, cy, cz};
    for (int o = 0; o < 27; ++o) {
      const int off[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
      // home first, then the forward half (z, then y, then x decides)
      const bool fwd = off[2] > 0 || (off[2] == 0 && (off[1] > 0 || (off[1] == 0 && off[0] > 0)));
      if (!fwd) continue;
      int X = c3[0] + off[0], Y = c3[1] + off[1], Z = c3[2] + off[2];
      if (box.pbc) {
        X = (X + g.n[0]) % g.n[0]; Y = (Y + g.n[1]) % g.n[1]; Z = (Z + g.n[2]) % g.n[2];
      } else if (X < 0 || Y < 0 || Z < 0 || X >= g.n[0] || Y >= g.n[1] || Z >= g.n[2]) {
        continue;
      }
      sm.ncl[1 + cnt++] = (Z * g.n[1] + Y) * g.n[0] + X;
    }
    sm.ncl[0] = cell;
    sm.nn = 1 + cnt;
  }
  if (threadIdx.x == 0 && !half) {
    int cnt = 0;
    int lo[3], hi[3];
    int c3[3] = {cx, cy, cz};
    for (int k = 0; k < 3; ++k) {
      if (box.pbc && (g.n[k] < 3 || all_pairs)) {
        lo[k] = 0; hi[k] = g.n[k] - 1;
      } else {
        lo[k] = c3[k] - 1; hi[k] = c3[k] + 1;
      }
    }
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int x = lo[0]; x <= hi[0]; ++x) {
          int X = x, Y = y, Z = z;
          if (box.pbc) {
            X = (X + g.n[0]) % g.n[0]; Y = (Y + g.n[1]) % g.n[1]; Z = (Z + g.n[2]) % g.n[2];
          } else if (X < 0 || Y < 0 || Z < 0 || X >= g.n[0] || Y >= g.n[1] || Z >= g.n[2]) {
            continue;
          }
          if (cnt < 27) sm.ncl[cnt++] = (Z * g.n[1] + Y) * g.n[0] + X;
        }
    sm.nn = cnt;
  }
  __syncthreads();
  const int nn = sm.nn;
  if ((int)threadIdx.x < nn) {
    const int c = sm.ncl[threadIdx.x];
    sm.nstart[threadIdx.x] = cell_start[c];
    sm.npre[threadIdx.x + 1] = cell_start[c + 1] - cell_start[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.npre[0] = 0;
    for (int c = 0; c < nn; ++c) sm.npre[c + 1] += sm.npre[c];
  }
  // (read after the barrier at the top of the home-tile loop)
  const int hs = cell_start[cell], he = cell_start[cell + 1];
  for (int h0 = hs; h0 < he; h0 += kTile) {
    const int H = he - h0 < kTile ? he - h0 : kTile;
    // G threads per home rod, each scanning every G-th rod of a tile: no
    // per-pair index division, the home rod's centre stays in registers
    const int G = (int)blockDim.x / H > 0 ? (int)blockDim.x / H : 1;
    const int hslot = (int)threadIdx.x / G, sub = (int)threadIdx.x - hslot * G;
    __syncthreads();
    if ((int)threadIdx.x < H) {
      int i = cell_rods[h0 + threadIdx.x];
      sm.hidx[threadIdx.x] = i;
      sm.home.put(threadIdx.x, seg[i]);
    }
    __syncthreads();
    const bool mine = hslot < H;
    const int i = mine ? sm.hidx[hslot] : 0;
    const double hcx = mine ? sm.home.cx[hslot] : 0.0, hcy = mine ? sm.home.cy[hslot] : 0.0;
    const double hcz = mine ? sm.home.cz[hslot] : 0.0;
    const double hhr = mine ? sm.home.h[hslot] : 0.0, hrr = mine ? sm.home.r[hslot] : 0.0;
    // the neighbourhood's rods as one sequence (cell after cell), staged in
    // full tiles: fewer, fuller tiles than one per neighbour cell
    const int total = sm.npre[nn];
    {
      for (int t0 = 0; t0 < total; t0 += kTile) {
        const int m = total - t0 < kTile ? total - t0 : kTile;
        __syncthreads();
        if ((int)threadIdx.x < m) {
          const int v = t0 + (int)threadIdx.x;
          int lo = 0, hi = nn;  // last cell with npre <= v
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (sm.npre[mid] <= v) lo = mid;
            else hi = mid;
          }
          int j = cell_rods[sm.nstart[lo] + (v - sm.npre[lo])];
          sm.tidx[threadIdx.x] = j;
          sm.tile.put(threadIdx.x, seg[j]);
        }
        __syncthreads();
        if (all_pairs) {
          // tiny periodic boxes: every pair is listed
          if (!mine) continue;
          for (int u = sub; u < m; u += G) {
            const int j = sm.tidx[u];
            if (j <= i) continue;
            int pos = atomicAdd(&nbr_cnt[i], 1);
            if (pos < maxnb) nbr[(size_t)i * maxnb + pos] = j;
            else overflow = 1;
          }
          continue;
        }
        // Three block-wide stages per round, each over compacted work, so a
        // warp's lanes run the same test: centre test of every candidate ->
        // queue q1; axial/line prefilter of q1 -> queue q2; exact distance
        // of q2 -> lists.  (Tested lane by lane, one lane's exact test held
        // up its whole warp.)  per = candidates per thread and round.
        constexpr int kAhead = 4;
        const int per = (qcap / (int)blockDim.x) / kAhead * kAhead;
        const int cand = (m + G - 1) / G;  // most candidates of any thread
        const int rounds = (cand + per - 1) / per;
        const unsigned lane = threadIdx.x & 31u;
        for (int rd = 0; rd < rounds; ++rd) {
          if (threadIdx.x == 0) { sm.qn[0] = 0; sm.qn[1] = 0; }
          __syncthreads();
          for (int c0 = 0; c0 < per; c0 += kAhead) {
            // kAhead candidates with independent loads and FP64 chains
            bool pass[kAhead];
#pragma unroll
            for (int k = 0; k < kAhead; ++k) {
              const int u = sub + (rd * per + c0 + k) * G;
              const bool ok = mine && u < m;
              const int uu = ok ? u : 0;
              const int j = sm.tidx[uu];
              // centre test from the staged centres only (same arithmetic as
              // centre_offset)
              d3 d{sm.tile.cx[uu] - hcx, sm.tile.cy[uu] - hcy, sm.tile.cz[uu] - hcz};
              if (box.pbc) {
                if (box.L[0] > 0.0) d.x -= box.L[0] * rint(d.x * invL[0]);
                if (box.L[1] > 0.0) d.y -= box.L[1] * rint(d.y * invL[1]);
                if (box.L[2] > 0.0) d.z -= box.L[2] * rint(d.z * invL[2]);
              }
              const double hr = hhr + sm.tile.h[uu] + hrr + sm.tile.r[uu];
              const double cc = hr + margin + skin;
              const bool order = (half && t0 + uu >= sm.npre[1]) ? j != i : j > i;
              pass[k] = ok && order && !(dot(d, d) > cc * cc * (1.0 + 1e-9));
            }
#pragma unroll
            for (int k = 0; k < kAhead; ++k) {
              const unsigned bal = __ballot_sync(0xffffffffu, pass[k]);
              int base = 0;
              if (lane == 0 && bal) base = atomicAdd(&sm.qn[0], __popc(bal));
              base = __shfl_sync(0xffffffffu, base, 0);
              const int u = sub + (rd * per + c0 + k) * G;
              if (pass[k]) q1[base + __popc(bal & ((1u << lane) - 1u))] = ((unsigned)hslot << 16) | (unsigned)u;
            }
          }
          __syncthreads();
          const int n1 = sm.qn[0];
          for (int e = threadIdx.x; e < n1; e += blockDim.x) {
            const unsigned w = q1[e];
            const int h = (int)(w >> 16), u = (int)(w & 0xffffu);
            const Seg A = sm.home.get(h);
            const Seg B = sm.tile.get(u);
            d3 d{B.cx - A.cx, B.cy - A.cy, B.cz - A.cz};
            if (box.pbc) {
              if (box.L[0] > 0.0) d.x -= box.L[0] * rint(d.x * invL[0]);
              if (box.L[1] > 0.0) d.y -= box.L[1] * rint(d.y * invL[1]);
              if (box.L[2] > 0.0) d.z -= box.L[2] * rint(d.z * invL[2]);
            }
            const double lim = A.r + B.r + margin + skin;
            if (!seg_far(A, B, d, lim)) q2[atomicAdd(&sm.qn[1], 1)] = w;
          }
          __syncthreads();
          const int n2 = sm.qn[1];
          for (int e = threadIdx.x; e < n2; e += blockDim.x) {
            const unsigned w = q2[e];
            const int h = (int)(w >> 16), u = (int)(w & 0xffffu);
            const Seg A = sm.home.get(h);
            const Seg B = sm.tile.get(u);
            const double lim = A.r + B.r + margin + skin;
            Narrow nr = narrow_pair(A, B, box);
            if (!(nr.d2 < lim * lim)) continue;
            const int a = sm.hidx[h], b = sm.tidx[u];
            const int ii = a < b ? a : b, j = a < b ? b : a;  // listed under the lower index
            int pos = atomicAdd(&nbr_cnt[ii], 1);
            if (pos < maxnb) nbr[(size_t)ii * maxnb + pos] = j;
            else overflow = 1;
          }
          __syncthreads();
        }
      }
    }
  }
  __syncthreads();
}

// Rod-parallel list build (one thread per home rod, no block barriers):
// the candidates of rod i are the rods of its cell's neighbourhood, read
// from the cell arrays; accepted j > i are appended to i's own list (sorted
// afterwards by sort_list).  Same acceptance as build_cell_pairs.  Suits
// sparse cells, where staging a tile per neighbouring cell costs a memory
// round trip and a barrier for a handful of pairs.
__device__ inline void build_rod_list(int i, const Seg* seg, const GridDev& g, const Box& box, const double* invL,
                                      const int* cell_of, const int* cell_start, const int* cell_rods, double margin,
                                      double skin, int all_pairs, int* nbr_cnt, int* nbr, int maxnb, int& overflow) {
  const int cell = cell_of[i];
  const int c3[3] = {cell % g.n[0], (cell / g.n[0]) % g.n[1], cell / (g.n[0] * g.n[1])};
  int lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    if (box.pbc && (g.n[k] < 3 || all_pairs)) {
      lo[k] = 0; hi[k] = g.n[k] - 1;
    } else {
      lo[k] = c3[k] - 1; hi[k] = c3[k] + 1;
    }
  }
  const Seg A = seg[i];
  int* L = nbr + (size_t)i * maxnb;
  int cnt = 0;
  for (int z = lo[2]; z <= hi[2]; ++z)
    for (int y = lo[1]; y <= hi[1]; ++y)
      for (int x = lo[0]; x <= hi[0]; ++x) {
        int X = x, Y = y, Z = z;
        if (box.pbc) {
          X = (X + g.n[0]) % g.n[0]; Y = (Y + g.n[1]) % g.n[1]; Z = (Z + g.n[2]) % g.n[2];
        } else if (X < 0 || Y < 0 || Z < 0 || X >= g.n[0] || Y >= g.n[1] || Z >= g.n[2]) {
          continue;
        }
        const int c = (Z * g.n[1] + Y) * g.n[0] + X;
        const int e = cell_start[c + 1];
        for (int q = cell_start[c]; q < e; ++q) {
          const int j = cell_rods[q];
          if (j <= i) continue;
          const Seg B = seg[j];
          if (!all_pairs) {
            const d3 d = centre_offset(A, B, box, invL);
            const double cc = A.h + B.h + A.r + B.r + margin + skin;
            if (dot(d, d) > cc * cc * (1.0 + 1e-9)) continue;
            const double lim = A.r + B.r + margin + skin;
            if (seg_far(A, B, d, lim)) continue;
            const Narrow nr = narrow_pair(A, B, box);
            if (!(nr.d2 < lim * lim)) continue;
          }
          if (cnt < maxnb) L[cnt] = j;
          else overflow = 1;
          ++cnt;
        }
      }
  nbr_cnt[i] = cnt;
}

// Sorts rod i's neighbour list ascending (insertion sort; lists are short).
__device__ inline void sort_list(int* nbr, int* nbr_cnt, int maxnb, int i, int& overflow) {
  int cnt = nbr_cnt[i];
  if (cnt > maxnb) {
    overflow = 1;
    cnt = maxnb;
    nbr_cnt[i] = cnt;
  }
  int* L = nbr + (size_t)i * maxnb;
  for (int k = 1; k < cnt; ++k) {
    int v = L[k];
    int m = k;
    while (m > 0 && L[m - 1] > v) {
      L[m] = L[m - 1];
      --m;
    }
    L[m] = v;
  }
}

// Narrow-phase count with G lanes per rod (G divides 32): lane l tests list
// entries l, l+G, ...; contacts set bits in the rod's mask words (zeroed by
// lane 0 first) and the group's hit count is returned to every lane.
// prefilter: skip list entries that seg_far proves out of reach.  1: the
// centre offset uses the division-free image (valid when the box is not in
// all-pairs mode, where any other image is farther than the list cut-off);
// 2: the exact image of the narrow phase (valid always, costs 3 divisions).
template <int G>
__device__ inline int narrow_count_lanes(int i, bool valid, const Seg* seg, const double* inv_mass,
                                         const Box& box, double delta, const int* nbr_cnt, const int* nbr,
                                         int maxnb, int words, unsigned long long* mask, int prefilter = 0) {
  const int l = threadIdx.x & (G - 1);
  const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (threadIdx.x & 31 & ~(G - 1)));
  int cnt = valid ? nbr_cnt[i] : 0;
  if (valid && l == 0)
    for (int w = 0; w < words && w * 64 < cnt; ++w) mask[(size_t)i * words + w] = 0ull;
  __syncwarp();
  int hits = 0;
  if (valid) {
    const int* list = nbr + (size_t)i * maxnb;
    Seg A = seg[i];
    bool a_static = !(inv_mass[i] > 0.0);
    double invL[3] = {1.0, 1.0, 1.0};
    if (prefilter == 1)
      for (int k = 0; k < 3; ++k)
        if (box.L[k] > 0.0) invL[k] = 1.0 / box.L[k];
    for (int k = l; k < cnt; k += G) {
      int j = list[k];
      if (a_static && !(inv_mass[j] > 0.0)) continue;
      Seg B = seg[j];
      if (prefilter == 1 && seg_far(A, B, centre_offset(A, B, box, invL), A.r + B.r + delta)) continue;
      if (prefilter == 2) {
        d3 xa{A.cx, A.cy, A.cz}, xb{B.cx, B.cy, B.cz};
        if (seg_far(A, B, (xb - xa) + min_image_shift(box, xa, xb), A.r + B.r + delta)) continue;
      }
      Narrow nr = narrow_pair(A, B, box);
      if (contact_test(nr.d2, A.r + B.r, delta)) {
        atomicOr(&mask[(size_t)i * words + (k >> 6)], 1ull << (k & 63));
        ++hits;
      }
    }
  }
#pragma unroll
  for (int o = 1; o < G; o <<= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
  (void)gmask;
  return hits;
}

// Exact FP64 narrow phase of rod i against its list: sets one mask bit per
// contacting list entry and returns the number of contacts.
__device__ inline int narrow_count_rod(int i, const Seg* seg, const double* inv_mass, const Box& box,
                                       double delta, const int* nbr_cnt, const int* nbr, int maxnb,
                                       int words, unsigned long long* mask) {
  int cnt = nbr_cnt[i];
  const int* list = nbr + (size_t)i * maxnb;
  Seg A = seg[i];
  bool a_static = !(inv_mass[i] > 0.0);
  int hits = 0;
  unsigned long long wbits = 0;
  int w = 0;
  for (int k = 0; k < cnt; ++k) {
    int j = list[k];
    bool hit = false;
    if (!(a_static && !(inv_mass[j] > 0.0))) {
      Seg B = seg[j];
      Narrow nr = narrow_pair(A, B, box);
      hit = contact_test(nr.d2, A.r + B.r, delta);
    }
    if (hit) {
      wbits |= 1ull << (k & 63);
      ++hits;
    }
    if ((k & 63) == 63) {
      mask[(size_t)i * words + w] = wbits;
      wbits = 0;
      ++w;
    }
  }
  if (w < words && (cnt & 63)) mask[(size_t)i * words + w] = wbits;
  return hits;
}

// Centre offset B - A for seg_far: division-free image (mode 1, valid when
// the box is not in all-pairs mode) or the narrow phase's exact image (2).
__device__ inline d3 prefilter_offset(const Seg& A, const Seg& B, const Box& box, const double* invL, int mode) {
  if (mode == 1) return centre_offset(A, B, box, invL);
  d3 xa{A.cx, A.cy, A.cz}, xb{B.cx, B.cy, B.cz};
  return (xb - xa) + min_image_shift(box, xa, xb);
}

// Near-list count with G lanes per rod: list entries that seg_far cannot
// place beyond r_a + r_b + extra set their bit in the rod's mask words; the
// group's count is returned to every lane.
template <int G>
__device__ inline int near_count_lanes(int i, bool valid, const Seg* seg, const double* inv_mass, const Box& box,
                                       const double* invL, int mode, double extra, const int* nbr_cnt,
                                       const int* nbr, int maxnb, int words, unsigned long long* mask) {
  const int l = threadIdx.x & (G - 1);
  int cnt = valid ? nbr_cnt[i] : 0;
  if (valid && l == 0)
    for (int w = 0; w < words && w * 64 < cnt; ++w) mask[(size_t)i * words + w] = 0ull;
  __syncwarp();
  int hits = 0;
  if (valid) {
    const int* list = nbr + (size_t)i * maxnb;
    const Seg A = seg[i];
    const bool a_static = !(inv_mass[i] > 0.0);
    // two entries per round: both gathers are in flight before either test
    for (int k = l; k < cnt; k += 2 * G) {
      const bool has1 = k + G < cnt;
      const int j0 = list[k];
      const int j1 = has1 ? list[k + G] : j0;
      const Seg B0 = seg[j0];
      const Seg B1 = seg[j1];
      if (!(a_static && !(inv_mass[j0] > 0.0)) &&
          !seg_far(A, B0, prefilter_offset(A, B0, box, invL, mode), A.r + B0.r + extra)) {
        atomicOr(&mask[(size_t)i * words + (k >> 6)], 1ull << (k & 63));
        ++hits;
      }
      if (has1 && !(a_static && !(inv_mass[j1] > 0.0)) &&
          !seg_far(A, B1, prefilter_offset(A, B1, box, invL, mode), A.r + B1.r + extra)) {
        atomicOr(&mask[(size_t)i * words + ((k + G) >> 6)], 1ull << ((k + G) & 63));
        ++hits;
      }
    }
  }
#pragma unroll
  for (int o = 1; o < G; o <<= 1) hits += __shfl_xor_sync(0xffffffffu, hits, o);
  return hits;
}

// Writes rod i's marked list entries as (i, j) pairs from slot o on.
__device__ inline void near_write_rod(int i, int o, const int* nbr_cnt, const int* nbr, int maxnb, int words,
                                      const unsigned long long* mask, int2* out) {
  const int cnt = nbr_cnt[i];
  const int* list = nbr + (size_t)i * maxnb;
  for (int w = 0; w < words && w * 64 < cnt; ++w)
    for (unsigned long long m = __ldcg(&mask[(size_t)i * words + w]); m; m &= m - 1)
      out[o++] = make_int2(i, list[w * 64 + __ffsll((long long)m) - 1]);
}

// Contact record o of pair (i, j) from its narrow-phase result.
__device__ inline void write_contact(const Contacts& con, int o, int i, int j, double rsum, const Narrow& nr) {
  double dist = sqrt(nr.d2);
  d3 diff = nr.pb - nr.pa;
  d3 nv = dist > 1e-10 ? diff / dist : mk3(1, 0, 0);
  con.a[o] = i;
  con.b[o] = j;
  con.type[o] = contact_type(nr.s, nr.t);
  con.comp(0)[o] = nr.pa.x; con.comp(1)[o] = nr.pa.y; con.comp(2)[o] = nr.pa.z;
  con.comp(3)[o] = nr.pb.x; con.comp(4)[o] = nr.pb.y; con.comp(5)[o] = nr.pb.z;
  con.comp(6)[o] = nv.x; con.comp(7)[o] = nv.y; con.comp(8)[o] = nv.z;
  con.comp(9)[o] = nr.sh.x; con.comp(10)[o] = nr.sh.y; con.comp(11)[o] = nr.sh.z;
  con.comp(12)[o] = dist;
  con.comp(13)[o] = rsum;
}

// Writes the contacts of rod i (in list order: ascending b) from slot o on.
__device__ inline void narrow_write_rod(int i, int o, const Seg* seg, const Box& box, const int* nbr_cnt,
                                        const int* nbr, int maxnb, int words,
                                        const unsigned long long* mask, const Contacts& con) {
  int cnt = nbr_cnt[i];
  const int* list = nbr + (size_t)i * maxnb;
  Seg A = seg[i];
  for (int k = 0; k < cnt; ++k) {
    if (!((mask[(size_t)i * words + (k >> 6)] >> (k & 63)) & 1ull)) continue;
    int j = list[k];
    Seg B = seg[j];
    Narrow nr = narrow_pair(A, B, box);
    double dist = sqrt(nr.d2);
    d3 diff = nr.pb - nr.pa;
    d3 nv = dist > 1e-10 ? diff / dist : mk3(1, 0, 0);
    con.a[o] = i;
    con.b[o] = j;
    con.type[o] = contact_type(nr.s, nr.t);
    con.comp(0)[o] = nr.pa.x; con.comp(1)[o] = nr.pa.y; con.comp(2)[o] = nr.pa.z;
    con.comp(3)[o] = nr.pb.x; con.comp(4)[o] = nr.pb.y; con.comp(5)[o] = nr.pb.z;
    con.comp(6)[o] = nv.x; con.comp(7)[o] = nv.y; con.comp(8)[o] = nv.z;
    con.comp(9)[o] = nr.sh.x; con.comp(10)[o] = nr.sh.y; con.comp(11)[o] = nr.sh.z;
    con.comp(12)[o] = dist;
    con.comp(13)[o] = A.r + B.r;
    ++o;
  }
}

__device__ inline Seg make_seg(const State& st, int i) {
  dq q = st.q.ld(i);
  d3 u = axis_y(q);
  Seg s;
  s.cx = st.x.x[i]; s.cy = st.x.y[i]; s.cz = st.x.z[i]; s.h = st.h[i];
  s.ux = u.x; s.uy = u.y; s.uz = u.z; s.r = st.r[i];
  return s;
}

// |Δx| + h|Δu| since the last list build (non-finite state -> huge).
__device__ inline double seg_disp(const Seg& s, const double* ref, int n, int i, const Box& box) {
  d3 dx{s.cx - ref[i], s.cy - ref[n + i], s.cz - ref[2 * n + i]};
  if (box.pbc) {
    if (box.L[0] > 0.0) dx.x -= floor(dx.x / box.L[0] + 0.5) * box.L[0];
    if (box.L[1] > 0.0) dx.y -= floor(dx.y / box.L[1] + 0.5) * box.L[1];
    if (box.L[2] > 0.0) dx.z -= floor(dx.z / box.L[2] + 0.5) * box.L[2];
  }
  d3 du{s.ux - ref[3 * n + i], s.uy - ref[4 * n + i], s.uz - ref[5 * n + i]};
  double d = len(dx) + s.h * len(du);
  return (d == d) ? d : 1e300;
}

}  // namespace rg
