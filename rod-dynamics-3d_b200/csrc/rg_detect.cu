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
// Exclusive scan (three launches, capacity-sized grids, device-side n).
// ---------------------------------------------------------------------------
constexpr int kScanBS = 1024;
constexpr int kScanItems = 2;
constexpr int kScanTile = kScanBS * kScanItems;

__global__ void k_scan_tiles(const int* in, int* out, const int* n_dev, int* blocks) {
  __shared__ int shw[32];
  int n = *n_dev;
  int ntile = (n + kScanTile - 1) / kScanTile;
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    int base = t * kScanTile + threadIdx.x * kScanItems;
    int v0 = base < n ? in[base] : 0;
    int v1 = base + 1 < n ? in[base + 1] : 0;
    int tot;
    int ex = block_excl_scan(v0 + v1, shw, tot);
    if (base < n) out[base] = ex;
    if (base + 1 < n) out[base + 1] = ex + v0;
    if (threadIdx.x == 0) blocks[t] = tot;
  }
}

__global__ void k_scan_blocks(int* blocks, const int* n_dev, int* out) {
  __shared__ int shw[32];
  int n = *n_dev;
  int ntile = (n + kScanTile - 1) / kScanTile;
  int carry = 0;
  for (int base = 0; base < ntile; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < ntile ? blocks[i] : 0;
    int tot;
    int ex = block_excl_scan(v, shw, tot);
    if (i < ntile) blocks[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void k_scan_add(int* out, const int* n_dev, const int* blocks) {
  int n = *n_dev;
  int ntile = (n + kScanTile - 1) / kScanTile;
  for (int t = blockIdx.x; t < ntile; t += gridDim.x) {
    int add = blocks[t];
    if (add == 0) continue;
    int base = t * kScanTile + threadIdx.x * kScanItems;
    if (base < n) out[base] += add;
    if (base + 1 < n) out[base + 1] += add;
  }
}

cudaError_t Scan::alloc(int cap_) {
  cap = cap_;
  return cudaMalloc(&d_blocks, sizeof(int) * ((cap + kScanTile - 1) / kScanTile + 1));
}
void Scan::free_() {
  if (d_blocks) cudaFree(d_blocks);
  d_blocks = nullptr;
}
void Scan::run(const int* in, int* out, const int* n_dev, cudaStream_t s) const {
  int tiles = (cap + kScanTile - 1) / kScanTile;
  int g = tiles < 148 * 4 ? tiles : 148 * 4;
  if (g < 1) g = 1;
  RGL k_scan_tiles<<<g, kScanBS, 0, s>>>(in, out, n_dev, d_blocks);
  RGL k_scan_blocks<<<1, kScanBS, 0, s>>>(d_blocks, n_dev, out);
  RGL k_scan_add<<<g, kScanBS, 0, s>>>(out, n_dev, d_blocks);
}

// ---------------------------------------------------------------------------
// Segment records, displacement check, cell grid.
// ---------------------------------------------------------------------------
__global__ void k_seg(State st, Seg* seg) {
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
// rebuild flag when it reaches skin/2.
__global__ void k_disp_check(State st, const Seg* seg, const double* ref, Box box, double skin,
                             Ctl* ctl) {
  if (ctl->err) return;
  __shared__ double sm[32];
  double m = 0.0;
  const int n = st.n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Seg s = seg[i];
    d3 dx{s.cx - ref[i], s.cy - ref[n + i], s.cz - ref[2 * n + i]};
    if (box.pbc) {
      if (box.L[0] > 0.0) dx.x -= floor(dx.x / box.L[0] + 0.5) * box.L[0];
      if (box.L[1] > 0.0) dx.y -= floor(dx.y / box.L[1] + 0.5) * box.L[1];
      if (box.L[2] > 0.0) dx.z -= floor(dx.z / box.L[2] + 0.5) * box.L[2];
    }
    d3 du{s.ux - ref[3 * n + i], s.uy - ref[4 * n + i], s.uz - ref[5 * n + i]};
    double d = len(dx) + s.h * len(du);
    if (!(d == d)) d = 1e300;  // non-finite state forces a rebuild
    m = fmax(m, d);
  }
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    v = warp_max(v);
    if (threadIdx.x == 0) {
      atomic_max_nonneg(&ctl->maxdisp, v);
      if (v >= 0.5 * skin * (1.0 - 1e-9)) atomicExch(&ctl->rebuild, 1);
    }
  }
}

__global__ void k_cell_fill(int n, const int* cell_of, const int* cell_start, int* cell_fill,
                            int* cell_rods, const Ctl* ctl) {
  if (ctl->err || !ctl->rebuild) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = cell_of[i];
    int p = atomicAdd(&cell_fill[c], 1);
    cell_rods[cell_start[c] + p] = i;
  }
}

__global__ void k_zero_cells(int* cnt, int* fill, int ncells, int* nbr_cnt, int n, const Ctl* ctl) {
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
  if (ctl->err) return;
  if (ctl->rebuild) {
    ctl->rebuilds += 1;
    ctl->rebuild = 0;
  }
  ctl->maxdisp = 0.0;
}

__global__ void k_bounds(const Seg* seg, int n, unsigned long long* mn, unsigned long long* mx,
                         const Ctl* ctl) {
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
  if (ctl->err || !ctl->rebuild) return;
  open_grid(mn, mx, cut, maxdim, g);
}

// Reads the device grid descriptor into each thread (open systems).
__global__ void k_cell_count_dyn(const Seg* seg, int n, const GridDev* gd, int pbc, int* cell_of,
                                 int* cell_cnt, const Ctl* ctl) {
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
__global__ void k_narrow_count(const Seg* seg, State st, Box box, double delta, const int* nbr_cnt,
                               const int* nbr, int maxnb, int words, unsigned long long* mask,
                               int* hit_cnt, const Ctl* ctl) {
  if (ctl->err) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x)
    hit_cnt[i] = narrow_count_rod(i, seg, st.inv_mass, box, delta, nbr_cnt, nbr, maxnb, words, mask);
}

__global__ void k_narrow_write(const Seg* seg, int n, Box box, const int* nbr_cnt, const int* nbr,
                               int maxnb, int words, const unsigned long long* mask, const int* hit_off,
                               Contacts con, Ctl* ctl) {
  if (ctl->err) return;
  int total = hit_off[n];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->contacts = total < con.cap ? total : con.cap;
    if (total > con.cap) atomicOr(&ctl->err, ERR_CONTACT_CAP);
  }
  if (total > con.cap) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (hit_off[i + 1] == hit_off[i]) continue;
    narrow_write_rod(i, hit_off[i], seg, box, nbr_cnt, nbr, maxnb, words, mask, con);
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
  if (ctl->err || !ctl->rebuild) return;
  dd->ncells = dd->grid.ncells;
}

cudaError_t detector_alloc(rg_system* s) {
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
  d = Detector();
}

void force_rebuild(rg_system* s) {
  int one = 1;
  cudaMemcpyAsync(&s->d_ctl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice, s->stream);
}

// Full detection at the current state with activation margin `delta`:
// segment records, (optional) displacement check and list rebuild, narrow
// phase.  Result: s->con sorted by (a,b) and ctl->contacts.
void detect_launch(rg_system* s, double delta, bool check_rebuild) {
  Detector& d = s->det;
  const int n = s->n;
  cudaStream_t st = s->stream;
  Ctl* ctl = s->d_ctl;
  DetDev* dd = det_dev(s);
  const int bs = 256;
  const int g = grid_for(n, bs);
  RGL k_seg<<<g, bs, 0, st>>>(s->st, d.seg);
  if (check_rebuild && !d.all_pairs)
    RGL k_disp_check<<<g, bs, 0, st>>>(s->st, d.seg, d.ref, s->box, d.skin, ctl);
  // --- rebuild: every kernel below returns at once unless ctl->rebuild ---
  if (!s->box.pbc) {
    cudaMemsetAsync(dd->mn, 0xff, sizeof(dd->mn), st);
    cudaMemsetAsync(dd->mx, 0x00, sizeof(dd->mx), st);
    RGL k_bounds<<<g, bs, 0, st>>>(d.seg, n, dd->mn, dd->mx, ctl);
    RGL k_open_grid<<<1, 1, 0, st>>>(dd->mn, dd->mx, d.cut_center, 64, &dd->grid, ctl);
    RGL k_grid_ncells<<<1, 1, 0, st>>>(dd, ctl);
  }
  RGL k_zero_cells<<<grid_for((d.ncells + 1 > n ? d.ncells + 1 : n), bs), bs, 0, st>>>(d.cell_cnt, d.cell_fill, d.ncells,
                                                                                     d.nbr_cnt, n, ctl);
  RGL k_cell_count_dyn<<<g, bs, 0, st>>>(d.seg, n, &dd->grid, s->box.pbc, d.cell_of, d.cell_cnt, ctl);
  s->scan.run(d.cell_cnt, d.cell_start, &dd->ncells, st);
  RGL k_cell_fill<<<g, bs, 0, st>>>(n, d.cell_of, d.cell_start, d.cell_fill, d.cell_rods, ctl);
  int gb = d.ncells < s->sm_count * 8 ? d.ncells : s->sm_count * 8;
  RGL k_build_lists<<<gb, kTile, 0, st>>>(d.seg, n, &dd->grid, s->box, d.cell_start, d.cell_rods,
                                       d.margin, d.skin, d.cut_center, d.all_pairs ? 1 : 0,
                                       d.nbr_cnt, d.nbr, d.maxnb, ctl);
  RGL k_save_ref<<<g, bs, 0, st>>>(d.seg, n, d.ref, d.nbr, d.nbr_cnt, d.maxnb, ctl);
  RGL k_build_done<<<1, 1, 0, st>>>(ctl);
  // --- narrow phase ---
  RGL k_narrow_count<<<g, bs, 0, st>>>(d.seg, s->st, s->box, delta, d.nbr_cnt, d.nbr, d.maxnb,
                                   d.mask_words, d.hit_mask, d.hit_cnt, ctl);
  s->scan.run(d.hit_cnt, d.hit_off, &dd->n, st);
  RGL k_narrow_write<<<g, bs, 0, st>>>(d.seg, n, s->box, d.nbr_cnt, d.nbr, d.maxnb, d.mask_words,
                                   d.hit_mask, d.hit_off, s->con, ctl);
}

}  // namespace rg
