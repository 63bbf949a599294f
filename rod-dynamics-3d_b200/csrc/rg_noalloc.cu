// rg_noalloc.cu - contact detection that allocates no device memory.
//
// For callers that cannot call cudaMalloc (code that runs under another
// framework's device allocator, inside a memory budget it does not own, or
// in a process whose allocator must not be touched), rg_detect_noalloc
// finds the same contacts as rg_detect from device buffers the caller
// already has.  Every intermediate array lives in one file-scope
// __device__ array of fixed size (RG_NOALLOC_MAX_BODIES bodies), which each
// GPU that loads the library keeps until the process exits.
//
// The contact predicate and its FP64 arithmetic are the ones of the main
// narrow phase (narrow_pair / contact_test), so the pair list and contact
// geometry equal rg_detect's bit for bit.  Candidate pairs are all j > i
// (brute force), filtered by a conservative centre-distance test.
#include <mutex>

#include "rg_detect_dev.cuh"

namespace rg {

namespace {

constexpr int kNaMax = RG_NOALLOC_MAX_BODIES;
constexpr int kNaBS = 256;

// Scratch layout: segment records, per-rod contact counts, exclusive
// offsets (kNaMax + 1) and the scan's block totals.
struct NoAllocScratch {
  Seg seg[kNaMax];
  int count[kNaMax + 1];
  int offset[kNaMax + 1];
  int blocks[64];
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_na_mutex;
NoAllocScratch* g_na_ptr[64] = {nullptr};  // device address per device ordinal

__global__ void k_na_seg(const double* x, const double* q, const double* r, const double* h, int n,
                         NoAllocScratch* S) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    dq qq{q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]};
    d3 u = axis_y(qq);
    Seg s;
    s.cx = x[3 * i]; s.cy = x[3 * i + 1]; s.cz = x[3 * i + 2]; s.h = h[i];
    s.ux = u.x; s.uy = u.y; s.uz = u.z; s.r = r[i];
    S->seg[i] = s;
  }
}

__device__ inline bool na_pair(const Seg& A, const Seg& B, const Box& box, double delta, Narrow& nr) {
  d3 d{B.cx - A.cx, B.cy - A.cy, B.cz - A.cz};
  d = d + min_image_shift(box, mk3(A.cx, A.cy, A.cz), mk3(B.cx, B.cy, B.cz));
  double cc = A.h + B.h + A.r + B.r + delta;
  if (dot(d, d) > cc * cc * (1.0 + 1e-9) + 1e-12) return false;
  nr = narrow_pair(A, B, box);
  return contact_test(nr.d2, A.r + B.r, delta);
}

// Contacts of rod i with every j > i (both static: skipped, as the naive
// detector does, contact_detector.cpp:236-239).  One warp per rod i, its
// lanes striding over j: rows are triangular (rod 0 tests n-1 partners, rod
// n-1 none), and many small warp tasks keep the SMs evenly loaded.
__device__ inline bool na_candidate(int i, int j, const Seg& A, const Seg* seg, const Box& box, double delta,
                                    const double* inv_mass, bool a_static, Narrow& nr) {
  if (a_static && !(inv_mass[j] > 0.0)) return false;
  return na_pair(A, seg[j], box, delta, nr);
}

__global__ void k_na_count(int n, Box box, double delta, const double* inv_mass, NoAllocScratch* S) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const Seg A = S->seg[i];
    const bool a_static = inv_mass && !(inv_mass[i] > 0.0);
    int c = 0;
    for (int j = i + 1 + lane; j < n; j += 32) {
      Narrow nr;
      if (na_candidate(i, j, A, S->seg, box, delta, inv_mass, a_static, nr)) ++c;
    }
    c = warp_sum_i(c);
    if (lane == 0) S->count[i] = c;
  }
}

// Exclusive scan of count[0..n) into offset[0..n], one block.
__global__ void k_na_scan(int n, NoAllocScratch* S) {
  __shared__ int shw[32];
  int carry = 0;
  for (int base = 0; base < n; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < n ? S->count[i] : 0;
    int tot;
    int ex = block_excl_scan(v, shw, tot);
    if (i < n) S->offset[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) S->offset[n] = carry;
}

// Writes rod i's contacts in ascending j: each round of 32 candidates is
// ballot-compacted, so the output order is the (i, j) order of rg_detect.
__global__ void k_na_write(int n, Box box, double delta, const double* inv_mass, NoAllocScratch* S,
                           int32_t* pairs, double* geom, int cap, int32_t* count_out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *count_out = S->offset[n];
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    if (S->count[i] == 0) continue;
    const Seg A = S->seg[i];
    const bool a_static = inv_mass && !(inv_mass[i] > 0.0);
    int o = S->offset[i];
    for (int j0 = i + 1; j0 < n; j0 += 32) {
      const int j = j0 + lane;
      Narrow nr;
      const bool hit = j < n && na_candidate(i, j, A, S->seg, box, delta, inv_mass, a_static, nr);
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      const int slot = o + __popc(m & lt);
      if (hit && slot < cap) {
        pairs[2 * slot] = i;
        pairs[2 * slot + 1] = j;
        if (geom) {
          const Seg B = S->seg[j];
          double dist = sqrt(nr.d2);
          d3 diff = nr.pb - nr.pa;
          d3 nv = dist > 1e-10 ? diff / dist : mk3(1, 0, 0);
          double* gg = geom + 12 * (size_t)slot;
          gg[0] = nr.pa.x; gg[1] = nr.pa.y; gg[2] = nr.pa.z;
          gg[3] = nr.pb.x; gg[4] = nr.pb.y; gg[5] = nr.pb.z;
          gg[6] = nv.x; gg[7] = nv.y; gg[8] = nv.z;
          gg[9] = dist; gg[10] = A.r + B.r; gg[11] = (double)contact_type(nr.s, nr.t);
        }
      }
      o += __popc(m);
    }
  }
}

// Device address of the scratch array on the current device, looked up once
// per device with that device current.
int na_scratch(NoAllocScratch** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return RG_ERR_CUDA;
    }
    g_na_ptr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *out = g_na_ptr[dev];
  return RG_OK;
}

}  // namespace

}  // namespace rg

extern "C" int rg_detect_noalloc(const double* x, const double* q, const double* radius,
                                 const double* half_height, const double* inv_mass, int n, int pbc_enabled,
                                 const double* pbc_min, const double* pbc_max, double delta, int32_t* pairs,
                                 double* geom, int cap, int32_t* count, void* stream) {
  using namespace rg;
  if (n > kNaMax) return RG_ERR_CAPACITY;  // more bodies than the fixed scratch holds
  if (n < 0 || cap < 0 || !count || (n > 0 && (!x || !q || !radius || !half_height)) || (cap > 0 && !pairs) ||
      !(delta >= 0.0) || (pbc_enabled && (!pbc_min || !pbc_max)))
    return RG_ERR_ARG;
  Box box{};
  box.pbc = pbc_enabled ? 1 : 0;
  for (int k = 0; k < 3 && pbc_enabled; ++k) {
    box.lo[k] = pbc_min[k];
    box.hi[k] = pbc_max[k];
    box.L[k] = pbc_max[k] - pbc_min[k];
    if (!(box.L[k] > 0.0)) return RG_ERR_ARG;
  }
  NoAllocScratch* S = nullptr;
  int rc = na_scratch(&S);
  if (rc != RG_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int g = n > 0 ? (n + kNaBS - 1) / kNaBS : 1;
  const int gw = n > 0 ? (n + kNaBS / 32 - 1) / (kNaBS / 32) : 1;  // one warp per rod
  if (n > 0) {
    RGL k_na_seg<<<g, kNaBS, 0, st>>>(x, q, radius, half_height, n, S);
    RGL k_na_count<<<gw, kNaBS, 0, st>>>(n, box, delta, inv_mass, S);
  }
  RGL k_na_scan<<<1, 1024, 0, st>>>(n, S);
  RGL k_na_write<<<gw, kNaBS, 0, st>>>(n, box, delta, inv_mass, S, pairs, geom, cap, count);
  return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}
