// rg_api.cu - the C ABI of librodgpu.so (declared in include/rodgpu.h).
//
// Owns the device buffers of one system, sequences the per-step kernels of
// App::physicsStep (src/app/main.cpp:4333-4858) for the configured model, and
// turns device-side error bits into rg_status codes.  Capacity overflows
// (contacts, neighbour lists, history, colours) are recovered transparently:
// the state at the start of the call is kept in a device snapshot, the
// buffers grow, and the call re-runs from the snapshot.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "rg_internal.cuh"

using namespace rg;

namespace rg {

const char* kStatus[] = {"ok", "bad argument", "CUDA error", "capacity exceeded",
                         "non-finite state", "PSOR not converged", "no CUDA device",
                         "device wait timed out", "call out of order"};

int fail(rg_system* s, int code, const std::string& msg) {
  if (s) s->err_text = msg;
  return code;
}

int cuda_fail(rg_system* s, cudaError_t e, const char* where) {
  cudaGetLastError();
  return fail(s, RG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define RG_TRY2(sys, call, where)                   \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(sys, e_, where); \
  } while (0)
#define RG_TRY(call, where)                         \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(s, e_, where); \
  } while (0)

void bind_state(rg_system* s) {
  const int n = s->n;
  double* b = s->d_state;
  State& st = s->st;
  st.n = n;
  st.x = {b, b + n, b + 2 * n};
  st.q = {b + 3 * n, b + 4 * n, b + 5 * n, b + 6 * n};
  st.v = {b + 7 * n, b + 8 * n, b + 9 * n};
  st.w = {b + 10 * n, b + 11 * n, b + 12 * n};
  st.f = {b + 13 * n, b + 14 * n, b + 15 * n};
  st.tau = {b + 16 * n, b + 17 * n, b + 18 * n};
  double* p = s->d_props;
  st.r = p; st.h = p + n; st.mass = p + 2 * n; st.inv_mass = p + 3 * n; st.rest = p + 4 * n;
  st.I = {p + 5 * n, p + 6 * n, p + 7 * n};
  st.Iinv = {p + 8 * n, p + 9 * n, p + 10 * n};
  st.sbase = b;
  st.pbase = p;
}

size_t ctl_size(const rg_config& c) {
  int slots = c.nsc_velocity_iters;
  if (c.nsc_position_psor_iters + 2 > slots) slots = c.nsc_position_psor_iters + 2;
  if (slots < 4) slots = 4;
  return sizeof(Ctl) + sizeof(double) * (size_t)slots;
}

void free_contact_buffers(rg_system* s) {
  s->con.free_();
  cudaFree(s->csr.cnt); cudaFree(s->csr.off); cudaFree(s->csr.fill); cudaFree(s->csr.ent);
  s->csr = BodyCSR();
  History& H = s->hist;
  for (int k = 0; k < 2; ++k) { cudaFree(H.key[k]); cudaFree(H.val[k]); cudaFree(H.frame[k]); }
  cudaFree(H.touched); cudaFree(H.touched_off); cudaFree(H.kept);
  cudaFree(H.kept_off); cudaFree(H.newval);
  H = History();
  Nsc& N = s->nsc;
  cudaFree(N.row); cudaFree(N.lam); cudaFree(N.color); cudaFree(N.color_tmp); cudaFree(N.order);
  cudaFree(N.color_cnt); cudaFree(N.color_off); cudaFree(N.wkey); cudaFree(N.wlam); cudaFree(N.wn);
  cudaFree(N.xrow);
  cudaFree(N.dx); cudaFree(N.prow); cudaFree(N.pactive);
  cudaFree(N.pmax); cudaFree(N.cmask); cudaFree(N.owner); cudaFree(N.cursor); cudaFree(N.remaining);
  cudaFree(N.blk); cudaFree(N.slot_of); cudaFree(N.bar); cudaFree(N.view_dev); cudaFree(N.team_dev);
  N = Nsc();
  cudaFree(s->d_cf);
  s->d_cf = nullptr;
  s->scan.free_();
  cudaFree(s->d_feat); cudaFree(s->d_pred);
  s->d_feat = nullptr; s->d_pred = nullptr;
}

// Allocates every contact-sized buffer for capacity ccap and history hcap.
cudaError_t alloc_contact_buffers(rg_system* s, int ccap, int hcap) {
  const int n = s->n;
  s->ccap = ccap;
  ++s->buf_gen;
  cudaError_t e;
  if ((e = s->con.alloc(ccap))) return e;
  if ((e = cudaMalloc(&s->csr.cnt, sizeof(int) * (n + 1)))) return e;
  if ((e = cudaMalloc(&s->csr.off, sizeof(int) * (n + 1)))) return e;
  if ((e = cudaMalloc(&s->csr.fill, sizeof(int) * n))) return e;
  if ((e = cudaMalloc(&s->csr.ent, sizeof(int) * 2 * (size_t)ccap))) return e;
  History& H = s->hist;
  H.cap = hcap;
  for (int k = 0; k < 2; ++k) {
    if ((e = cudaMalloc(&H.key[k], sizeof(unsigned long long) * hcap))) return e;
    if ((e = cudaMalloc(&H.val[k], sizeof(double) * 3 * (size_t)hcap))) return e;
    if ((e = cudaMalloc(&H.frame[k], sizeof(long long) * hcap))) return e;
  }
  if ((e = cudaMalloc(&H.touched, sizeof(int) * (ccap + 1)))) return e;
  if ((e = cudaMalloc(&H.touched_off, sizeof(int) * (ccap + 1)))) return e;
  if ((e = cudaMalloc(&H.kept, sizeof(int) * (hcap + 1)))) return e;
  if ((e = cudaMalloc(&H.kept_off, sizeof(int) * (hcap + 1)))) return e;
  if ((e = cudaMalloc(&H.newval, sizeof(double) * 3 * (size_t)ccap))) return e;
  Nsc& N = s->nsc;
  if ((e = cudaMalloc(&N.row, sizeof(double) * kRowComps * (size_t)ccap))) return e;
  if ((e = cudaMalloc(&N.lam, sizeof(double) * 3 * (size_t)ccap))) return e;
  if ((e = cudaMalloc(&N.color, sizeof(int) * (ccap + 1)))) return e;
  if ((e = cudaMalloc(&N.color_tmp, sizeof(int) * ((size_t)ccap + 1024)))) return e;
  if ((e = cudaMalloc(&N.order, sizeof(int) * (ccap + 1)))) return e;
  if ((e = cudaMalloc(&N.color_cnt, sizeof(int) * (kMaxColors + 2)))) return e;
  if ((e = cudaMalloc(&N.color_off, sizeof(int) * (kMaxColors + 2)))) return e;
  N.wcap = ccap;
  if ((e = cudaMalloc(&N.wkey, sizeof(unsigned long long) * ccap))) return e;
  if ((e = cudaMalloc(&N.wlam, sizeof(double) * 3 * (size_t)ccap + sizeof(int) * (size_t)ccap))) return e;
  if ((e = cudaMalloc(&N.wn, sizeof(int)))) return e;
  if ((e = cudaMemset(N.wn, 0, sizeof(int)))) return e;
  if (s->export_on && (e = cudaMalloc(&N.xrow, sizeof(double) * kExportComps * (size_t)ccap))) return e;
  if ((e = cudaMalloc(&N.dx, sizeof(double) * 6 * (size_t)n))) return e;
  if ((e = cudaMemset(N.dx, 0, sizeof(double) * 6 * (size_t)n))) return e;
  if ((e = cudaMalloc(&N.prow, sizeof(double) * kPosComps * (size_t)ccap))) return e;
  if ((e = cudaMalloc(&N.pactive, sizeof(int) * ccap))) return e;
  if ((e = cudaMalloc(&N.pmax, sizeof(unsigned long long) * 2 * (size_t)n))) return e;
  if ((e = cudaMalloc(&N.cmask, sizeof(unsigned long long) * (size_t)n))) return e;
  if ((e = cudaMalloc(&N.owner, sizeof(int) * (size_t)n))) return e;
  if ((e = cudaMalloc(&N.cursor, sizeof(int) * (kMaxColors + 2)))) return e;
  if ((e = cudaMalloc(&N.remaining, sizeof(int) * 1024))) return e;
  if ((e = cudaMalloc(&N.blk, sizeof(int) * (s->coop_blocks + 32)))) return e;
  if ((e = cudaMalloc(&N.slot_of, sizeof(int) * (size_t)n))) return e;
  if ((e = cudaMemset(N.slot_of, 0xff, sizeof(int) * (size_t)n))) return e;
  if ((e = cudaMalloc(&N.bar, sizeof(unsigned int) * 8))) return e;
  if ((e = cudaMemset(N.bar, 0, sizeof(unsigned int) * 8))) return e;
  if ((e = cudaMalloc(&N.view_dev, nsc_view_bytes()))) return e;
  if ((e = cudaMalloc(&N.team_dev, nsc_team_bytes()))) return e;
  if ((e = cudaMalloc(&s->d_cf, sizeof(double) * (13 * (size_t)ccap + 64)))) return e;
  if ((e = cudaMalloc(&s->d_feat, sizeof(float) * 8 * (size_t)ccap))) return e;
  if ((e = cudaMalloc(&s->d_pred, sizeof(float) * 3 * (size_t)ccap))) return e;
  int scap = ccap + 1;
  if (hcap + 1 > scap) scap = hcap + 1;
  if (n + 1 > scap) scap = n + 1;
  if (s->det.ncells + 1 > scap) scap = s->det.ncells + 1;
  return s->scan.alloc(scap);
}

__global__ void k_ke(State st, Ctl* ctl, double* out) {
  __shared__ double sm[32];
  double ke = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n; i += gridDim.x * blockDim.x) {
    d3 v = st.v.ld(i), w = st.w.ld(i);
    ke += 0.5 * st.mass[i] * dot(v, v);
    ke += 0.5 * dot(w, rot_diag_apply(st.q.ld(i), st.I.ld(i), w));
  }
  ke = warp_sum(ke);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = ke;
  __syncthreads();
  if (threadIdx.x < 32) {
    double u = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 0.0;
    u = warp_sum(u);
    if (threadIdx.x == 0) out[blockIdx.x] = u;
  }
  (void)ctl;
}

constexpr int kKeBlocks = 64;

void ke_launch(rg_system* s) {
  if (!s->d_ke && cudaMalloc(&s->d_ke, sizeof(double) * kKeBlocks) != cudaSuccess) return;
  RGL k_ke<<<kKeBlocks, 256, 0, s->stream>>>(s->st, s->d_ctl, s->d_ke);
  cudaMemcpyAsync(s->h_ke, s->d_ke, sizeof(double) * kKeBlocks, cudaMemcpyDeviceToHost, s->stream);
}

double ke_sum(const rg_system* s) {
  if (!s->d_ke) return NAN;
  double ke = 0;
  for (int i = 0; i < kKeBlocks; ++i) ke += s->h_ke[i];
  return ke;
}

double kinetic_energy(rg_system* s) {
  ke_launch(s);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) return NAN;
  return ke_sum(s);
}

// Device snapshot of everything a step mutates: state, control words,
// current history table and the NSC warm cache.
cudaError_t snapshot_alloc(rg_system* s) {
  const int n = s->n;
  cudaError_t e = cudaSuccess;
  size_t need = sizeof(double) * 19 * (size_t)n;
  if (!s->d_snap && (e = cudaMalloc(&s->d_snap, need))) return e;
  const History& H = s->hist;
  if (s->snap_hcap != H.cap) {
    cudaFree(s->snap_hkey); cudaFree(s->snap_hval); cudaFree(s->snap_hframe);
    if ((e = cudaMalloc(&s->snap_hkey, sizeof(unsigned long long) * H.cap))) return e;
    if ((e = cudaMalloc(&s->snap_hval, sizeof(double) * 3 * (size_t)H.cap))) return e;
    if ((e = cudaMalloc(&s->snap_hframe, sizeof(long long) * H.cap))) return e;
    s->snap_hcap = H.cap;
  }
  const Nsc& N = s->nsc;
  const size_t wl_bytes = sizeof(double) * 3 * (size_t)N.wcap + sizeof(int) * (size_t)N.wcap;
  if (s->snap_wcap != N.wcap) {
    cudaFree(s->snap_wkey); cudaFree(s->snap_wlam);
    if ((e = cudaMalloc(&s->snap_wkey, sizeof(unsigned long long) * N.wcap))) return e;
    if ((e = cudaMalloc(&s->snap_wlam, wl_bytes))) return e;
    s->snap_wcap = N.wcap;
  }
  return e;
}

// The snapshot copies of one system: the whole state, and of the history
// table and the warm cache only their live entries (counts read on the
// device; restore_snapshot copies whole arrays back, and nothing reads an
// entry beyond the live count).
void snapshot_segments(rg_system* s, std::vector<CopySeg>& out) {
  const History& H = s->hist;
  const Nsc& N = s->nsc;
  const int* hn = &s->d_ctl->hist_n;
  const size_t hc = (size_t)H.cap, wc = (size_t)N.wcap;
  out.push_back({s->d_state, s->d_snap, sizeof(double) * 19 * (size_t)s->n, nullptr, 0, 0});
  out.push_back({H.key[H.cur], s->snap_hkey, sizeof(unsigned long long) * hc, hn, 8, 0});
  for (int c = 0; c < 3; ++c)
    out.push_back({H.val[H.cur] + c * hc, s->snap_hval + c * hc, sizeof(double) * hc, hn, 8, 0});
  out.push_back({H.frame[H.cur], s->snap_hframe, sizeof(long long) * hc, hn, 8, 0});
  out.push_back({N.wkey, s->snap_wkey, sizeof(unsigned long long) * wc, N.wn, 8, 0});
  for (int c = 0; c < 3; ++c)
    out.push_back({N.wlam + c * wc, s->snap_wlam + c * wc, sizeof(double) * wc, N.wn, 8, 0});
  out.push_back({N.wlam + 3 * wc, s->snap_wlam + 3 * wc, sizeof(int) * wc, N.wn, 4, 0});
}

// One block per segment (strided; segments are split into pieces of at most
// kCopyChunk bytes by the caller): 16-byte words when both ends allow it,
// each thread loading all of its words before storing any, else 4-byte
// words (every buffer here is 4-byte aligned and sized).
__global__ void k_copy_segments(const CopySeg* segs, int n) {
  constexpr int kPer = kCopyChunk / 16 / 256;  // 16-byte words per thread
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    CopySeg g = segs[k];
    if (g.count) {  // live part only
      const int c = *g.count;
      const unsigned long long live = c > 0 ? (unsigned long long)c * g.elem : 0ull;
      if (g.off >= live) continue;
      if (g.bytes > live - g.off) g.bytes = live - g.off;
    }
    const unsigned long long a = (unsigned long long)g.src | (unsigned long long)g.dst | g.bytes;
    if ((a & 15ull) == 0 && g.bytes <= (unsigned long long)kCopyChunk && blockDim.x == 256) {
      const uint4* src = static_cast<const uint4*>(g.src);
      uint4* dst = static_cast<uint4*>(g.dst);
      const int nv = (int)(g.bytes / 16);
      uint4 r[kPer];
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int i = threadIdx.x + u * 256;
        if (i < nv) r[u] = src[i];
      }
#pragma unroll
      for (int u = 0; u < kPer; ++u) {
        const int i = threadIdx.x + u * 256;
        if (i < nv) dst[i] = r[u];
      }
    } else if ((a & 15ull) == 0) {
      const uint4* src = static_cast<const uint4*>(g.src);
      uint4* dst = static_cast<uint4*>(g.dst);
      for (unsigned long long i = threadIdx.x; i < g.bytes / 16; i += blockDim.x) dst[i] = src[i];
    } else {
      const unsigned* src = static_cast<const unsigned*>(g.src);
      unsigned* dst = static_cast<unsigned*>(g.dst);
      for (unsigned long long i = threadIdx.x; i < g.bytes / 4; i += blockDim.x) dst[i] = src[i];
    }
  }
}

void split_segments(const std::vector<CopySeg>& in, std::vector<CopySeg>& out) {
  out.clear();
  for (const CopySeg& g : in)
    for (unsigned long long off = 0; off < g.bytes; off += kCopyChunk) {
      const unsigned long long nb = g.bytes - off < (unsigned long long)kCopyChunk ? g.bytes - off : kCopyChunk;
      out.push_back({static_cast<const char*>(g.src) + off, static_cast<char*>(g.dst) + off, nb, g.count, g.elem,
                     g.off + off});
    }
}

void copy_segments_launch(const CopySeg* d_segs, int n, cudaStream_t st) {
  if (n <= 0) return;
  RGL k_copy_segments<<<n < 2048 ? n : 2048, 256, 0, st>>>(d_segs, n);
}

__global__ void k_ctl_reset(Ctl* const* ctls, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    Ctl* c = ctls[k];
    c->err = 0;
    c->rebuilds = 0;
    c->sweeps_sum = 0;
    c->not_conv = 0;
    c->max_residual = 0;
    c->row_sweeps = 0;
    c->contact_steps = 0;
    c->near_rebuilds = 0;
    c->member_ns = 0;
    c->serial_ns = 0;
    c->det_valid = 0;
    c->bar_count = 0;
  }
}

__global__ void k_ctl_zero_time(Ctl* const* ctls, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    ctls[k]->member_ns = 0;
    ctls[k]->serial_ns = 0;
  }
}

void ctl_zero_time_launch(Ctl* const* d_ctls, int n, cudaStream_t st) {
  if (n <= 0) return;
  RGL k_ctl_zero_time<<<(n + 127) / 128, 128, 0, st>>>(d_ctls, n);
}

void ctl_reset_launch(Ctl* const* d_ctls, int n, cudaStream_t st) {
  if (n <= 0) return;
  RGL k_ctl_reset<<<(n + 127) / 128, 128, 0, st>>>(d_ctls, n);
}

cudaError_t take_snapshot(rg_system* s, Snapshot& sn, bool sync) {
  cudaError_t e = snapshot_alloc(s);
  if (e) return e;
  const int n = s->n;
  const size_t need = sizeof(double) * 19 * (size_t)n;
  const History& H = s->hist;
  const Nsc& N = s->nsc;
  const size_t wl_bytes = sizeof(double) * 3 * (size_t)N.wcap + sizeof(int) * (size_t)N.wcap;
  cudaStream_t st = s->stream;
  cudaMemcpyAsync(s->d_snap, s->d_state, need, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->snap_hkey, H.key[H.cur], sizeof(unsigned long long) * H.cap, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->snap_hval, H.val[H.cur], sizeof(double) * 3 * (size_t)H.cap, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->snap_hframe, H.frame[H.cur], sizeof(long long) * H.cap, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->snap_wkey, N.wkey, sizeof(unsigned long long) * N.wcap, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->snap_wlam, N.wlam, wl_bytes, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(s->h_snapctl, s->d_ctl, s->ctl_bytes, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(s->h_wn, N.wn, sizeof(int), cudaMemcpyDeviceToHost, st);
  sn.hist_cur = H.cur;
  if (!sync) return cudaGetLastError();
  e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) finish_snapshot(s, sn);
  return e;
}

void finish_snapshot(rg_system* s, Snapshot& sn) {
  sn.ctl.resize(s->ctl_bytes);
  std::memcpy(sn.ctl.data(), s->h_snapctl, s->ctl_bytes);
  sn.wn = *s->h_wn;
}

// Puts the snapshot back into the live buffers (same capacities).
cudaError_t restore_snapshot(rg_system* s, const Snapshot& sn) {
  History& H = s->hist;
  const Nsc& N = s->nsc;
  H.cur = sn.hist_cur;
  const size_t wl_bytes = sizeof(double) * 3 * (size_t)N.wcap + sizeof(int) * (size_t)N.wcap;
  cudaMemcpy(s->d_state, s->d_snap, sizeof(double) * 19 * (size_t)s->n, cudaMemcpyDeviceToDevice);
  cudaMemcpy(H.key[H.cur], s->snap_hkey, sizeof(unsigned long long) * H.cap, cudaMemcpyDeviceToDevice);
  cudaMemcpy(H.val[H.cur], s->snap_hval, sizeof(double) * 3 * (size_t)H.cap, cudaMemcpyDeviceToDevice);
  cudaMemcpy(H.frame[H.cur], s->snap_hframe, sizeof(long long) * H.cap, cudaMemcpyDeviceToDevice);
  cudaMemcpy(N.wkey, s->snap_wkey, sizeof(unsigned long long) * N.wcap, cudaMemcpyDeviceToDevice);
  cudaMemcpy(N.wlam, s->snap_wlam, wl_bytes, cudaMemcpyDeviceToDevice);
  cudaMemcpy(N.wn, &sn.wn, sizeof(int), cudaMemcpyHostToDevice);
  std::memcpy(s->h_ctl, sn.ctl.data(), s->ctl_bytes);
  return cudaMemcpy(s->d_ctl, sn.ctl.data(), s->ctl_bytes, cudaMemcpyHostToDevice);
}

}  // namespace rg

extern "C" {

int rg_abi_version(void) { return RG_ABI_VERSION; }

const char* rg_status_string(int status) {
  if (status < 0 || status > RG_ERR_STATE) return "unknown status";
  return kStatus[status];
}

const char* rg_last_error(const rg_system* s) { return s ? s->err_text.c_str() : ""; }

int rg_create(const rg_config* cfg, rg_system** out) {
  if (!cfg || !out) return RG_ERR_ARG;
  *out = nullptr;
  if (cfg->n_bodies <= 0 || cfg->model < RG_MODEL_NONE || cfg->model > RG_MODEL_HERTZ_MINDLIN ||
      !(cfg->dt > 0.0))
    return RG_ERR_ARG;
  if (cfg->psor_order != RG_ORDER_COLORED) return RG_ERR_ARG;  // device order is coloured
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  rg_system* s = new rg_system();
  s->cfg = *cfg;
  s->n = cfg->n_bodies;
  cudaGetDevice(&s->device);
  cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device);
  s->box.pbc = cfg->pbc_enabled ? 1 : 0;
  for (int k = 0; k < 3; ++k) {
    s->box.lo[k] = cfg->pbc_min[k];
    s->box.hi[k] = cfg->pbc_max[k];
    s->box.L[k] = cfg->pbc_max[k] - cfg->pbc_min[k];
  }
  if (s->box.pbc && !(s->box.L[0] > 0 && s->box.L[1] > 0 && s->box.L[2] > 0)) {
    delete s;
    return RG_ERR_ARG;
  }
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) ||
      (e = cudaMalloc(&s->d_state, sizeof(double) * 19 * (size_t)s->n)) ||
      (e = cudaMalloc(&s->d_props, sizeof(double) * 11 * (size_t)s->n)) ||
      (e = cudaMemset(s->d_state, 0, sizeof(double) * 19 * (size_t)s->n)) ||
      (e = cudaMemset(s->d_props, 0, sizeof(double) * 11 * (size_t)s->n)) ||
      (e = cudaMallocHost(&s->h_stage, sizeof(double) * 19 * (size_t)s->n))) {
    rg_destroy(s);
    return RG_ERR_CUDA;
  }
  s->ctl_bytes = ctl_size(*cfg);
  if ((e = cudaMalloc(&s->d_ctl, s->ctl_bytes)) || (e = cudaMemset(s->d_ctl, 0, s->ctl_bytes)) ||
      (e = cudaMallocHost(&s->h_ctl, s->ctl_bytes)) || (e = cudaMallocHost(&s->h_snapctl, s->ctl_bytes)) ||
      (e = cudaMallocHost(&s->h_wn, sizeof(int))) || (e = cudaMallocHost(&s->h_ke, sizeof(double) * 64))) {
    rg_destroy(s);
    return RG_ERR_CUDA;
  }
  bind_state(s);
  // identity orientations
  std::vector<double> one(s->n, 1.0);
  cudaMemcpy(s->st.q.w, one.data(), sizeof(double) * s->n, cudaMemcpyHostToDevice);
  // persistent kernels run as many blocks per SM as fit (co-residency is
  // guaranteed by the cooperative launch attribute)
  s->coop_blocks = s->sm_count * nsc_blocks_per_sm();
  s->team_blocks = cfg->team_blocks;  // NSC team size; 0 = automatic
  *out = s;
  return RG_OK;
}

int rg_destroy(rg_system* s) {
  if (!s) return RG_ERR_ARG;
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->vgraph) cudaGraphExecDestroy(s->vgraph);
  free_contact_buffers(s);
  detector_free(s);
  cudaFree(s->d_state); cudaFree(s->d_props); cudaFree(s->d_ctl); cudaFree(s->d_snap);
  cudaFree(s->snap_hkey); cudaFree(s->snap_hval); cudaFree(s->snap_hframe);
  cudaFree(s->snap_wkey); cudaFree(s->snap_wlam);
  mlp_free(s);
  cudaFree(s->d_rec_x); cudaFree(s->d_rec_y); cudaFree(s->d_ke);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_snapctl) cudaFreeHost(s->h_snapctl);
  if (s->h_wn) cudaFreeHost(s->h_wn);
  if (s->h_ke) cudaFreeHost(s->h_ke);
  if (s->h_stage) cudaFreeHost(s->h_stage);
  for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return RG_OK;
}

int rg_get_config(const rg_system* s, rg_config* cfg) {
  if (!s || !cfg) return RG_ERR_ARG;
  *cfg = s->cfg;
  return RG_OK;
}

int rg_set_bodies(rg_system* s, const double* radius, const double* half_height,
                  const double* mass, const double* inertia, const double* restitution) {
  if (!s || !radius || !half_height || !mass || !inertia) return RG_ERR_ARG;
  const int n = s->n;
  std::vector<double> p(11 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    if (!(radius[i] > 0) || !(half_height[i] >= 0)) return fail(s, RG_ERR_ARG, "radius must be > 0 and half height >= 0");
    bool dyn = mass[i] > 0;
    p[i] = radius[i];
    p[n + i] = half_height[i];
    p[2 * n + i] = dyn ? mass[i] : 0.0;
    p[3 * n + i] = dyn ? 1.0 / mass[i] : 0.0;
    p[4 * n + i] = restitution ? restitution[i] : 0.2;
    for (int k = 0; k < 3; ++k) {
      double I = dyn ? inertia[3 * i + k] : 0.0;
      p[(5 + k) * (size_t)n + i] = I;
      p[(8 + k) * (size_t)n + i] = (dyn && I > 0) ? 1.0 / I : 0.0;
    }
  }
  RG_TRY(cudaMemcpy(s->d_props, p.data(), sizeof(double) * p.size(), cudaMemcpyHostToDevice), "upload bodies");
  free_contact_buffers(s);
  detector_free(s);
  cudaError_t e = detector_alloc(s);
  if (e == cudaErrorInvalidValue)
    return fail(s, RG_ERR_ARG, "periodic box smaller than twice the contact range with more than 4096 bodies");
  if (e) return cuda_fail(s, e, "detector_alloc");
  int ccap = 4 * n > 4096 ? 4 * n : 4096;
  RG_TRY(alloc_contact_buffers(s, ccap, 2 * ccap), "alloc contact buffers");
  force_rebuild(s);
  RG_TRY(cudaStreamSynchronize(s->stream), "set_bodies sync");
  s->bodies_set = true;
  s->contacts_fresh = false;
  return RG_OK;
}

int rg_set_state(rg_system* s, const double* x, const double* q, const double* v, const double* w,
                 const double* f, const double* tau) {
  if (!s || !x || !q || !v || !w) return RG_ERR_ARG;
  const int n = s->n;
  double* b = s->h_stage;
  std::memset(b, 0, sizeof(double) * 19 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      b[(size_t)k * n + i] = x[3 * i + k];
      b[(size_t)(7 + k) * n + i] = v[3 * i + k];
      b[(size_t)(10 + k) * n + i] = w[3 * i + k];
      if (f) b[(size_t)(13 + k) * n + i] = f[3 * i + k];
      if (tau) b[(size_t)(16 + k) * n + i] = tau[3 * i + k];
    }
    for (int k = 0; k < 4; ++k) b[(size_t)(3 + k) * n + i] = q[4 * i + k];
  }
  // A NaN or infinite component would reach the cell grid and every force
  // law; it is refused here, before any device work, and the device state
  // stays what it was.
  for (size_t k = 0; k < 19 * (size_t)n; ++k)
    if (!std::isfinite(b[k])) return fail(s, RG_ERR_NONFINITE, "non-finite component in the uploaded state");
  // The neighbour lists need no forced rebuild: the displacement check
  // against the positions of the last build catches any jump of the state.
  RG_TRY(cudaMemcpyAsync(s->d_state, b, sizeof(double) * 19 * (size_t)n, cudaMemcpyHostToDevice,
                         s->stream), "upload state");
  RG_TRY(cudaStreamSynchronize(s->stream), "set_state sync");
  s->state_set = true;
  s->contacts_fresh = false;
  return RG_OK;
}

int rg_get_state(const rg_system* s, double* x, double* q, double* v, double* w, double* f, double* tau) {
  if (!s) return RG_ERR_ARG;
  const int n = s->n;
  const double* b = s->h_stage;
  cudaError_t e = cudaMemcpyAsync(s->h_stage, s->d_state, sizeof(double) * 19 * (size_t)n,
                                  cudaMemcpyDeviceToHost, s->stream);
  if (!e) e = cudaStreamSynchronize(s->stream);
  if (e) return cuda_fail(const_cast<rg_system*>(s), e, "download state");
  for (int i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k) {
      if (x) x[3 * i + k] = b[(size_t)k * n + i];
      if (v) v[3 * i + k] = b[(size_t)(7 + k) * n + i];
      if (w) w[3 * i + k] = b[(size_t)(10 + k) * n + i];
      if (f) f[3 * i + k] = b[(size_t)(13 + k) * n + i];
      if (tau) tau[3 * i + k] = b[(size_t)(16 + k) * n + i];
    }
    if (q)
      for (int k = 0; k < 4; ++k) q[4 * i + k] = b[(size_t)(3 + k) * n + i];
  }
  return RG_OK;
}

}  // extern "C"

namespace rg {

// One velocity-Verlet step (main.cpp:4610-4810): forces at t, half kick and
// drift, forces at t + dt, second half kick.  Each evaluation starts from
// zero forces (integrateSecondHalf clears them for the next frame,
// integrator.cpp:156-158, and the step clears them again before the second
// evaluation); the per-body sums are fused into the two kick kernels.
static void verlet_step(rg_system* s) {
  force_eval_launch(s, EvalTail::kHalfPos);  // forces at t (reuses fresh contacts), kick and drift
  s->contacts_fresh = false;
  force_eval_launch(s, EvalTail::kSecondHalf, true);  // forces at t + dt, second kick
  s->contacts_fresh = true;  // positions unchanged until the next drift
}

// Captures one Verlet step (entered with fresh contacts) as a CUDA graph.
// Every launch of the step is decided on the host from state that a whole
// step leaves as it found it (fresh contacts, the history ping-pong index),
// so the same graph serves every step until buffers are reallocated.
static bool capture_verlet_step(rg_system* s) {
  if (s->vgraph) {
    cudaGraphExecDestroy(s->vgraph);
    s->vgraph = nullptr;
  }
  const long long l0 = g_launches;
  const int cur = s->hist.cur;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  verlet_step(s);
  cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  s->vgraph_kernels = g_launches - l0;
  g_launches = l0;  // counted when the graph runs
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s->vgraph, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess || s->hist.cur != cur || !s->contacts_fresh) {
    cudaGetLastError();
    if (s->vgraph) cudaGraphExecDestroy(s->vgraph);
    s->vgraph = nullptr;
    s->hist.cur = cur;
    return false;
  }
  s->vgraph_gen = s->buf_gen;
  s->vgraph_cur = cur;
  return true;
}

void launch_steps(rg_system* s, int nsteps) {
  const int model = s->cfg.model;
  if (model == RG_MODEL_NSC) {
    if (nsteps > 0) nsc_run_launch(s, nsteps);  // one persistent launch for all steps
    return;
  }
  if (model != RG_MODEL_HARMONIC && model != RG_MODEL_HERTZ_MINDLIN) return;
  int k = 0;
  if (nsteps > 0 && !s->contacts_fresh) {  // the first evaluation detects
    verlet_step(s);
    k = 1;
  }
  // The rest replay one captured step (stage timers need the plain launches).
  if (nsteps - k >= 2 && !s->prof_on) {
    bool ok = s->vgraph && s->vgraph_gen == s->buf_gen && s->vgraph_cur == s->hist.cur;
    if (!ok) ok = capture_verlet_step(s);
    if (ok)
      for (; k < nsteps; ++k) {
        RGL cudaGraphLaunch(s->vgraph, s->stream);
        g_launches += s->vgraph_kernels - 1;
      }
  }
  for (; k < nsteps; ++k) verlet_step(s);
}

// Grows the buffer named by the error bits.  Returns false if nothing grew.
bool grow(rg_system* s, int err) {
  bool grew = false;
  if (err & (ERR_CONTACT_CAP | ERR_HIST_CAP)) {
    // keep the history table contents: copy the current table to host
    History& H = s->hist;
    int hn = s->h_ctl->hist_n;
    std::vector<unsigned long long> hk(hn);
    std::vector<double> hv(3 * (size_t)hn);
    std::vector<long long> hf(hn);
    int cur = H.cur;
    cudaMemcpy(hk.data(), H.key[cur], sizeof(unsigned long long) * hn, cudaMemcpyDeviceToHost);
    for (int k = 0; k < 3; ++k)
      cudaMemcpy(hv.data() + (size_t)k * hn, H.val[cur] + (size_t)k * H.cap, sizeof(double) * hn,
                 cudaMemcpyDeviceToHost);
    cudaMemcpy(hf.data(), H.frame[cur], sizeof(long long) * hn, cudaMemcpyDeviceToHost);
    // warm cache
    int wn = 0;
    cudaMemcpy(&wn, s->nsc.wn, sizeof(int), cudaMemcpyDeviceToHost);
    std::vector<unsigned long long> wk(wn);
    std::vector<double> wl(3 * (size_t)wn);
    cudaMemcpy(wk.data(), s->nsc.wkey, sizeof(unsigned long long) * wn, cudaMemcpyDeviceToHost);
    for (int k = 0; k < 3; ++k)
      cudaMemcpy(wl.data() + (size_t)k * wn, s->nsc.wlam + (size_t)k * s->nsc.wcap, sizeof(double) * wn,
                 cudaMemcpyDeviceToHost);
    int ccap = s->ccap, hcap = H.cap;
    if (err & ERR_CONTACT_CAP) ccap *= 2;
    if (err & ERR_HIST_CAP) hcap *= 2;
    if (hcap < 2 * ccap) hcap = 2 * ccap;
    free_contact_buffers(s);
    if (alloc_contact_buffers(s, ccap, hcap)) return false;
    History& G = s->hist;
    G.cur = 0;
    cudaMemcpy(G.key[0], hk.data(), sizeof(unsigned long long) * hn, cudaMemcpyHostToDevice);
    for (int k = 0; k < 3; ++k)
      cudaMemcpy(G.val[0] + (size_t)k * G.cap, hv.data() + (size_t)k * hn, sizeof(double) * hn,
                 cudaMemcpyHostToDevice);
    cudaMemcpy(G.frame[0], hf.data(), sizeof(long long) * hn, cudaMemcpyHostToDevice);
    cudaMemcpy(s->nsc.wkey, wk.data(), sizeof(unsigned long long) * wn, cudaMemcpyHostToDevice);
    for (int k = 0; k < 3; ++k)
      cudaMemcpy(s->nsc.wlam + (size_t)k * s->nsc.wcap, wl.data() + (size_t)k * wn, sizeof(double) * wn,
                 cudaMemcpyHostToDevice);
    cudaMemcpy(s->nsc.wn, &wn, sizeof(int), cudaMemcpyHostToDevice);
    grew = true;
  }
  if (err & ERR_NBR_CAP) {
    int nb = s->det.maxnb * 2;
    detector_free(s);
    s->det.maxnb = nb;
    if (detector_alloc(s)) return false;
    if (s->det.ncells + 1 > s->scan.cap) {
      s->scan.free_();
      s->scan.alloc(s->det.ncells + 1);
    }
    grew = true;
  }
  return grew;
}

// Per-call counters start from the snapshot's control words.
cudaError_t reset_call_ctl(rg_system* s, const Snapshot& sn) {
  Ctl* h = s->h_ctl;
  std::memcpy(h, sn.ctl.data(), s->ctl_bytes);
  h->err = 0;
  h->rebuilds = 0;
  h->sweeps_sum = 0;
  h->not_conv = 0;
  h->max_residual = 0;
  h->row_sweeps = 0;
  h->contact_steps = 0;
  h->near_rebuilds = 0;
  h->member_ns = 0;
  h->serial_ns = 0;
  h->det_valid = 0;
  h->bar_count = 0;
  return cudaMemcpyAsync(s->d_ctl, h, s->ctl_bytes, cudaMemcpyHostToDevice, s->stream);
}

// Turns the error bits of a finished call into a status.  Capacity errors
// restore the snapshot, grow the buffers and ask for a retry (RG_OK with
// *retry set).
int resolve_call(rg_system* s, Snapshot& sn, int err, bool* retry) {
  *retry = false;
  if (!err) return RG_OK;
  // Every failure puts back the state, history and warm cache the call
  // started from, so the handle stays usable after an error status.
  cudaError_t e = restore_snapshot(s, sn);
  if (e) return cuda_fail(s, e, "restore");
  if (err & (ERR_TIMEOUT | ERR_NONFINITE | ERR_COLOR)) {
    std::memcpy(s->h_ctl, sn.ctl.data(), s->ctl_bytes);
    reinterpret_cast<Ctl*>(s->h_ctl)->rebuild = 1;
    s->contacts_fresh = false;
    e = cudaMemcpyAsync(s->d_ctl, s->h_ctl, s->ctl_bytes, cudaMemcpyHostToDevice, s->stream);
    if (!e) e = cudaStreamSynchronize(s->stream);
    if (e) return cuda_fail(s, e, "restore control words");
  }
  if (err & ERR_TIMEOUT) return fail(s, RG_ERR_TIMEOUT, "a device-side barrier timed out");
  if (err & ERR_NONFINITE) return fail(s, RG_ERR_NONFINITE, "non-finite body state");
  if (err & ERR_COLOR) return fail(s, RG_ERR_CAPACITY, "contact graph needs more than 64 colours");
  if (!grow(s, err)) return fail(s, RG_ERR_CAPACITY, "could not grow device buffers");
  e = take_snapshot(s, sn);
  if (e) return cuda_fail(s, e, "snapshot");
  reinterpret_cast<Ctl*>(sn.ctl.data())->rebuild = 1;
  s->contacts_fresh = false;
  *retry = true;
  return RG_OK;
}

void fill_stats(rg_system* s, int nsteps, rg_step_stats* stats, bool ke_launched) {
  Ctl* h = s->h_ctl;
  std::memset(stats, 0, sizeof(*stats));
  stats->steps = nsteps;
  stats->contacts = s->cfg.model == RG_MODEL_NSC ? h->vel_contacts : h->contacts;
  stats->collisions = h->collisions;
  stats->psor_sweeps = h->sweeps_sum;
  stats->psor_sweeps_last = h->sweeps_last;
  stats->list_rebuilds = h->rebuilds;
  stats->colors = h->colors;
  stats->history_size = h->hist_n;
  stats->residual = h->residual;
  stats->jn_sum = h->jn_sum;
  stats->jt_sum = h->jt_sum;
  stats->potential_energy = h->pe;
  stats->max_residual = h->max_residual;
  stats->not_converged = h->not_conv;
  stats->device_ms = s->last_call_ms;
  stats->psor_row_sweeps = h->row_sweeps;
  stats->kernel_launches = s->last_call_launches;
  stats->contact_steps = h->contact_steps;
  stats->near_rebuilds = h->near_rebuilds;
  stats->kinetic_energy = ke_launched ? ke_sum(s) : kinetic_energy(s);
}

}  // namespace rg

extern "C" {

int rg_step(rg_system* s, int nsteps, rg_step_stats* stats) {
  if (!s || nsteps < 0) return RG_ERR_ARG;
  if (!s->bodies_set || !s->state_set) return fail(s, RG_ERR_STATE, "set bodies and state before stepping");
  if (s->cfg.model == RG_MODEL_NSC && s->cfg.nsc_warm_start == RG_WARM_MLP && !s->mlp_ready)
    return fail(s, RG_ERR_STATE, "learned warm start selected but no network is loaded (rg_mlp_train or rg_mlp_set_params)");
  Snapshot sn;
  RG_TRY(take_snapshot(s, sn), "snapshot");
  for (int attempt = 0; attempt < 8; ++attempt) {
    RG_TRY(reset_call_ctl(s, sn), "ctl upload");
    s->rec_stage.clear(); s->rec_a.clear(); s->rec_b.clear(); s->ev_used = 0;
    int ev0 = prof_event(s), ev1 = prof_event(s);
    const long long l0 = g_launches;
    cudaEventRecord(s->ev_pool[ev0], s->stream);
    launch_steps(s, nsteps);
    cudaEventRecord(s->ev_pool[ev1], s->stream);
    cudaError_t e = cudaGetLastError();
    if (e) return cuda_fail(s, e, "kernel launch");
    Ctl* h = s->h_ctl;
    RG_TRY(cudaMemcpyAsync(h, s->d_ctl, s->ctl_bytes, cudaMemcpyDeviceToHost, s->stream), "ctl download");
    RG_TRY(cudaStreamSynchronize(s->stream), "step");
    float call_ms = 0;
    cudaEventElapsedTime(&call_ms, s->ev_pool[ev0], s->ev_pool[ev1]);
    s->last_call_ms = call_ms;
    s->last_call_launches = g_launches - l0;
    if (!h->err) {
      prof_resolve(s);
      break;
    }
    s->rec_stage.clear(); s->rec_a.clear(); s->rec_b.clear(); s->ev_used = 0;
    bool retry = false;
    int rc = resolve_call(s, sn, h->err, &retry);
    if (rc != RG_OK) return rc;
    if (attempt == 7) return fail(s, RG_ERR_CAPACITY, "capacity retries exhausted");
  }
  if (stats) fill_stats(s, nsteps, stats);
  return RG_OK;
}

int rg_detect(rg_system* s, double delta, int32_t* pairs, double* geom, double* shift, size_t cap,
              size_t* n) {
  if (!s || !n) return RG_ERR_ARG;
  if (!s->bodies_set || !s->state_set) return fail(s, RG_ERR_STATE, "set bodies and state first");
  if (delta > s->det.margin) return fail(s, RG_ERR_ARG, "delta exceeds the neighbour-list margin of this model");
  for (int attempt = 0; attempt < 8; ++attempt) {
    Ctl* h = s->h_ctl;
    RG_TRY(cudaMemcpy(h, s->d_ctl, s->ctl_bytes, cudaMemcpyDeviceToHost), "ctl");
    h->err = 0;
    RG_TRY(cudaMemcpy(s->d_ctl, h, s->ctl_bytes, cudaMemcpyHostToDevice), "ctl");
    detect_launch(s, delta, true);
    RG_TRY(cudaGetLastError(), "detect launch");
    RG_TRY(cudaMemcpyAsync(h, s->d_ctl, s->ctl_bytes, cudaMemcpyDeviceToHost, s->stream), "ctl");
    RG_TRY(cudaStreamSynchronize(s->stream), "detect");
    if (!h->err) break;
    if (h->err & ERR_TIMEOUT) return fail(s, RG_ERR_TIMEOUT, "a device-side wait timed out in detection");
    if (h->err & ERR_NONFINITE) return fail(s, RG_ERR_NONFINITE, "non-finite body state");
    if (attempt == 7) return fail(s, RG_ERR_CAPACITY, "capacity retries exhausted");
    if (!grow(s, h->err)) return fail(s, RG_ERR_CAPACITY, "could not grow device buffers");
    force_rebuild(s);
  }
  s->contacts_fresh = false;  // the force path must rebuild its CSR
  const int C = s->h_ctl->contacts;
  if (C < 0 || C > s->ccap) return fail(s, RG_ERR_CAPACITY, "contact count exceeds the contact buffer");
  *n = (size_t)C;
  size_t m = cap < (size_t)C ? cap : (size_t)C;
  if (m) {
    std::vector<int> a(m), b(m), t(m);
    RG_TRY(cudaMemcpy(a.data(), s->con.a, sizeof(int) * m, cudaMemcpyDeviceToHost), "contacts");
    RG_TRY(cudaMemcpy(b.data(), s->con.b, sizeof(int) * m, cudaMemcpyDeviceToHost), "contacts");
    RG_TRY(cudaMemcpy(t.data(), s->con.type, sizeof(int) * m, cudaMemcpyDeviceToHost), "contacts");
    std::vector<double> g(14 * m);
    for (int k = 0; k < 14; ++k)
      RG_TRY(cudaMemcpy(g.data() + (size_t)k * m, s->con.comp(k), sizeof(double) * m, cudaMemcpyDeviceToHost),
             "contacts");
    for (size_t i = 0; i < m; ++i) {
      if (pairs) { pairs[2 * i] = a[i]; pairs[2 * i + 1] = b[i]; }
      if (geom) {
        double* o = geom + 12 * i;
        for (int k = 0; k < 9; ++k) o[k] = g[(size_t)k * m + i];
        o[9] = g[12 * m + i];
        o[10] = g[13 * m + i];
        o[11] = (double)t[i];
      }
      if (shift)
        for (int k = 0; k < 3; ++k) shift[3 * i + k] = g[(size_t)(9 + k) * m + i];
    }
  }
  return (size_t)C > cap ? RG_ERR_CAPACITY : RG_OK;
}

int rg_get_impulses(const rg_system* s, int32_t* pairs, double* lambda, int32_t* color, size_t cap,
                    size_t* n) {
  if (!s || !n) return RG_ERR_ARG;
  int wn = 0;
  cudaMemcpy(&wn, s->nsc.wn, sizeof(int), cudaMemcpyDeviceToHost);
  *n = (size_t)wn;
  size_t m = cap < (size_t)wn ? cap : (size_t)wn;
  if (m) {
    std::vector<unsigned long long> k(m);
    std::vector<double> l(3 * m);
    std::vector<int> c(m);
    cudaMemcpy(k.data(), s->nsc.wkey, sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost);
    for (int j = 0; j < 3; ++j)
      cudaMemcpy(l.data() + (size_t)j * m, s->nsc.wlam + (size_t)j * s->nsc.wcap, sizeof(double) * m,
                 cudaMemcpyDeviceToHost);
    const int* wcol = reinterpret_cast<const int*>(s->nsc.wlam + 3 * (size_t)s->nsc.wcap);
    cudaMemcpy(c.data(), wcol, sizeof(int) * m, cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < m; ++i) {
      if (pairs) { pairs[2 * i] = (int32_t)(k[i] >> 32); pairs[2 * i + 1] = (int32_t)(k[i] & 0xffffffffu); }
      if (lambda) for (int j = 0; j < 3; ++j) lambda[3 * i + j] = l[(size_t)j * m + i];
      if (color) color[i] = c[i];
    }
  }
  return (size_t)wn > cap ? RG_ERR_CAPACITY : RG_OK;
}

int rg_set_network_export(rg_system* s, int enable) {
  if (!s) return RG_ERR_ARG;
  if (s->cfg.model != RG_MODEL_NSC) return fail(s, RG_ERR_ARG, "the contact-network export needs the nsc model");
  s->export_on = enable != 0;
  if (s->export_on && !s->nsc.xrow) {
    RG_TRY(cudaMalloc(&s->nsc.xrow, sizeof(double) * kExportComps * (size_t)s->nsc.wcap), "export buffer");
    RG_TRY(cudaMemset(s->nsc.xrow, 0, sizeof(double) * kExportComps * (size_t)s->nsc.wcap), "export buffer");
  }
  return RG_OK;
}

int rg_get_contact_network(const rg_system* s, int32_t* pairs, double* rows, size_t cap, size_t* n) {
  if (!s || !n) return RG_ERR_ARG;
  rg_system* m = const_cast<rg_system*>(s);
  if (!s->export_on || !s->nsc.xrow) return fail(m, RG_ERR_STATE, "enable the export before stepping");
  int wn = 0;
  RG_TRY2(m, cudaMemcpy(&wn, s->nsc.wn, sizeof(int), cudaMemcpyDeviceToHost), "network count");
  *n = (size_t)wn;
  const size_t k = cap < (size_t)wn ? cap : (size_t)wn;
  if (k) {
    const size_t W = (size_t)s->nsc.wcap;
    std::vector<unsigned long long> key(k);
    std::vector<double> lam(3 * k), xr(kExportComps * k);
    RG_TRY2(m, cudaMemcpy(key.data(), s->nsc.wkey, sizeof(unsigned long long) * k, cudaMemcpyDeviceToHost), "keys");
    for (int j = 0; j < 3; ++j)
      RG_TRY2(m, cudaMemcpy(lam.data() + j * k, s->nsc.wlam + j * W, sizeof(double) * k, cudaMemcpyDeviceToHost),
              "impulses");
    for (int j = 0; j < kExportComps; ++j)
      RG_TRY2(m, cudaMemcpy(xr.data() + j * k, s->nsc.xrow + j * W, sizeof(double) * k, cudaMemcpyDeviceToHost),
              "export rows");
    // contact point and post-solve normal velocity from the current state
    // (App::logNetworkFrame, main.cpp:3670-3684)
    const size_t N = (size_t)s->n;
    std::vector<double> st(19 * N);
    RG_TRY2(m, cudaMemcpy(st.data(), s->d_state, sizeof(double) * 19 * N, cudaMemcpyDeviceToHost), "state");
    auto comp = [&](int c, size_t i) { return st[(size_t)c * N + i]; };
    for (size_t i = 0; i < k; ++i) {
      const size_t a = (size_t)(key[i] >> 32), b = (size_t)(key[i] & 0xffffffffu);
      const double nv[3] = {xr[0 * k + i], xr[1 * k + i], xr[2 * k + i]};
      const double ra[3] = {xr[3 * k + i], xr[4 * k + i], xr[5 * k + i]};
      const double rb[3] = {xr[6 * k + i], xr[7 * k + i], xr[8 * k + i]};
      double va[3], vb[3];
      for (int d = 0; d < 3; ++d) {
        const int e = (d + 1) % 3, f = (d + 2) % 3;  // (w x r)_d = w_e r_f - w_f r_e
        va[d] = comp(7 + d, a) + (comp(10 + e, a) * ra[f] - comp(10 + f, a) * ra[e]);
        vb[d] = comp(7 + d, b) + (comp(10 + e, b) * rb[f] - comp(10 + f, b) * rb[e]);
      }
      double vn_post = 0.0;
      for (int d = 0; d < 3; ++d) vn_post += nv[d] * (vb[d] - va[d]);
      if (pairs) { pairs[2 * i] = (int32_t)a; pairs[2 * i + 1] = (int32_t)b; }
      if (rows) {
        double* o = rows + 12 * i;
        for (int d = 0; d < 3; ++d) { o[d] = comp(d, a) + ra[d]; o[3 + d] = nv[d]; }
        o[6] = xr[9 * k + i];
        o[7] = lam[i]; o[8] = lam[k + i]; o[9] = lam[2 * k + i];
        o[10] = xr[10 * k + i];
        o[11] = vn_post;
      }
    }
  }
  return (size_t)wn > cap ? RG_ERR_CAPACITY : RG_OK;
}

int rg_compute_forces(rg_system* s, double* f, double* tau, double* pe) {
  if (!s) return RG_ERR_ARG;
  if (!s->bodies_set || !s->state_set) return fail(s, RG_ERR_STATE, "set bodies and state first");
  if (s->cfg.model != RG_MODEL_HARMONIC && s->cfg.model != RG_MODEL_HERTZ_MINDLIN)
    return fail(s, RG_ERR_ARG, "force evaluation needs the harmonic or hertz-mindlin model");
  Snapshot sn;
  RG_TRY(take_snapshot(s, sn), "snapshot");
  for (int attempt = 0; attempt < 8; ++attempt) {
    Ctl* h = s->h_ctl;
    std::memcpy(h, sn.ctl.data(), s->ctl_bytes);
    h->err = 0;
    RG_TRY(cudaMemcpyAsync(s->d_ctl, h, s->ctl_bytes, cudaMemcpyHostToDevice, s->stream), "ctl");
    clear_forces_launch(s);
    s->contacts_fresh = false;
    force_eval_launch(s);
    RG_TRY(cudaGetLastError(), "force launch");
    RG_TRY(cudaMemcpyAsync(h, s->d_ctl, s->ctl_bytes, cudaMemcpyDeviceToHost, s->stream), "ctl");
    RG_TRY(cudaStreamSynchronize(s->stream), "forces");
    if (!h->err) break;
    if (h->err & ERR_TIMEOUT) return fail(s, RG_ERR_TIMEOUT, "a device-side wait timed out in force evaluation");
    if (h->err & ERR_NONFINITE) return fail(s, RG_ERR_NONFINITE, "non-finite body state");
    if (h->err & ERR_COLOR) return fail(s, RG_ERR_CAPACITY, "force evaluation failed");
    if (attempt == 7) return fail(s, RG_ERR_CAPACITY, "capacity retries exhausted");
    int err = h->err;
    RG_TRY(restore_snapshot(s, sn), "restore");
    if (!grow(s, err)) return fail(s, RG_ERR_CAPACITY, "could not grow device buffers");
    RG_TRY(take_snapshot(s, sn), "snapshot");
    reinterpret_cast<Ctl*>(sn.ctl.data())->rebuild = 1;
  }
  s->contacts_fresh = true;
  if (pe) *pe = s->h_ctl->pe;
  return rg_get_state(s, nullptr, nullptr, nullptr, nullptr, f, tau);
}

int rg_set_profiling(rg_system* s, int enable) {
  if (!s) return RG_ERR_ARG;
  s->prof_on = enable != 0;
  for (int k = 0; k < 8; ++k) { s->prof_ms[k] = 0; s->prof_cnt[k] = 0; }
  // persistent-step phase timers live in the control block
  Ctl h;
  cudaMemcpy(&h, s->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
  h.prof_phases = s->prof_on ? 1 : 0;
  for (int k = 0; k < 12; ++k) h.phase_ns[k] = 0;
  cudaMemcpy(s->d_ctl, &h, sizeof(Ctl), cudaMemcpyHostToDevice);
  return RG_OK;
}

int rg_get_phase_times(const rg_system* s, double* ms, int n) {
  if (!s || !ms) return RG_ERR_ARG;
  Ctl h;
  cudaMemcpy(&h, s->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
  for (int k = 0; k < n && k < 12; ++k) ms[k] = h.phase_ns[k] * 1e-6;
  return RG_OK;
}

int rg_get_profile(const rg_system* s, double* ms, int64_t* launches) {
  if (!s) return RG_ERR_ARG;
  for (int k = 0; k < 8; ++k) {
    if (ms) ms[k] = s->prof_ms[k];
    if (launches) launches[k] = s->prof_cnt[k];
  }
  return RG_OK;
}

int rg_get_history(const rg_system* s, int32_t* pairs, double* value, int64_t* last_frame, size_t cap,
                   size_t* n) {
  if (!s || !n) return RG_ERR_ARG;
  Ctl h;
  cudaMemcpy(&h, s->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost);
  const History& H = s->hist;
  int hn = h.hist_n;
  *n = (size_t)hn;
  size_t m = cap < (size_t)hn ? cap : (size_t)hn;
  if (m) {
    std::vector<unsigned long long> k(m);
    std::vector<double> v(3 * m);
    std::vector<long long> fr(m);
    cudaMemcpy(k.data(), H.key[H.cur], sizeof(unsigned long long) * m, cudaMemcpyDeviceToHost);
    for (int j = 0; j < 3; ++j)
      cudaMemcpy(v.data() + (size_t)j * m, H.val[H.cur] + (size_t)j * H.cap, sizeof(double) * m,
                 cudaMemcpyDeviceToHost);
    cudaMemcpy(fr.data(), H.frame[H.cur], sizeof(long long) * m, cudaMemcpyDeviceToHost);
    for (size_t i = 0; i < m; ++i) {
      if (pairs) { pairs[2 * i] = (int32_t)(k[i] >> 32); pairs[2 * i + 1] = (int32_t)(k[i] & 0xffffffffu); }
      if (value) for (int j = 0; j < 3; ++j) value[3 * i + j] = v[(size_t)j * m + i];
      if (last_frame) last_frame[i] = fr[i];
    }
  }
  return (size_t)hn > cap ? RG_ERR_CAPACITY : RG_OK;
}

}  // extern "C"
