// rg_internal.cuh - host-side layout of an rg_system and the launch helpers
// each .cu file provides.  Not part of the public ABI (include/rodgpu.h).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

#include "rg_common.cuh"

namespace rg {

// Exclusive scan of int32 counts: out[0..n] with out[n] = total, n read
// from the device (n_dev) so launches do not depend on host-known sizes.
// One pass (decoupled look-back); a wait that runs out sets ERR_TIMEOUT in
// *err.
struct Scan {
  int cap = 0;
  void* d_blocks = nullptr;  // tile counter and tile status words
  cudaError_t alloc(int cap_);
  void free_();
  void run(const int* in, int* out, const int* n_dev, int* err, cudaStream_t s) const;
  // two independent arrays (each of at most cap elements) in one launch
  void run2(const int* in0, int* out0, const int* n0_dev, const int* in1, int* out1, const int* n1_dev, int* err,
            cudaStream_t s) const;
};

// Device-resident control words of one system (one cudaMalloc).
struct Ctl {
  int err;              // error bits
  int rebuild;          // 1: neighbour list must be rebuilt before next use
  int contacts;         // contacts of the last detection
  int hist_n;           // live history entries (current table)
  int hist_touched;     // scratch
  int colors;           // colours of the last colouring
  int proj_active;      // projection rows active in the current pass
  int sweeps_last;      // PSOR sweeps of the last solve
  double maxdisp;       // max displacement since the last list build
  double near_disp;     // max displacement since the last near-list build
  int near_valid;       // 1: the near list matches the current lists
  int near_n;           // pairs in the near list
  double residual;      // last PSOR residual
  long long frame;      // force-evaluation counter (HM / Cundall frames)
  long long rebuilds;   // list rebuilds (cumulative)
  long long sweeps_sum; // PSOR sweeps (cumulative)
  long long not_conv;   // steps whose PSOR stopped at max sweeps
  double max_residual;  // worst final residual (cumulative)
  long long collisions; // NSC impacts of the last step
  double jn_sum, jt_sum, pe;
  long long row_sweeps; // Σ contacts x sweeps (cumulative)
  long long member_ns;  // device time of this system's steps in the call (batch cost model)
  long long serial_ns;  // of which in the single-block solves (no team speed-up)
  long long contact_steps;  // Σ velocity-solve contacts over steps
  long long near_rebuilds;  // near-list rebuilds (per call)
  int vel_contacts;     // NSC: contacts of the last velocity solve (lastHitCount)
  int prof_phases;      // 1: the persistent step records phase times
  long long phase_ns[12];  // persistent-step phase time accumulators
  int rec_n;            // MLP records stored
  int det_valid;        // 1: the near-pair hit bits hold the position-level
                        // detection of this call's last step
  unsigned int bar_count, bar_gen;  // grid barrier
  double res_sweep[1];  // per-sweep residual slots follow (velocity_iters)
};

struct Contacts {  // sorted by (a,b)
  int cap = 0;
  int *a = nullptr, *b = nullptr, *type = nullptr;
  double* g = nullptr;  // 14 component arrays of cap: pa(3) pb(3) n(3) sh(3) dist surf
  cudaError_t alloc(int cap_);
  void free_();
  __host__ __device__ double* comp(int k) const { return g + (size_t)k * cap; }
};

struct Detector {
  int maxnb = 0;
  int* nbr_cnt = nullptr;   // n
  int* nbr = nullptr;       // n * maxnb (j > i, ascending)
  double* ref = nullptr;    // 6n: x_ref(3n), u_ref(3n)
  Seg* seg = nullptr;       // n
  int ncell[3] = {1, 1, 1};
  int ncells = 1;
  double cell[3] = {1, 1, 1};
  int *cell_of = nullptr, *cell_cnt = nullptr, *cell_start = nullptr, *cell_fill = nullptr,
      *cell_rods = nullptr;
  // near list (persistent NSC step): the list entries within the contact
  // reach plus near_skin, as sorted (i, j) pairs, and the segments at its build
  int2* near = nullptr;           // n * maxnb
  double* ref2 = nullptr;         // 6n
  double near_skin = 0;
  // near lists of the multi-kernel detection (soft / HM models): per rod,
  // the ascending list entries within reach + near_skin (same layout as
  // nbr); null when the full lists are used (NSC models, all-pairs boxes)
  int* near_cnt = nullptr;        // n
  int* near_nbr = nullptr;        // n * maxnb
  // 1: rod moved (position projection or periodic wrap) since the
  // position-level detection of the step; cleared by the position update
  unsigned char* moved = nullptr;  // n
  int* hit_cnt = nullptr;         // n+1
  int* hit_off = nullptr;         // n+1
  unsigned long long* hit_mask = nullptr;  // n * words
  int mask_words = 1;
  double skin = 0, margin = 0;    // skin and the largest activation margin
  double cut_center = 0;          // centre-distance cutoff for list building
  bool all_pairs = false;         // tiny periodic box: scan every cell
};

// Closes a history merge: the new table size from the two offset scans
// (touched contacts + retained entries), and the call's contact-evaluation
// count (k_hist_finish, or the first thread of the kick kernel after it).
struct HistFinish {
  const int* toff;
  const int* koff;
};
__device__ inline void hist_finish(const HistFinish& h, Ctl* ctl) {
  const int T = h.toff[ctl->contacts], K = h.koff[ctl->hist_n];
  ctl->hist_n = T + K;
  ctl->contact_steps += ctl->contacts;  // contact-evaluations of the call
}

struct BodyCSR {  // contacts incident to each body, in contact order
  int* cnt = nullptr;   // n+1
  int* off = nullptr;   // n+1
  int* fill = nullptr;  // n
  int* ent = nullptr;   // 2*ccap: 2c (side a) or 2c+1 (side b)
};

struct History {  // sorted by key (a<<32|b)
  int cap = 0;
  unsigned long long* key[2] = {nullptr, nullptr};
  double* val[2] = {nullptr, nullptr};       // 3 * cap each (SoA)
  long long* frame[2] = {nullptr, nullptr};
  int cur = 0;
  int* touched = nullptr;      // ccap+1 flags -> scan
  int* touched_off = nullptr;  // ccap+1
  int* kept = nullptr;         // cap+1
  int* kept_off = nullptr;     // cap+1
  double* newval = nullptr;    // 3*ccap
};

struct Nsc {
  // manifold rows, SoA, ccap each
  double* row = nullptr;  // kRowComps * ccap
  double* lam = nullptr;  // 3*ccap (λn, λt1, λt2)
  int* color = nullptr;   // ccap
  int* color_tmp = nullptr;
  int* order = nullptr;   // colour-major contact order
  int* color_cnt = nullptr;   // kMaxColors+1
  int* color_off = nullptr;   // kMaxColors+1
  // warm cache: previous step's sorted keys and impulses
  unsigned long long* wkey = nullptr;
  double* wlam = nullptr;
  int* wn = nullptr;  // device count of the warm cache
  int wcap = 0;
  // contact-network export (enabled per system): kExportComps component
  // arrays of wcap, warm-cache order - normal, r_a, r_b, phi, v_n_pre
  double* xrow = nullptr;
  // projection scratch
  double* dx = nullptr;   // 6n: dx(3n), dθ(3n)
  double* prow = nullptr; // kPosComps * ccap
  int* pactive = nullptr; // ccap
  // colouring scratch of the persistent step (per body)
  unsigned long long* pmax = nullptr;   // 2n priority maxima (two rounds)
  unsigned long long* cmask = nullptr;  // n colour masks
  int* owner = nullptr;                 // n lowest contact index per body
  int* cursor = nullptr;                // kMaxColors+1
  int* remaining = nullptr;             // colouring rounds
  int* blk = nullptr;                   // per-block scan scratch
  int* slot_of = nullptr;               // n per-body local slots (-1)
  unsigned int* bar = nullptr;          // team barrier words
  void* view_dev = nullptr;             // device copy of the step view
  void* team_dev = nullptr;             // device team descriptor
};
constexpr int kRowComps = 42;
constexpr int kExportComps = 11;
constexpr int kPosComps = 12;

}  // namespace rg

struct rg_system {
  rg_config cfg;
  int n = 0;
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string err_text;
  bool bodies_set = false, state_set = false;
  bool contacts_fresh = false;  // contacts match the current positions

  double* d_state = nullptr;  // 19 n
  double* d_props = nullptr;  // 11 n
  rg::State st;
  rg::Box box;
  rg::Ctl* d_ctl = nullptr;
  rg::Ctl* h_ctl = nullptr;   // pinned mirror
  size_t ctl_bytes = 0;

  int ccap = 0;
  rg::Contacts con;
  rg::Detector det;
  rg::BodyCSR csr;
  rg::History hist;
  rg::Nsc nsc;
  rg::Scan scan;
  double* d_cf = nullptr;     // per-contact force/torque addends, 12 * ccap

  // snapshot for capacity retry: state, current history table, warm cache
  double* d_snap = nullptr;
  unsigned long long* snap_hkey = nullptr;
  double* snap_hval = nullptr;
  long long* snap_hframe = nullptr;
  int snap_hcap = 0;
  unsigned long long* snap_wkey = nullptr;
  double* snap_wlam = nullptr;  // 3*wcap doubles + wcap ints (colours)
  int snap_wcap = 0;

  // MLP (learned warm start)
  void* mlp_host = nullptr;   // network parameters and training workspace (rg_mlp.cu)
  double* d_ke = nullptr;     // kinetic-energy block partials
  // page-locked host words for asynchronous snapshots and statistics
  rg::Ctl* h_snapctl = nullptr;  // ctl_bytes
  int* h_wn = nullptr;
  double* h_ke = nullptr;        // 64 partial sums
  bool mlp_ready = false;
  bool recording = false;
  bool export_on = false;     // contact-network export rows saved by the NSC step
  int rec_cap = 0;
  float* d_rec_x = nullptr;
  float* d_rec_y = nullptr;
  float* d_feat = nullptr;    // 8 * ccap scratch
  float* d_pred = nullptr;    // 3 * ccap scratch

  int coop_blocks = 0;        // co-resident blocks for the persistent kernels
  int team_blocks = 0;        // blocks of the NSC team (0: automatic)
  cudaGraphExec_t graph = nullptr;
  int graph_kind = -1;
  // one velocity-Verlet step (soft / HM) captured as a CUDA graph; valid
  // while the buffers it names are the current ones (buf_gen) and the
  // history table starts in the same ping-pong buffer (vgraph_cur)
  cudaGraphExec_t vgraph = nullptr;
  long long vgraph_gen = -1;
  int vgraph_cur = -1;
  long long vgraph_kernels = 0;  // kernel nodes of the graph
  long long buf_gen = 0;         // bumped by every (re)allocation of device buffers

  // pinned staging for host <-> device state copies (19 n doubles)
  double* h_stage = nullptr;
  double last_call_ms = 0;
  long long last_call_launches = 0;

  // stage timers
  bool prof_on = false;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<int> rec_stage, rec_a, rec_b;
  double prof_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  long long prof_cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

namespace rg {
// Kernel launches issued by this library (all systems), for run statistics.
extern long long g_launches;
// Counts the launch written after it; one expression (comma operator), so
// `if (c) RGL k<<<...>>>(...)` guards the count and the launch together.
#define RGL ++::rg::g_launches,

// Launches k with programmatic stream serialization: the grid may be
// scheduled while the previous kernel in the stream drains, which hides the
// launch gap between the short dependent kernels of a step (inside a CUDA
// graph as well).  k must call griddep_wait() before it touches memory.
template <typename... K, typename... A>
inline cudaError_t launch_dep(void (*k)(K...), unsigned grid, unsigned block, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, static_cast<A&&>(args)...);
}

enum Stage { ST_INTEGRATE = 0, ST_DETECT, ST_COLOR, ST_MANIFOLDS, ST_PSOR, ST_PROJECT, ST_FORCES, ST_OTHER };

inline int prof_event(rg_system* s) {
  if (s->ev_used == s->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    s->ev_pool.push_back(e);
  }
  return (int)s->ev_used++;
}
// Records CUDA events around a group of launches of one stage.
struct ProfScope {
  rg_system* s;
  int stage, a;
  ProfScope(rg_system* s_, int st) : s(s_), stage(st), a(-1) {
    if (!s->prof_on) return;
    a = prof_event(s);
    cudaEventRecord(s->ev_pool[a], s->stream);
  }
  ~ProfScope() { end(); }
  void end() {
    if (a < 0) return;
    int b = prof_event(s);
    cudaEventRecord(s->ev_pool[b], s->stream);
    s->rec_stage.push_back(stage);
    s->rec_a.push_back(a);
    s->rec_b.push_back(b);
    a = -1;
  }
};
// Folds recorded event pairs into the accumulators (after a stream sync).
inline void prof_resolve(rg_system* s) {
  for (size_t i = 0; i < s->rec_stage.size(); ++i) {
    float ms = 0;
    cudaEventElapsedTime(&ms, s->ev_pool[s->rec_a[i]], s->ev_pool[s->rec_b[i]]);
    s->prof_ms[s->rec_stage[i]] += ms;
    s->prof_cnt[s->rec_stage[i]] += 1;
  }
  s->rec_stage.clear();
  s->rec_a.clear();
  s->rec_b.clear();
  s->ev_used = 0;
}

// rg_detect.cu
cudaError_t detector_alloc(rg_system* s);
void detector_free(rg_system* s);
// seg_ready: the segment records and the displacement check of the current
// positions were written by the drift kernel (reduce_drift_launch)
// body_csr: the narrow phase also zeroes and counts the body CSR (csr_launch
// then starts at its scan)
void detect_launch(rg_system* s, double delta, bool check_rebuild, bool seg_ready = false,
                   bool body_csr = false);
void force_rebuild(rg_system* s);
// rg_forces.cu
enum class EvalTail { kForces, kHalfPos, kSecondHalf };
// detect (unless fresh) + forces; the tail (force_eval_launch in rg_forces.cu)
void force_eval_launch(rg_system* s, EvalTail tail = EvalTail::kForces, bool seg_ready = false);
// forces at t reduced per body, first half kick and drift, segment records
// and displacement check of the drifted positions (velocity Verlet)
void reduce_drift_launch(rg_system* s, bool wall, rg::HistFinish hf);
// forces at t + dt reduced per body (kept in f, tau) and the second half kick
void reduce_kick_launch(rg_system* s, bool wall, rg::HistFinish hf);
void csr_launch(rg_system* s, bool counted = false);  // body CSR of the current contacts
// rg_integrate.cu
void clear_forces_launch(rg_system* s);
void nsc_free_flight_launch(rg_system* s);
void nsc_position_update_launch(rg_system* s);
void wrap_launch(rg_system* s);
// rg_nsc.cu
void nsc_run_launch(rg_system* s, int nsteps);
int nsc_team_blocks(const rg_system* s);
int nsc_blocks_per_sm();
size_t nsc_view_bytes();
size_t nsc_team_bytes();
// rg_mlp.cu
void mlp_free(rg_system* s);

// rg_api.cu: one call of rg_step, in pieces the batch driver reuses.
// Control words and the replay snapshot taken at the start of a call:
struct Snapshot {
  std::vector<char> ctl;
  int hist_cur = 0;
  int wn = 0;
};
int fail(rg_system* s, int code, const std::string& msg);
int cuda_fail(rg_system* s, cudaError_t e, const char* where);
cudaError_t take_snapshot(rg_system* s, Snapshot& sn, bool sync = true);
// Pieces of a snapshot for callers that gather many systems' copies into one
// device copy kernel (rg_batch): buffer set-up and the device-to-device
// copies a snapshot makes.
struct CopySeg {
  const void* src;
  void* dst;
  unsigned long long bytes;
  // optional: only the first (*count) x elem bytes of the whole segment are
  // live (read on the device when the copy runs); off = this piece's offset
  // within the segment
  const int* count;
  unsigned elem;
  unsigned long long off;
};
constexpr int kCopyChunk = 32768;  // largest piece one block of k_copy_segments moves
// Splits segments into pieces of at most kCopyChunk bytes (same copies).
void split_segments(const std::vector<CopySeg>& in, std::vector<CopySeg>& out);
cudaError_t snapshot_alloc(rg_system* s);
void snapshot_segments(rg_system* s, std::vector<CopySeg>& out);
void copy_segments_launch(const CopySeg* d_segs, int n, cudaStream_t st);
// Zeroes the per-call counters (as reset_call_ctl does from a snapshot)
// of n systems' control blocks on the device.
void ctl_reset_launch(rg::Ctl* const* d_ctls, int n, cudaStream_t st);
void ctl_zero_time_launch(rg::Ctl* const* d_ctls, int n, cudaStream_t st);  // member_ns, serial_ns
void finish_snapshot(rg_system* s, Snapshot& sn);  // after the stream synchronised
cudaError_t restore_snapshot(rg_system* s, const Snapshot& sn);
cudaError_t reset_call_ctl(rg_system* s, const Snapshot& sn);
int resolve_call(rg_system* s, Snapshot& sn, int err, bool* retry);
void launch_steps(rg_system* s, int nsteps);
void fill_stats(rg_system* s, int nsteps, rg_step_stats* stats, bool ke_launched = false);
double kinetic_energy(rg_system* s);
void ke_launch(rg_system* s);  // partials to h_ke; read them with ke_sum after a stream sync
double ke_sum(const rg_system* s);
// launch geometry helper
inline int grid_for(long long n, int bs, int maxb = 148 * 16) {
  long long g = (n + bs - 1) / bs;
  if (g < 1) g = 1;
  if (g > maxb) g = maxb;
  return (int)g;
}
}  // namespace rg
