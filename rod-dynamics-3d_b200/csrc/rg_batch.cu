// rg_batch.cu - many independent systems of uneven size in one persistent
// launch.
//
// No reference counterpart: the reference steps one system per process
// (App::physicsStep, src/app/main.cpp:4333-4858; its CUDA state is a
// file-static singleton, src/physics/cuda_broadphase.cu:658).  A batch owns
// one rg_system per member (its own box, model, dt, friction, buffers and
// error words) on one shared stream.  NSC members run as teams of the
// persistent step kernel in ONE cooperative launch for all requested
// steps; that launch (with the reset of the team barriers) is captured in a
// CUDA graph and replayed.  Members with the Verlet models run their
// multi-kernel step on the same stream after it.
//
// Schedule: each member's work is its rod count until the device has timed
// its steps (every call records each member's own step time), then that
// measured cost in rod units.  Members of at least 1.5 R work units (R =
// rods per block) get a team of round(work/R) blocks to themselves; the rest
// share single-block teams, assigned longest-first to the least-loaded
// block.  The balanced plan (R = -1) models each member's step on a team of
// nb blocks as s + p / nb (+ a team overhead when nb > 1), from its measured
// time in the single-block solves (s) and the rest of its single-block step
// (p), and finds the smallest makespan that fits the blocks.
// rg_batch_autotune first measures the costs, then times a few schedules on
// the live systems (from a snapshot, restored afterwards) and keeps the
// fastest.  The schedule changes time only: every member's results are the
// same for any schedule.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "rg_internal.cuh"
#include "rg_nsc_dev.cuh"

using namespace rg;

struct rg_batch {
  int n = 0;
  std::vector<rg_system*> sys;
  cudaStream_t stream = nullptr;
  int coop_blocks = 0;
  // schedule
  int rods_per_block = 0;  // 0: every NSC member in single-block teams; -1: balanced
  bool use_graph = true;
  bool plan_dirty = true;
  std::vector<TeamDesc> teams;
  std::vector<int> members;
  int grid = 0;
  NscView* d_views = nullptr;
  TeamDesc* d_teams = nullptr;
  int* d_members = nullptr;
  unsigned int* d_bars = nullptr;
  long long* d_team_ns = nullptr;
  int cap_members = 0, cap_teams = 0;
  // what the device holds now (uploads are skipped when nothing changed)
  std::vector<NscView> up_views;
  std::vector<TeamDesc> up_teams;
  std::vector<int> up_members;
  // graph of (barrier reset + persistent launch) for graph_steps steps
  cudaGraphExec_t graph = nullptr;
  int graph_steps = -1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0;
  std::string err;
  // measured cost per member: block-milliseconds per step (0: not measured)
  std::vector<double> cost;
  std::vector<int> team_nb;  // blocks of the member's team in the last plan
  // balanced-plan model per member (ms per step): single-block solves and
  // the rest of a single-block step; team overhead of a multi-block team
  std::vector<double> ser, par;
  double team_ms = 0.05;
  bool cost_frozen = false;  // autotuner trials compare schedules on one cost model
  // control plane: copy segments, member control blocks gathered into one
  // device buffer and one page-locked host buffer (control words + wn)
  CopySeg* d_segs = nullptr;
  int cap_segs = 0;
  Ctl** d_ctls = nullptr;
  unsigned char* d_ctlbuf = nullptr;
  unsigned char* h_ctlbuf = nullptr;
  std::vector<size_t> ctl_off;
  size_t ctlbuf_bytes = 0;
  // bulk state transfer: member table and device staging (x, q, v, w)
  void* d_bulk = nullptr;
  double* d_stage = nullptr;
  int* d_bulk_bad = nullptr;   // non-finite flag of the last bulk upload
  int* h_bulk_bad = nullptr;   // page-locked mirror
  long long total = 0;
};

namespace {
struct BulkMember {
  double* state;  // 19 n component arrays of the member
  int n;
  long long off;  // first rod in the concatenated arrays
};

__device__ inline int bulk_find(const BulkMember* m, int nm, long long g) {
  int lo = 0, hi = nm;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (m[mid].off <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Concatenated host-layout arrays (x[3T], q[4T], v[3T], w[3T]) into every
// member's component arrays; forces and torques are cleared, as
// rg_set_state does without them.
// Flags a non-finite value among the staged x, q, v, w (13 T doubles,
// contiguous); the scatter that follows leaves every member's state as it
// was when the flag is set.
__global__ void k_bulk_check(const double* staged, long long count, int* bad) {
  int any = 0;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < count;
       g += (long long)gridDim.x * blockDim.x)
    any |= !isfinite(staged[g]);
  if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(bad, 1);
}

__global__ void k_bulk_scatter(const BulkMember* m, int nm, long long T, const double* x, const double* q,
                               const double* v, const double* w, const int* bad) {
  if (*(volatile const int*)bad) return;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < T;
       g += (long long)gridDim.x * blockDim.x) {
    const BulkMember M = m[bulk_find(m, nm, g)];
    const size_t n = (size_t)M.n, i = (size_t)(g - M.off);
    double* b = M.state;
    for (int k = 0; k < 3; ++k) {
      b[k * n + i] = x[3 * g + k];
      b[(7 + k) * n + i] = v[3 * g + k];
      b[(10 + k) * n + i] = w[3 * g + k];
      b[(13 + k) * n + i] = 0.0;
      b[(16 + k) * n + i] = 0.0;
    }
    for (int k = 0; k < 4; ++k) b[(3 + k) * n + i] = q[4 * g + k];
  }
}

__global__ void k_bulk_gather(const BulkMember* m, int nm, long long T, double* x, double* q, double* v,
                              double* w) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < T;
       g += (long long)gridDim.x * blockDim.x) {
    const BulkMember M = m[bulk_find(m, nm, g)];
    const size_t n = (size_t)M.n, i = (size_t)(g - M.off);
    const double* b = M.state;
    for (int k = 0; k < 3; ++k) {
      x[3 * g + k] = b[k * n + i];
      v[3 * g + k] = b[(7 + k) * n + i];
      w[3 * g + k] = b[(10 + k) * n + i];
    }
    for (int k = 0; k < 4; ++k) q[4 * g + k] = b[(3 + k) * n + i];
  }
}
}  // namespace

namespace {

int bfail(rg_batch* b, int code, const std::string& msg) {
  b->err = msg;
  return code;
}

// Work of member k in rod units: its rod count, or, once measured, its
// device cost converted to rods at the batch's average cost per rod (so a
// system of thin rods or a tiny all-pairs box weighs what it costs).
std::vector<double> work_of(const rg_batch* b, const std::vector<int>& which) {
  double cn = 0, cc = 0;
  for (int k : which)
    if (b->cost[k] > 0) { cn += b->sys[k]->n; cc += b->cost[k]; }
  std::vector<double> w(b->n, 0.0);
  for (int k : which) w[k] = (cc > 0 && b->cost[k] > 0) ? b->cost[k] * (cn / cc) : (double)b->sys[k]->n;
  return w;
}

// Packs `small` (sorted by decreasing w) longest-first onto nbins blocks.
void pack_lpt(const std::vector<int>& small, const std::vector<double>& w, int nbins,
              std::vector<std::vector<int>>& bins) {
  bins.assign(nbins, {});
  std::vector<double> load(nbins, 0.0);
  for (int k : small) {
    int m = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    bins[m].push_back(k);
    load[m] += w[k];
  }
}

// Blocks needed for makespan M (member k on nb blocks: ser + par / nb, plus
// team_ms when nb > 1; single-block members first-fit into blocks of
// capacity M); nb_out gets each large member's team size.  Returns a count
// above the budget when M is not reachable.
long long balanced_blocks(const rg_batch* b, const std::vector<int>& order, double M, int budget,
                          std::vector<int>* nb_out) {
  long long blocks = 0;
  std::vector<double> bins;
  for (int k : order) {
    const double w1 = b->ser[k] + b->par[k];
    if (w1 <= M) {
      bool placed = false;
      for (double& l : bins)
        if (l + w1 <= M) {
          l += w1;
          placed = true;
          break;
        }
      if (!placed) bins.push_back(w1);
      if (nb_out) (*nb_out)[k] = 1;
      continue;
    }
    const double room = M - b->ser[k] - b->team_ms;
    if (room <= 0.0) return (long long)budget + 1;
    const long long nb = std::max<long long>(2, (long long)std::ceil(b->par[k] / room));
    if (nb > budget) return (long long)budget + 1;
    blocks += nb;
    if (nb_out) (*nb_out)[k] = (int)nb;
  }
  return blocks + (long long)bins.size();
}

// Balanced plan: the smallest makespan whose teams fit the blocks (bisection
// on M), then the single-block members packed over all remaining blocks.
// Returns false when a member has no measured cost yet.
bool plan_balanced(rg_batch* b, const std::vector<int>& which, std::vector<TeamDesc>& teams,
                   std::vector<int>& members, int& grid) {
  const int budget = b->coop_blocks;
  double sum = 0.0, lo = 0.0, hi = 0.0;
  for (int k : which) {
    if (!(b->par[k] > 0.0)) return false;
    sum += b->ser[k] + b->par[k];
    lo = std::max(lo, b->ser[k]);
    hi = std::max(hi, b->ser[k] + b->par[k]);
  }
  std::vector<int> order(which);
  std::sort(order.begin(), order.end(), [&](int x, int y) {
    const double wx = b->ser[x] + b->par[x], wy = b->ser[y] + b->par[y];
    return wx != wy ? wx > wy : x < y;
  });
  lo = std::max(lo, sum / budget);
  hi = std::max(hi, sum);  // one block holds everything
  if (balanced_blocks(b, order, lo, budget, nullptr) > budget) {
    for (int it = 0; it < 48 && hi - lo > 1e-6 * hi; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (balanced_blocks(b, order, mid, budget, nullptr) <= budget) hi = mid;
      else lo = mid;
    }
  } else {
    hi = lo;
  }
  std::vector<int> nb(b->n, 1);
  balanced_blocks(b, order, hi, budget, &nb);
  teams.clear();
  members.clear();
  int b0 = 0;
  std::vector<int> small;
  for (int k : order) {
    if (nb[k] > 1) {
      teams.push_back(TeamDesc{b0, nb[k], (int)members.size(), 1, nullptr});
      members.push_back(k);
      b0 += nb[k];
    } else {
      small.push_back(k);
    }
  }
  if (!small.empty()) {
    std::vector<double> w(b->n, 0.0);
    for (int k : small) w[k] = b->ser[k] + b->par[k];
    std::vector<std::vector<int>> bins;
    pack_lpt(small, w, std::min<int>((int)small.size(), std::max(1, budget - b0)), bins);
    for (auto& bin : bins) {
      teams.push_back(TeamDesc{b0, 1, (int)members.size(), (int)bin.size(), nullptr});
      for (int k : bin) members.push_back(k);
      ++b0;
    }
  }
  grid = b0;
  for (const TeamDesc& t : teams)
    for (int m = t.first; m < t.first + t.count; ++m) b->team_nb[members[m]] = t.nb;
  return true;
}

// Team plan for the NSC members in `which` with R (work in rod units) per
// block: members of at least 1.5 R get round(work / R) blocks, the rest are
// packed longest-first onto the least-loaded single blocks.  R = -1: the
// balanced plan once every member has been timed on one block (all
// single-block before, which times them).
void plan(rg_batch* b, const std::vector<int>& which, int R, std::vector<TeamDesc>& teams,
          std::vector<int>& members, int& grid) {
  if (R < 0) {
    if (plan_balanced(b, which, teams, members, grid)) return;
    R = 0;
  }
  teams.clear();
  members.clear();
  const int budget = b->coop_blocks;
  const std::vector<double> W = work_of(b, which);
  std::vector<int> big, small;
  for (int k : which) {
    if (R > 0 && W[k] >= 1.5 * R) big.push_back(k);
    else small.push_back(k);
  }
  if ((int)big.size() > budget / 2) {  // too many large members: pack everything
    small.insert(small.end(), big.begin(), big.end());
    big.clear();
  }
  std::sort(big.begin(), big.end(), [&](int x, int y) { return W[x] != W[y] ? W[x] > W[y] : x < y; });
  std::sort(small.begin(), small.end(), [&](int x, int y) { return W[x] != W[y] ? W[x] > W[y] : x < y; });
  std::vector<int> nb(big.size());
  long long want = 0;
  for (size_t i = 0; i < big.size(); ++i) {
    nb[i] = std::max(1, (int)(W[big[i]] / R + 0.5));
    want += nb[i];
  }
  // blocks for the packed members: their work at R per block
  double small_work = 0.0;
  for (int k : small) small_work += W[k];
  const int reserve = small.empty() ? 0
                                    : std::min<int>((int)small.size(),
                                                    std::max(1, (int)std::ceil(small_work / std::max(1, R))));
  const int avail = std::max<int>((int)big.size(), budget - reserve);
  if (want > avail) {  // scale the large teams down to fit
    for (size_t i = 0; i < big.size(); ++i) nb[i] = std::max(1, (int)((long long)nb[i] * avail / want));
    want = std::accumulate(nb.begin(), nb.end(), 0LL);
    for (size_t i = 0; want > avail && i < big.size(); ++i)
      while (nb[i] > 1 && want > avail) { --nb[i]; --want; }
  }
  int b0 = 0;
  for (size_t i = 0; i < big.size(); ++i) {
    teams.push_back(TeamDesc{b0, nb[i], (int)members.size(), 1, nullptr});
    members.push_back(big[i]);
    b0 += nb[i];
  }
  const int nsb = std::min<int>((int)small.size(), std::max(1, budget - b0));
  if (!small.empty()) {
    std::vector<std::vector<int>> bins(nsb);
    std::vector<double> load(nsb, 0.0);
    for (int k : small) {
      int m = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      bins[m].push_back(k);
      load[m] += W[k];
    }
    for (int i = 0; i < nsb; ++i) {
      teams.push_back(TeamDesc{b0, 1, (int)members.size(), (int)bins[i].size(), nullptr});
      for (int k : bins[i]) members.push_back(k);
      ++b0;
    }
  }
  grid = b0;
  for (const TeamDesc& t : teams)
    for (int m = t.first; m < t.first + t.count; ++m) b->team_nb[members[m]] = t.nb;
}

cudaError_t ensure_dev(rg_batch* b, size_t nteams, size_t nmembers) {
  cudaError_t e = cudaSuccess;
  if ((int)nmembers > b->cap_members) {
    cudaFree(b->d_views);
    cudaFree(b->d_members);
    b->cap_members = (int)std::max<size_t>(nmembers, (size_t)b->n);
    if ((e = cudaMalloc(&b->d_views, sizeof(NscView) * b->cap_members))) return e;
    if ((e = cudaMalloc(&b->d_members, sizeof(int) * b->cap_members))) return e;
  }
  if ((int)nteams > b->cap_teams) {
    cudaFree(b->d_teams);
    cudaFree(b->d_bars);
    b->cap_teams = (int)std::max<size_t>(nteams, (size_t)b->coop_blocks);
    if ((e = cudaMalloc(&b->d_teams, sizeof(TeamDesc) * b->cap_teams))) return e;
    if ((e = cudaMalloc(&b->d_bars, sizeof(unsigned int) * 4 * b->cap_teams))) return e;
    cudaFree(b->d_team_ns);
    if ((e = cudaMalloc(&b->d_team_ns, sizeof(long long) * b->cap_teams))) return e;
  }
  return e;
}

// Uploads the views of all members (buffer addresses change when buffers
// grow) and the team plan.  The views array is indexed by member number.
cudaError_t upload(rg_batch* b, std::vector<TeamDesc>& teams, const std::vector<int>& members) {
  const int cm = b->cap_members, ct = b->cap_teams;
  cudaError_t e = ensure_dev(b, teams.size(), members.size());
  if (e) return e;
  const bool moved = cm != b->cap_members || ct != b->cap_teams;  // device tables reallocated
  std::vector<NscView> views(b->n);
  for (int k = 0; k < b->n; ++k) {
    std::memset(&views[k], 0, sizeof(NscView));
    if (b->sys[k]->cfg.model == RG_MODEL_NSC) views[k] = make_view(b->sys[k]);
  }
  for (size_t t = 0; t < teams.size(); ++t) {
    teams[t].bar = b->d_bars + 4 * t;
    teams[t].t_ns = b->d_team_ns + t;
  }
  bool any = false;
  if (moved || b->up_views.size() != views.size() ||
      std::memcmp(b->up_views.data(), views.data(), sizeof(NscView) * views.size()) != 0) {
    cudaMemcpyAsync(b->d_views, views.data(), sizeof(NscView) * b->n, cudaMemcpyHostToDevice, b->stream);
    b->up_views = views;
    any = true;
  }
  if (moved || b->up_teams.size() != teams.size() ||
      std::memcmp(b->up_teams.data(), teams.data(), sizeof(TeamDesc) * teams.size()) != 0 ||
      b->up_members != members) {
    cudaMemcpyAsync(b->d_teams, teams.data(), sizeof(TeamDesc) * teams.size(), cudaMemcpyHostToDevice, b->stream);
    cudaMemcpyAsync(b->d_members, members.data(), sizeof(int) * members.size(), cudaMemcpyHostToDevice, b->stream);
    b->up_teams = teams;
    b->up_members = members;
    any = true;
  }
  return any ? cudaStreamSynchronize(b->stream) : cudaSuccess;
}

void drop_graph(rg_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_steps = -1;
}

// Barrier reset + persistent launch, through the graph when enabled.
cudaError_t launch_nsc(rg_batch* b, int nteams, int grid, int nsteps, bool graph_ok) {
  if (grid <= 0 || nsteps <= 0) return cudaSuccess;
  if (!(graph_ok && b->use_graph)) {
    cudaMemsetAsync(b->d_bars, 0, sizeof(unsigned int) * 4 * nteams, b->stream);
    nsc_batch_launch(b->d_views, b->d_teams, nteams, b->d_members, grid, nsteps, b->stream);
    return cudaGetLastError();
  }
  if (!b->graph || b->graph_steps != nsteps) {
    drop_graph(b);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e) return e;
    cudaMemsetAsync(b->d_bars, 0, sizeof(unsigned int) * 4 * nteams, b->stream);
    nsc_batch_launch(b->d_views, b->d_teams, nteams, b->d_members, grid, nsteps, b->stream);
    e = cudaStreamEndCapture(b->stream, &g);
    if (e) return e;
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e) { b->graph = nullptr; return e; }
    b->graph_steps = nsteps;
  }
  RGL cudaGraphLaunch(b->graph, b->stream);
  return cudaGetLastError();
}

// Gathered control-plane buffers (allocated on first use).
int ctl_setup(rg_batch* b) {
  if (b->d_ctlbuf) return RG_OK;
  b->ctl_off.resize(b->n + 1);
  size_t off = 0;
  for (int k = 0; k < b->n; ++k) {
    b->ctl_off[k] = off;
    off += (b->sys[k]->ctl_bytes + sizeof(int) + 15) & ~(size_t)15;  // control words, then wn
  }
  b->ctl_off[b->n] = off;
  b->ctlbuf_bytes = off;
  std::vector<Ctl*> ctls(b->n);
  for (int k = 0; k < b->n; ++k) ctls[k] = b->sys[k]->d_ctl;
  if (cudaMalloc(&b->d_ctlbuf, off) || cudaMallocHost(&b->h_ctlbuf, off) ||
      cudaMalloc(&b->d_ctls, sizeof(Ctl*) * b->n)) {
    cudaGetLastError();
    return bfail(b, RG_ERR_CUDA, "control-plane buffers");
  }
  cudaMemcpy(b->d_ctls, ctls.data(), sizeof(Ctl*) * b->n, cudaMemcpyHostToDevice);
  return RG_OK;
}

// Runs the copy segments on the device (one upload, one kernel).
int run_segments(rg_batch* b, const std::vector<CopySeg>& whole) {
  std::vector<CopySeg> segs;
  split_segments(whole, segs);
  if ((int)segs.size() > b->cap_segs) {
    cudaFree(b->d_segs);
    b->cap_segs = (int)segs.size() * 2;
    if (cudaMalloc(&b->d_segs, sizeof(CopySeg) * b->cap_segs)) {
      cudaGetLastError();
      b->cap_segs = 0;
      return bfail(b, RG_ERR_CUDA, "copy segments");
    }
  }
  cudaMemcpyAsync(b->d_segs, segs.data(), sizeof(CopySeg) * segs.size(), cudaMemcpyHostToDevice, b->stream);
  copy_segments_launch(b->d_segs, (int)segs.size(), b->stream);
  return RG_OK;
}

// Snapshots of all members with one copy kernel and one host read.
int snapshot_all(rg_batch* b, std::vector<Snapshot>& sn) {
  int rc = ctl_setup(b);
  if (rc != RG_OK) return rc;
  std::vector<CopySeg> segs;
  segs.reserve(8 * b->n);
  for (int k = 0; k < b->n; ++k) {
    rg_system* s = b->sys[k];
    if (snapshot_alloc(s)) return bfail(b, RG_ERR_CUDA, "snapshot buffers");
    snapshot_segments(s, segs);
    segs.push_back({s->d_ctl, b->d_ctlbuf + b->ctl_off[k], s->ctl_bytes});
    segs.push_back({s->nsc.wn, b->d_ctlbuf + b->ctl_off[k] + s->ctl_bytes, sizeof(int)});
    sn[k].hist_cur = s->hist.cur;
  }
  if ((rc = run_segments(b, segs)) != RG_OK) return rc;
  cudaMemcpyAsync(b->h_ctlbuf, b->d_ctlbuf, b->ctlbuf_bytes, cudaMemcpyDeviceToHost, b->stream);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e) return bfail(b, RG_ERR_CUDA, std::string("snapshot: ") + cudaGetErrorString(e));
  for (int k = 0; k < b->n; ++k) {
    rg_system* s = b->sys[k];
    sn[k].ctl.assign(b->h_ctlbuf + b->ctl_off[k], b->h_ctlbuf + b->ctl_off[k] + s->ctl_bytes);
    std::memcpy(&sn[k].wn, b->h_ctlbuf + b->ctl_off[k] + s->ctl_bytes, sizeof(int));
  }
  return RG_OK;
}

// Control blocks of the members in `which` into their host mirrors: one
// copy kernel and one read (the caller synchronises the stream).
int read_ctls(rg_batch* b, const std::vector<int>& which) {
  std::vector<CopySeg> segs;
  segs.reserve(which.size());
  for (int k : which) segs.push_back({b->sys[k]->d_ctl, b->d_ctlbuf + b->ctl_off[k], b->sys[k]->ctl_bytes});
  int rc = run_segments(b, segs);
  if (rc != RG_OK) return rc;
  cudaMemcpyAsync(b->h_ctlbuf, b->d_ctlbuf, b->ctlbuf_bytes, cudaMemcpyDeviceToHost, b->stream);
  return RG_OK;
}

// One batch call: snapshot, launch, error resolution with replay of the
// members that need larger buffers.  With restore_after (autotuner trials)
// every member is put back to its state at the start of the call and its
// neighbour lists are rebuilt at the next step.
int batch_call(rg_batch* b, int nsteps, rg_step_stats* per, bool restore_after = false, int warm_steps = 0) {
  for (int k = 0; k < b->n; ++k) {
    rg_system* s = b->sys[k];
    if (!s->bodies_set || !s->state_set) return bfail(b, RG_ERR_STATE, "member " + std::to_string(k) + ": set bodies and state before stepping");
    if (s->cfg.model == RG_MODEL_NSC && s->cfg.nsc_warm_start == RG_WARM_MLP && !s->mlp_ready)
      return bfail(b, RG_ERR_STATE, "member " + std::to_string(k) + ": learned warm start without a network");
  }
  std::vector<Snapshot> sn(b->n);
  int rc0 = snapshot_all(b, sn);
  if (rc0 != RG_OK) return rc0;
  std::vector<int> todo(b->n);
  std::iota(todo.begin(), todo.end(), 0);
  double total_ms = 0;
  for (int attempt = 0; attempt < 8 && !todo.empty(); ++attempt) {
    if (attempt == 0) {
      // the device control blocks equal the snapshots: zero the per-call
      // counters in place
      ctl_reset_launch(b->d_ctls, b->n, b->stream);
    } else {
      for (int k : todo)  // replays start from the (edited) snapshot words
        if (reset_call_ctl(b->sys[k], sn[k])) return bfail(b, RG_ERR_CUDA, "ctl upload");
    }
    std::vector<int> nsc;
    for (int k : todo)
      if (b->sys[k]->cfg.model == RG_MODEL_NSC) nsc.push_back(k);
    const bool full = attempt == 0;
    std::vector<TeamDesc> teams;
    std::vector<int> members;
    int grid = 0;
    if (full && !b->plan_dirty) {
      teams = b->teams;
      members = b->members;
      grid = b->grid;
    } else {
      plan(b, nsc, b->rods_per_block, teams, members, grid);
      if (full) {
        b->teams = teams;
        b->members = members;
        b->grid = grid;
        b->plan_dirty = false;
        drop_graph(b);
      }
    }
    if (upload(b, teams, members)) return bfail(b, RG_ERR_CUDA, "upload views");
    if (warm_steps > 0) {  // untimed lead-in (autotuner trials)
      cudaError_t ew = launch_nsc(b, (int)teams.size(), grid, warm_steps, false);
      if (ew) return bfail(b, RG_ERR_CUDA, std::string("persistent launch: ") + cudaGetErrorString(ew));
      for (int k : todo)
        if (b->sys[k]->cfg.model != RG_MODEL_NSC) launch_steps(b->sys[k], warm_steps);
      ctl_zero_time_launch(b->d_ctls, b->n, b->stream);  // costs count the timed steps only
    }
    const long long l0 = g_launches;
    cudaEventRecord(b->ev0, b->stream);
    cudaError_t e = launch_nsc(b, (int)teams.size(), grid, nsteps, full);
    if (e) return bfail(b, RG_ERR_CUDA, std::string("persistent launch: ") + cudaGetErrorString(e));
    for (int k : todo)
      if (b->sys[k]->cfg.model != RG_MODEL_NSC) launch_steps(b->sys[k], nsteps);
    cudaEventRecord(b->ev1, b->stream);
    if ((e = cudaGetLastError())) return bfail(b, RG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (read_ctls(b, todo) != RG_OK) return RG_ERR_CUDA;
    if ((e = cudaStreamSynchronize(b->stream))) return bfail(b, RG_ERR_CUDA, std::string("step: ") + cudaGetErrorString(e));
    for (int k : todo) std::memcpy(b->sys[k]->h_ctl, b->h_ctlbuf + b->ctl_off[k], b->sys[k]->ctl_bytes);
    float ms = 0;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    total_ms += ms;
    const long long launches = g_launches - l0;
    std::vector<int> again;
    std::vector<double> over;  // team overhead samples of multi-block members
    for (int k : todo) {
      rg_system* s = b->sys[k];
      s->last_call_ms = ms;
      s->last_call_launches = launches;
      const int err = s->h_ctl->err;
      if (!err && full && !b->cost_frozen && s->cfg.model == RG_MODEL_NSC && nsteps > 0 && s->h_ctl->member_ns > 0) {
        // block-ms per step, averaged with the previous estimate: list
        // rebuilds and steps that run to the sweep limit make single calls
        // noisy
        const int nb = b->team_nb[k];
        const double t = 1e-6 * (double)s->h_ctl->member_ns / nsteps;
        const double sv = std::min(t, 1e-6 * (double)s->h_ctl->serial_ns / nsteps);
        const double c = t * nb;
        b->cost[k] = b->cost[k] > 0 ? 0.5 * (b->cost[k] + c) : c;
        b->ser[k] = b->ser[k] > 0 ? 0.5 * (b->ser[k] + sv) : sv;
        if (nb == 1) {
          const double p = std::max(1e-6, t - sv);
          b->par[k] = b->par[k] > 0 ? 0.5 * (b->par[k] + p) : p;
        } else if (b->par[k] > 0) {
          over.push_back(t - sv - b->par[k] / nb);
        }
      }
      if (!err) continue;
      bool retry = false;
      int rc = resolve_call(s, sn[k], err, &retry);
      if (rc != RG_OK) return bfail(b, rc, "member " + std::to_string(k) + ": " + s->err_text);
      again.push_back(k);
    }
    if (!over.empty()) {
      std::nth_element(over.begin(), over.begin() + over.size() / 2, over.end());
      const double m = std::min(1.0, std::max(0.0, over[over.size() / 2]));
      b->team_ms = 0.5 * (b->team_ms + m);
    }
    todo.swap(again);
  }
  if (!todo.empty()) return bfail(b, RG_ERR_CAPACITY, "capacity retries exhausted");
  b->last_ms = total_ms;
  if (restore_after) {
    for (int k = 0; k < b->n; ++k) {
      rg_system* s = b->sys[k];
      const int one = 1;
      if (restore_snapshot(s, sn[k]) || cudaMemcpy(&s->d_ctl->rebuild, &one, sizeof(int), cudaMemcpyHostToDevice))
        return bfail(b, RG_ERR_CUDA, "restore");
      s->contacts_fresh = false;
    }
    return RG_OK;
  }
  if (per) {
    for (int k = 0; k < b->n; ++k) ke_launch(b->sys[k]);
    if (cudaStreamSynchronize(b->stream)) return bfail(b, RG_ERR_CUDA, "statistics");
    for (int k = 0; k < b->n; ++k) {
      fill_stats(b->sys[k], nsteps, &per[k], true);
      per[k].device_ms = total_ms;
    }
  }
  return RG_OK;
}

}  // namespace

extern "C" {

int rg_batch_create(const rg_config* cfgs, int n_systems, rg_batch** out) {
  if (!cfgs || n_systems <= 0 || !out) return RG_ERR_ARG;
  *out = nullptr;
  rg_batch* b = new rg_batch();
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) || cudaEventCreate(&b->ev0) ||
      cudaEventCreate(&b->ev1)) {
    cudaGetLastError();
    rg_batch_destroy(b);
    return RG_ERR_CUDA;
  }
  for (int k = 0; k < n_systems; ++k) {
    rg_system* s = nullptr;
    int rc = rg_create(&cfgs[k], &s);
    if (rc != RG_OK) {
      rg_batch_destroy(b);
      return rc;
    }
    cudaStreamDestroy(s->stream);  // members share the batch stream
    s->stream = b->stream;
    b->sys.push_back(s);
    ++b->n;
  }
  b->coop_blocks = b->sys[0]->coop_blocks;
  b->cost.assign(b->n, 0.0);
  b->ser.assign(b->n, 0.0);
  b->par.assign(b->n, 0.0);
  b->team_nb.assign(b->n, 1);
  *out = b;
  return RG_OK;
}

int rg_batch_destroy(rg_batch* b) {
  if (!b) return RG_ERR_ARG;
  drop_graph(b);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (rg_system* s : b->sys) {
    s->stream = nullptr;
    rg_destroy(s);
  }
  cudaFree(b->d_views); cudaFree(b->d_teams); cudaFree(b->d_members); cudaFree(b->d_bars); cudaFree(b->d_team_ns);
  cudaFree(b->d_bulk); cudaFree(b->d_stage); cudaFree(b->d_bulk_bad);
  if (b->h_bulk_bad) cudaFreeHost(b->h_bulk_bad);
  cudaFree(b->d_segs); cudaFree(b->d_ctls); cudaFree(b->d_ctlbuf);
  if (b->h_ctlbuf) cudaFreeHost(b->h_ctlbuf);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return RG_OK;
}

int rg_batch_size(const rg_batch* b) { return b ? b->n : 0; }

rg_system* rg_batch_member(rg_batch* b, int k) {
  if (!b || k < 0 || k >= b->n) return nullptr;
  return b->sys[k];
}

const char* rg_batch_last_error(const rg_batch* b) { return b ? b->err.c_str() : ""; }

int rg_batch_set_bodies(rg_batch* b, int k, const double* radius, const double* half_height, const double* mass,
                        const double* inertia, const double* restitution) {
  if (!b || k < 0 || k >= b->n) return RG_ERR_ARG;
  b->plan_dirty = true;
  return rg_set_bodies(b->sys[k], radius, half_height, mass, inertia, restitution);
}

int rg_batch_set_state(rg_batch* b, int k, const double* x, const double* q, const double* v, const double* w) {
  if (!b || k < 0 || k >= b->n) return RG_ERR_ARG;
  return rg_set_state(b->sys[k], x, q, v, w, nullptr, nullptr);
}

int rg_batch_get_state(const rg_batch* b, int k, double* x, double* q, double* v, double* w) {
  if (!b || k < 0 || k >= b->n) return RG_ERR_ARG;
  return rg_get_state(b->sys[k], x, q, v, w, nullptr, nullptr);
}

namespace {
// Member table and staging for the bulk transfers (allocated on first use).
int bulk_setup(rg_batch* b) {
  if (b->d_bulk) return RG_OK;
  std::vector<BulkMember> t(b->n);
  long long off = 0;
  for (int k = 0; k < b->n; ++k) {
    t[k] = BulkMember{b->sys[k]->d_state, b->sys[k]->n, off};
    off += b->sys[k]->n;
  }
  b->total = off;
  if (cudaMalloc(&b->d_bulk, sizeof(BulkMember) * b->n) ||
      cudaMalloc(&b->d_stage, sizeof(double) * 13 * (size_t)off) ||
      cudaMalloc(&b->d_bulk_bad, sizeof(int)) || cudaMallocHost(&b->h_bulk_bad, sizeof(int))) {
    cudaGetLastError();
    return bfail(b, RG_ERR_CUDA, "bulk staging allocation");
  }
  cudaMemcpy(b->d_bulk, t.data(), sizeof(BulkMember) * b->n, cudaMemcpyHostToDevice);
  return RG_OK;
}
}  // namespace

// States of all members at once: x[3T], q[4T], v[3T], w[3T] with the
// members' rods concatenated in member order (T = total rods).  One copy per
// array and one device kernel, instead of per-member host staging; page-
// locked host arrays transfer at full link speed.
int rg_batch_set_state_all(rg_batch* b, const double* x, const double* q, const double* v, const double* w) {
  if (!b || !x || !q || !v || !w) return RG_ERR_ARG;
  int rc = bulk_setup(b);
  if (rc != RG_OK) return rc;
  const long long T = b->total;
  double* sx = b->d_stage;
  double* sq = sx + 3 * T;
  double* sv = sq + 4 * T;
  double* sw = sv + 3 * T;
  cudaMemcpyAsync(sx, x, sizeof(double) * 3 * T, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(sq, q, sizeof(double) * 4 * T, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(sv, v, sizeof(double) * 3 * T, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(sw, w, sizeof(double) * 3 * T, cudaMemcpyHostToDevice, b->stream);
  cudaMemsetAsync(b->d_bulk_bad, 0, sizeof(int), b->stream);
  RGL k_bulk_check<<<592, 256, 0, b->stream>>>(sx, 13 * T, b->d_bulk_bad);
  RGL k_bulk_scatter<<<592, 256, 0, b->stream>>>(static_cast<const BulkMember*>(b->d_bulk), b->n, T, sx, sq, sv, sw,
                                                 b->d_bulk_bad);
  cudaMemcpyAsync(b->h_bulk_bad, b->d_bulk_bad, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e) return bfail(b, RG_ERR_CUDA, std::string("bulk set_state: ") + cudaGetErrorString(e));
  if (*b->h_bulk_bad) return bfail(b, RG_ERR_NONFINITE, "non-finite component in the uploaded states (nothing changed)");
  for (rg_system* s : b->sys) {
    s->state_set = true;
    s->contacts_fresh = false;
  }
  return RG_OK;
}

int rg_batch_get_state_all(rg_batch* b, double* x, double* q, double* v, double* w) {
  if (!b || !x || !q || !v || !w) return RG_ERR_ARG;
  int rc = bulk_setup(b);
  if (rc != RG_OK) return rc;
  const long long T = b->total;
  double* sx = b->d_stage;
  double* sq = sx + 3 * T;
  double* sv = sq + 4 * T;
  double* sw = sv + 3 * T;
  RGL k_bulk_gather<<<592, 256, 0, b->stream>>>(static_cast<const BulkMember*>(b->d_bulk), b->n, T, sx, sq, sv, sw);
  cudaMemcpyAsync(x, sx, sizeof(double) * 3 * T, cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(q, sq, sizeof(double) * 4 * T, cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(v, sv, sizeof(double) * 3 * T, cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(w, sw, sizeof(double) * 3 * T, cudaMemcpyDeviceToHost, b->stream);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e) return bfail(b, RG_ERR_CUDA, std::string("bulk get_state: ") + cudaGetErrorString(e));
  return RG_OK;
}

int rg_batch_set_mlp(rg_batch* b, const float* params, size_t n) {
  if (!b || !params) return RG_ERR_ARG;
  for (rg_system* s : b->sys) {
    if (s->cfg.model != RG_MODEL_NSC) continue;
    int rc = rg_mlp_set_params(s, params, n);
    if (rc != RG_OK) return rc;
  }
  return RG_OK;
}

int rg_batch_set_schedule(rg_batch* b, int rods_per_block, int use_graph) {
  if (!b || rods_per_block < -1) return RG_ERR_ARG;
  b->rods_per_block = rods_per_block;
  b->use_graph = use_graph != 0;
  b->plan_dirty = true;
  drop_graph(b);
  return RG_OK;
}

int rg_batch_get_schedule(const rg_batch* b, int* rods_per_block, int* grid, int* nteams) {
  if (!b) return RG_ERR_ARG;
  if (rods_per_block) *rods_per_block = b->rods_per_block;
  if (grid) *grid = b->grid;
  if (nteams) *nteams = (int)b->teams.size();
  return RG_OK;
}

int rg_batch_get_team_times(const rg_batch* b, double* ms, int* blocks, int* members, int cap, int* nteams) {
  if (!b || !nteams) return RG_ERR_ARG;
  const int nt = (int)b->teams.size();
  *nteams = nt;
  if (nt == 0 || !b->d_team_ns) return RG_OK;
  std::vector<long long> ns(nt);
  cudaMemcpy(ns.data(), b->d_team_ns, sizeof(long long) * nt, cudaMemcpyDeviceToHost);
  for (int t = 0; t < nt && t < cap; ++t) {
    if (ms) ms[t] = 1e-6 * (double)ns[t];
    if (blocks) blocks[t] = b->teams[t].nb;
    if (members) members[t] = b->teams[t].count;
  }
  return RG_OK;
}

int rg_batch_get_costs(const rg_batch* b, double* cost_ms, int* team_blocks) {
  if (!b) return RG_ERR_ARG;
  for (int k = 0; k < b->n; ++k) {
    if (cost_ms) cost_ms[k] = b->cost[k];
    if (team_blocks) team_blocks[k] = b->team_nb[k];
  }
  return RG_OK;
}

int rg_batch_step(rg_batch* b, int nsteps, rg_step_stats* per_system) {
  if (!b || nsteps < 0) return RG_ERR_ARG;
  return batch_call(b, nsteps, per_system);
}

// Times trial_steps steps for each candidate R (bodies per block; 0 = all
// single-block teams) after two untimed steps (the first step after the state
// is put back rebuilds every neighbour list, which a running batch rarely
// does), puts the state back after each trial and keeps the fastest R.
// ms_out (optional, n_cand entries) receives the trial times.
int rg_batch_autotune(rg_batch* b, const int* candidates, int n_cand, int trial_steps, int* best_out,
                      double* ms_out) {
  if (!b || !candidates || n_cand <= 0 || trial_steps <= 0) return RG_ERR_ARG;
  for (int c = 0; c < n_cand; ++c)
    if (candidates[c] < -1) return RG_ERR_ARG;
  // cost model first: every member's own step time on the device, measured
  // with all members in single-block teams
  rg_batch_set_schedule(b, 0, b->use_graph);
  const int rc0 = batch_call(b, 2 * trial_steps, nullptr, true, 2);
  if (rc0 != RG_OK) return rc0;
  int best = candidates[0];
  double best_ms = 1e300;
  b->cost_frozen = true;
  for (int c = 0; c < n_cand; ++c) {
    rg_batch_set_schedule(b, candidates[c], b->use_graph);
    int rc = batch_call(b, trial_steps, nullptr, true, 2);  // grows buffers, builds the graph
    if (rc == RG_OK) rc = batch_call(b, trial_steps, nullptr, true, 2);
    if (rc != RG_OK) {
      b->cost_frozen = false;
      return rc;
    }
    const double ms = b->last_ms;
    if (ms_out) ms_out[c] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = candidates[c];
    }
  }
  b->cost_frozen = false;
  rg_batch_set_schedule(b, best, b->use_graph);
  if (best_out) *best_out = best;
  return RG_OK;
}

}  // extern "C"
