// ref_cuda_harness.cu - drives the reference's own FP32 CUDA broad phase.
//
// TEST INFRASTRUCTURE / SECONDARY GPU BASELINE ONLY.  Compiled by
// oracle/Makefile (target refcuda) with the reference's
// src/physics/cuda_broadphase.cu and rigid_body.cpp, in place, for sm_100a;
// only bench.py's secondary-baseline leg loads it.  The product never does.
//
// refcuda_detect builds the std::vector<RigidBody> the reference's solvers
// pass (capsules: x, q, cap.r, cap.h) and calls
// cudaDetectCapsulePairsTwoPass (include/physics/cuda_broadphase.hpp:95-101):
// host upload, AABB kernel, O(N^2) AABB pair kernel, Lumelsky narrow-phase
// kernel, download.  It returns the pairs (a < b, in the kernel's atomic
// order, then sorted here), the reference's own per-stage timings and the
// wall time of the call.
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "physics/cuda_broadphase.hpp"
#include "physics/rigid_body.hpp"

extern "C" int refcuda_detect(int n, const double* x, const double* q, const double* radius,
                              const double* half_height, double margin, int pbc, double sx, double sy,
                              double sz, int32_t* pairs, size_t cap, size_t* n_out, double* stats,
                              double* wall_ms) {
  if (n < 0 || !x || !q || !radius || !half_height || !n_out) return 1;
  std::vector<RigidBody> bodies(n);
  for (int i = 0; i < n; ++i) {
    RigidBody& b = bodies[i];
    b.type = ShapeType::Capsule;
    b.x = glm::vec3((float)x[3 * i], (float)x[3 * i + 1], (float)x[3 * i + 2]);
    b.q = glm::quat((float)q[4 * i], (float)q[4 * i + 1], (float)q[4 * i + 2], (float)q[4 * i + 3]);
    b.cap.r = (float)radius[i];
    b.cap.h = (float)half_height[i];
  }
  std::vector<GpuContactRaw> raw;
  CudaTwoPassStats st;
  const auto t0 = std::chrono::steady_clock::now();
  cudaDetectCapsulePairsTwoPass(bodies, (float)margin, pbc != 0, (float)sx, (float)sy, (float)sz, raw, &st);
  const auto t1 = std::chrono::steady_clock::now();
  if (wall_ms) *wall_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  if (stats) {
    stats[0] = st.upload_ms; stats[1] = st.aabb_ms; stats[2] = st.broadphase_ms;
    stats[3] = st.narrowphase_ms; stats[4] = st.download_ms;
    stats[5] = st.candidates; stats[6] = st.contacts;
  }
  std::vector<std::pair<int, int>> pr(raw.size());
  for (size_t k = 0; k < raw.size(); ++k) pr[k] = {std::min(raw[k].a, raw[k].b), std::max(raw[k].a, raw[k].b)};
  std::sort(pr.begin(), pr.end());
  *n_out = pr.size();
  for (size_t k = 0; k < pr.size() && k < cap && pairs; ++k) {
    pairs[2 * k] = pr[k].first;
    pairs[2 * k + 1] = pr[k].second;
  }
  return 0;
}
