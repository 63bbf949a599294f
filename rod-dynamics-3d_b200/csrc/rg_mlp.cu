// rg_mlp.cu - training and batch inference of the learned PSOR warm start.
//
// No reference counterpart: the reference warm-starts PSOR from a hash map of
// last-step impulses only (src/physics/nsc_contact.cpp:305-317, :646-654).
// The network (rg_mlp_dev.cuh) is trained on records of converged impulses
// that the plain PSOR path itself produces (rg_mlp_record), with this file's
// own forward and backward kernels: a strided, shared-memory-tiled GEMM on
// tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulation), SiLU
// and loss kernels, and Adam on FP32 master weights.  BF16 copies of the
// weights feed both training and the in-step inference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "rg_internal.cuh"
#include "rg_mlp_dev.cuh"

namespace rg {

// ---------------------------------------------------------------------------
// GEMM: C[M x N] (FP32) = A[M x K] * B[K x N] (+ C), A and B BF16 with
// arbitrary element strides: A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn].
// Block 128 threads (4 warps) computes a 64 x 64 tile, K in steps of 32.
// ---------------------------------------------------------------------------
constexpr int kGM = 64, kGN = 64, kGK = 32, kGPad = 8;

__global__ void __launch_bounds__(128) k_gemm_bf16(const __nv_bfloat16* A, long sam, long sak,
                                                   const __nv_bfloat16* B, long sbk, long sbn, float* C,
                                                   long ldc, int M, int N, int K, int accumulate) {
  __shared__ __align__(16) __nv_bfloat16 As[kGM][kGK + kGPad];
  __shared__ __align__(16) __nv_bfloat16 Bs[kGN][kGK + kGPad];  // [n][k]
  const int m0 = blockIdx.y * kGM, n0 = blockIdx.x * kGN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  float acc[2][4][4];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 4; ++j)
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;
  const __nv_bfloat16 zero = __float2bfloat16(0.0f);
  for (int k0 = 0; k0 < K; k0 += kGK) {
    for (int e = threadIdx.x; e < kGM * kGK; e += blockDim.x) {
      int mm = e / kGK, kk = e % kGK;
      int m = m0 + mm, k = k0 + kk;
      As[mm][kk] = (m < M && k < K) ? A[m * sam + k * sak] : zero;
    }
    for (int e = threadIdx.x; e < kGN * kGK; e += blockDim.x) {
      int nn = e / kGK, kk = e % kGK;
      int n = n0 + nn, k = k0 + kk;
      Bs[nn][kk] = (n < N && k < K) ? B[k * sbk + n * sbn] : zero;
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < kGK; ks += 16) {
      unsigned a[2][4], b[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + g;
        a[i][0] = *reinterpret_cast<const unsigned*>(&As[r][ks + 2 * t]);
        a[i][1] = *reinterpret_cast<const unsigned*>(&As[r + 8][ks + 2 * t]);
        a[i][2] = *reinterpret_cast<const unsigned*>(&As[r][ks + 2 * t + 8]);
        a[i][3] = *reinterpret_cast<const unsigned*>(&As[r + 8][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + g;
        b[j][0] = *reinterpret_cast<const unsigned*>(&Bs[c][ks + 2 * t]);
        b[j][1] = *reinterpret_cast<const unsigned*>(&Bs[c][ks + 2 * t + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i][0], a[i][1], a[i][2], a[i][3], b[j][0], b[j][1]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        int m = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0);
        int n = n0 + wn + j * 8 + 2 * t + (r & 1);
        if (m < M && n < N) {
          float v = acc[i][j][r];
          if (accumulate) v += C[m * ldc + n];
          C[m * ldc + n] = v;
        }
      }
}

static void gemm(const __nv_bfloat16* A, long sam, long sak, const __nv_bfloat16* B, long sbk, long sbn, float* C,
                 long ldc, int M, int N, int K, cudaStream_t st, int accumulate = 0) {
  dim3 grid((N + kGN - 1) / kGN, (M + kGM - 1) / kGM);
  RGL k_gemm_bf16<<<grid, 128, 0, st>>>(A, sam, sak, B, sbk, sbn, C, ldc, M, N, K, accumulate);
}

// ---------------------------------------------------------------------------
// Elementwise kernels.
// ---------------------------------------------------------------------------
// X[b][0..15] = normalised features (8..15 zero), rows gathered by idx.
__global__ void k_mlp_input(const float* feat, const int* idx, int n, const float* P, __nv_bfloat16* X) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * kW1Pad; e += gridDim.x * blockDim.x) {
    int b = e / kW1Pad, k = e % kW1Pad;
    float v = 0.0f;
    if (k < kMlpIn) {
      int r = idx ? idx[b] : b;
      v = (feat[(size_t)r * kMlpIn + k] - P[kOffInMean + k]) * P[kOffInScale + k];
    }
    X[e] = __float2bfloat16(v);
  }
}
// Z += bias; H = bf16(silu(Z)).
__global__ void k_bias_silu(float* Z, const float* bias, int n, int w, __nv_bfloat16* H) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * w; e += gridDim.x * blockDim.x) {
    float z = Z[e] + bias[e % w];
    Z[e] = z;
    H[e] = __float2bfloat16(silu(z));
  }
}
// Output layer: Y = Z4 + b4 against the normalised impulse change
// T = (λ - λ_prev) / s; dY = 2 (Y - T) / (n * 3); per-block loss sums.
__global__ void k_out_loss(float* Z4, const float* P, const float* feat, const float* tgt, const int* idx, int n,
                           float* dY, __nv_bfloat16* dYb, float* loss_part) {
  __shared__ float sm[32];
  float l = 0.0f;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * kW4Pad; e += gridDim.x * blockDim.x) {
    int b = e / kW4Pad, o = e % kW4Pad;
    float d = 0.0f;
    if (o < kMlpOut) {
      float y = Z4[e] + P[kOffB4 + o];
      Z4[e] = y;
      int r = idx ? idx[b] : b;
      float tn = (tgt[(size_t)r * kMlpOut + o] - feat[(size_t)r * kMlpIn + 4 + o]) / P[kOffOutScale + o];
      float diff = y - tn;
      l += diff * diff;
      d = 2.0f * diff / (float)(n * kMlpOut);
    }
    dY[e] = d;
    dYb[e] = __float2bfloat16(d);
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    float s = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[w];
    loss_part[blockIdx.x] = s;
  }
}
// dZ = dH * silu'(Z), FP32 and BF16 copies.
__global__ void k_silu_back(const float* dH, const float* Z, int n, float* dZ, __nv_bfloat16* dZb) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n * kMlpH; e += gridDim.x * blockDim.x) {
    float z = Z[e];
    float s = 1.0f / (1.0f + __expf(-z));
    float d = dH[e] * (s * (1.0f + z * (1.0f - s)));
    dZ[e] = d;
    dZb[e] = __float2bfloat16(d);
  }
}
// db[c] = Σ_b dZ[b][c] for c < w_out (one block per column).
__global__ void k_bias_grad(const float* dZ, int n, int w, int w_out, float* db) {
  __shared__ float sm[32];
  const int c = blockIdx.x;
  if (c >= w_out) return;
  float s = 0.0f;
  for (int b = threadIdx.x; b < n; b += blockDim.x) s += dZ[(size_t)b * w + c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) t += sm[w2];
    db[c] = t;
  }
}
// Copies a padded gradient block ([rows][ldp]) into the parameter layout.
__global__ void k_unpad(const float* src, int rows, int cols, int ldp, float* dst) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < rows * cols; e += gridDim.x * blockDim.x)
    dst[e] = src[(e / cols) * ldp + (e % cols)];
}
// Adam on the network parameters [0, kOffInMean).
__global__ void k_adam(float* P, const float* G, float* m, float* v, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kOffInMean; i += gridDim.x * blockDim.x) {
    float g = G[i];
    float mi = b1 * m[i] + (1.0f - b1) * g;
    float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}
// BF16 padded weight copies from the FP32 parameter vector.
__global__ void k_weights_bf16(const float* P, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3,
                               __nv_bfloat16* w4) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, str = gridDim.x * blockDim.x;
  for (int e = tid; e < kMlpH * kW1Pad; e += str) {
    int n = e / kW1Pad, k = e % kW1Pad;
    w1[e] = __float2bfloat16(k < kMlpIn ? P[kOffW1 + n * kMlpIn + k] : 0.0f);
  }
  for (int e = tid; e < kMlpH * kMlpH; e += str) {
    w2[e] = __float2bfloat16(P[kOffW2 + e]);
    w3[e] = __float2bfloat16(P[kOffW3 + e]);
  }
  for (int e = tid; e < kW4Pad * kMlpH; e += str) {
    int n = e / kMlpH;
    w4[e] = __float2bfloat16(n < kMlpOut ? P[kOffW4 + e] : 0.0f);
  }
}
// Batch inference with the in-step warp routine (feature-major input):
// predicted impulse = previous impulse (features 4-6) + network output.
__global__ void k_mlp_infer(MlpDev M, const float* featT, int n, float* outT) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int row0 = warp * 16; row0 < n; row0 += nw * 16) {
    mlp_warp(M, featT, n, row0, n, outT, lane);
    __syncwarp();
    if (lane < 16 && row0 + lane < n)
      for (int o = 0; o < kMlpOut; ++o) outT[(size_t)o * n + row0 + lane] += featT[(size_t)(4 + o) * n + row0 + lane];
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Host-side network state.
// ---------------------------------------------------------------------------
struct MlpHost {
  float* P = nullptr;              // FP32 parameters (kMlpParams)
  __nv_bfloat16* wb = nullptr;     // w1 | w2 | w3 | w4 (padded)
  // training workspace (sized for cap rows)
  int cap = 0;
  __nv_bfloat16 *X = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr, *dZb = nullptr, *dYb = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *Z4 = nullptr, *dZ = nullptr, *dH = nullptr, *dY = nullptr;
  float *G = nullptr, *Gpad = nullptr, *Am = nullptr, *Av = nullptr, *loss = nullptr;
  int* idx = nullptr;
  float *feat = nullptr, *tgt = nullptr;  // dataset on the device
  size_t nfeat = 0;
};

static MlpHost& host_of(rg_system* s) { return *reinterpret_cast<MlpHost*>(s->mlp_host); }

static cudaError_t ensure_net(rg_system* s) {
  if (!s->mlp_host) s->mlp_host = new MlpHost();
  MlpHost& H = host_of(s);
  cudaError_t e = cudaSuccess;
  if (!H.P) {
    if ((e = cudaMalloc(&H.P, sizeof(float) * kMlpParams))) return e;
    if ((e = cudaMemset(H.P, 0, sizeof(float) * kMlpParams))) return e;
    size_t nb = kMlpH * kW1Pad + 2 * kMlpH * kMlpH + kW4Pad * kMlpH;
    if ((e = cudaMalloc(&H.wb, sizeof(__nv_bfloat16) * nb))) return e;
  }
  return e;
}

MlpDev mlp_dev(rg_system* s) {
  MlpHost& H = host_of(s);
  MlpDev M;
  M.w1 = H.wb;
  M.w2 = M.w1 + kMlpH * kW1Pad;
  M.w3 = M.w2 + kMlpH * kMlpH;
  M.w4 = M.w3 + kMlpH * kMlpH;
  M.p = H.P;
  return M;
}

static void refresh_bf16(rg_system* s) {
  MlpHost& H = host_of(s);
  MlpDev M = mlp_dev(s);
  RGL k_weights_bf16<<<64, 256, 0, s->stream>>>(H.P, const_cast<__nv_bfloat16*>(M.w1),
                                                 const_cast<__nv_bfloat16*>(M.w2),
                                                 const_cast<__nv_bfloat16*>(M.w3),
                                                 const_cast<__nv_bfloat16*>(M.w4));
}

static cudaError_t ensure_workspace(rg_system* s, int rows) {
  MlpHost& H = host_of(s);
  if (H.cap >= rows) return cudaSuccess;
  cudaFree(H.X); cudaFree(H.H1); cudaFree(H.H2); cudaFree(H.H3); cudaFree(H.dZb); cudaFree(H.dYb);
  cudaFree(H.Z1); cudaFree(H.Z2); cudaFree(H.Z3); cudaFree(H.Z4); cudaFree(H.dZ); cudaFree(H.dH);
  cudaFree(H.dY); cudaFree(H.G); cudaFree(H.Gpad); cudaFree(H.Am); cudaFree(H.Av); cudaFree(H.loss);
  cudaFree(H.idx);
  H.cap = rows;
  const size_t r = rows;
  cudaError_t e;
  if ((e = cudaMalloc(&H.X, sizeof(__nv_bfloat16) * r * kW1Pad))) return e;
  if ((e = cudaMalloc(&H.H1, sizeof(__nv_bfloat16) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.H2, sizeof(__nv_bfloat16) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.H3, sizeof(__nv_bfloat16) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.dZb, sizeof(__nv_bfloat16) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.dYb, sizeof(__nv_bfloat16) * r * kW4Pad))) return e;
  if ((e = cudaMalloc(&H.Z1, sizeof(float) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.Z2, sizeof(float) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.Z3, sizeof(float) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.Z4, sizeof(float) * r * kW4Pad))) return e;
  if ((e = cudaMalloc(&H.dZ, sizeof(float) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.dH, sizeof(float) * r * kMlpH))) return e;
  if ((e = cudaMalloc(&H.dY, sizeof(float) * r * kW4Pad))) return e;
  if ((e = cudaMalloc(&H.G, sizeof(float) * kMlpParams))) return e;
  if ((e = cudaMalloc(&H.Gpad, sizeof(float) * kMlpH * kMlpH))) return e;
  if ((e = cudaMalloc(&H.Am, sizeof(float) * kMlpParams))) return e;
  if ((e = cudaMalloc(&H.Av, sizeof(float) * kMlpParams))) return e;
  if ((e = cudaMalloc(&H.loss, sizeof(float) * 256))) return e;
  return cudaMalloc(&H.idx, sizeof(int) * r);
}

// Forward + backward on rows (feat/tgt row-major, gathered by idx when
// given); gradients into H.G, loss (mean squared error in normalised target
// units) returned through the loss partials.
static void forward_backward(rg_system* s, const float* feat, const float* tgt, const int* idx, int n) {
  MlpHost& H = host_of(s);
  MlpDev M = mlp_dev(s);
  cudaStream_t st = s->stream;
  const int eb = 256, eg = grid_for((long long)n * kMlpH, eb, 1024);
  RGL k_mlp_input<<<grid_for((long long)n * kW1Pad, eb, 1024), eb, 0, st>>>(feat, idx, n, H.P, H.X);
  // forward: Z = H_prev W^T (W row-major [out][in])
  gemm(H.X, kW1Pad, 1, M.w1, 1, kW1Pad, H.Z1, kMlpH, n, kMlpH, kW1Pad, st);
  RGL k_bias_silu<<<eg, eb, 0, st>>>(H.Z1, H.P + kOffB1, n, kMlpH, H.H1);
  gemm(H.H1, kMlpH, 1, M.w2, 1, kMlpH, H.Z2, kMlpH, n, kMlpH, kMlpH, st);
  RGL k_bias_silu<<<eg, eb, 0, st>>>(H.Z2, H.P + kOffB2, n, kMlpH, H.H2);
  gemm(H.H2, kMlpH, 1, M.w3, 1, kMlpH, H.Z3, kMlpH, n, kMlpH, kMlpH, st);
  RGL k_bias_silu<<<eg, eb, 0, st>>>(H.Z3, H.P + kOffB3, n, kMlpH, H.H3);
  gemm(H.H3, kMlpH, 1, M.w4, 1, kMlpH, H.Z4, kW4Pad, n, kW4Pad, kMlpH, st);
  RGL k_out_loss<<<128, 256, 0, st>>>(H.Z4, H.P, feat, tgt, idx, n, H.dY, H.dYb, H.loss);
  // backward
  cudaMemsetAsync(H.G, 0, sizeof(float) * kMlpParams, st);
  // layer 4: dW4 = dY^T H3 ([8 x 128]), db4, dH3 = dY W4
  gemm(H.dYb, 1, kW4Pad, H.H3, kMlpH, 1, H.Gpad, kMlpH, kW4Pad, kMlpH, n, st);
  RGL k_unpad<<<4, 256, 0, st>>>(H.Gpad, kMlpOut, kMlpH, kMlpH, H.G + kOffW4);
  RGL k_bias_grad<<<kW4Pad, 256, 0, st>>>(H.dY, n, kW4Pad, kMlpOut, H.G + kOffB4);
  gemm(H.dYb, kW4Pad, 1, M.w4, kMlpH, 1, H.dH, kMlpH, n, kMlpH, kW4Pad, st);
  // layer 3
  RGL k_silu_back<<<eg, eb, 0, st>>>(H.dH, H.Z3, n, H.dZ, H.dZb);
  gemm(H.dZb, 1, kMlpH, H.H2, kMlpH, 1, H.G + kOffW3, kMlpH, kMlpH, kMlpH, n, st);
  RGL k_bias_grad<<<kMlpH, 256, 0, st>>>(H.dZ, n, kMlpH, kMlpH, H.G + kOffB3);
  gemm(H.dZb, kMlpH, 1, M.w3, kMlpH, 1, H.dH, kMlpH, n, kMlpH, kMlpH, st);
  // layer 2
  RGL k_silu_back<<<eg, eb, 0, st>>>(H.dH, H.Z2, n, H.dZ, H.dZb);
  gemm(H.dZb, 1, kMlpH, H.H1, kMlpH, 1, H.G + kOffW2, kMlpH, kMlpH, kMlpH, n, st);
  RGL k_bias_grad<<<kMlpH, 256, 0, st>>>(H.dZ, n, kMlpH, kMlpH, H.G + kOffB2);
  gemm(H.dZb, kMlpH, 1, M.w2, kMlpH, 1, H.dH, kMlpH, n, kMlpH, kMlpH, st);
  // layer 1: dW1 = dZ1^T X ([128 x 16] -> first 8 columns)
  RGL k_silu_back<<<eg, eb, 0, st>>>(H.dH, H.Z1, n, H.dZ, H.dZb);
  gemm(H.dZb, 1, kMlpH, H.X, kW1Pad, 1, H.Gpad, kW1Pad, kMlpH, kW1Pad, n, st);
  RGL k_unpad<<<8, 256, 0, st>>>(H.Gpad, kMlpH, kMlpIn, kW1Pad, H.G + kOffW1);
  RGL k_bias_grad<<<kMlpH, 256, 0, st>>>(H.dZ, n, kMlpH, kMlpH, H.G + kOffB1);
}

static double read_loss(rg_system* s, int n) {
  MlpHost& H = host_of(s);
  float part[128];
  cudaMemcpyAsync(part, H.loss, sizeof(part), cudaMemcpyDeviceToHost, s->stream);
  cudaStreamSynchronize(s->stream);
  double l = 0;
  for (int i = 0; i < 128; ++i) l += part[i];
  return l / ((double)n * kMlpOut);
}

// Normalisation from the data; He-uniform weights from the seed.
static void init_params(std::vector<float>& P, const float* feat, const float* tgt, size_t n, uint64_t seed) {
  P.assign(kMlpParams, 0.0f);
  for (int k = 0; k < kMlpIn; ++k) {
    double m = 0, v = 0;
    for (size_t i = 0; i < n; ++i) m += feat[i * kMlpIn + k];
    m /= (double)n;
    for (size_t i = 0; i < n; ++i) { double d = feat[i * kMlpIn + k] - m; v += d * d; }
    double sd = std::sqrt(v / (double)n);
    P[kOffInMean + k] = (float)m;
    P[kOffInScale + k] = sd > 1e-30 ? (float)(1.0 / sd) : 1.0f;
  }
  for (int o = 0; o < kMlpOut; ++o) {
    double v = 0;
    for (size_t i = 0; i < n; ++i) {
      double d = (double)tgt[i * kMlpOut + o] - feat[i * kMlpIn + 4 + o];
      v += d * d;
    }
    double rms = std::sqrt(v / (double)n);
    P[kOffOutScale + o] = rms > 1e-30 ? (float)rms : 1.0f;
  }
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_in, int count) {
    double lim = std::sqrt(6.0 / fan_in);
    std::uniform_real_distribution<double> U(-lim, lim);
    for (int i = 0; i < count; ++i) P[off + i] = (float)U(rng);
  };
  fill(kOffW1, kMlpIn, kMlpH * kMlpIn);
  fill(kOffW2, kMlpH, kMlpH * kMlpH);
  fill(kOffW3, kMlpH, kMlpH * kMlpH);
  fill(kOffW4, kMlpH, kMlpOut * kMlpH);
  for (int i = 0; i < kMlpOut * kMlpH; ++i) P[kOffW4 + i] *= 0.1f;
}

void mlp_free(rg_system* s) {
  if (!s->mlp_host) return;
  MlpHost& H = host_of(s);
  cudaFree(H.P); cudaFree(H.wb);
  cudaFree(H.X); cudaFree(H.H1); cudaFree(H.H2); cudaFree(H.H3); cudaFree(H.dZb); cudaFree(H.dYb);
  cudaFree(H.Z1); cudaFree(H.Z2); cudaFree(H.Z3); cudaFree(H.Z4); cudaFree(H.dZ); cudaFree(H.dH);
  cudaFree(H.dY); cudaFree(H.G); cudaFree(H.Gpad); cudaFree(H.Am); cudaFree(H.Av); cudaFree(H.loss);
  cudaFree(H.idx); cudaFree(H.feat); cudaFree(H.tgt);
  delete &H;
  s->mlp_host = nullptr;
}

}  // namespace rg

using namespace rg;

extern "C" {

size_t rg_mlp_param_count(void) { return (size_t)kMlpParams; }

int rg_mlp_set_params(rg_system* s, const float* params, size_t n) {
  if (!s || !params || n != (size_t)kMlpParams) return RG_ERR_ARG;
  if (ensure_net(s)) return RG_ERR_CUDA;
  cudaMemcpy(host_of(s).P, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
  refresh_bf16(s);
  if (cudaStreamSynchronize(s->stream)) return RG_ERR_CUDA;
  s->mlp_ready = true;
  return RG_OK;
}

int rg_mlp_get_params(const rg_system* s, float* params, size_t n) {
  if (!s || !params || n != (size_t)kMlpParams || !s->mlp_host) return RG_ERR_ARG;
  cudaMemcpy(params, reinterpret_cast<MlpHost*>(s->mlp_host)->P, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost);
  return RG_OK;
}

int rg_mlp_record(rg_system* s, int enable, size_t cap) {
  if (!s) return RG_ERR_ARG;
  if (!enable) {
    s->recording = false;
    return RG_OK;
  }
  if (cap == 0 || cap > (size_t)1 << 30) return RG_ERR_ARG;
  cudaFree(s->d_rec_x);
  cudaFree(s->d_rec_y);
  if (cudaMalloc(&s->d_rec_x, sizeof(float) * kMlpIn * cap) || cudaMalloc(&s->d_rec_y, sizeof(float) * kMlpOut * cap))
    return RG_ERR_CUDA;
  s->rec_cap = (int)cap;
  s->recording = true;
  int zero = 0;
  cudaMemcpy(&s->d_ctl->rec_n, &zero, sizeof(int), cudaMemcpyHostToDevice);
  return RG_OK;
}

int rg_mlp_records(const rg_system* s, float* features, float* targets, size_t cap, size_t* n) {
  if (!s || !n) return RG_ERR_ARG;
  int rn = 0;
  cudaMemcpy(&rn, &s->d_ctl->rec_n, sizeof(int), cudaMemcpyDeviceToHost);
  if (rn > s->rec_cap) rn = s->rec_cap;
  *n = (size_t)rn;
  size_t m = cap < (size_t)rn ? cap : (size_t)rn;
  if (m && features) cudaMemcpy(features, s->d_rec_x, sizeof(float) * kMlpIn * m, cudaMemcpyDeviceToHost);
  if (m && targets) cudaMemcpy(targets, s->d_rec_y, sizeof(float) * kMlpOut * m, cudaMemcpyDeviceToHost);
  return (size_t)rn > cap ? RG_ERR_CAPACITY : RG_OK;
}

// Loss and gradient (parameter layout) of one batch at the current weights.
int rg_mlp_grad(rg_system* s, const float* features, const float* targets, size_t n, float* grad, float* loss) {
  if (!s || !features || !targets || n == 0 || n > (1u << 24)) return RG_ERR_ARG;
  if (!s->mlp_host || !reinterpret_cast<MlpHost*>(s->mlp_host)->P) return RG_ERR_STATE;
  MlpHost& H = host_of(s);
  if (ensure_workspace(s, (int)n)) return RG_ERR_CUDA;
  float *df = nullptr, *dt = nullptr;
  if (cudaMalloc(&df, sizeof(float) * kMlpIn * n) || cudaMalloc(&dt, sizeof(float) * kMlpOut * n)) return RG_ERR_CUDA;
  cudaMemcpy(df, features, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dt, targets, sizeof(float) * kMlpOut * n, cudaMemcpyHostToDevice);
  forward_backward(s, df, dt, nullptr, (int)n);
  double l = read_loss(s, (int)n);
  if (grad) cudaMemcpy(grad, H.G, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost);
  if (loss) *loss = (float)l;
  cudaFree(df);
  cudaFree(dt);
  return cudaGetLastError() == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}

int rg_mlp_train(rg_system* s, const float* features, const float* targets, size_t n, int epochs, int batch,
                 float lr, uint64_t seed, float* final_loss) {
  if (!s || !features || !targets || n < 16 || epochs <= 0 || batch < 16 || !(lr > 0)) return RG_ERR_ARG;
  if (ensure_net(s)) return RG_ERR_CUDA;
  MlpHost& H = host_of(s);
  std::vector<float> P;
  init_params(P, features, targets, n, seed);
  cudaMemcpy(H.P, P.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice);
  refresh_bf16(s);
  if (batch > (int)n) batch = (int)n;
  if (ensure_workspace(s, batch)) return RG_ERR_CUDA;
  if (H.nfeat < n) {
    cudaFree(H.feat);
    cudaFree(H.tgt);
    if (cudaMalloc(&H.feat, sizeof(float) * kMlpIn * n) || cudaMalloc(&H.tgt, sizeof(float) * kMlpOut * n))
      return RG_ERR_CUDA;
    H.nfeat = n;
  }
  cudaMemcpy(H.feat, features, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice);
  cudaMemcpy(H.tgt, targets, sizeof(float) * kMlpOut * n, cudaMemcpyHostToDevice);
  cudaMemset(H.Am, 0, sizeof(float) * kMlpParams);
  cudaMemset(H.Av, 0, sizeof(float) * kMlpParams);
  std::mt19937_64 rng(seed ^ 0xA5A5A5A5ull);
  std::vector<int> perm(n);
  for (size_t i = 0; i < n; ++i) perm[i] = (int)i;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  long step = 0;
  double last = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    double ep_loss = 0;
    int nb = 0;
    for (size_t b0 = 0; b0 + batch <= n; b0 += batch) {
      cudaMemcpyAsync(H.idx, perm.data() + b0, sizeof(int) * batch, cudaMemcpyHostToDevice, s->stream);
      forward_backward(s, H.feat, H.tgt, H.idx, batch);
      ++step;
      float bc1 = 1.0f - std::pow(b1, (float)step), bc2 = 1.0f - std::pow(b2, (float)step);
      RGL k_adam<<<64, 256, 0, s->stream>>>(H.P, H.G, H.Am, H.Av, lr, b1, b2, eps, bc1, bc2);
      refresh_bf16(s);
      if (ep == epochs - 1) {
        ep_loss += read_loss(s, batch);
        ++nb;
      }
    }
    if (nb) last = ep_loss / nb;
  }
  if (cudaStreamSynchronize(s->stream) || cudaGetLastError()) return RG_ERR_CUDA;
  s->mlp_ready = true;
  if (final_loss) *final_loss = (float)last;
  return RG_OK;
}

int rg_mlp_infer(rg_system* s, const float* features, float* out, size_t n) {
  if (!s || !features || !out || n == 0) return RG_ERR_ARG;
  if (!s->mlp_ready) return RG_ERR_STATE;
  float *fT = nullptr, *oT = nullptr;
  if (cudaMalloc(&fT, sizeof(float) * kMlpIn * n) || cudaMalloc(&oT, sizeof(float) * kMlpOut * n)) return RG_ERR_CUDA;
  std::vector<float> t(kMlpIn * n);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < kMlpIn; ++k) t[(size_t)k * n + i] = features[i * kMlpIn + k];
  cudaMemcpy(fT, t.data(), sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice);
  int warps = (int)((n + 15) / 16);
  RGL k_mlp_infer<<<(warps + 7) / 8, 256, 0, s->stream>>>(mlp_dev(s), fT, (int)n, oT);
  std::vector<float> o(kMlpOut * n);
  cudaMemcpyAsync(o.data(), oT, sizeof(float) * kMlpOut * n, cudaMemcpyDeviceToHost, s->stream);
  cudaError_t e = cudaStreamSynchronize(s->stream);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < kMlpOut; ++k) out[i * kMlpOut + k] = o[(size_t)k * n + i];
  cudaFree(fT);
  cudaFree(oT);
  return e == cudaSuccess ? RG_OK : RG_ERR_CUDA;
}

// Batched systems: implemented in rg_batch.cu.

}  // extern "C"
