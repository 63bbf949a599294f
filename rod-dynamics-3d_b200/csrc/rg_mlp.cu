// rg_mlp.cu - training and batch inference of the learned PSOR warm start.
//
// No reference counterpart: the reference warm-starts PSOR from a hash map of
// last-step impulses only (src/physics/nsc_contact.cpp:305-317, :646-654).
// The network (rg_mlp_dev.cuh) is trained on records of converged impulses
// that the plain PSOR path itself produces (rg_mlp_record), with this file's
// own kernels: one fused forward + loss + backward + weight-gradient kernel
// per minibatch on tensor cores (mma.sync m16n8k16, BF16 operands, FP32
// accumulation) and one kernel that sums the blocks' partial gradients and
// applies Adam to the FP32 master weights.  BF16 copies of the weights feed
// both training and the in-step inference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "rg_internal.cuh"
#include "rg_mlp_dev.cuh"

namespace rg {

// ---------------------------------------------------------------------------
// Training: one fused kernel per minibatch.  A block of kTrainWarps warps
// takes tiles of kTrainRows rows (16 per warp) and runs, for its rows, the
// forward pass (pre-activations Z kept in shared memory, activations in
// registers: the accumulator fragment of a layer is the A fragment of the
// next), the loss, the backward pass (dH = dZ W with W read transposed from
// shared memory, dZ = dH * silu'(Z)) and the block's share of the weight
// gradients dW = dZ^T H as block-level mma.sync products over the tile's
// rows (H recomputed from Z).  Each block writes its partial gradient (and
// loss) to its own slice of a partial buffer, summing over its tiles in a
// fixed order; one reduction kernel then adds the slices in block order
// (deterministic) and applies Adam and the BF16 weight copies.
// ---------------------------------------------------------------------------
constexpr int kTrainWarps = 4;
constexpr int kTrainThreads = 32 * kTrainWarps;
constexpr int kTrainRows = 16 * kTrainWarps;      // 64 rows per tile
constexpr int kZLd = kMlpH + 8;                   // FP32 pre-activation rows (136)
constexpr int kXLd = kW1Pad + 8;                  // BF16 input rows (24)
constexpr int kDyLd = 16;                         // BF16 output-gradient rows
constexpr int kGradParams = kOffInMean;           // trained parameters
constexpr int kTrainMaxBlocks = 296;

// Shared-memory carve-up of the training kernel (byte offsets, 16-aligned).
constexpr int kTsW2 = 0;
constexpr int kTsW3 = kTsW2 + 2 * kStageWh;
constexpr int kTsSmall = kTsW3 + 2 * kStageWh;                         // W1, W4, floats (MlpStage)
constexpr int kTsX = kTsSmall + ((kStageSmallBytes + 15) / 16) * 16;
constexpr int kTsZ = kTsX + 2 * kTrainRows * kXLd;                     // Z1, Z2, Z3
constexpr int kTsDzA = kTsZ + 3 * 4 * kTrainRows * kZLd;
constexpr int kTsDzB = kTsDzA + 2 * kTrainRows * kWhLd;
constexpr int kTsDy = kTsDzB + 2 * kTrainRows * kWhLd;
constexpr int kTsBias = kTsDy + 2 * kTrainRows * kDyLd;                // [warp][b1|b2|b3|b4(8)]
constexpr int kTsLoss = kTsBias + 4 * kTrainWarps * (3 * kMlpH + 8);
constexpr int kTrainSmem = kTsLoss + 16 * kTrainWarps;
static_assert(kTrainSmem <= 227 * 1024, "training kernel shared memory");
static_assert(kTsSmall % 16 == 0 && kTsX % 16 == 0 && kTsZ % 16 == 0 && kTsDzA % 16 == 0 && kTsDzB % 16 == 0 &&
                  kTsDy % 16 == 0 && kTsBias % 16 == 0,
              "16-byte aligned regions");

struct TrainSmem {
  __nv_bfloat16 *w2, *w3;  // [128][kWhLd]
  MlpStage st;             // W1 [128][kW1Ld], W4 [8][kWhLd], biases and scales
  __nv_bfloat16* x;        // [64][kXLd] normalised inputs (columns 8..15 zero)
  float* z[3];             // [64][kZLd] pre-activations of layers 1..3
  __nv_bfloat16 *dza, *dzb;  // [64][kWhLd] BF16 dZ of two layers
  __nv_bfloat16* dy;       // [64][kDyLd] BF16 dY (columns 3..15 zero)
  float* bias;             // [warp][3 * 128 + 8] bias-gradient partial sums
  float* loss;             // [warp]
};
__device__ inline TrainSmem train_smem(unsigned char* b) {
  TrainSmem s;
  s.w2 = reinterpret_cast<__nv_bfloat16*>(b + kTsW2);
  s.w3 = reinterpret_cast<__nv_bfloat16*>(b + kTsW3);
  s.st = mlp_stage_at(b + kTsSmall);
  s.x = reinterpret_cast<__nv_bfloat16*>(b + kTsX);
  for (int l = 0; l < 3; ++l) s.z[l] = reinterpret_cast<float*>(b + kTsZ) + (size_t)l * kTrainRows * kZLd;
  s.dza = reinterpret_cast<__nv_bfloat16*>(b + kTsDzA);
  s.dzb = reinterpret_cast<__nv_bfloat16*>(b + kTsDzB);
  s.dy = reinterpret_cast<__nv_bfloat16*>(b + kTsDy);
  s.bias = reinterpret_cast<float*>(b + kTsBias);
  s.loss = reinterpret_cast<float*>(b + kTsLoss);
  return s;
}

__device__ inline unsigned short bf16_bits(__nv_bfloat16 v) { return *reinterpret_cast<unsigned short*>(&v); }
// Two BF16 values from different rows packed into one fragment register.
__device__ inline unsigned pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (unsigned)bf16_bits(lo) | ((unsigned)bf16_bits(hi) << 16);
}
// B fragment of W^T for the backward product dH = dZ W (W row-major
// [out][in] with leading dimension ldw): k = out (k-tile kt), n = in
// (n-tile nt); elements of a register come from two rows of W.
__device__ inline void load_bt(const __nv_bfloat16* W, int ldw, int nt, int kt, int lane, unsigned& b0,
                               unsigned& b1) {
  const int g = lane >> 2, t = lane & 3;
  const int n = nt * 8 + g, k = kt * 16 + 2 * t;
  b0 = pack2(W[(size_t)k * ldw + n], W[(size_t)(k + 1) * ldw + n]);
  b1 = pack2(W[(size_t)(k + 8) * ldw + n], W[(size_t)(k + 9) * ldw + n]);
}
__device__ inline float silu_grad(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}
// Accumulator fragments (16 n-tiles) -> A fragments of the next product.
__device__ inline void acc_to_a(const float (&c)[16][4], unsigned (&a)[8][4], bool act) {
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
    const float* p = c[2 * kk];
    const float* q = c[2 * kk + 1];
    if (act) {
      a[kk][0] = pack_bf16(silu(p[0]), silu(p[1]));
      a[kk][1] = pack_bf16(silu(p[2]), silu(p[3]));
      a[kk][2] = pack_bf16(silu(q[0]), silu(q[1]));
      a[kk][3] = pack_bf16(silu(q[2]), silu(q[3]));
    } else {
      a[kk][0] = pack_bf16(p[0], p[1]);
      a[kk][1] = pack_bf16(p[2], p[3]);
      a[kk][2] = pack_bf16(q[0], q[1]);
      a[kk][3] = pack_bf16(q[2], q[3]);
    }
  }
}
// Stores a warp's 16 x 128 FP32 accumulator block at rows lr0.. of Z.
__device__ inline void store_z(float* z, int lr0, const float (&c)[16][4], int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const int col = nt * 8 + 2 * t;
    *reinterpret_cast<float2*>(&z[(size_t)(lr0 + g) * kZLd + col]) = make_float2(c[nt][0], c[nt][1]);
    *reinterpret_cast<float2*>(&z[(size_t)(lr0 + g + 8) * kZLd + col]) = make_float2(c[nt][2], c[nt][3]);
  }
}

__device__ inline float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Partial gradient slice of a block: '=' on its first tile, '+=' after.
__device__ inline void part_put(float* p, int i, float v, bool first) { p[i] = first ? v : p[i] + v; }

// Block-level weight gradient dW[o][i] = Σ_r dZ[r][o] H[r][i] over the
// tile's 64 rows: output rows o in m-tiles [0, mtiles) (warp w takes m-tiles
// w, w + 4, ...), input columns [0, 8 * NTN).  dZ: BF16 rows of leading
// dimension ldz.  H: the BF16 copy of silu(Z) (Z FP32 [64][kZLd]) or, when
// zs is null, the BF16 inputs xs [64][kXLd].  Rows o < nrows and columns
// i < ncols go to part[off + o * ncols + i].
template <int NTN>
__device__ inline void block_dw(const __nv_bfloat16* dz, int ldz, int mtiles, int nrows, const float* zs,
                                const __nv_bfloat16* xs, int ncols, float* part, int off, bool first, int warp,
                                int lane) {
  const int g = lane >> 2, t = lane & 3;
  for (int mt = warp; mt < mtiles; mt += kTrainWarps) {
    const int m0 = mt * 16;
    float c[NTN][4];
#pragma unroll
    for (int j = 0; j < NTN; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < kTrainRows / 16; ++ks) {
      const int r = ks * 16 + 2 * t;
      const __nv_bfloat16* d0 = dz + (size_t)r * ldz + m0 + g;
      const unsigned a0 = pack2(d0[0], d0[ldz]);
      const unsigned a1 = pack2(d0[8], d0[ldz + 8]);
      const unsigned a2 = pack2(d0[8 * ldz], d0[9 * ldz]);
      const unsigned a3 = pack2(d0[8 * ldz + 8], d0[9 * ldz + 8]);
#pragma unroll
      for (int j = 0; j < NTN; ++j) {
        const int n = j * 8 + g;
        unsigned b0, b1;
        if (zs) {
          const float* z0 = zs + (size_t)r * kZLd + n;
          b0 = pack_bf16(silu(z0[0]), silu(z0[kZLd]));
          b1 = pack_bf16(silu(z0[8 * kZLd]), silu(z0[9 * kZLd]));
        } else {
          const __nv_bfloat16* x0 = xs + (size_t)r * kXLd + n;
          b0 = pack2(x0[0], x0[kXLd]);
          b1 = pack2(x0[8 * kXLd], x0[9 * kXLd]);
        }
        mma_bf16(c[j], a0, a1, a2, a3, b0, b1);
      }
    }
#pragma unroll
    for (int j = 0; j < NTN; ++j) {
      const int col = j * 8 + 2 * t;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int o = m0 + g + (e >= 2 ? 8 : 0), i = col + (e & 1);
        if (o < nrows && i < ncols) part_put(part, off + o * ncols + i, c[j][e], first);
      }
    }
  }
}

// Column sums over a warp's 16 rows of a 16 x 128 FP32 fragment block,
// added to sums[0..127] ('=' on the block's first tile); lanes with g = 0
// write.
__device__ inline void warp_colsum_acc(const float (&c)[16][4], float* sums, int lane, bool first) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      float v = c[nt][cc] + c[nt][2 + cc];
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 16);
      if (g == 0) {
        float* s = &sums[nt * 8 + 2 * t + cc];
        *s = first ? v : *s + v;
      }
    }
  }
}

// dZ = dH * silu'(Z) in place on the accumulator block (Z rows lr0..), and
// its BF16 copy into dzs.
__device__ inline void dz_from_dh(float (&c)[16][4], const float* z, __nv_bfloat16* dzs, int lr0, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const int col = nt * 8 + 2 * t;
    const float2 z0 = *reinterpret_cast<const float2*>(&z[(size_t)(lr0 + g) * kZLd + col]);
    const float2 z1 = *reinterpret_cast<const float2*>(&z[(size_t)(lr0 + g + 8) * kZLd + col]);
    c[nt][0] *= silu_grad(z0.x);
    c[nt][1] *= silu_grad(z0.y);
    c[nt][2] *= silu_grad(z1.x);
    c[nt][3] *= silu_grad(z1.y);
    *reinterpret_cast<unsigned*>(&dzs[(size_t)(lr0 + g) * kWhLd + col]) = pack_bf16(c[nt][0], c[nt][1]);
    *reinterpret_cast<unsigned*>(&dzs[(size_t)(lr0 + g + 8) * kWhLd + col]) = pack_bf16(c[nt][2], c[nt][3]);
  }
}
// dH = dZ W for a warp's 16 rows: dZ A fragments from dzs (BF16 rows lr0..),
// W staged [out][kWhLd].
__device__ inline void dh_product(const __nv_bfloat16* dzs, int lr0, const __nv_bfloat16* W, float (&c)[16][4],
                                  int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0f;
#pragma unroll
  for (int kt = 0; kt < 8; ++kt) {
    const __nv_bfloat16* r0 = dzs + (size_t)(lr0 + g) * kWhLd + kt * 16 + 2 * t;
    const __nv_bfloat16* r1 = r0 + 8 * kWhLd;
    const unsigned a0 = *reinterpret_cast<const unsigned*>(r0), a1 = *reinterpret_cast<const unsigned*>(r1);
    const unsigned a2 = *reinterpret_cast<const unsigned*>(r0 + 8), a3 = *reinterpret_cast<const unsigned*>(r1 + 8);
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
      unsigned b0, b1;
      load_bt(W, kWhLd, nt, kt, lane, b0, b1);
      mma_bf16(c[nt], a0, a1, a2, a3, b0, b1);
    }
  }
}
// Forward through one hidden layer from A fragments a (16 x 128) with W
// staged [out][kWhLd]: c = a W^T + bias (FP32).
__device__ inline void fwd_product(const unsigned (&a)[8][4], const __nv_bfloat16* W, const float* bias,
                                   float (&c)[16][4], int lane) {
  const int t = lane & 3;
#pragma unroll
  for (int nt = 0; nt < 16; ++nt) {
    const float bl = bias[nt * 8 + 2 * t], bh = bias[nt * 8 + 2 * t + 1];
    c[nt][0] = bl; c[nt][1] = bh; c[nt][2] = bl; c[nt][3] = bh;
  }
#pragma unroll
  for (int kt = 0; kt < 8; ++kt) {
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
      unsigned b0, b1;
      load_b(W, kWhLd, nt, kt, lane, b0, b1);
      mma_bf16(c[nt], a[kt][0], a[kt][1], a[kt][2], a[kt][3], b0, b1);
    }
  }
}

// One minibatch: rows [0, n) of feat/tgt (row-major [n][8] / [n][3]),
// gathered by idx when given.  Block b handles tiles b, b + gridDim.x, ...
// and leaves its partial gradient in part[b * kGradParams ...] and its
// partial loss (Σ squared error) in loss_part[b].
__global__ void __launch_bounds__(kTrainThreads, 1)
    k_mlp_train_fb(MlpDev M, const float* feat, const float* tgt, const int* idx, int n, float* part,
                   float* loss_part) {
  extern __shared__ __align__(16) unsigned char tsm[];
  const TrainSmem S = train_smem(tsm);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  stage_bf16(S.w2, kWhLd, M.w2, kMlpH, kMlpH);
  stage_bf16(S.w3, kWhLd, M.w3, kMlpH, kMlpH);
  stage_small(S.st, M);
  stage_wait();
  __syncthreads();
  const MlpSmall q = S.st.small();
  float* mypart = part + (size_t)blockIdx.x * kGradParams;
  const int ntiles = (n + kTrainRows - 1) / kTrainRows;
  const float inv_n3 = 1.0f / (float)(n * kMlpOut);
  const int lr0 = warp * 16;
  float* bsum = S.bias + warp * (3 * kMlpH + 8);
  float lsum = 0.0f;
  bool first = true;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, first = false) {
    const int row0 = tile * kTrainRows;
    // ---- forward (per warp, rows lr0..lr0+15 of the tile) ----
    unsigned x0, x1;
    {
      float v[4];
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const int lr = lr0 + g + 8 * rr, r = row0 + lr;
        const int rid = r < n ? (idx ? idx[r] : r) : 0;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int k = 2 * t + cc;
          v[rr * 2 + cc] = r < n ? (feat[(size_t)rid * kMlpIn + k] - q.in_mean[k]) * q.in_scale[k] : 0.0f;
        }
        *reinterpret_cast<unsigned*>(&S.x[(size_t)lr * kXLd + 2 * t]) = pack_bf16(v[rr * 2], v[rr * 2 + 1]);
        *reinterpret_cast<unsigned*>(&S.x[(size_t)lr * kXLd + 8 + 2 * t]) = 0u;
      }
      x0 = pack_bf16(v[0], v[1]);
      x1 = pack_bf16(v[2], v[3]);
    }
    unsigned a[8][4];
    float c[16][4];
#pragma unroll
    for (int nt = 0; nt < 16; ++nt) {
      const float bl = q.b1[nt * 8 + 2 * t], bh = q.b1[nt * 8 + 2 * t + 1];
      c[nt][0] = bl; c[nt][1] = bh; c[nt][2] = bl; c[nt][3] = bh;
      unsigned b0, b1;
      load_b(S.st.w1, kW1Ld, nt, 0, lane, b0, b1);
      mma_bf16(c[nt], x0, x1, 0u, 0u, b0, b1);
    }
    store_z(S.z[0], lr0, c, lane);
    acc_to_a(c, a, true);
    fwd_product(a, S.w2, q.b2, c, lane);
    store_z(S.z[1], lr0, c, lane);
    acc_to_a(c, a, true);
    fwd_product(a, S.w3, q.b3, c, lane);
    store_z(S.z[2], lr0, c, lane);
    acc_to_a(c, a, true);
    // output layer, loss and dY (outputs 2t, 2t + 1 of rows g, g + 8)
    float dy[4];
    {
      float y[4];
      const float bl = 2 * t < kMlpOut ? q.b4[2 * t] : 0.0f, bh = 2 * t + 1 < kMlpOut ? q.b4[2 * t + 1] : 0.0f;
      y[0] = bl; y[1] = bh; y[2] = bl; y[3] = bh;
#pragma unroll
      for (int kt = 0; kt < 8; ++kt) {
        unsigned b0, b1;
        load_b(S.st.w4, kWhLd, 0, kt, lane, b0, b1);
        mma_bf16(y, a[kt][0], a[kt][1], a[kt][2], a[kt][3], b0, b1);
      }
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const int lr = lr0 + g + 8 * rr, r = row0 + lr;
        const int rid = r < n ? (idx ? idx[r] : r) : 0;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int o = 2 * t + cc;
          float d = 0.0f;
          if (o < kMlpOut && r < n) {
            const float tn = (tgt[(size_t)rid * kMlpOut + o] - feat[(size_t)rid * kMlpIn + 4 + o]) / q.out_scale[o];
            const float diff = y[rr * 2 + cc] - tn;
            lsum += diff * diff;
            d = 2.0f * diff * inv_n3;
          }
          dy[rr * 2 + cc] = d;
        }
        *reinterpret_cast<unsigned*>(&S.dy[(size_t)lr * kDyLd + 2 * t]) = pack_bf16(dy[rr * 2], dy[rr * 2 + 1]);
        *reinterpret_cast<unsigned*>(&S.dy[(size_t)lr * kDyLd + 8 + 2 * t]) = 0u;
      }
    }
    // ---- backward through the output layer: db4, dH3 = dY W4 ----
    {
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        float v = dy[cc] + dy[2 + cc];
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        if (g == 0) {
          float* s = &bsum[3 * kMlpH + 2 * t + cc];
          *s = first ? v : *s + v;
        }
      }
      const unsigned ya0 = pack_bf16(dy[0], dy[1]), ya1 = pack_bf16(dy[2], dy[3]);
#pragma unroll
      for (int nt = 0; nt < 16; ++nt) {
        c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0f;
        const int nn = nt * 8 + g;
        const unsigned b0 = pack2(S.st.w4[(size_t)(2 * t) * kWhLd + nn], S.st.w4[(size_t)(2 * t + 1) * kWhLd + nn]);
        mma_bf16(c[nt], ya0, ya1, 0u, 0u, b0, 0u);
      }
    }
    // layer 3: dZ3 -> dza, db3; dH2 = dZ3 W3
    dz_from_dh(c, S.z[2], S.dza, lr0, lane);
    warp_colsum_acc(c, bsum + 2 * kMlpH, lane, first);
    __syncwarp();
    dh_product(S.dza, lr0, S.w3, c, lane);
    // layer 2: dZ2 -> dzb, db2
    dz_from_dh(c, S.z[1], S.dzb, lr0, lane);
    warp_colsum_acc(c, bsum + kMlpH, lane, first);
    __syncthreads();  // every warp's dZ3, dZ2 and dY are in shared memory
    block_dw<16>(S.dza, kWhLd, kMlpH / 16, kMlpH, S.z[1], nullptr, kMlpH, mypart, kOffW3, first, warp, lane);
    block_dw<16>(S.dy, kDyLd, 1, kMlpOut, S.z[2], nullptr, kMlpH, mypart, kOffW4, first, warp, lane);
    __syncthreads();  // dza is free again
    // layer 1: dH1 = dZ2 W2, dZ1 -> dza, db1
    dh_product(S.dzb, lr0, S.w2, c, lane);
    dz_from_dh(c, S.z[0], S.dza, lr0, lane);
    warp_colsum_acc(c, bsum, lane, first);
    __syncthreads();
    block_dw<16>(S.dzb, kWhLd, kMlpH / 16, kMlpH, S.z[0], nullptr, kMlpH, mypart, kOffW2, first, warp, lane);
    block_dw<2>(S.dza, kWhLd, kMlpH / 16, kMlpH, nullptr, S.x, kMlpIn, mypart, kOffW1, first, warp, lane);
    __syncthreads();  // shared tiles are reused by the next tile
  }
  // bias gradients and loss: sum the warps' partial sums in warp order
  lsum = warp_sum_f(lsum);
  if (lane == 0) S.loss[warp] = lsum;
  __syncthreads();
  const bool any = blockIdx.x < ntiles;
  for (int i = threadIdx.x; i < 3 * kMlpH + kMlpOut; i += blockDim.x) {
    float v = 0.0f;
    if (any)
      for (int w = 0; w < kTrainWarps; ++w) v += S.bias[w * (3 * kMlpH + 8) + i];
    const int off = i < kMlpH ? kOffB1 + i : i < 2 * kMlpH ? kOffB2 + i - kMlpH
                  : i < 3 * kMlpH ? kOffB3 + i - 2 * kMlpH : kOffB4 + i - 3 * kMlpH;
    mypart[off] = v;
  }
  if (threadIdx.x == 0) {
    float l = 0.0f;
    for (int w = 0; w < kTrainWarps; ++w) l += S.loss[w];
    loss_part[blockIdx.x] = any ? l : 0.0f;
  }
  if (!any) {  // a block without a tile contributes zero weight gradients
    for (int i = threadIdx.x; i < kGradParams; i += blockDim.x) {
      const bool bias = (i >= kOffB1 && i < kOffW2) || (i >= kOffB2 && i < kOffW3) || (i >= kOffB3 && i < kOffW4) ||
                        i >= kOffB4;
      if (!bias) mypart[i] = 0.0f;
    }
  }
}

// g_i = Σ_b part[b][i] in block order (deterministic), i < kGradParams.
__device__ inline float grad_sum(const float* part, int nblk, int i) {
  float g = 0.0f;
  for (int b = 0; b < nblk; ++b) g += part[(size_t)b * kGradParams + i];
  return g;
}
__global__ void k_mlp_grad_sum(const float* part, int nblk, float* G) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGradParams; i += gridDim.x * blockDim.x)
    G[i] = grad_sum(part, nblk, i);
}
// Adam on the trained parameters from the summed partial gradients, then
// the BF16 weight copies the next minibatch and the in-step inference read
// (their padding stays zero from the full copy).
__global__ void k_mlp_adam(const float* part, int nblk, float* P, float* m, float* v, float lr, float b1, float b2,
                           float eps, float bc1, float bc2, __nv_bfloat16* w1, __nv_bfloat16* w2,
                           __nv_bfloat16* w3, __nv_bfloat16* w4) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGradParams; i += gridDim.x * blockDim.x) {
    const float g = grad_sum(part, nblk, i);
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float p = P[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    P[i] = p;
    const __nv_bfloat16 pb = __float2bfloat16(p);
    if (i < kOffB1) {
      w1[(i / kMlpIn) * kW1Pad + i % kMlpIn] = pb;
    } else if (i >= kOffW2 && i < kOffB2) {
      w2[i - kOffW2] = pb;
    } else if (i >= kOffW3 && i < kOffB3) {
      w3[i - kOffW3] = pb;
    } else if (i >= kOffW4 && i < kOffB4) {
      w4[i - kOffW4] = pb;
    }
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
  // training workspace
  float *part = nullptr, *loss = nullptr;  // per-block partial gradients / losses
  float *G = nullptr, *Am = nullptr, *Av = nullptr;
  int* idx = nullptr;              // minibatch order of an epoch (n)
  size_t nidx = 0;
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

static cudaError_t ensure_workspace(rg_system* s) {
  MlpHost& H = host_of(s);
  if (H.part) return cudaSuccess;
  cudaError_t e;
  if ((e = cudaMalloc(&H.part, sizeof(float) * (size_t)kTrainMaxBlocks * kGradParams))) return e;
  if ((e = cudaMalloc(&H.loss, sizeof(float) * kTrainMaxBlocks))) return e;
  if ((e = cudaMalloc(&H.G, sizeof(float) * kMlpParams))) return e;
  if ((e = cudaMalloc(&H.Am, sizeof(float) * kMlpParams))) return e;
  if ((e = cudaMalloc(&H.Av, sizeof(float) * kMlpParams))) return e;
  return cudaFuncSetAttribute(k_mlp_train_fb, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
}

// Forward + backward of rows [0, n) (feat/tgt row-major, gathered by idx
// when given) into the per-block partial gradients and losses; returns the
// number of blocks (partial slices) used.
static int forward_backward(rg_system* s, const float* feat, const float* tgt, const int* idx, int n) {
  MlpHost& H = host_of(s);
  const int tiles = (n + kTrainRows - 1) / kTrainRows;
  const int nblk = tiles < kTrainMaxBlocks ? tiles : kTrainMaxBlocks;
  RGL k_mlp_train_fb<<<nblk, kTrainThreads, kTrainSmem, s->stream>>>(mlp_dev(s), feat, tgt, idx, n, H.part,
                                                                     H.loss);
  return nblk;
}

static double read_loss(rg_system* s, int n, int nblk) {
  MlpHost& H = host_of(s);
  std::vector<float> part(nblk);
  cudaMemcpyAsync(part.data(), H.loss, sizeof(float) * nblk, cudaMemcpyDeviceToHost, s->stream);
  cudaStreamSynchronize(s->stream);
  double l = 0;
  for (int i = 0; i < nblk; ++i) l += part[i];
  return l / ((double)n * kMlpOut);
}

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
  cudaFree(H.part); cudaFree(H.loss); cudaFree(H.G); cudaFree(H.Am); cudaFree(H.Av);
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
  if (ensure_workspace(s)) return RG_ERR_CUDA;
  float *df = nullptr, *dt = nullptr;
  if (cudaMalloc(&df, sizeof(float) * kMlpIn * n) || cudaMalloc(&dt, sizeof(float) * kMlpOut * n)) return RG_ERR_CUDA;
  cudaMemcpy(df, features, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice);
  cudaMemcpy(dt, targets, sizeof(float) * kMlpOut * n, cudaMemcpyHostToDevice);
  const int nblk = forward_backward(s, df, dt, nullptr, (int)n);
  cudaMemsetAsync(H.G, 0, sizeof(float) * kMlpParams, s->stream);
  RGL k_mlp_grad_sum<<<grid_for(kGradParams, 256), 256, 0, s->stream>>>(H.part, nblk, H.G);
  double l = read_loss(s, (int)n, nblk);
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
  if (ensure_workspace(s)) return RG_ERR_CUDA;
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
  if (H.nidx < n) {
    cudaFree(H.idx);
    if (cudaMalloc(&H.idx, sizeof(int) * n)) return RG_ERR_CUDA;
    H.nidx = n;
  }
  std::mt19937_64 rng(seed ^ 0xA5A5A5A5ull);
  std::vector<int> perm(n);
  for (size_t i = 0; i < n; ++i) perm[i] = (int)i;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const MlpDev M = mlp_dev(s);
  long step = 0;
  double last = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    // the epoch's order goes up once; each minibatch reads its slice
    if (cudaMemcpyAsync(H.idx, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s->stream)) return RG_ERR_CUDA;
    double ep_loss = 0;
    int nb = 0;
    for (size_t b0 = 0; b0 + batch <= n; b0 += batch) {
      const int nblk = forward_backward(s, H.feat, H.tgt, H.idx + b0, batch);
      ++step;
      float bc1 = 1.0f - std::pow(b1, (float)step), bc2 = 1.0f - std::pow(b2, (float)step);
      RGL k_mlp_adam<<<grid_for(kGradParams, 256), 256, 0, s->stream>>>(
          H.part, nblk, H.P, H.Am, H.Av, lr, b1, b2, eps, bc1, bc2, const_cast<__nv_bfloat16*>(M.w1),
          const_cast<__nv_bfloat16*>(M.w2), const_cast<__nv_bfloat16*>(M.w3), const_cast<__nv_bfloat16*>(M.w4));
      if (ep == epochs - 1) {
        ep_loss += read_loss(s, batch, nblk);
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
