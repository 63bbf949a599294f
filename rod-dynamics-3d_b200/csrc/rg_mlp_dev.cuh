// rg_mlp_dev.cuh - the learned PSOR warm start on tensor cores.
//
// MLP 8 -> 128 -> 128 -> 128 -> 3, SiLU, BF16 weights and activations, FP32
// accumulation.  One warp evaluates 16 contacts with mma.sync m16n8k16
// (BF16 x BF16 -> FP32): the accumulator fragment of one layer is exactly the
// A fragment of the next (rows g, g+8; columns 2t, 2t+1 of two adjacent
// n-tiles), so hidden activations never leave registers.
//
// Features per contact (computed where the manifold row is built):
//   0 gap φ, 1 v_n, 2 v_t1, 3 v_t2 (pre-solve relative velocity in the
//   contact frame), 4-6 previous-step impulses (λn, λt1, λt2; 0 for a new
//   contact), 7 contact-graph degree (other contacts on the two dynamic
//   bodies).  Targets: converged (λn, λt1, λt2) of plain PSOR.  The network
//   predicts the change from the previous impulse (features 4-6), so a
//   persistent contact starts from its cached impulse plus a correction and
//   a new one from the prediction alone; the change is scaled by the
//   output scales (its RMS over the training records).
#pragma once
#include <cuda_bf16.h>

#include "rg_common.cuh"

namespace rg {

constexpr int kMlpIn = 8, kMlpH = 128, kMlpOut = 3;
// Float parameter vector layout (rg_mlp_param_count in include/rodgpu.h).
constexpr int kOffW1 = 0;                          // 128 x 8
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;    // 128
constexpr int kOffW2 = kOffB1 + kMlpH;             // 128 x 128
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;             // 128 x 128
constexpr int kOffB3 = kOffW3 + kMlpH * kMlpH;
constexpr int kOffW4 = kOffB3 + kMlpH;             // 3 x 128
constexpr int kOffB4 = kOffW4 + kMlpOut * kMlpH;   // 3
constexpr int kOffInMean = kOffB4 + kMlpOut;       // 8
constexpr int kOffInScale = kOffInMean + kMlpIn;   // 8
constexpr int kOffOutScale = kOffInScale + kMlpIn; // 3
constexpr int kMlpParams = kOffOutScale + kMlpOut;

// BF16 device copy used by inference: weights padded to mma tiles,
// row-major [out][in]; W1 is 128 x 16 (inputs zero-padded), W4 is 8 x 128.
struct MlpDev {
  const __nv_bfloat16 *w1, *w2, *w3, *w4;
  const float* p;  // FP32 parameter vector (biases, normalisation)
};
constexpr int kW1Pad = 16, kW4Pad = 8;

__device__ inline unsigned pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}
// SiLU with the fast exponential and division: the network runs in BF16, so
// their few-ulp FP32 error is far below its resolution, and a warp's
// inference is a long chain of these (three layers x 64 values per lane).
__device__ inline float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }

// Not volatile: the MMA has no side effects, so the compiler may interleave
// independent accumulator chains (a volatile statement keeps every MMA in
// program order, and each then waits for the one before it).
__device__ inline void mma_bf16(float* c, unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                unsigned b1) {
  asm(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// B fragment of W (row-major [n][k], leading dimension ldk) for n-tile nt,
// k-tile kt: (k = 2t..2t+1, n = g) and (k = 2t+8.., n = g).
__device__ inline void load_b(const __nv_bfloat16* W, int ldk, int nt, int kt, int lane, unsigned& b0,
                              unsigned& b1) {
  const int g = lane >> 2, t = lane & 3;
  const __nv_bfloat16* row = W + (size_t)(nt * 8 + g) * ldk + kt * 16 + 2 * t;
  b0 = *reinterpret_cast<const unsigned*>(row);
  b1 = *reinterpret_cast<const unsigned*>(row + 8);
}

// One hidden layer 128 -> 128: a[kt] (4 regs each, 8 k-tiles) -> out a;
// W row-major [n][k] with leading dimension ldw.  Four n-tiles at a time:
// their accumulation chains are independent, so four MMAs are in flight
// (each chain still adds its k-tiles in order).
__device__ inline void hidden_layer(unsigned (&a)[8][4], const __nv_bfloat16* W, int ldw, const float* bias,
                                    int lane) {
  const int t = lane & 3;
  unsigned na[8][4];
#pragma unroll
  for (int grp = 0; grp < 4; ++grp) {
    float acc[4][4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int nt = 4 * grp + h;
      const float bl = bias[nt * 8 + 2 * t], bh = bias[nt * 8 + 2 * t + 1];
      acc[h][0] = bl; acc[h][1] = bh; acc[h][2] = bl; acc[h][3] = bh;
    }
#pragma unroll
    for (int kt = 0; kt < 8; ++kt) {
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        unsigned b0, b1;
        load_b(W, ldw, 4 * grp + h, kt, lane, b0, b1);
        mma_bf16(acc[h], a[kt][0], a[kt][1], a[kt][2], a[kt][3], b0, b1);
      }
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int kk = 2 * grp + q;
      na[kk][0] = pack_bf16(silu(acc[2 * q][0]), silu(acc[2 * q][1]));
      na[kk][1] = pack_bf16(silu(acc[2 * q][2]), silu(acc[2 * q][3]));
      na[kk][2] = pack_bf16(silu(acc[2 * q + 1][0]), silu(acc[2 * q + 1][1]));
      na[kk][3] = pack_bf16(silu(acc[2 * q + 1][2]), silu(acc[2 * q + 1][3]));
    }
  }
#pragma unroll
  for (int kk = 0; kk < 8; ++kk)
#pragma unroll
    for (int r = 0; r < 4; ++r) a[kk][r] = na[kk][r];
}

// Small parameters of one evaluation: biases, b4 padded to 8 with zeros,
// input normalisation and output scales (global parameter vector or a
// staged shared-memory copy).
struct MlpSmall {
  const float *b1, *b2, *b3, *b4, *in_mean, *in_scale, *out_scale;
};
__device__ inline MlpSmall mlp_small_global(const float* P) {
  return MlpSmall{P + kOffB1, P + kOffB2, P + kOffB3, P + kOffB4, P + kOffInMean, P + kOffInScale,
                  P + kOffOutScale};
}

// Layer 1 (8 -> 128, SiLU) for rows row0..row0+15 of feat (float, [8][ld]);
// rows >= n read as zero.  w1 row-major [128][k], leading dimension ld1.
__device__ inline void mlp_layer1(const __nv_bfloat16* w1, int ld1, const MlpSmall& q, const float* feat, int ld,
                                  int row0, int n, int lane, unsigned (&a)[8][4]) {
  const int g = lane >> 2, t = lane & 3;
  // layer 1 input fragment: X (16 rows x 16 k, inputs 8..15 are zero)
  unsigned x0, x1;
  {
    float v[4];
    const int rows[2] = {row0 + g, row0 + g + 8};
    for (int rr = 0; rr < 2; ++rr) {
      for (int cc = 0; cc < 2; ++cc) {
        int k = 2 * t + cc;
        int r = rows[rr];
        float f = r < n ? feat[(size_t)k * ld + r] : 0.0f;
        v[rr * 2 + cc] = (f - q.in_mean[k]) * q.in_scale[k];
      }
    }
    x0 = pack_bf16(v[0], v[1]);
    x1 = pack_bf16(v[2], v[3]);
  }
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
    float acc[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kk + h;
      const float bl = q.b1[nt * 8 + 2 * t], bh = q.b1[nt * 8 + 2 * t + 1];
      acc[h][0] = bl; acc[h][1] = bh; acc[h][2] = bl; acc[h][3] = bh;
      unsigned b0, b1;
      load_b(w1, ld1, nt, 0, lane, b0, b1);
      mma_bf16(acc[h], x0, x1, 0u, 0u, b0, b1);
    }
    a[kk][0] = pack_bf16(silu(acc[0][0]), silu(acc[0][1]));
    a[kk][1] = pack_bf16(silu(acc[0][2]), silu(acc[0][3]));
    a[kk][2] = pack_bf16(silu(acc[1][0]), silu(acc[1][1]));
    a[kk][3] = pack_bf16(silu(acc[1][2]), silu(acc[1][3]));
  }
}

// Output layer (128 -> 3): writes the outputs times out_scale to out
// ([3][ld]); rows >= n are skipped.  w4 row-major [8][128], leading
// dimension ld4 (rows 3..7 zero).
__device__ inline void mlp_layer4(const unsigned (&a)[8][4], const __nv_bfloat16* w4, int ld4, const MlpSmall& q,
                                  float* out, int ld, int row0, int n, int lane) {
  const int g = lane >> 2, t = lane & 3;
  float acc[4];
  {
    const float bl = 2 * t < kMlpOut ? q.b4[2 * t] : 0.0f;
    const float bh = 2 * t + 1 < kMlpOut ? q.b4[2 * t + 1] : 0.0f;
    acc[0] = bl; acc[1] = bh; acc[2] = bl; acc[3] = bh;
#pragma unroll
    for (int kt = 0; kt < 8; ++kt) {
      unsigned b0, b1;
      load_b(w4, ld4, 0, kt, lane, b0, b1);
      mma_bf16(acc, a[kt][0], a[kt][1], a[kt][2], a[kt][3], b0, b1);
    }
  }
  // c0,c1: row g, outputs 2t, 2t+1; c2,c3: row g+8
  const int rows[2] = {row0 + g, row0 + g + 8};
  for (int rr = 0; rr < 2; ++rr) {
    int r = rows[rr];
    if (r >= n) continue;
    for (int cc = 0; cc < 2; ++cc) {
      int o = 2 * t + cc;
      if (o < kMlpOut) out[(size_t)o * ld + r] = acc[rr * 2 + cc] * q.out_scale[o];
    }
  }
}

// Evaluates the MLP for rows row0..row0+15 of feat (float, [8][ld]) and
// writes the unscaled outputs times out_scale to out ([3][ld]); rows >= n
// are ignored.  All 32 lanes of the warp must call it.  Weights are read
// from global memory.
__device__ inline void mlp_warp(const MlpDev& M, const float* feat, int ld, int row0, int n, float* out,
                                int lane) {
  const MlpSmall q = mlp_small_global(M.p);
  unsigned a[8][4];
  mlp_layer1(M.w1, kW1Pad, q, feat, ld, row0, n, lane, a);
  hidden_layer(a, M.w2, kMlpH, q.b2, lane);
  hidden_layer(a, M.w3, kMlpH, q.b3, lane);
  mlp_layer4(a, M.w4, kMlpH, q, out, ld, row0, n, lane);
}

// ---- shared-memory staging of the weights ---------------------------------
// Padded row strides: eight rows of a B fragment fall in distinct banks.
constexpr int kW1Ld = kW1Pad + 8;          // 24 (48 B rows)
constexpr int kWhLd = kMlpH + 8;           // 136 (272 B rows)
constexpr int kStageW1 = kMlpH * kW1Ld;    // elements
constexpr int kStageW4 = kW4Pad * kWhLd;
constexpr int kStageWh = kMlpH * kWhLd;    // one hidden layer
constexpr int kStageFloats = 3 * kMlpH + 8 + 8 + 8 + 8;  // b1 b2 b3 b4(8) mean scale outscale(8)
// bytes of the small part (W1, W4, floats)
constexpr int kStageSmallBytes = 2 * (kStageW1 + kStageW4) + 4 * kStageFloats;

struct MlpStage {
  __nv_bfloat16* w1;  // kStageW1
  __nv_bfloat16* w4;  // kStageW4
  float* f;           // kStageFloats
  __device__ MlpSmall small() const {
    return MlpSmall{f, f + kMlpH, f + 2 * kMlpH, f + 3 * kMlpH, f + 3 * kMlpH + 8, f + 3 * kMlpH + 16,
                    f + 3 * kMlpH + 24};
  }
};
// Carves the small part from a 16-byte aligned buffer of kStageSmallBytes.
__device__ inline MlpStage mlp_stage_at(void* buf) {
  MlpStage s;
  s.w1 = reinterpret_cast<__nv_bfloat16*>(buf);
  s.w4 = s.w1 + kStageW1;
  s.f = reinterpret_cast<float*>(s.w4 + kStageW4);
  return s;
}

// 16-byte asynchronous copy global -> shared (no register round trip; all
// of a thread's copies are in flight together until stage_wait).
__device__ inline void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// Waits for this thread's asynchronous copies; a block barrier must follow
// before other threads read them.
__device__ inline void stage_wait() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Block-cooperative asynchronous copy of rows x cols BF16 (cols a multiple
// of 8, both 16-byte aligned) into a padded shared-memory matrix; complete
// after stage_wait and a block barrier.
__device__ inline void stage_bf16(__nv_bfloat16* dst, int ldd, const __nv_bfloat16* src, int rows, int cols) {
  const int vpr = cols / 8;
  for (int v = threadIdx.x; v < rows * vpr; v += blockDim.x) {
    const int r = v / vpr, c = v - r * vpr;
    cp_async16(dst + (size_t)r * ldd + c * 8, src + (size_t)r * cols + c * 8);
  }
}
// Block-cooperative copy of W1, W4 (asynchronous, see stage_bf16) and the
// small parameters.
__device__ inline void stage_small(const MlpStage& s, const MlpDev& M) {
  stage_bf16(s.w1, kW1Ld, M.w1, kMlpH, kW1Pad);
  stage_bf16(s.w4, kWhLd, M.w4, kW4Pad, kMlpH);
  const float* P = M.p;
  for (int i = threadIdx.x; i < kStageFloats; i += blockDim.x) {
    float v = 0.0f;
    if (i < 3 * kMlpH) v = P[(i < kMlpH ? kOffB1 : i < 2 * kMlpH ? kOffB2 - kMlpH : kOffB3 - 2 * kMlpH) + i];
    else if (i < 3 * kMlpH + 8) v = i - 3 * kMlpH < kMlpOut ? P[kOffB4 + i - 3 * kMlpH] : 0.0f;
    else if (i < 3 * kMlpH + 16) v = P[kOffInMean + i - 3 * kMlpH - 8];
    else if (i < 3 * kMlpH + 24) v = P[kOffInScale + i - 3 * kMlpH - 16];
    else v = i - 3 * kMlpH - 24 < kMlpOut ? P[kOffOutScale + i - 3 * kMlpH - 24] : 0.0f;
    s.f[i] = v;
  }
}

// Impulse prediction projected onto the admissible set: λn >= 0 and the
// Coulomb cone |λt| <= μ λn.
__device__ inline void cone_clamp(double& ln, double& l1, double& l2, double mu) {
  ln = ln > 0.0 ? ln : 0.0;
  double lim = mu * ln;
  double m = sqrt(l1 * l1 + l2 * l2);
  if (m > lim) {
    double s = m > 0.0 ? lim / m : 0.0;
    l1 *= s;
    l2 *= s;
  }
}

}  // namespace rg
