// Learned far-field order selector: a 3 x 32 tanh MLP (FP32 weights) that predicts, for an
// M2L pair, log10 of the relative acceleration error of an order-q M2L for every order class q
// (error relative to the source's monopole acceleration M_s / r^2).
//
// Features (TC_NFEAT = 8, standardised with the training set's mean and deviation):
//   log(Rt/r), log(Rs/r), log(Pn_s[2] / (Pn_s[0] Rs^2)), log(Pn_s[4] / (Pn_s[0] Rs^4)),
//   log(Pn_s[6] / (Pn_s[0] Rs^6)), log(Pn_s[8] / (Pn_s[0] Rs^8)), log(N_s), log(N_t)
// i.e. distance over cell radii, the per-degree multipole power of the source and the two
// cells' particle counts.  Training data come from the FMM itself (tc_train.cuh): M2L at each
// order class against exact P2P for pairs drawn from a real interaction list.
//
// Forward, backward (mean-squared error on the log errors) and Adam are hand-written kernels;
// one thread per sample, weights staged in shared memory.
#pragma once
#include "tc_select.cuh"

namespace tc {

constexpr int kMlpIn = TC_NFEAT, kMlpH = 32, kMlpOutMax = TC_MAX_CLASSES;
// parameter layout: W1[H][IN] b1[H] W2[H][H] b2[H] W3[H][H] b3[H] W4[OUT][H] b4[OUT]
__host__ __device__ constexpr int tc_mlp_nparam(int nout) {
  return kMlpH * kMlpIn + kMlpH + 2 * (kMlpH * kMlpH + kMlpH) + nout * kMlpH + nout;
}
constexpr int kMlpParamMax = kMlpH * kMlpIn + kMlpH + 2 * (kMlpH * kMlpH + kMlpH) + kMlpOutMax * kMlpH + kMlpOutMax;

struct TcMlpNorm {
  float mean[kMlpIn], inv_std[kMlpIn];
  float out_mean;  // outputs are learned as offsets from this value
};

__device__ __forceinline__ float tc_clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// hardware tanh approximation (one MUFU op), used for inference over every pair
__device__ __forceinline__ float tc_tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// raw features of one pair (before standardisation)
__device__ __forceinline__ void tc_pair_features(const TcCells& c, int t, int s, const double* pn, int P, float* f) {
  double dx = c.X[t] - c.X[s], dy = c.Y[t] - c.Y[s], dz = c.Z[t] - c.Z[s];
  double r = sqrt(dx * dx + dy * dy + dz * dz);
  double rt = c.R[t], rs = c.R[s];
  const double* ps = pn + (size_t)s * (P + 1);
  double p0 = fmax(ps[0], 1e-300);
  f[0] = (float)log(rt / r);
  f[1] = (float)log(rs / r);
  for (int j = 0; j < 4; j++) {
    int deg = 2 * (j + 1);
    double v = deg <= P ? ps[deg] / (p0 * pow(rs, (double)deg)) : 0.0;
    f[2 + j] = tc_clampf((float)log(fmax(v, 1e-30)), -69.f, 10.f);
  }
  f[6] = (float)log((double)c.nbody[s]);
  f[7] = (float)log((double)c.nbody[t]);
}

// forward pass; a1..a3 hold the hidden activations (for the backward pass).  FAST uses the
// hardware tanh approximation (inference only; training uses tanhf).
template <bool FAST = false>
__device__ __forceinline__ void tc_mlp_forward(const float* __restrict__ w, int nout, const float* x, float* a1,
                                               float* a2, float* a3, float* y) {
  const float* W1 = w;
  const float* b1 = W1 + kMlpH * kMlpIn;
  const float* W2 = b1 + kMlpH;
  const float* b2 = W2 + kMlpH * kMlpH;
  const float* W3 = b2 + kMlpH;
  const float* b3 = W3 + kMlpH * kMlpH;
  const float* W4 = b3 + kMlpH;
  const float* b4 = W4 + nout * kMlpH;
  for (int j = 0; j < kMlpH; j++) {
    float s = b1[j];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) s += W1[j * kMlpIn + i] * x[i];
    a1[j] = FAST ? tc_tanh_fast(s) : tanhf(s);
  }
  for (int j = 0; j < kMlpH; j++) {
    float s = b2[j];
#pragma unroll 8
    for (int i = 0; i < kMlpH; i++) s += W2[j * kMlpH + i] * a1[i];
    a2[j] = FAST ? tc_tanh_fast(s) : tanhf(s);
  }
  for (int j = 0; j < kMlpH; j++) {
    float s = b3[j];
#pragma unroll 8
    for (int i = 0; i < kMlpH; i++) s += W3[j * kMlpH + i] * a2[i];
    a3[j] = FAST ? tc_tanh_fast(s) : tanhf(s);
  }
  for (int j = 0; j < nout; j++) {
    float s = b4[j];
#pragma unroll 8
    for (int i = 0; i < kMlpH; i++) s += W4[j * kMlpH + i] * a3[i];
    y[j] = s;
  }
}

// The same network on the tensor cores, for the 32 pairs of a warp at once: each layer is a
// [32 pairs x K] x [K x 32] product in mma.sync m16n8k8 TF32 tiles with FP32 accumulation; the
// activations pass between layers through the warp's shared buffer.  TF32 keeps 10 bits of the
// operands, so the outputs (log10 errors) differ from the FP32 forward by about 1e-3 -- far below
// the network's own scatter (0.2 dex).
struct TcMlpTc {
  static constexpr int S1 = 12, S = 36;  // padded row strides (conflict-free fragment loads)
  float W1[kMlpH * S1], W2[kMlpH * S], W3[kMlpH * S], W4[8 * S];
  float b1[kMlpH], b2[kMlpH], b3[kMlpH], b4[8];
};
constexpr int kMlpActS = 36;  // row stride of a warp's activation buffer (32 rows)

__device__ __forceinline__ float tc_to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// weights (the flat layout of tc_mlp_forward) -> TF32, padded rows; W4 / b4 rows >= nout zero
__device__ __forceinline__ void tc_mlp_tc_load(TcMlpTc& T, const float* __restrict__ w, int nout, int tid,
                                               int nthr) {
  const float* W1 = w;
  const float* b1 = W1 + kMlpH * kMlpIn;
  const float* W2 = b1 + kMlpH;
  const float* b2 = W2 + kMlpH * kMlpH;
  const float* W3 = b2 + kMlpH;
  const float* b3 = W3 + kMlpH * kMlpH;
  const float* W4 = b3 + kMlpH;
  const float* b4 = W4 + nout * kMlpH;
  for (int i = tid; i < kMlpH * kMlpIn; i += nthr) T.W1[(i / kMlpIn) * TcMlpTc::S1 + i % kMlpIn] = tc_to_tf32(W1[i]);
  for (int i = tid; i < kMlpH * kMlpH; i += nthr) {
    T.W2[(i / kMlpH) * TcMlpTc::S + i % kMlpH] = tc_to_tf32(W2[i]);
    T.W3[(i / kMlpH) * TcMlpTc::S + i % kMlpH] = tc_to_tf32(W3[i]);
  }
  for (int i = tid; i < 8 * kMlpH; i += nthr)
    T.W4[(i / kMlpH) * TcMlpTc::S + i % kMlpH] = i / kMlpH < nout ? tc_to_tf32(W4[i]) : 0.f;
  for (int i = tid; i < kMlpH; i += nthr) {
    T.b1[i] = b1[i];
    T.b2[i] = b2[i];
    T.b3[i] = b3[i];
  }
  for (int i = tid; i < 8; i += nthr) T.b4[i] = i < nout ? b4[i] : 0.f;
}

__device__ __forceinline__ void tc_mma_tf32(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// one layer in place in act (32 rows): out[r][n] = f(bias[n] + sum_k act[r][k] W[n][k]) for the
// NT * 8 outputs; fragment layouts of m16n8k8: A (g, t) (g + 8, t) (g, t + 4) (g + 8, t + 4),
// B (k = t, n = g) (k = t + 4, n = g), C (g, 2t) (g, 2t + 1) (g + 8, 2t) (g + 8, 2t + 1), with
// g = lane / 4, t = lane % 4
template <int K, int NT, bool TANH>
__device__ __forceinline__ void tc_mlp_tc_layer(float* act, const float* W, int ws, const float* bias, int lane) {
  const int g = lane >> 2, t = lane & 3;
  float acc[2][NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; nt++) {
    const float b0 = bias[nt * 8 + 2 * t], b1 = bias[nt * 8 + 2 * t + 1];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      acc[mt][nt][0] = acc[mt][nt][2] = b0;
      acc[mt][nt][1] = acc[mt][nt][3] = b1;
    }
  }
  // each weight fragment is loaded once and feeds both 16-row tiles
#pragma unroll
  for (int kt = 0; kt < K / 8; kt++) {
    uint32_t a[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
      const float* r0 = act + (mt * 16 + g) * kMlpActS + kt * 8;
      const float* r1 = r0 + 8 * kMlpActS;
      a[mt][0] = __float_as_uint(tc_to_tf32(r0[t]));
      a[mt][1] = __float_as_uint(tc_to_tf32(r1[t]));
      a[mt][2] = __float_as_uint(tc_to_tf32(r0[t + 4]));
      a[mt][3] = __float_as_uint(tc_to_tf32(r1[t + 4]));
    }
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      const float* wr = W + (nt * 8 + g) * ws + kt * 8;
      const uint32_t b[2] = {__float_as_uint(wr[t]), __float_as_uint(wr[t + 4])};
      tc_mma_tf32(acc[0][nt], a[0], b);
      tc_mma_tf32(acc[1][nt], a[1], b);
    }
  }
  __syncwarp();  // every row is read by every lane before any is overwritten
#pragma unroll
  for (int mt = 0; mt < 2; mt++) {
#pragma unroll
    for (int nt = 0; nt < NT; nt++) {
      float* o0 = act + (mt * 16 + g) * kMlpActS + nt * 8 + 2 * t;
      float* o1 = o0 + 8 * kMlpActS;
      o0[0] = TANH ? tc_tanh_fast(acc[mt][nt][0]) : acc[mt][nt][0];
      o0[1] = TANH ? tc_tanh_fast(acc[mt][nt][1]) : acc[mt][nt][1];
      o1[0] = TANH ? tc_tanh_fast(acc[mt][nt][2]) : acc[mt][nt][2];
      o1[1] = TANH ? tc_tanh_fast(acc[mt][nt][3]) : acc[mt][nt][3];
    }
  }
  __syncwarp();
}

// warp-wide: every lane passes its pair's standardised features x and gets its outputs y
template <int NOUT>
__device__ __forceinline__ void tc_mlp_infer_tc(const TcMlpTc& T, float* act, const float* x, float* y, int lane) {
  static_assert(NOUT <= 8, "one output tile");
#pragma unroll
  for (int i = 0; i < kMlpIn; i++) act[lane * kMlpActS + i] = x[i];
  __syncwarp();
  tc_mlp_tc_layer<kMlpIn, 4, true>(act, T.W1, TcMlpTc::S1, T.b1, lane);
  tc_mlp_tc_layer<kMlpH, 4, true>(act, T.W2, TcMlpTc::S, T.b2, lane);
  tc_mlp_tc_layer<kMlpH, 4, true>(act, T.W3, TcMlpTc::S, T.b3, lane);
  tc_mlp_tc_layer<kMlpH, 1, false>(act, T.W4, TcMlpTc::S, T.b4, lane);
#pragma unroll
  for (int j = 0; j < NOUT; j++) y[j] = act[lane * kMlpActS + j];
  __syncwarp();
}

// The per-cell part of the selector's features (tc_pair_features): the source spectrum ratios
// (f2..f5) and log of the body count, feat[c * 5 + k]
template <int P>
__global__ void k_cell_feat(int ncell, const TcCells c, const double* __restrict__ pn, float* __restrict__ feat,
                            const int* ncdev = nullptr) {
  if (ncdev) ncell = *ncdev;  // device-sized launch (graph)
  for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < ncell; ci += gridDim.x * blockDim.x) {
    const double* ps = pn + (size_t)ci * (P + 1);
    const double p0 = fmax(ps[0], 1e-300), rs = c.R[ci];
    for (int j = 0; j < 4; j++) {
      const int deg = 2 * (j + 1);
      const double v = deg <= P ? ps[deg] / (p0 * pow(rs, (double)deg)) : 0.0;
      feat[(size_t)ci * 5 + j] = tc_clampf((float)log(fmax(v, 1e-30)), -69.f, 10.f);
    }
    feat[(size_t)ci * 5 + 4] = (float)log((double)c.nbody[ci]);
  }
}

// loss = mean over samples and outputs of (y - target)^2; gradients accumulated into g
__global__ void k_mlp_grad(int ns, int nout, const float* __restrict__ feat, const float* __restrict__ target,
                           const float* __restrict__ w, TcMlpNorm norm, float* __restrict__ g,
                           float* __restrict__ loss) {
  __shared__ float sw[kMlpParamMax];
  __shared__ float sg[kMlpParamMax];
  __shared__ float sloss;
  const int np = tc_mlp_nparam(nout);
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    sw[i] = w[i];
    sg[i] = 0.f;
  }
  if (threadIdx.x == 0) sloss = 0.f;
  __syncthreads();
  const float* W2 = sw + kMlpH * kMlpIn + kMlpH;
  const float* W3 = W2 + kMlpH * kMlpH + kMlpH;
  const float* W4 = W3 + kMlpH * kMlpH + kMlpH;
  float* gW1 = sg;
  float* gb1 = gW1 + kMlpH * kMlpIn;
  float* gW2 = gb1 + kMlpH;
  float* gb2 = gW2 + kMlpH * kMlpH;
  float* gW3 = gb2 + kMlpH;
  float* gb3 = gW3 + kMlpH * kMlpH;
  float* gW4 = gb3 + kMlpH;
  float* gb4 = gW4 + nout * kMlpH;
  const float scale = 2.f / ((float)ns * (float)nout);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ns; k += gridDim.x * blockDim.x) {
    float x[kMlpIn], a1[kMlpH], a2[kMlpH], a3[kMlpH], y[kMlpOutMax], d4[kMlpOutMax], d3[kMlpH], d2[kMlpH];
    for (int i = 0; i < kMlpIn; i++) x[i] = (feat[(size_t)k * kMlpIn + i] - norm.mean[i]) * norm.inv_std[i];
    tc_mlp_forward(sw, nout, x, a1, a2, a3, y);
    float l = 0.f;
    for (int j = 0; j < nout; j++) {
      float e = y[j] - (target[(size_t)k * nout + j] - norm.out_mean);
      l += e * e;
      d4[j] = scale * e;
      atomicAdd(&gb4[j], d4[j]);
      for (int i = 0; i < kMlpH; i++) atomicAdd(&gW4[j * kMlpH + i], d4[j] * a3[i]);
    }
    atomicAdd(&sloss, l / ((float)ns * (float)nout));
    for (int i = 0; i < kMlpH; i++) {
      float s = 0.f;
      for (int j = 0; j < nout; j++) s += W4[j * kMlpH + i] * d4[j];
      d3[i] = s * (1.f - a3[i] * a3[i]);
      atomicAdd(&gb3[i], d3[i]);
    }
    for (int j = 0; j < kMlpH; j++)
      for (int i = 0; i < kMlpH; i++) atomicAdd(&gW3[j * kMlpH + i], d3[j] * a2[i]);
    for (int i = 0; i < kMlpH; i++) {
      float s = 0.f;
      for (int j = 0; j < kMlpH; j++) s += W3[j * kMlpH + i] * d3[j];
      d2[i] = s * (1.f - a2[i] * a2[i]);
      atomicAdd(&gb2[i], d2[i]);
    }
    for (int j = 0; j < kMlpH; j++)
      for (int i = 0; i < kMlpH; i++) atomicAdd(&gW2[j * kMlpH + i], d2[j] * a1[i]);
    for (int i = 0; i < kMlpH; i++) {
      float s = 0.f;
      for (int j = 0; j < kMlpH; j++) s += W2[j * kMlpH + i] * d2[j];
      float d1 = s * (1.f - a1[i] * a1[i]);
      atomicAdd(&gb1[i], d1);
      for (int q = 0; q < kMlpIn; q++) atomicAdd(&gW1[i * kMlpIn + q], d1 * x[q]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < np; i += blockDim.x)
    if (sg[i] != 0.f) atomicAdd(&g[i], sg[i]);
  if (threadIdx.x == 0) atomicAdd(loss, sloss);
}

__global__ void k_mlp_adam(int np, float* __restrict__ w, float* __restrict__ g, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float b1, float b2, float eps, int step) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  float gi = g[i];
  float a = b1 * m1[i] + (1.f - b1) * gi;
  float b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  float ah = a / (1.f - powf(b1, (float)step)), bh = b / (1.f - powf(b2, (float)step));
  w[i] -= lr * ah / (sqrtf(bh) + eps);
  g[i] = 0.f;
}

}  // namespace tc
