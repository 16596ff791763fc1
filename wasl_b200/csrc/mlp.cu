// The learned troubled-cell indicator: a small MLP over normalised modal
// coefficients of a cell and its limiter-stencil neighbours, trained on the
// flags the reference modal-decay sensor (cpp/src/limiting/euler_modal_limiter.cpp:18-24)
// produces on the method's own runs, with that sensor as the fallback for
// cells the network is not confident about.
//
// Network: x[F] -> 64 (ReLU) -> 64 (ReLU) -> 1 (logit), F = 4 (M - 1) + 3
// padded to a multiple of 16.  Weights and the two matrix operands (inputs,
// first hidden layer) are BF16, accumulation and biases FP32; training keeps
// FP32 master weights and runs the forward pass with the same BF16 rounding
// the inference kernel applies (gradients pass straight through it).
//
// Kernels: features (shared by data collection and inference), the training
// forward/backward over a block's mini-batch with atomic gradient
// accumulation, Adam, an FP32 prediction pass, and the inference kernel on
// the tensor cores (mma.sync m16n8k16 BF16, FP32 accumulate).
#include <cuda_bf16.h>

#include <algorithm>
#include <stdexcept>
#include <string>

#include "mlp.hpp"

namespace wasl_b200 {

namespace {

__device__ __forceinline__ float clamp8(float x) { return fminf(fmaxf(x, -8.0f), 8.0f); }

__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

} // namespace

// Features of element e into x[F] (zero padded): density modes m >= 1 over
// the mean, for the cell then each stencil neighbour (zeros for a missing
// one), then neighbour mean / cell mean - 1; every value clamped to [-8, 8].
__device__ __forceinline__ void mlp_features_of(const double *state, std::int64_t ne, int M,
                                                const std::int32_t *neighbors, std::int64_t e,
                                                int F, float *x) {
  for (int i = 0; i < F; ++i)
    x[i] = 0.0f;
  const double c0 = state[e];
  const double inv = c0 != 0.0 ? 1.0 / c0 : 0.0;
  for (int m = 1; m < M; ++m)
    x[m - 1] = clamp8(static_cast<float>(state[m * ne + e] * inv));
  for (int j = 0; j < 3; ++j) {
    const std::int32_t nb = neighbors[e * 3 + j];
    if (nb < 0)
      continue;
    const double n0 = state[nb];
    const double ninv = n0 != 0.0 ? 1.0 / n0 : 0.0;
    for (int m = 1; m < M; ++m)
      x[(j + 1) * (M - 1) + m - 1] = clamp8(static_cast<float>(state[m * ne + nb] * ninv));
    x[4 * (M - 1) + j] = clamp8(static_cast<float>(__dadd_rn(__dmul_rn(n0, inv), -1.0)));
  }
}

// The reference modal-decay decision on density (modal_decay.hpp:23-33).
__device__ __forceinline__ bool reference_troubled(const double *state, std::int64_t ne, int M,
                                                   std::int64_t e, double threshold,
                                                   int highest_degree_begin) {
  double total = 0.0, high = 0.0;
  for (int m = 0; m < M; ++m) {
    const double value = state[m * ne + e];
    total += value * value;
    if (m >= highest_degree_begin)
      high += value * value;
  }
  return !(total == 0.0 || high / total <= threshold);
}

__global__ void mlp_features_kernel(const double *state, std::int64_t ne, int M,
                                    const std::int32_t *neighbors, int F, double threshold,
                                    int highest_degree_begin, float *features,
                                    std::uint8_t *labels) {
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= ne)
    return;
  float x[kMlpMaxFeatures];
  mlp_features_of(state, ne, M, neighbors, e, F, x);
  for (int i = 0; i < F; ++i)
    features[e * F + i] = x[i];
  labels[e] = reference_troubled(state, ne, M, e, threshold, highest_degree_begin) ? 1 : 0;
}

// ---- training ------------------------------------------------------------------

// One block: kMlpBatch samples [first, first + kMlpBatch) of the data (cyclic),
// forward with BF16-rounded weights and operands, weighted binary
// cross-entropy on the logit (positives weighted pos_weight), backward, and
// the gradient of the summed loss added to grad; the summed loss to loss.
__global__ void __launch_bounds__(256) mlp_train_kernel(const MlpShape sh, const float *params,
                                                        const float *features,
                                                        const std::uint8_t *labels,
                                                        std::int64_t n, std::int64_t first,
                                                        float pos_weight, float *grad,
                                                        double *loss) {
  constexpr int B = kMlpBatch, Hd = kMlpHidden;
  const int F = sh.features;
  extern __shared__ float smem[];
  float *X = smem;            // [B][F]
  float *H1 = X + B * F;      // [B][Hd]
  float *H2 = H1 + B * Hd;    // [B][Hd]
  float *D2 = H2 + B * Hd;    // [B][Hd] dLoss/d(pre-activation 2)
  float *D1 = D2 + B * Hd;    // [B][Hd]
  float *d3 = D1 + B * Hd;    // [B] dLoss/dlogit
  const float *W1 = params + sh.w1, *b1 = params + sh.b1, *W2 = params + sh.w2,
              *b2 = params + sh.b2, *w3 = params + sh.w3;
  const float b3 = params[sh.b3];
  const std::int64_t base = first + static_cast<std::int64_t>(blockIdx.x) * B;
  const int t = threadIdx.x;
  for (int i = t; i < B * F; i += blockDim.x) {
    const std::int64_t s = (base + i / F) % n;
    X[i] = bf16_round(features[s * F + i % F]);
  }
  __syncthreads();
  for (int i = t; i < B * Hd; i += blockDim.x) {
    const int b = i / Hd, j = i % Hd;
    float acc = b1[j];
    for (int k = 0; k < F; ++k)
      acc = fmaf(bf16_round(W1[j * F + k]), X[b * F + k], acc);
    H1[i] = bf16_round(fmaxf(acc, 0.0f));
  }
  __syncthreads();
  for (int i = t; i < B * Hd; i += blockDim.x) {
    const int b = i / Hd, j = i % Hd;
    float acc = b2[j];
    for (int k = 0; k < Hd; ++k)
      acc = fmaf(bf16_round(W2[j * Hd + k]), H1[b * Hd + k], acc);
    H2[i] = fmaxf(acc, 0.0f);
  }
  __syncthreads();
  if (t < B) {
    float z = b3;
    for (int k = 0; k < Hd; ++k)
      z = fmaf(bf16_round(w3[k]), H2[t * Hd + k], z);
    const std::int64_t s = (base + t) % n;
    const float y = labels[s] ? 1.0f : 0.0f;
    const float w = labels[s] ? pos_weight : 1.0f;
    // loss = w (softplus(z) - y z), stable form; dloss/dz = w (sigmoid(z) - y)
    const float sp = fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z)));
    atomicAdd(loss, static_cast<double>(w * (sp - y * z)));
    d3[t] = w * (1.0f / (1.0f + expf(-z)) - y);
  }
  __syncthreads();
  for (int i = t; i < B * Hd; i += blockDim.x) {
    const int b = i / Hd, k = i % Hd;
    D2[i] = H2[i] > 0.0f ? d3[b] * bf16_round(w3[k]) : 0.0f;
  }
  __syncthreads();
  for (int i = t; i < B * Hd; i += blockDim.x) {
    const int b = i / Hd, j = i % Hd;
    float acc = 0.0f;
    for (int k = 0; k < Hd; ++k)
      acc = fmaf(D2[b * Hd + k], bf16_round(W2[k * Hd + j]), acc);
    D1[i] = H1[i] > 0.0f ? acc : 0.0f;
  }
  __syncthreads();
  // Weight gradients, one entry per thread and pass, summed over the batch.
  for (int i = t; i < Hd; i += blockDim.x) {
    float gw3 = 0.0f, gb2 = 0.0f, gb1 = 0.0f;
    for (int b = 0; b < B; ++b) {
      gw3 = fmaf(d3[b], H2[b * Hd + i], gw3);
      gb2 += D2[b * Hd + i];
      gb1 += D1[b * Hd + i];
    }
    atomicAdd(grad + sh.w3 + i, gw3);
    atomicAdd(grad + sh.b2 + i, gb2);
    atomicAdd(grad + sh.b1 + i, gb1);
  }
  if (t == 0) {
    float gb3 = 0.0f;
    for (int b = 0; b < B; ++b)
      gb3 += d3[b];
    atomicAdd(grad + sh.b3, gb3);
  }
  for (int i = t; i < Hd * Hd; i += blockDim.x) {
    const int k = i / Hd, j = i % Hd;
    float acc = 0.0f;
    for (int b = 0; b < B; ++b)
      acc = fmaf(D2[b * Hd + k], H1[b * Hd + j], acc);
    atomicAdd(grad + sh.w2 + i, acc);
  }
  for (int i = t; i < Hd * F; i += blockDim.x) {
    const int j = i / F, k = i % F;
    float acc = 0.0f;
    for (int b = 0; b < B; ++b)
      acc = fmaf(D1[b * Hd + j], X[b * F + k], acc);
    atomicAdd(grad + sh.w1 + i, acc);
  }
}

// Adam on the FP32 master weights with the summed gradient scaled by
// `scale` (1 / samples), then the gradient is zeroed.
__global__ void mlp_adam_kernel(std::int64_t count, float *params, float *grad, float *m1,
                                float *m2, float lr, float beta1, float beta2, float eps,
                                float bias1, float bias2, float scale) {
  const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count)
    return;
  const float g = grad[i] * scale;
  m1[i] = beta1 * m1[i] + (1.0f - beta1) * g;
  m2[i] = beta2 * m2[i] + (1.0f - beta2) * g * g;
  params[i] -= lr * (m1[i] / bias1) / (sqrtf(m2[i] / bias2) + eps);
  grad[i] = 0.0f;
}

// Logits of samples with the training forward pass (FP32 SIMT, BF16 rounding).
__global__ void mlp_predict_kernel(const MlpShape sh, const float *params, const float *features,
                                   std::int64_t n, float *logits) {
  const std::int64_t s = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n)
    return;
  constexpr int Hd = kMlpHidden;
  const int F = sh.features;
  float x[kMlpMaxFeatures], h1[Hd];
  for (int k = 0; k < F; ++k)
    x[k] = bf16_round(features[s * F + k]);
  for (int j = 0; j < Hd; ++j) {
    float acc = params[sh.b1 + j];
    for (int k = 0; k < F; ++k)
      acc = fmaf(bf16_round(params[sh.w1 + j * F + k]), x[k], acc);
    h1[j] = bf16_round(fmaxf(acc, 0.0f));
  }
  float z = params[sh.b3];
  for (int j = 0; j < Hd; ++j) {
    float acc = params[sh.b2 + j];
    for (int k = 0; k < Hd; ++k)
      acc = fmaf(bf16_round(params[sh.w2 + j * Hd + k]), h1[k], acc);
    z = fmaf(bf16_round(params[sh.w3 + j]), fmaxf(acc, 0.0f), z);
  }
  logits[s] = z;
}

// ---- inference on the tensor cores ------------------------------------------------

namespace {

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned *>(&v);
}

// D = A B + D, A 16x16 row-major BF16 (4 registers), B 16x8 column-major BF16
// (2 registers), D 16x8 FP32.
__device__ __forceinline__ void mma_bf16(float *d, const unsigned *a, const unsigned *b) {
  asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
               "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

} // namespace

// Per element, the part of the features and of the reference decision that
// depends on it alone, packed into 32 bytes: its density mean (FP64), its
// density modes m >= 1 over the mean (clamped to [-8, 8], BF16: the values
// the network's input rows hold), and the reference modal-decay decision.
// The inference kernel builds each element's input row from its own record
// and its three neighbours' (one 32-byte read each) instead of gathering
// 4 M scattered FP64 modes.
struct __align__(16) IndicatorRecord {
  double mean;
  __nv_bfloat16 high[kMlpMaxModes - 1];
  unsigned char reference;
  unsigned char pad[32 - 8 - 2 * (kMlpMaxModes - 1) - 1];
};
static_assert(sizeof(IndicatorRecord) == 32, "indicator record is 32 bytes");

__global__ void __launch_bounds__(128) mlp_records_kernel(const MlpIndicatorArgs a) {
  const std::int64_t e = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= a.ne)
    return;
  IndicatorRecord r{};
  const double c0 = a.state[e];
  const double inv = c0 != 0.0 ? 1.0 / c0 : 0.0;
  r.mean = c0;
  for (int m = 1; m < a.M; ++m)
    r.high[m - 1] = __float2bfloat16_rn(clamp8(static_cast<float>(a.state[m * a.ne + e] * inv)));
  r.reference = reference_troubled(a.state, a.ne, a.M, e, a.threshold, a.highest_degree_begin);
  reinterpret_cast<IndicatorRecord *>(a.records)[e] = r;
}

// ---- the fifth-generation tensor cores (tcgen05), for the inference kernel ----
//
// Operands in shared memory in the canonical K-major layout without swizzle:
// 8 x 8 BF16 core matrices of 128 contiguous bytes (8 rows of 16 bytes), the
// core matrices of one 8-row group consecutive along K.  Element (r, k) of a
// rows x K operand sits at byte umma_offset(r, k, K).  The matrix descriptor
// gives the start address, the byte step between core matrices along K
// (leading byte offset, 128) and between 8-row groups (stride byte offset,
// K / 8 x 128), all in 16-byte units, with the descriptor version of this
// architecture (bit 46) and no swizzle.
__device__ __forceinline__ unsigned umma_offset(int r, int k, int K) {
  return static_cast<unsigned>(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ unsigned long long umma_desc(unsigned smem_address, int K) {
  const unsigned long long lbo = 128 >> 4, sbo = static_cast<unsigned long long>((K >> 3) * 128) >> 4;
  return static_cast<unsigned long long>((smem_address >> 4) & 0x3FFFu) | (lbo << 16) |
         (sbo << 32) | (1ULL << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32
// accumulator, M = 128 rows, N = 64 columns.
constexpr unsigned kUmmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) |
                                ((128u >> 4) << 24);

// D (TMEM) (+)= A B^T for one K = 16 step; issued by one thread.
__device__ __forceinline__ void umma_bf16(unsigned d_tmem, unsigned long long a_desc,
                                          unsigned long long b_desc, bool accumulate) {
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
               :
               : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(kUmmaIdesc),
                 "r"(accumulate ? 1u : 0u)
               : "memory");
}

// The MMAs issued so far by this thread arrive on the mbarrier when done.
__device__ __forceinline__ void umma_commit(unsigned mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void tmem_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Plain shared-memory stores made visible to the tensor cores' reads.
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Waits until the mbarrier's phase of the given parity has completed, for at
// most about `cycles` SM clocks; false when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned mbar, unsigned parity, long long cycles) {
  const long long start = clock64();
  for (;;) {
    unsigned done = 0;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(mbar), "r"(parity)
                 : "memory");
    if (done)
      return true;
    if (clock64() - start > cycles)
      return false;
  }
}

// This thread's TMEM lane, 64 consecutive 32-bit columns from taddr (the
// load and its wait in one statement: the registers are defined after both).
__device__ __forceinline__ void tmem_load64(unsigned taddr, float (&v)[64]) {
  unsigned r[64];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x64.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
      "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
      "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
        "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]),
        "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]),
        "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]),
        "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
        "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]),
        "=r"(r[62]), "=r"(r[63])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 64; ++i)
    v[i] = __uint_as_float(r[i]);
}

// One element's network input row (BF16, zero padded to F values) from its
// own record and its three neighbours': its high modes, each neighbour's,
// then each neighbour's mean over its own minus 1; returns the element's
// reference decision.  H: high modes per element (P1, P2, P3 by F / 16).
template <int F> union IndicatorRow {
  uint4 v[F / 8];
  __nv_bfloat16 h[F];
};

template <int KF>
__device__ __forceinline__ bool indicator_row(const MlpIndicatorArgs &a, std::int64_t e,
                                              bool active, IndicatorRow<KF * 16> &row) {
  constexpr int F = KF * 16, H = KF == 1 ? 2 : KF == 2 ? 5 : 9;
  static_assert(4 * H + 3 <= F, "features do not fit the row");
  const IndicatorRecord *records = reinterpret_cast<const IndicatorRecord *>(a.records);
#pragma unroll
  for (int k = 0; k < F / 8; ++k)
    row.v[k] = make_uint4(0u, 0u, 0u, 0u);
  if (!active)
    return false;
  const IndicatorRecord own = records[e];
  const double inv = own.mean != 0.0 ? 1.0 / own.mean : 0.0;
#pragma unroll
  for (int m = 0; m < H; ++m)
    row.h[m] = own.high[m];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const std::int32_t nb = a.neighbors[e * 3 + j];
    if (nb < 0)
      continue;
    const IndicatorRecord n = records[nb];
#pragma unroll
    for (int m = 0; m < H; ++m)
      row.h[(j + 1) * H + m] = n.high[m];
    row.h[4 * H + j] = __float2bfloat16_rn(
        clamp8(static_cast<float>(__dadd_rn(__dmul_rn(n.mean, inv), -1.0))));
  }
  return own.reference;
}

// The decision for element e from its logit: troubled when sigmoid(logit) >=
// hi, smooth when <= lo, else the reference decision; the flag, the
// compacted troubled list (one atomic per warp) and the CTA's counters.
__device__ __forceinline__ void indicator_decide(const MlpIndicatorArgs &a, std::int64_t e,
                                                 float logit, bool reference,
                                                 unsigned long long *counts, int lane) {
  const float p = 1.0f / (1.0f + expf(-logit));
  bool troubled;
  int kind;
  if (p >= a.hi) {
    troubled = true;
    kind = 0;
  } else if (p <= a.lo) {
    troubled = false;
    kind = 1;
  } else {
    troubled = reference;
    kind = 2;
  }
  if (a.logits)
    a.logits[e] = logit;
  a.flags[e] = troubled ? 1 : 0;
  atomicAdd(&counts[kind], 1ULL);
  if (reference)
    atomicAdd(&counts[3], 1ULL);
  if (reference && !troubled)
    atomicAdd(&counts[4], 1ULL);
  if (!reference && troubled)
    atomicAdd(&counts[5], 1ULL);
  const unsigned mask = __activemask();
  const unsigned ballot = __ballot_sync(mask, troubled);
  if (ballot) {
    const int leader = __ffs(ballot) - 1;
    int base = 0;
    if (lane == leader)
      base = atomicAdd(a.troubled_count, __popc(ballot));
    base = __shfl_sync(mask, base, leader);
    if (troubled)
      a.troubled[base + __popc(ballot & ((1u << lane) - 1u))] = static_cast<std::int32_t>(e);
  }
}

// A persistent kernel: each CTA of 128 threads loads the network once (BF16
// in shared memory) and then takes 128-element tiles in turn.  Per tile, each
// thread builds its element's input row (BF16, shared memory) from the
// element's and its neighbours' records; each warp runs its 32 rows through
// the network as two 16-row tiles of m16n8k16 MMAs (the first layer's
// accumulators become the second layer's A fragments in registers), and the
// last layer as a quad reduction.  A cell is troubled when sigmoid(logit) >=
// hi, smooth when <= lo, and otherwise takes the reference decision.  Flags
// and the compacted troubled list as the sensor writes them; counters: [0]
// network troubled, [1] network smooth, [2] fallback, [3] reference
// troubled, [4] missed (reference troubled, decided smooth), [5] false
// (reference smooth, decided troubled).
template <int KF>
__global__ void __launch_bounds__(128) mlp_indicator_kernel(const MlpIndicatorArgs a) {
  constexpr int Hd = kMlpHidden, F = KF * 16, ROW = F + 8; // +8: fewer bank conflicts
  __shared__ __align__(16) __nv_bfloat16 X[128 * ROW];
  __shared__ __align__(16) __nv_bfloat16 W1[Hd * ROW];
  __shared__ __align__(16) __nv_bfloat16 W2[Hd * (Hd + 8)];
  __shared__ float b1[Hd], b2[Hd], w3[Hd], logit[128];
  __shared__ unsigned long long counts[6];
  const int t = threadIdx.x;
  const float *P = a.params;
  for (int i = t; i < Hd * F; i += 128)
    W1[(i / F) * ROW + i % F] = __float2bfloat16_rn(P[a.shape.w1 + i]);
  for (int i = t; i < Hd * Hd; i += 128)
    W2[(i / Hd) * (Hd + 8) + i % Hd] = __float2bfloat16_rn(P[a.shape.w2 + i]);
  for (int i = t; i < Hd; i += 128) {
    b1[i] = P[a.shape.b1 + i];
    b2[i] = P[a.shape.b2 + i];
    w3[i] = bf16_round(P[a.shape.w3 + i]);
  }
  if (t < 6)
    counts[t] = 0;
  const float b3 = P[a.shape.b3];
  const int warp = t >> 5, lane = t & 31, g = lane >> 2, q = lane & 3;
  const std::int64_t tiles = (a.ne + 127) / 128;
  for (std::int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const std::int64_t e = tile * 128 + t;
    const bool active = e < a.ne;
    bool reference = false;
    {
      // The row in registers (zero padded), then 16-byte stores: a row is
      // (F + 8) x 2 bytes, a multiple of 16, and eight consecutive rows fill
      // distinct 16-byte bank groups.
      IndicatorRow<F> row;
      reference = indicator_row<KF>(a, e, active, row);
      uint4 *dst = reinterpret_cast<uint4 *>(X + t * ROW);
#pragma unroll
      for (int k = 0; k < F / 8; ++k)
        dst[k] = row.v[k];
    }
    __syncthreads(); // rows built (and, the first time, the network loaded)

    for (int mt = 0; mt < 2; ++mt) {
      const int row0 = warp * 32 + mt * 16;
      // Layer 1: 16 rows x 64 outputs, K = F.
      float h[8][4];
      for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * q;
        h[nt][0] = h[nt][2] = b1[c];
        h[nt][1] = h[nt][3] = b1[c + 1];
      }
      for (int kk = 0; kk < KF; ++kk) {
        unsigned af[4];
        const __nv_bfloat16 *r0 = X + (row0 + g) * ROW + kk * 16 + 2 * q;
        const __nv_bfloat16 *r8 = X + (row0 + g + 8) * ROW + kk * 16 + 2 * q;
        af[0] = *reinterpret_cast<const unsigned *>(r0);
        af[1] = *reinterpret_cast<const unsigned *>(r8);
        af[2] = *reinterpret_cast<const unsigned *>(r0 + 8);
        af[3] = *reinterpret_cast<const unsigned *>(r8 + 8);
        for (int nt = 0; nt < 8; ++nt) {
          const __nv_bfloat16 *wb = W1 + (nt * 8 + g) * ROW + kk * 16 + 2 * q;
          const unsigned bf[2] = {*reinterpret_cast<const unsigned *>(wb),
                                  *reinterpret_cast<const unsigned *>(wb + 8)};
          mma_bf16(h[nt], af, bf);
        }
      }
      // Layer 2: A fragments straight from layer 1's accumulators (ReLU, BF16).
      float o[8][4];
      for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * q;
        o[nt][0] = o[nt][2] = b2[c];
        o[nt][1] = o[nt][3] = b2[c + 1];
      }
      for (int kk = 0; kk < 4; ++kk) {
        const float *lo = h[2 * kk], *hi = h[2 * kk + 1];
        const unsigned af[4] = {pack_bf16(fmaxf(lo[0], 0.0f), fmaxf(lo[1], 0.0f)),
                                pack_bf16(fmaxf(lo[2], 0.0f), fmaxf(lo[3], 0.0f)),
                                pack_bf16(fmaxf(hi[0], 0.0f), fmaxf(hi[1], 0.0f)),
                                pack_bf16(fmaxf(hi[2], 0.0f), fmaxf(hi[3], 0.0f))};
        for (int nt = 0; nt < 8; ++nt) {
          const __nv_bfloat16 *wb = W2 + (nt * 8 + g) * (Hd + 8) + kk * 16 + 2 * q;
          const unsigned bf[2] = {*reinterpret_cast<const unsigned *>(wb),
                                  *reinterpret_cast<const unsigned *>(wb + 8)};
          mma_bf16(o[nt], af, bf);
        }
      }
      // Layer 3: rows g and g + 8, columns 2q, 2q+1 of each n-tile, then the quad.
      float z0 = 0.0f, z8 = 0.0f;
      for (int nt = 0; nt < 8; ++nt) {
        const int c = nt * 8 + 2 * q;
        z0 = fmaf(w3[c], fmaxf(o[nt][0], 0.0f), fmaf(w3[c + 1], fmaxf(o[nt][1], 0.0f), z0));
        z8 = fmaf(w3[c], fmaxf(o[nt][2], 0.0f), fmaf(w3[c + 1], fmaxf(o[nt][3], 0.0f), z8));
      }
      z0 += __shfl_xor_sync(0xffffffffu, z0, 1);
      z0 += __shfl_xor_sync(0xffffffffu, z0, 2);
      z8 += __shfl_xor_sync(0xffffffffu, z8, 1);
      z8 += __shfl_xor_sync(0xffffffffu, z8, 2);
      if (q == 0) {
        logit[row0 + g] = z0 + b3;
        logit[row0 + g + 8] = z8 + b3;
      }
    }
    __syncthreads(); // logits written; the next tile's rows may overwrite X

    if (active)
      indicator_decide(a, e, logit[t], reference, counts, lane);
    // The logits of this tile are read above before the next tile's MMAs
    // write them: those come after the next tile's first barrier.
  }
  __syncthreads();
  if (t < 6 && a.stats && counts[t])
    atomicAdd(a.stats + t, counts[t]);
}

// The inference on the fifth-generation tensor cores: the persistent kernel's
// work per 128-element tile, with the two hidden layers as single-CTA
// tcgen05 MMAs (M = 128 rows, N = 64, K = F then 64; BF16 operands in shared
// memory, FP32 accumulators in 64 TMEM columns).  One thread issues the MMAs
// and commits them to an mbarrier; every thread then reads its own row (its
// TMEM lane) with tcgen05.ld, adds the bias and applies ReLU; layer 1's BF16
// activations become layer 2's A operand in shared memory, and the last
// layer is each thread's dot product over its row.  Waits on the mbarrier
// are bounded (about a second of SM clock): a wait that runs out records
// kIndicatorWait in the error word, the CTA leaves its loop, waits once more
// (bounded) for the MMAs it issued and frees its TMEM.
template <int KF>
__global__ void __launch_bounds__(128) mlp_indicator_tc_kernel(const MlpIndicatorArgs a) {
  constexpr int Hd = kMlpHidden, F = KF * 16;
  __shared__ __align__(1024) __nv_bfloat16 A[128 * Hd]; // the rows (K = F), then layer 1's output
  __shared__ __align__(1024) __nv_bfloat16 W1[Hd * F];
  __shared__ __align__(1024) __nv_bfloat16 W2[Hd * Hd];
  __shared__ float b1[Hd], b2[Hd], w3[Hd];
  __shared__ unsigned long long counts[6];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ unsigned tmem_base;
  __shared__ int failed; // 0, or 1 + the parity of the wait that ran out
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const float *P = a.params;
  unsigned char *a_bytes = reinterpret_cast<unsigned char *>(A);
  unsigned char *w1_bytes = reinterpret_cast<unsigned char *>(W1);
  unsigned char *w2_bytes = reinterpret_cast<unsigned char *>(W2);
  for (int i = t; i < Hd * F; i += 128)
    *reinterpret_cast<__nv_bfloat16 *>(w1_bytes + umma_offset(i / F, i % F, F)) =
        __float2bfloat16_rn(P[a.shape.w1 + i]);
  for (int i = t; i < Hd * Hd; i += 128)
    *reinterpret_cast<__nv_bfloat16 *>(w2_bytes + umma_offset(i / Hd, i % Hd, Hd)) =
        __float2bfloat16_rn(P[a.shape.w2 + i]);
  for (int i = t; i < Hd; i += 128) {
    b1[i] = P[a.shape.b1 + i];
    b2[i] = P[a.shape.b2 + i];
    w3[i] = bf16_round(P[a.shape.w3 + i]);
  }
  if (t < 6)
    counts[t] = 0;
  const unsigned bar = static_cast<unsigned>(__cvta_generic_to_shared(&mbar));
  if (t == 0) {
    failed = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const unsigned slot = static_cast<unsigned>(__cvta_generic_to_shared(&tmem_base));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(slot)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_shared(); // the weights, for the tensor cores
  tmem_fence_before_sync();
  __syncthreads();
  tmem_fence_after_sync();
  const unsigned tmem = tmem_base;
  const unsigned my_lanes = tmem + (static_cast<unsigned>(warp * 32) << 16);
  const unsigned a_addr = static_cast<unsigned>(__cvta_generic_to_shared(A));
  const unsigned w1_addr = static_cast<unsigned>(__cvta_generic_to_shared(W1));
  const unsigned w2_addr = static_cast<unsigned>(__cvta_generic_to_shared(W2));
  const float b3 = P[a.shape.b3];
  constexpr long long kWaitCycles = 1LL << 31;
  const std::int64_t tiles = (a.ne + 127) / 128;
  for (std::int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const std::int64_t e = tile * 128 + t;
    const bool active = e < a.ne;
    bool reference;
    {
      IndicatorRow<F> row;
      reference = indicator_row<KF>(a, e, active, row);
#pragma unroll
      for (int c = 0; c < F / 8; ++c)
        *reinterpret_cast<uint4 *>(a_bytes + umma_offset(t, 8 * c, F)) = row.v[c];
    }
    fence_async_shared();
    tmem_fence_before_sync();
    __syncthreads(); // rows in place; last tile's TMEM reads done
    if (t == 0) {
      tmem_fence_after_sync();
#pragma unroll
      for (int k = 0; k < KF; ++k)
        umma_bf16(tmem, umma_desc(a_addr + 256 * k, F), umma_desc(w1_addr + 256 * k, F), k > 0);
      umma_commit(bar);
    }
    if (!mbar_wait(bar, 0, kWaitCycles))
      atomicCAS(&failed, 0, 1);
    __syncthreads();
    if (failed)
      break;
    tmem_fence_after_sync();
    float v[64];
    tmem_load64(my_lanes, v);
#pragma unroll
    for (int c = 0; c < Hd / 8; ++c) {
      uint4 packed;
      unsigned *u = reinterpret_cast<unsigned *>(&packed);
#pragma unroll
      for (int j = 0; j < 4; ++j)
        u[j] = pack_bf16(fmaxf(v[8 * c + 2 * j] + b1[8 * c + 2 * j], 0.0f),
                         fmaxf(v[8 * c + 2 * j + 1] + b1[8 * c + 2 * j + 1], 0.0f));
      *reinterpret_cast<uint4 *>(a_bytes + umma_offset(t, 8 * c, Hd)) = packed;
    }
    fence_async_shared();
    tmem_fence_before_sync();
    __syncthreads(); // layer 1's activations in place; its TMEM reads done
    if (t == 0) {
      tmem_fence_after_sync();
#pragma unroll
      for (int k = 0; k < Hd / 16; ++k)
        umma_bf16(tmem, umma_desc(a_addr + 256 * k, Hd), umma_desc(w2_addr + 256 * k, Hd), k > 0);
      umma_commit(bar);
    }
    if (!mbar_wait(bar, 1, kWaitCycles))
      atomicCAS(&failed, 0, 2);
    __syncthreads();
    if (failed)
      break;
    tmem_fence_after_sync();
    tmem_load64(my_lanes, v);
    float z = 0.0f;
#pragma unroll
    for (int c = 0; c < Hd; ++c)
      z = fmaf(w3[c], fmaxf(v[c] + b2[c], 0.0f), z);
    if (active)
      indicator_decide(a, e, z + b3, reference, counts, lane);
  }
  __syncthreads();
  if (failed && t == 0) {
    mbar_wait(bar, static_cast<unsigned>(failed - 1), kWaitCycles); // the MMAs still in flight
    if (a.error)
      atomicCAS(a.error, 0ULL, static_cast<unsigned long long>(kMlpWaitCode) << 56);
  }
  tmem_fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tmem_fence_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
  }
  if (t < 6 && a.stats && counts[t])
    atomicAdd(a.stats + t, counts[t]);
}

// ---- host launchers -------------------------------------------------------------

MlpShape mlp_shape(int features) {
  if (features <= 0 || features % 16 != 0 || features > kMlpMaxFeatures)
    throw std::invalid_argument("indicator network: features must be a multiple of 16, at most " +
                                std::to_string(kMlpMaxFeatures));
  MlpShape s;
  s.features = features;
  s.w1 = 0;
  s.b1 = s.w1 + kMlpHidden * features;
  s.w2 = s.b1 + kMlpHidden;
  s.b2 = s.w2 + kMlpHidden * kMlpHidden;
  s.w3 = s.b2 + kMlpHidden;
  s.b3 = s.w3 + kMlpHidden;
  s.count = s.b3 + 1;
  return s;
}

int mlp_features_for_modes(int M) {
  const int raw = 4 * (M - 1) + 3;
  return (raw + 15) / 16 * 16;
}

void launch_mlp_features(const double *state, std::int64_t ne, int M,
                         const std::int32_t *neighbors, int F, double threshold,
                         int highest_degree_begin, float *features, std::uint8_t *labels,
                         cudaStream_t s) {
  if (ne > 0)
    mlp_features_kernel<<<static_cast<unsigned>((ne + 127) / 128), 128, 0, s>>>(
        state, ne, M, neighbors, F, threshold, highest_degree_begin, features, labels);
}

std::size_t mlp_train_smem(int F) {
  return sizeof(float) * (kMlpBatch * F + 4 * kMlpBatch * kMlpHidden + kMlpBatch);
}

void launch_mlp_train(const MlpShape &sh, const float *params, const float *features,
                      const std::uint8_t *labels, std::int64_t n, std::int64_t first,
                      std::int64_t blocks, float pos_weight, float *grad, double *loss,
                      cudaStream_t s) {
  const std::size_t smem = mlp_train_smem(sh.features);
  cudaError_t rc = cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        static_cast<int>(smem));
  if (rc != cudaSuccess)
    throw std::runtime_error(std::string("indicator training: ") + cudaGetErrorString(rc));
  if (blocks > 0)
    mlp_train_kernel<<<static_cast<unsigned>(blocks), 256, smem, s>>>(
        sh, params, features, labels, n, first, pos_weight, grad, loss);
}

void launch_mlp_adam(std::int64_t count, float *params, float *grad, float *m1, float *m2,
                     float lr, float beta1, float beta2, float eps, std::int64_t step, float scale,
                     cudaStream_t s) {
  const float bias1 = 1.0f - powf(beta1, static_cast<float>(step));
  const float bias2 = 1.0f - powf(beta2, static_cast<float>(step));
  mlp_adam_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, s>>>(
      count, params, grad, m1, m2, lr, beta1, beta2, eps, bias1, bias2, scale);
}

void launch_mlp_predict(const MlpShape &sh, const float *params, const float *features,
                        std::int64_t n, float *logits, cudaStream_t s) {
  if (n > 0)
    mlp_predict_kernel<<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(sh, params, features,
                                                                              n, logits);
}

void launch_mlp_indicator(const MlpIndicatorArgs &a, cudaStream_t s) {
  if (a.ne <= 0)
    return;
  if (!a.records)
    throw std::invalid_argument("indicator network: no record scratch");
  mlp_records_kernel<<<static_cast<unsigned>((a.ne + 127) / 128), 128, 0, s>>>(a);
  const int KF = a.shape.features / 16;
  if (KF < 1 || KF > 3 || a.M != (KF == 1 ? 3 : KF == 2 ? 6 : 10))
    throw std::invalid_argument("indicator network: unsupported feature count");
  // Persistent CTAs, every one resident at once, each loading the network once
  // (the tcgen05 kernel holds 64 TMEM columns, so at most 8 fit an SM).
  const bool tc = a.kernel == 0;
  const void *kernel =
      tc ? (KF == 1   ? reinterpret_cast<const void *>(mlp_indicator_tc_kernel<1>)
            : KF == 2 ? reinterpret_cast<const void *>(mlp_indicator_tc_kernel<2>)
                      : reinterpret_cast<const void *>(mlp_indicator_tc_kernel<3>))
         : (KF == 1   ? reinterpret_cast<const void *>(mlp_indicator_kernel<1>)
            : KF == 2 ? reinterpret_cast<const void *>(mlp_indicator_kernel<2>)
                      : reinterpret_cast<const void *>(mlp_indicator_kernel<3>));
  static int resident[64][2][4] = {};
  int device = 0;
  cudaGetDevice(&device);
  int &slots = resident[device & 63][tc ? 0 : 1][KF];
  if (!slots) {
    int per_sm = 0, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (tc) {
      // The occupancy calculator cannot see how much tensor memory a kernel
      // allocates, and answers one CTA per SM; count the registers, the shared
      // memory and the 64 TMEM columns (512 per SM) instead.
      cudaFuncAttributes attr{};
      int smem_sm = 0, reserved = 0;
      cudaFuncGetAttributes(&attr, kernel);
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device);
      const int warp_regs = (attr.numRegs * 32 + 255) / 256 * 256;
      const int by_regs = attr.numRegs > 0 ? 65536 / (4 * warp_regs) : 1;
      const int by_smem =
          static_cast<int>(smem_sm / (attr.sharedSizeBytes + static_cast<std::size_t>(reserved)));
      per_sm = std::min({by_regs, by_smem, 512 / 64, 16});
    } else {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
    }
    slots = std::max(1, per_sm) * std::max(1, sms);
  }
  const std::int64_t tiles = (a.ne + 127) / 128;
  const unsigned blocks = static_cast<unsigned>(std::min<std::int64_t>(tiles, slots));
  if (tc) {
    switch (KF) {
    case 1: mlp_indicator_tc_kernel<1><<<blocks, 128, 0, s>>>(a); break;
    case 2: mlp_indicator_tc_kernel<2><<<blocks, 128, 0, s>>>(a); break;
    default: mlp_indicator_tc_kernel<3><<<blocks, 128, 0, s>>>(a); break;
    }
  } else {
    switch (KF) {
    case 1: mlp_indicator_kernel<1><<<blocks, 128, 0, s>>>(a); break;
    case 2: mlp_indicator_kernel<2><<<blocks, 128, 0, s>>>(a); break;
    default: mlp_indicator_kernel<3><<<blocks, 128, 0, s>>>(a); break;
    }
  }
}

} // namespace wasl_b200
