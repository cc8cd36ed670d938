// Partition cost model: a 24 -> 128 -> 128 -> 1 ReLU MLP that predicts the
// log of a partition's kernel time from its features.  BF16 weights and
// activations, FP32 accumulation; training (forward + backward + Adam) and
// inference are hand-written kernels here.
//
// Parameter vector theta (fp32 master copy, NP floats):
//   W1 [128][24] | b1 [128] | W2 [128][128] | b2 [128] | W3 [128] | b3
// theta16 is its bf16 copy used by the forward passes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/jacquard_b200.h"

namespace jqm {

constexpr int NF = JQ_MLP_FEATURES, H = JQ_MLP_HIDDEN;
constexpr int OW1 = 0, OB1 = OW1 + H * NF, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H,
              OB3 = OW3 + H, NP = OB3 + 1;
static_assert(NP == JQ_MLP_PARAMS, "parameter count");
constexpr int TPB = 256;

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float round_bf(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// Shared-memory copy of the bf16 parameters.
struct SmemW {
  __nv_bfloat16 w1[H * NF], w2[H * H], w3[H];
  float b1[H], b2[H], b3;
};

__device__ void load_weights(SmemW &W, const __nv_bfloat16 *theta16, const float *theta) {
  for (int i = threadIdx.x; i < H * NF; i += blockDim.x) W.w1[i] = theta16[OW1 + i];
  for (int i = threadIdx.x; i < H * H; i += blockDim.x) W.w2[i] = theta16[OW2 + i];
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    W.w3[i] = theta16[OW3 + i];
    W.b1[i] = theta[OB1 + i];
    W.b2[i] = theta[OB2 + i];
  }
  if (threadIdx.x == 0) W.b3 = theta[OB3];
}

// Forward of one row by 128 threads (j = hidden unit).  h1/h2 are bf16-rounded
// activations in shared memory; returns y in thread 0 of the group.
__device__ float forward_row(const SmemW &W, const __nv_bfloat16 *x, float *h1, float *h2,
                             float *red, int j) {
  float a = W.b1[j];
#pragma unroll
  for (int i = 0; i < NF; ++i) a = fmaf(bf(W.w1[j * NF + i]), bf(x[i]), a);
  h1[j] = round_bf(a > 0.f ? a : 0.f);
  __syncthreads();
  float c = W.b2[j];
#pragma unroll 8
  for (int k = 0; k < H; ++k) c = fmaf(bf(W.w2[j * H + k]), h1[k], c);
  h2[j] = round_bf(c > 0.f ? c : 0.f);
  float p = bf(W.w3[j]) * h2[j];
  // reduce over the 128 threads of the row group (4 warps)
  for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
  if ((j & 31) == 0) red[j >> 5] = p;
  __syncthreads();
  float y = W.b3 + red[0] + red[1] + red[2] + red[3];
  __syncthreads();
  return y;
}

// Inference: 128 threads per row, two rows per CTA pass.
__global__ void __launch_bounds__(TPB) mlp_forward_kernel(const float *theta,
                                                          const __nv_bfloat16 *theta16,
                                                          const __nv_bfloat16 *X, size_t n,
                                                          float *y) {
  __shared__ SmemW W;
  __shared__ float h1[2][H], h2[2][H], red[2][4];
  load_weights(W, theta16, theta);
  __syncthreads();
  const int g = threadIdx.x / H, j = threadIdx.x % H;
  for (size_t r0 = (size_t)blockIdx.x * 2; r0 < n; r0 += (size_t)gridDim.x * 2) {
    const size_t r = r0 + g;
    const size_t rr = r < n ? r : n - 1;  // both groups run the barriers
    const float v = forward_row(W, X + rr * NF, h1[g], h2[g], red[g], j);
    if (j == 0 && r < n) y[r] = v;
  }
}

// Gradient of the mean squared error over a batch: each CTA takes a slice of
// the batch, accumulates its parameter gradient in shared memory, and writes
// it to its row of `partial` (scratch, grid x NP floats).
struct SmemG {
  float g_w1[H * NF], g_w2[H * H], g_b1[H], g_b2[H], g_w3[H], g_b3;
  float h1[H], h2[H], dh2[H], dh1[H], red[4];
  float loss;
};

__global__ void __launch_bounds__(TPB, 1) mlp_grad_kernel(const float *theta,
                                                          const __nv_bfloat16 *theta16,
                                                          const __nv_bfloat16 *X, const float *T,
                                                          const uint32_t *idx, uint32_t batch,
                                                          float *partial, float *loss_partial) {
  extern __shared__ __align__(16) uint8_t dyn[];
  SmemW &W = *reinterpret_cast<SmemW *>(dyn);
  SmemG &G = *reinterpret_cast<SmemG *>(dyn + ((sizeof(SmemW) + 15) & ~size_t(15)));
  const int t = threadIdx.x;
  load_weights(W, theta16, theta);
  for (int i = t; i < H * NF; i += TPB) G.g_w1[i] = 0.f;
  for (int i = t; i < H * H; i += TPB) G.g_w2[i] = 0.f;
  for (int i = t; i < H; i += TPB) {
    G.g_b1[i] = 0.f;
    G.g_b2[i] = 0.f;
    G.g_w3[i] = 0.f;
  }
  if (t == 0) {
    G.g_b3 = 0.f;
    G.loss = 0.f;
  }
  __syncthreads();
  const uint32_t per = (batch + gridDim.x - 1) / gridDim.x;
  const uint32_t lo = blockIdx.x * per, hi = min(batch, lo + per);
  const float scale = 2.f / (float)batch;
  for (uint32_t b = lo; b < hi; ++b) {
    const uint32_t r = idx[b];
    const __nv_bfloat16 *x = X + (size_t)r * NF;
    // forward (threads 0..127 do the row; 128..255 follow the barriers)
    const int j = t & (H - 1);
    float y = 0.f;
    {
      float a = W.b1[j];
#pragma unroll
      for (int i = 0; i < NF; ++i) a = fmaf(bf(W.w1[j * NF + i]), bf(x[i]), a);
      if (t < H) G.h1[j] = round_bf(a > 0.f ? a : 0.f);
      __syncthreads();
      float c = W.b2[j];
#pragma unroll 8
      for (int k = 0; k < H; ++k) c = fmaf(bf(W.w2[j * H + k]), G.h1[k], c);
      float p = 0.f;
      if (t < H) {
        G.h2[j] = round_bf(c > 0.f ? c : 0.f);
        p = bf(W.w3[j]) * G.h2[j];
      }
      for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
      if (t < H && (t & 31) == 0) G.red[t >> 5] = p;
      __syncthreads();
      y = W.b3 + G.red[0] + G.red[1] + G.red[2] + G.red[3];
    }
    const float e = y - T[r];
    const float dy = scale * e;
    if (t == 0) {
      G.loss += e * e;
      G.g_b3 += dy;
    }
    // output layer and dh2
    if (t < H) {
      G.g_w3[t] += dy * G.h2[t];
      G.dh2[t] = G.h2[t] > 0.f ? dy * bf(W.w3[t]) : 0.f;
      G.g_b2[t] += G.dh2[t];
    }
    __syncthreads();
    // dW2[j][k] += dh2[j] * h1[k]: thread t owns 64 entries (fixed set)
    for (int q = t; q < H * H; q += TPB) G.g_w2[q] += G.dh2[q / H] * G.h1[q % H];
    // dh1[k] = sum_j W2[j][k] dh2[j], masked by h1 > 0
    if (t < H) {
      float s = 0.f;
#pragma unroll 8
      for (int jj = 0; jj < H; ++jj) s = fmaf(bf(W.w2[jj * H + t]), G.dh2[jj], s);
      G.dh1[t] = G.h1[t] > 0.f ? s : 0.f;
    }
    __syncthreads();
    for (int q = t; q < H * NF; q += TPB) G.g_w1[q] += G.dh1[q / NF] * bf(x[q % NF]);
    if (t < H) G.g_b1[t] += G.dh1[t];
    __syncthreads();
  }
  float *out = partial + (size_t)blockIdx.x * NP;
  for (int i = t; i < H * NF; i += TPB) out[OW1 + i] = G.g_w1[i];
  for (int i = t; i < H * H; i += TPB) out[OW2 + i] = G.g_w2[i];
  for (int i = t; i < H; i += TPB) {
    out[OB1 + i] = G.g_b1[i];
    out[OB2 + i] = G.g_b2[i];
    out[OW3 + i] = G.g_w3[i];
  }
  if (t == 0) {
    out[OB3] = G.g_b3;
    loss_partial[blockIdx.x] = G.loss;
  }
}

// Sum the per-CTA gradients; optionally write the gradient and/or apply Adam.
__global__ void mlp_reduce_adam_kernel(float *theta, __nv_bfloat16 *theta16, float *m, float *v,
                                       const float *partial, uint32_t parts, float *grad_out,
                                       int apply, float lr, float beta1, float beta2, float eps,
                                       uint32_t step, const float *loss_partial, float *loss_out,
                                       uint32_t batch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && loss_out) {
    float l = 0.f;
    for (uint32_t p = 0; p < parts; ++p) l += loss_partial[p];
    *loss_out = l / (float)batch;
  }
  if (i >= NP) return;
  float g = 0.f;
  for (uint32_t p = 0; p < parts; ++p) g += partial[(size_t)p * NP + i];
  if (grad_out) grad_out[i] = g;
  if (!apply) return;
  const float mi = beta1 * m[i] + (1.f - beta1) * g;
  const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.f - powf(beta1, (float)step));
  const float vh = vi / (1.f - powf(beta2, (float)step));
  const float w = theta[i] - lr * mh / (sqrtf(vh) + eps);
  theta[i] = w;
  theta16[i] = __float2bfloat16_rn(w);
}

__global__ void mlp_to_bf16_kernel(const float *theta, __nv_bfloat16 *theta16) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NP) theta16[i] = __float2bfloat16_rn(theta[i]);
}

size_t grad_smem() {
  return ((sizeof(SmemW) + 15) & ~size_t(15)) + sizeof(SmemG);
}

}  // namespace jqm

using namespace jqm;

extern "C" {

int jq_mlp_sync_bf16(const float *theta, uint16_t *theta16, void *stream) {
  mlp_to_bf16_kernel<<<(NP + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      theta, reinterpret_cast<__nv_bfloat16 *>(theta16));
  return cudaGetLastError() == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

int jq_mlp_forward(const float *theta, const uint16_t *theta16, const uint16_t *X, size_t n,
                   float *y, void *stream) {
  if (!theta || !theta16 || !X || !y) return JQ_ERR_INVALID_ARG;
  if (n == 0) return JQ_OK;
  size_t grid = (n + 1) / 2;
  if (grid > 1184) grid = 1184;
  mlp_forward_kernel<<<(unsigned)grid, TPB, 0, (cudaStream_t)stream>>>(
      theta, reinterpret_cast<const __nv_bfloat16 *>(theta16),
      reinterpret_cast<const __nv_bfloat16 *>(X), n, y);
  return cudaGetLastError() == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

size_t jq_mlp_scratch_floats(uint32_t ctas) { return (size_t)ctas * (NP + 1); }

int jq_mlp_train_step(const jq_mlp_step_args *a) {
  if (!a || !a->theta || !a->theta16 || !a->X || !a->T || !a->batch_index || a->batch == 0 ||
      !a->scratch || a->scratch_ctas == 0)
    return JQ_ERR_INVALID_ARG;
  if (a->apply && (!a->adam_m || !a->adam_v || a->step == 0)) return JQ_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)a->stream;
  const size_t smem = grad_smem();
  if (cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return JQ_ERR_LAUNCH;
  float *partial = a->scratch;
  float *loss_partial = a->scratch + (size_t)a->scratch_ctas * NP;
  mlp_grad_kernel<<<a->scratch_ctas, TPB, smem, st>>>(
      a->theta, reinterpret_cast<const __nv_bfloat16 *>(a->theta16),
      reinterpret_cast<const __nv_bfloat16 *>(a->X), a->T, a->batch_index, a->batch, partial,
      loss_partial);
  if (cudaGetLastError() != cudaSuccess) return JQ_ERR_LAUNCH;
  mlp_reduce_adam_kernel<<<(NP + 255) / 256, 256, 0, st>>>(
      a->theta, reinterpret_cast<__nv_bfloat16 *>(a->theta16), a->adam_m, a->adam_v, partial,
      a->scratch_ctas, a->grad_out, a->apply, a->lr, 0.9f, 0.999f, 1e-8f, a->step, loss_partial,
      a->loss_out, a->batch);
  return cudaGetLastError() == cudaSuccess ? JQ_OK : JQ_ERR_LAUNCH;
}

// ------------------------------------------------------------------------
// No-allocation variant of jq_mlp_train_step.
//
// Some hosts cannot call cudaMalloc (or any routine that allocates) once they
// are running: an embedding host that sizes one device pool at start-up and
// forbids allocation afterwards, or a host with hard latency limits where an
// allocation may stall on a device-wide synchronization.  For them the
// gradient workspace lives in this file-scope device array instead of a
// caller buffer.  It holds JQ_MLP_NOALLOC_MAX_CTAS partial-gradient rows
// (about 1.3 MB) on every GPU that loads the library, until the process
// exits.
static __device__ __align__(256) float g_mlp_noalloc_scratch[JQ_MLP_NOALLOC_MAX_CTAS * (JQ_MLP_PARAMS + 1)];

int jq_mlp_train_step_noalloc(const jq_mlp_step_args *a) {
  if (!a) return JQ_ERR_INVALID_ARG;
  if (a->scratch_ctas == 0 || a->scratch_ctas > JQ_MLP_NOALLOC_MAX_CTAS)
    return JQ_ERR_NOALLOC_LIMIT;
  // The array's device address, for the current device and context.  The
  // host-side symbol is only a stand-in and must never be handed to a kernel.
  // It is resolved on every call (this allocates nothing) rather than cached,
  // because the module's address changes when the context does (another
  // context made current by the host, or a device reset).
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_mlp_noalloc_scratch) != cudaSuccess || !p) return JQ_ERR_CUDA;
  jq_mlp_step_args b = *a;
  b.scratch = static_cast<float *>(p);
  return jq_mlp_train_step(&b);
}

}  // extern "C"
