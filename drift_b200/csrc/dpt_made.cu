// dpt_made.cu - the proposal network: a masked autoregressive MLP (MADE: Germain, Gregor, Murray,
// Larochelle, ICML 2015) over n spins with two hidden layers, and the exact Metropolis-Hastings step
// that lets its whole-configuration proposals enter a replica without changing the stationary
// distribution.
//
//   q(x) = prod_i sigma(x_i l_i(x_<i)),  l = W3 relu(W2 relu(W1 x + b1) + b2) + b3,
//   masks from unit degrees: input i has degree i+1, hidden units degrees in 1..n-1,
//   W1[k][i] != 0 only if m1(k) >= i+1, W2[k'][k] only if m2(k') >= m1(k), W3[i][k'] only if
//   i+1 > m2(k'), so l_i depends on x_0 .. x_{i-1} only.
//
// Training runs on the tensor cores (drift_pt_gemm_bf16) plus the element-wise kernels here
// (log-likelihood and its gradient, bias sums, transposes, Adam with the masks). Sampling and
// log q evaluation use one kernel that walks the spins in order and applies every weight exactly
// once (one forward pass of work per sample): at step i it draws or reads x_i from l_i, adds
// column i of W1 to the first layer, finishes the first-layer units of degree i+1 and adds their
// contributions to the second layer, finishes the second-layer units of degree i+1 and adds theirs
// to the logits. Each sum is accumulated in the same order whatever the launch shape, so log q(x)
// is one deterministic function of x and the weights: the value used to sample a proposal is the
// value the Metropolis-Hastings ratio divides by.
#include <cstring>
#include <cuda_bf16.h>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"

namespace dpt {
namespace {

constexpr uint32_t kTagMadeSample = 8u, kTagMadeMh = 9u;

// log sigma(z), stable for either sign
__device__ __forceinline__ float log_sigmoid(float z) { return fminf(z, 0.0f) - log1pf(expf(-fabsf(z))); }

// ------------------------------------------------------------------------------------------------
// training kernels
// ------------------------------------------------------------------------------------------------
// logq[b] = sum_i log sigma(x_i l_i); dlogits = d(-scale * sum_b logq[b]) / dl = -scale x sigma(-x l)
__global__ void made_loss_kernel(int B, int n, const float* logits, const int8_t* x, float* logq,
                                 __nv_bfloat16* dlogits, float scale) {
  const int b = blockIdx.x;
  if (b >= B) return;
  float acc = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float l = logits[(size_t)b * n + i];
    const float s = (float)x[(size_t)b * n + i];
    acc += log_sigmoid(s * l);
    if (dlogits) dlogits[(size_t)b * n + i] = __float2bfloat16_rn(-scale * s * (1.0f / (1.0f + expf(s * l))));
  }
  __shared__ float red[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    float t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0 && logq) logq[b] = t;
  }
}

__global__ void spins_to_bf16_kernel(size_t count, const int8_t* x, __nv_bfloat16* out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn((float)x[i]);
}

// out[c][r] = in[r][c], 32 x 32 tiles through shared memory
__global__ void transpose_bf16_kernel(int rows, int cols, const __nv_bfloat16* in, __nv_bfloat16* out) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = r0 + j, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[j][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int c = c0 + j, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][j];
  }
}

// out[c] = sum_r in[r][c]
__global__ void colsum_bf16_kernel(int rows, int cols, const __nv_bfloat16* in, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float acc = 0.0f;
  for (int r = 0; r < rows; ++r) acc += __bfloat162float(in[(size_t)r * cols + c]);
  out[c] = acc;
}

// Adam on a [rows][cols] weight (or a bias when w16 is NULL); masked entries stay zero. Writes the
// bf16 copy [rows][cols] and its transpose [cols][rows].
__global__ void adam_kernel(int rows, int cols, float* w, const float* g, float* m, float* v, const uint8_t* mask,
                            float lr, float b1, float b2, float eps, float c1, float c2, __nv_bfloat16* w16,
                            __nv_bfloat16* w16t) {
  const size_t count = (size_t)rows * cols;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < count; idx += (size_t)gridDim.x * blockDim.x) {
    float wi = w[idx];
    if (mask && !mask[idx]) {
      wi = 0.0f;
    } else {
      const float gi = g[idx];
      const float mi = b1 * m[idx] + (1.0f - b1) * gi;
      const float vi = b2 * v[idx] + (1.0f - b2) * gi * gi;
      m[idx] = mi;
      v[idx] = vi;
      wi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
    w[idx] = wi;
    if (w16) {
      const __nv_bfloat16 h = __float2bfloat16_rn(wi);
      w16[idx] = h;
      const size_t r = idx / cols, c = idx % cols;
      w16t[c * rows + r] = h;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// sampling / evaluation: one CTA per group of S samples, units processed in degree order
// ------------------------------------------------------------------------------------------------
struct MadeArgs {
  int n, h1, h2, S, count, mode;  // mode 0: sample x, 1: evaluate given x, 2: keep x_<keep, draw the rest
  int keep;
  const __nv_bfloat16* w1t;       // [n][h1]   column i of W1 = row i
  const __nv_bfloat16* w2t;       // [h1][h2]
  const __nv_bfloat16* w3t;       // [h2][n]
  const float *b1, *b2, *b3;
  const int* ord1;  // first-layer units sorted by degree
  const int* off1;  // [n+1] ord1[off1[d-1] .. off1[d]) have degree d (d = 1..n)
  const int* ord2;
  const int* off2;
  int8_t* x;        // [count][n]
  float* logq;      // [count]
  uint32_t k0, k1, stream;
};

// Thread t owns first-layer units t, t+T, ... (kH1 of them), second-layer units likewise (kH2) and
// logits likewise (kN): their partial sums for the S samples of the CTA live in its registers. It
// also holds its slices of the next step's weights, loaded one step ahead. Shared memory carries
// only what crosses threads in a step: the finished units' ReLU values, the next logit and the
// drawn spins.
template <int S, int kH1, int kH2, int kN>
__device__ __forceinline__ void made_sample_body(const MadeArgs& a) {
  __shared__ float r1[4][S], r2[4][S], lnext[S];
  __shared__ float xs[S];
  extern __shared__ int m_idx[];  // the degree orders: off1 [n+1], off2 [n+1], ord1 [H1], ord2 [H2]
  const int n = a.n, H1 = a.h1, H2 = a.h2;
  const int tid = threadIdx.x, T = blockDim.x;
  int* off1 = m_idx;
  int* off2 = off1 + (n + 1);
  int* ord1 = off2 + (n + 1);
  int* ord2 = ord1 + H1;
  for (int k = tid; k <= n; k += T) {
    off1[k] = a.off1[k];
    off2[k] = a.off2[k];
  }
  for (int k = tid; k < H1; k += T) ord1[k] = a.ord1[k];
  for (int k = tid; k < H2; k += T) ord2[k] = a.ord2[k];
  __syncthreads();
  const int base = blockIdx.x * S;
  const int ns = min(S, a.count - base);
  float h1[kH1][S], h2[kH2][S], lo[kN][S];
#pragma unroll
  for (int j = 0; j < kH1; ++j) {
    const float bv = tid + j * T < H1 ? a.b1[tid + j * T] : 0.0f;
#pragma unroll
    for (int s = 0; s < S; ++s) h1[j][s] = bv;
  }
#pragma unroll
  for (int j = 0; j < kH2; ++j) {
    const float bv = tid + j * T < H2 ? a.b2[tid + j * T] : 0.0f;
#pragma unroll
    for (int s = 0; s < S; ++s) h2[j][s] = bv;
  }
#pragma unroll
  for (int j = 0; j < kN; ++j) {
    const float bv = tid + j * T < n ? a.b3[tid + j * T] : 0.0f;
#pragma unroll
    for (int s = 0; s < S; ++s) lo[j][s] = bv;
  }
  // weight slices of a step: column i of W1, rows of W2 for the finishing first-layer units and rows
  // of W3 for the finishing second-layer units (at most 4 of each)
  float w1[kH1], w2[4][kH2], w3[4][kN];
  auto fetch = [&](int i, float (&v1)[kH1], float (&v2)[4][kH2], float (&v3)[4][kN]) {
    const __nv_bfloat16* col = a.w1t + (size_t)i * H1;
#pragma unroll
    for (int j = 0; j < kH1; ++j) v1[j] = tid + j * T < H1 ? __bfloat162float(col[tid + j * T]) : 0.0f;
    const int f1a = off1[i], nf1 = off1[i + 1] - f1a;
    const int f2a = off2[i], nf2 = off2[i + 1] - f2a;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const __nv_bfloat16* row2 = u < nf1 ? a.w2t + (size_t)ord1[f1a + u] * H2 : nullptr;
      const __nv_bfloat16* row3 = u < nf2 ? a.w3t + (size_t)ord2[f2a + u] * n : nullptr;
#pragma unroll
      for (int j = 0; j < kH2; ++j) v2[u][j] = row2 && tid + j * T < H2 ? __bfloat162float(row2[tid + j * T]) : 0.0f;
#pragma unroll
      for (int j = 0; j < kN; ++j) v3[u][j] = row3 && tid + j * T < n ? __bfloat162float(row3[tid + j * T]) : 0.0f;
    }
  };
  fetch(0, w1, w2, w3);
  // l_0 is b3[0]
  if (tid == 0)
#pragma unroll
    for (int s = 0; s < S; ++s) lnext[s] = lo[0][s];
  float lq = 0.0f;  // thread s < ns accumulates sample s
  __syncthreads();
  for (int i = 0; i < n; ++i) {
    // x_i from l_i (final: every second-layer unit of degree <= i is in)
    if (tid < ns) {
      const float l = lnext[tid];
      float sv;
      if (a.mode == 0 || (a.mode == 2 && i >= a.keep)) {
        const U4 u = philox(U4{(uint32_t)i, (uint32_t)(base + tid), a.stream, ctr3(kTagMadeSample, 0)}, a.k0, a.k1);
        const float uf = (float)(u.x >> 8) * 0x1.0p-24f;
        sv = uf < 1.0f / (1.0f + expf(-l)) ? 1.0f : -1.0f;
        a.x[(size_t)(base + tid) * n + i] = (int8_t)sv;
      } else {
        sv = (float)a.x[(size_t)(base + tid) * n + i];
      }
      xs[tid] = sv;
      lq += log_sigmoid(sv * l);
    }
    // the next step's weights, in flight during this step
    float nw1[kH1], nw2[4][kH2], nw3[4][kN];
    if (i + 1 < n) fetch(i + 1, nw1, nw2, nw3);
    const int f1a = off1[i], nf1 = off1[i + 1] - f1a;
    const int f2a = off2[i], nf2 = off2[i + 1] - f2a;
    __syncthreads();
    // first layer: += column i of W1 (zero where masked); owners of finishing units publish ReLU
    {
      float xv[S];
#pragma unroll
      for (int s = 0; s < S; ++s) xv[s] = xs[s];
#pragma unroll
      for (int j = 0; j < kH1; ++j)
#pragma unroll
        for (int s = 0; s < S; ++s) h1[j][s] += w1[j] * xv[s];
    }
    for (int u = 0; u < nf1; ++u) {
      const int k = ord1[f1a + u];
      if (k % T == tid) {
        const int jj = k / T;
#pragma unroll
        for (int j = 0; j < kH1; ++j)
          if (j == jj)
#pragma unroll
            for (int s = 0; s < S; ++s) r1[u][s] = fmaxf(h1[j][s], 0.0f);
      }
    }
    __syncthreads();
    // second layer: += finishing first-layer units; owners of finishing second-layer units publish
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (u >= nf1) break;
      float rv[S];
#pragma unroll
      for (int s = 0; s < S; ++s) rv[s] = r1[u][s];
#pragma unroll
      for (int j = 0; j < kH2; ++j)
#pragma unroll
        for (int s = 0; s < S; ++s) h2[j][s] += w2[u][j] * rv[s];
    }
    for (int u = 0; u < nf2; ++u) {
      const int k = ord2[f2a + u];
      if (k % T == tid) {
        const int jj = k / T;
#pragma unroll
        for (int j = 0; j < kH2; ++j)
          if (j == jj)
#pragma unroll
            for (int s = 0; s < S; ++s) r2[u][s] = fmaxf(h2[j][s], 0.0f);
      }
    }
    __syncthreads();
    // logits: += finishing second-layer units; the owner of l_{i+1} publishes it
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (u >= nf2) break;
      float rv[S];
#pragma unroll
      for (int s = 0; s < S; ++s) rv[s] = r2[u][s];
#pragma unroll
      for (int j = 0; j < kN; ++j)
#pragma unroll
        for (int s = 0; s < S; ++s) lo[j][s] += w3[u][j] * rv[s];
    }
    if (i + 1 < n && (i + 1) % T == tid) {
      const int jj = (i + 1) / T;
#pragma unroll
      for (int j = 0; j < kN; ++j)
        if (j == jj)
#pragma unroll
          for (int s = 0; s < S; ++s) lnext[s] = lo[j][s];
    }
    if (i + 1 < n) {
#pragma unroll
      for (int j = 0; j < kH1; ++j) w1[j] = nw1[j];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
#pragma unroll
        for (int j = 0; j < kH2; ++j) w2[u][j] = nw2[u][j];
#pragma unroll
        for (int j = 0; j < kN; ++j) w3[u][j] = nw3[u][j];
      }
    }
    __syncthreads();
  }
  if (tid < ns) a.logq[base + tid] = lq;
}

template <int S, int kH1, int kH2, int kN>
__global__ void __launch_bounds__(256) made_sample_kernel(const MadeArgs a) {
  made_sample_body<S, kH1, kH2, kN>(a);
}

// several networks in one launch: blocks (., g) run network g with its own arguments
template <int S, int kH1, int kH2, int kN>
__global__ void __launch_bounds__(256) made_sample_group_kernel(const MadeArgs* args, uint32_t stream_add) {
  MadeArgs a = args[blockIdx.y];
  a.stream += stream_add;
  if ((int)blockIdx.x * S >= a.count) return;
  made_sample_body<S, kH1, kH2, kN>(a);
}

constexpr int kSampleS = 8, kSampleT = 256;

// ------------------------------------------------------------------------------------------------
// exact Metropolis-Hastings for whole-configuration proposals (dense layer state)
// ------------------------------------------------------------------------------------------------
__global__ void made_mh_kernel(int n, int R, const int8_t* prop, const long long* e_prop, const float* lq_prop,
                               const float* lq_cur, const double* betas, double escale, uint32_t k0, uint32_t k1,
                               uint32_t inst, long long round, int8_t* spins, long long* energy, int8_t* best_spins,
                               long long* best_energy, const int* rung_of_slot, long long* tried, long long* accepted,
                               const uint8_t* active) {
  const int slot = blockIdx.x;
  if (slot >= R || (active && !active[slot])) return;
  __shared__ int acc_sm;
  if (threadIdx.x == 0) {
    const int rung = rung_of_slot[slot];
    // log A = -beta (E' - E) + log q(x) - log q(x'), in double; E exact
    const double de = d_mul((double)(e_prop[slot] - energy[slot]), escale);
    const double la = d_add(d_mul(-betas[rung], de), d_sub((double)lq_cur[slot], (double)lq_prop[slot]));
    bool acc = la >= 0.0;
    if (!acc) {
      const U4 u = philox(U4{(uint32_t)slot, (uint32_t)round, (uint32_t)((unsigned long long)round >> 32),
                             ctr3(kTagMadeMh, inst)},
                          k0, k1);
      acc = uniform53(u.x, u.y) < exp_neg_d(la);
    }
    tried[rung] += 1;
    if (acc) accepted[rung] += 1;
    acc_sm = acc ? 1 : 0;
  }
  __syncthreads();
  if (!acc_sm) return;
  const bool better = e_prop[slot] < best_energy[slot];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int8_t s = prop[(size_t)slot * n + i];
    spins[(size_t)slot * n + i] = s;
    if (better) best_spins[(size_t)slot * n + i] = s;
  }
  if (threadIdx.x == 0) {
    energy[slot] = e_prop[slot];
    if (better) best_energy[slot] = e_prop[slot];
  }
}

int made_fail(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DRIFT_PT_OK : set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace
}  // namespace dpt

using namespace dpt;

extern "C" int drift_pt_made_loss(int32_t batch, int32_t n, const float* logits, const int8_t* x, float* logq,
                                  void* dlogits_bf16, float scale, void* stream) {
  clear_error();
  if (batch < 1 || n < 1 || !logits || !x) return set_error(DRIFT_PT_EINVAL, "made_loss: bad arguments");
  made_loss_kernel<<<batch, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      batch, n, logits, x, logq, static_cast<__nv_bfloat16*>(dlogits_bf16), scale);
  return made_fail("made_loss_kernel");
}

extern "C" int drift_pt_made_spins_to_bf16(int64_t count, const int8_t* x, void* out_bf16, void* stream) {
  clear_error();
  if (count < 0 || (count && (!x || !out_bf16))) return set_error(DRIFT_PT_EINVAL, "spins_to_bf16: bad arguments");
  if (count == 0) return DRIFT_PT_OK;
  const int blocks = (int)((count + 255) / 256 < 4096 ? (count + 255) / 256 : 4096);
  spins_to_bf16_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>((size_t)count, x,
                                                                               static_cast<__nv_bfloat16*>(out_bf16));
  return made_fail("spins_to_bf16_kernel");
}

extern "C" int drift_pt_transpose_bf16(int32_t rows, int32_t cols, const void* in, void* out, void* stream) {
  clear_error();
  if (rows < 1 || cols < 1 || !in || !out) return set_error(DRIFT_PT_EINVAL, "transpose: bad arguments");
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_bf16_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, static_cast<const __nv_bfloat16*>(in), static_cast<__nv_bfloat16*>(out));
  return made_fail("transpose_bf16_kernel");
}

extern "C" int drift_pt_colsum_bf16(int32_t rows, int32_t cols, const void* in, float* out, void* stream) {
  clear_error();
  if (rows < 1 || cols < 1 || !in || !out) return set_error(DRIFT_PT_EINVAL, "colsum: bad arguments");
  colsum_bf16_kernel<<<(cols + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, static_cast<const __nv_bfloat16*>(in), out);
  return made_fail("colsum_bf16_kernel");
}

extern "C" int drift_pt_adam(int32_t rows, int32_t cols, float* w, const float* g, float* m, float* v,
                             const uint8_t* mask, float lr, float beta1, float beta2, float eps, int32_t step,
                             void* w_bf16, void* wt_bf16, void* stream) {
  clear_error();
  if (rows < 1 || cols < 1 || !w || !g || !m || !v || step < 1 || (!w_bf16) != (!wt_bf16))
    return set_error(DRIFT_PT_EINVAL, "adam: bad arguments");
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  const size_t count = (size_t)rows * cols;
  const int blocks = (int)((count + 255) / 256 < 4096 ? (count + 255) / 256 : 4096);
  adam_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      rows, cols, w, g, m, v, mask, lr, beta1, beta2, eps, c1, c2, static_cast<__nv_bfloat16*>(w_bf16),
      static_cast<__nv_bfloat16*>(wt_bf16));
  return made_fail("adam_kernel");
}

static int made_sample_launch(const DriftPtMadeNet* net, int32_t count, int32_t mode, int32_t keep, int8_t* x,
                              float* logq, uint64_t seed, uint32_t stream_id, void* stream);

extern "C" int drift_pt_made_sample(const DriftPtMadeNet* net, int32_t count, int32_t mode, int8_t* x, float* logq,
                                    uint64_t seed, uint32_t stream_id, void* stream) {
  clear_error();
  if (mode != 0 && mode != 1) return set_error(DRIFT_PT_EINVAL, "made_sample: mode must be 0 or 1");
  return made_sample_launch(net, count, mode, 0, x, logq, seed, stream_id, stream);
}

extern "C" int drift_pt_made_sample_suffix(const DriftPtMadeNet* net, int32_t count, int32_t keep, int8_t* x,
                                           float* logq, uint64_t seed, uint32_t stream_id, void* stream) {
  clear_error();
  if (!net || keep < 0 || keep > net->n) return set_error(DRIFT_PT_EINVAL, "made_sample_suffix: keep must be in [0, n]");
  return made_sample_launch(net, count, 2, keep, x, logq, seed, stream_id, stream);
}

static int made_sample_launch(const DriftPtMadeNet* net, int32_t count, int32_t mode, int32_t keep, int8_t* x,
                              float* logq, uint64_t seed, uint32_t stream_id, void* stream) {
  if (!net || !net->w1t || !net->w2t || !net->w3t || !net->b1 || !net->b2 || !net->b3 || !net->ord1 || !net->off1 ||
      !net->ord2 || !net->off2 || !x || !logq)
    return set_error(DRIFT_PT_EINVAL, "made_sample: null argument");
  if (net->n < 2 || net->h1 < 1 || net->h2 < 1 || count < 1)
    return set_error(DRIFT_PT_EINVAL, "made_sample: bad sizes");
  if (net->max_units_per_degree > 4) return set_error(DRIFT_PT_EINVAL, "made_sample: at most 4 hidden units per degree");
  MadeArgs a;
  std::memset(&a, 0, sizeof a);
  a.n = net->n;
  a.h1 = net->h1;
  a.h2 = net->h2;
  a.count = count;
  a.mode = mode;
  a.keep = keep;
  a.w1t = static_cast<const __nv_bfloat16*>(net->w1t);
  a.w2t = static_cast<const __nv_bfloat16*>(net->w2t);
  a.w3t = static_cast<const __nv_bfloat16*>(net->w3t);
  a.b1 = net->b1;
  a.b2 = net->b2;
  a.b3 = net->b3;
  a.ord1 = net->ord1;
  a.off1 = net->off1;
  a.ord2 = net->ord2;
  a.off2 = net->off2;
  a.x = x;
  a.logq = logq;
  a.k0 = (uint32_t)(seed & 0xffffffffu);
  a.k1 = (uint32_t)(seed >> 32);
  a.stream = stream_id;
  constexpr int S = kSampleS, T = kSampleT;
  a.S = S;
  // per-thread weight slices: up to 4 first-layer, 4 second-layer and 2 logit entries per unit
  if (a.h1 > 4 * T || a.h2 > 4 * T || a.n > 2 * T)
    return set_error(DRIFT_PT_EUNSUPPORTED, "made_sample: hidden widths up to %d and n up to %d", 4 * T, 2 * T);
  auto fn = made_sample_kernel<S, 4, 4, 2>;
  const size_t smem = (size_t)(2 * (a.n + 1) + a.h1 + a.h2) * sizeof(int);
  int per_sm = 0;
  int rc = prepare_kernel((const void*)fn, T, smem, &per_sm);
  if (rc) return rc;
  fn<<<(count + S - 1) / S, T, smem, static_cast<cudaStream_t>(stream)>>>(a);
  return made_fail("made_sample_kernel");
}

extern "C" int drift_pt_made_mh(const DriftPtSkProblem* problem, const DriftPtSkRunArgs* args, DriftPtSkState* state,
                                const int8_t* proposals, const int64_t* prop_energy, const float* logq_prop,
                                const float* logq_cur, const uint8_t* active, int64_t* prop_tried,
                                int64_t* prop_accepted, int64_t round, void* stream) {
  clear_error();
  if (!problem || !args || !state || !proposals || !prop_energy || !logq_prop || !logq_cur || !prop_tried ||
      !prop_accepted || !args->betas)
    return set_error(DRIFT_PT_EINVAL, "made_mh: null argument");
  if (problem->n < 1 || args->n_replicas < 1) return set_error(DRIFT_PT_EINVAL, "made_mh: bad sizes");
  made_mh_kernel<<<args->n_replicas, 128, 0, static_cast<cudaStream_t>(stream)>>>(
      problem->n, args->n_replicas, proposals, reinterpret_cast<const long long*>(prop_energy), logq_prop, logq_cur,
      args->betas, std::ldexp(1.0, -(problem->shift + 1)), (uint32_t)(args->seed & 0xffffffffu),
      (uint32_t)(args->seed >> 32), args->instance, (long long)round, state->spins,
      reinterpret_cast<long long*>(state->energy), state->best_spins, reinterpret_cast<long long*>(state->best_energy),
      state->rung_of_slot, reinterpret_cast<long long*>(prop_tried), reinterpret_cast<long long*>(prop_accepted), active);
  return made_fail("made_mh_kernel");
}

extern "C" int drift_pt_made_group_bytes(int32_t n_nets, size_t* bytes) {
  clear_error();
  if (n_nets < 1 || !bytes) return set_error(DRIFT_PT_EINVAL, "made_group_bytes: bad arguments");
  *bytes = sizeof(MadeArgs) * (size_t)n_nets;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_made_group_fill(int32_t n_nets, const DriftPtMadeNet* nets, const int32_t* counts, int32_t mode,
                                        int8_t* const* x, float* const* logq, uint64_t seed,
                                        const uint32_t* stream_id, void* table) {
  clear_error();
  if (n_nets < 1 || !nets || !counts || !x || !logq || !table || (mode != 0 && mode != 1) || (mode == 0 && !stream_id))
    return set_error(DRIFT_PT_EINVAL, "made_group_fill: bad arguments");
  std::vector<MadeArgs> v((size_t)n_nets);
  for (int g = 0; g < n_nets; ++g) {
    const DriftPtMadeNet* net = nets + g;
    if (!net->w1t || !net->w2t || !net->w3t || !net->b1 || !net->b2 || !net->b3 || !net->ord1 || !net->off1 ||
        !net->ord2 || !net->off2 || !x[g] || !logq[g])
      return set_error(DRIFT_PT_EINVAL, "made_group_fill: network %d: null array", g);
    if (net->n < 2 || net->h1 < 1 || net->h2 < 1 || counts[g] < 1 || net->max_units_per_degree > 4 ||
        net->h1 > 4 * kSampleT || net->h2 > 4 * kSampleT || net->n > 2 * kSampleT)
      return set_error(DRIFT_PT_EUNSUPPORTED, "made_group_fill: network %d: sizes (n <= %d, hidden <= %d)", g,
                       2 * kSampleT, 4 * kSampleT);
    MadeArgs& a = v[(size_t)g];
    std::memset(&a, 0, sizeof a);
    a.n = net->n;
    a.h1 = net->h1;
    a.h2 = net->h2;
    a.S = kSampleS;
    a.count = counts[g];
    a.mode = mode;
    a.w1t = static_cast<const __nv_bfloat16*>(net->w1t);
    a.w2t = static_cast<const __nv_bfloat16*>(net->w2t);
    a.w3t = static_cast<const __nv_bfloat16*>(net->w3t);
    a.b1 = net->b1;
    a.b2 = net->b2;
    a.b3 = net->b3;
    a.ord1 = net->ord1;
    a.off1 = net->off1;
    a.ord2 = net->ord2;
    a.off2 = net->off2;
    a.x = x[g];
    a.logq = logq[g];
    a.k0 = (uint32_t)(seed & 0xffffffffu);
    a.k1 = (uint32_t)(seed >> 32);
    a.stream = mode == 0 ? stream_id[g] : 0u;
  }
  const cudaError_t e = cudaMemcpy(table, v.data(), sizeof(MadeArgs) * v.size(), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? DRIFT_PT_OK : set_error(DRIFT_PT_ECUDA, "made_group_fill: upload: %s", cudaGetErrorString(e));
}

extern "C" int drift_pt_made_group_run(const void* table, int32_t n_nets, int32_t max_count, int32_t max_n,
                                       int32_t max_h1, int32_t max_h2, uint32_t stream_add, void* stream) {
  clear_error();
  if (!table || n_nets < 1 || n_nets > 65535 || max_count < 1 || max_n < 2 || max_h1 < 1 || max_h2 < 1)
    return set_error(DRIFT_PT_EINVAL, "made_group_run: bad arguments");
  if (max_h1 > 4 * kSampleT || max_h2 > 4 * kSampleT || max_n > 2 * kSampleT)
    return set_error(DRIFT_PT_EUNSUPPORTED, "made_group_run: hidden widths up to %d and n up to %d", 4 * kSampleT,
                     2 * kSampleT);
  auto fn = made_sample_group_kernel<kSampleS, 4, 4, 2>;
  const size_t smem = (size_t)(2 * (max_n + 1) + max_h1 + max_h2) * sizeof(int);
  int per_sm = 0;
  const int rc = prepare_kernel((const void*)fn, kSampleT, smem, &per_sm);
  if (rc) return rc;
  dim3 grid((unsigned)((max_count + kSampleS - 1) / kSampleS), (unsigned)n_nets);
  fn<<<grid, kSampleT, smem, static_cast<cudaStream_t>(stream)>>>(static_cast<const MadeArgs*>(table), stream_add);
  return made_fail("made_sample_group_kernel");
}
