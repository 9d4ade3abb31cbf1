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
  int n, h1, h2, S, count, mode;  // mode 0: sample x, 1: evaluate given x
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

template <int S>
__global__ void __launch_bounds__(256) made_sample_kernel(const MadeArgs a) {
  extern __shared__ __align__(16) unsigned char m_raw[];
  const int n = a.n, H1 = a.h1, H2 = a.h2;
  float* h1p = reinterpret_cast<float*>(m_raw);  // [S][H1]
  float* h2p = h1p + (size_t)S * H1;              // [S][H2]
  float* outp = h2p + (size_t)S * H2;             // [S][n]
  float* r1 = outp + (size_t)S * n;               // [S][4] finished first-layer values of this step
  float* r2 = r1 + 4 * S;                         // [S][4]
  int8_t* xs = reinterpret_cast<int8_t*>(r2 + 4 * S);  // [S] this step's spins
  const int tid = threadIdx.x, T = blockDim.x;
  const int base = blockIdx.x * S;
  const int ns = min(S, a.count - base);
  for (int idx = tid; idx < S * H1; idx += T) h1p[idx] = a.b1[idx % H1];
  for (int idx = tid; idx < S * H2; idx += T) h2p[idx] = a.b2[idx % H2];
  for (int idx = tid; idx < S * n; idx += T) outp[idx] = a.b3[idx % n];
  float lq = 0.0f;  // thread s < ns accumulates sample s
  __syncthreads();
  for (int i = 0; i < n; ++i) {
    // x_i from l_i (final: every second-layer unit of degree <= i is in)
    if (tid < ns) {
      const float l = outp[tid * n + i];
      int8_t s;
      if (a.mode == 0) {
        const U4 u = philox(U4{(uint32_t)i, (uint32_t)(base + tid), a.stream, ctr3(kTagMadeSample, 0)}, a.k0, a.k1);
        const float uf = (float)(u.x >> 8) * 0x1.0p-24f;
        s = uf < 1.0f / (1.0f + expf(-l)) ? (int8_t)1 : (int8_t)-1;
        a.x[(size_t)(base + tid) * n + i] = s;
      } else {
        s = a.x[(size_t)(base + tid) * n + i];
      }
      xs[tid] = s;
      lq += log_sigmoid((float)s * l);
    }
    __syncthreads();
    // first layer: += column i of W1 (zero where the mask excludes it)
    {
      const __nv_bfloat16* col = a.w1t + (size_t)i * H1;
      for (int k = tid; k < H1; k += T) {
        const float wv = __bfloat162float(col[k]);
        if (wv != 0.0f)
          for (int s = 0; s < ns; ++s) h1p[s * H1 + k] += wv * (float)xs[s];
      }
    }
    __syncthreads();
    // first-layer units of degree i+1 are finished: their ReLU feeds the second layer
    const int f1a = a.off1[i], f1b = a.off1[i + 1];
    for (int idx = tid; idx < (f1b - f1a) * ns; idx += T) {
      const int u = idx / ns, s = idx % ns;
      r1[s * 4 + u] = fmaxf(h1p[s * H1 + a.ord1[f1a + u]], 0.0f);
    }
    __syncthreads();
    for (int u = 0; u < f1b - f1a; ++u) {
      const __nv_bfloat16* row = a.w2t + (size_t)a.ord1[f1a + u] * H2;
      for (int k = tid; k < H2; k += T) {
        const float wv = __bfloat162float(row[k]);
        if (wv != 0.0f)
          for (int s = 0; s < ns; ++s) h2p[s * H2 + k] += wv * r1[s * 4 + u];
      }
    }
    __syncthreads();
    // second-layer units of degree i+1 are finished: their ReLU feeds the logits
    const int f2a = a.off2[i], f2b = a.off2[i + 1];
    for (int idx = tid; idx < (f2b - f2a) * ns; idx += T) {
      const int u = idx / ns, s = idx % ns;
      r2[s * 4 + u] = fmaxf(h2p[s * H2 + a.ord2[f2a + u]], 0.0f);
    }
    __syncthreads();
    for (int u = 0; u < f2b - f2a; ++u) {
      const __nv_bfloat16* row = a.w3t + (size_t)a.ord2[f2a + u] * n;
      for (int k = tid; k < n; k += T) {
        const float wv = __bfloat162float(row[k]);
        if (wv != 0.0f)
          for (int s = 0; s < ns; ++s) outp[s * n + k] += wv * r2[s * 4 + u];
      }
    }
    __syncthreads();
  }
  if (tid < ns) a.logq[base + tid] = lq;
}

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

extern "C" int drift_pt_made_sample(const DriftPtMadeNet* net, int32_t count, int32_t mode, int8_t* x, float* logq,
                                    uint64_t seed, uint32_t stream_id, void* stream) {
  clear_error();
  if (!net || !net->w1t || !net->w2t || !net->w3t || !net->b1 || !net->b2 || !net->b3 || !net->ord1 || !net->off1 ||
      !net->ord2 || !net->off2 || !x || !logq)
    return set_error(DRIFT_PT_EINVAL, "made_sample: null argument");
  if (net->n < 2 || net->h1 < 1 || net->h2 < 1 || count < 1 || (mode != 0 && mode != 1))
    return set_error(DRIFT_PT_EINVAL, "made_sample: bad sizes or mode");
  if (net->max_units_per_degree > 4) return set_error(DRIFT_PT_EINVAL, "made_sample: at most 4 hidden units per degree");
  MadeArgs a;
  std::memset(&a, 0, sizeof a);
  a.n = net->n;
  a.h1 = net->h1;
  a.h2 = net->h2;
  a.count = count;
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
  a.x = x;
  a.logq = logq;
  a.k0 = (uint32_t)(seed & 0xffffffffu);
  a.k1 = (uint32_t)(seed >> 32);
  a.stream = stream_id;
  constexpr int S = 8;
  a.S = S;
  const size_t smem = (size_t)S * (a.h1 + a.h2 + a.n) * 4 + 8 * S * 4 + 16;
  int per_sm = 0;
  int rc = prepare_kernel((const void*)made_sample_kernel<S>, 256, smem, &per_sm);
  if (rc) return rc;
  if (per_sm < 1) return set_error(DRIFT_PT_EUNSUPPORTED, "made_sample: network too wide for shared memory");
  made_sample_kernel<S><<<(count + S - 1) / S, 256, smem, static_cast<cudaStream_t>(stream)>>>(a);
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
