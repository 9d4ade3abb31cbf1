// dpt_gemm.cu - BF16 x BF16 -> FP32 GEMM on the tensor cores (tcgen05.mma kind::f16, accumulator in
// tensor memory) with fused epilogues, for training the proposal network.
//
//   C[m][n] = epi( sum_k A[m][k] B[n][k] ),  A [M][lda], B [N][ldb] bf16 row-major (K contiguous),
//   epi: + bias[n], then ReLU, or a multiply by (ref[m][n] > 0) (the ReLU derivative of a stored
//   activation), then a store as fp32 and / or bf16.
//
// One CTA computes a 128 x NT tile (NT = 64 or 128) with 128 threads. The K loop stages 64-element
// slabs of A and B in shared memory in the tensor cores' K-major no-swizzle layout (8-row x 16-byte
// core matrices; K chunk c of a tile of r rows at c * r * 16 bytes, row group at 128 bytes), two
// buffers deep: while the MMAs of slab k run, the threads load slab k+1. Thread 0 issues the MMAs
// (K = 16 each) and commits each slab to an mbarrier that frees its buffer. The epilogue reads the
// accumulator back with tcgen05.ld (warp w owns rows 32w..32w+31). Every wait is bounded.
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/drift_pt.h"
#include "dpt_internal.h"

namespace dpt {
namespace {

constexpr int kGM = 128;   // tile rows (MMA M)
constexpr int kGK = 64;    // K elements per staged slab
constexpr int kGThreads = 128;

__device__ __forceinline__ uint32_t g_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long g_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool g_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// every thread waits for itself; false after the time limit (the error flag is then set)
__device__ bool g_wait(uint32_t bar, uint32_t parity, int* err, long long timeout_ns) {
  if (g_test(bar, parity)) return true;
  const unsigned long long t0 = g_now();
  while (!g_test(bar, parity)) {
    if (g_now() - t0 > (unsigned long long)timeout_ns) {
      if (err) atomicExch(err, DRIFT_PT_ETIMEOUT);
      return false;
    }
  }
  return true;
}

// K-major, no swizzle: leading (K) offset = chunk stride, stride (row-group) offset = 128 bytes
__device__ __forceinline__ uint64_t g_desc(uint32_t addr, uint32_t chunk_stride) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((chunk_stride >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)(128u >> 4) << 32) | ((uint64_t)1 << 46);
}

struct GemmArgs {
  int M, N, K, lda, ldb, ldc, act;
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  const float* bias;
  const __nv_bfloat16* ref;
  float* out_f32;
  __nv_bfloat16* out_bf16;
  int* err;
  long long timeout_ns;
};

// stage one 64-element K slab of `rows` rows starting at (row0, k0) into shared memory
__device__ __forceinline__ void stage(unsigned char* dst, const __nv_bfloat16* src, int ld, int row0, int rows_valid,
                                      int k0, int K, int rows) {
  const int chunks = rows * (kGK / 8);  // 16-byte pieces
  for (int c = threadIdx.x; c < chunks; c += kGThreads) {
    const int r = c >> 3, kc = c & 7;  // row, K chunk
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    const int k = k0 + 8 * kc;
    if (r < rows_valid && k < K) v = *reinterpret_cast<const uint4*>(src + (size_t)(row0 + r) * ld + k);
    *reinterpret_cast<uint4*>(dst + kc * rows * 16 + (r >> 3) * 128 + (r & 7) * 16) = v;
  }
}

template <int NT>
__global__ void __launch_bounds__(kGThreads) gemm_bf16_kernel(const GemmArgs a) {
  extern __shared__ __align__(1024) unsigned char g_raw[];
  constexpr int kABytes = kGM * kGK * 2, kBBytes = NT * kGK * 2;
  unsigned char* bufA[2] = {g_raw, g_raw + kABytes + kBBytes};
  unsigned char* bufB[2] = {g_raw + kABytes, g_raw + 2 * kABytes + kBBytes};
  uint64_t* bars = reinterpret_cast<uint64_t*>(g_raw + 2 * (kABytes + kBBytes));
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 4);
  // instruction descriptor: kind::f16, D f32 (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1),
  // K-major, N = NT (bits 17-22 = N >> 3), M = 128 (bits 24-28 = M >> 4)
  constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(kGM >> 4) << 24);
  constexpr uint32_t kCols = NT < 32 ? 32 : NT;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kGM, n0 = blockIdx.y * NT;
  const int rows_a = min(kGM, a.M - m0), rows_b = min(NT, a.N - n0);
  if (tid == 0) {
    for (int i = 0; i < 3; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(g_smem(bars + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(g_smem(tslot)), "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tslot);

  const int nk = (a.K + kGK - 1) / kGK;
  bool ok = true;
  for (int it = 0; it < nk; ++it) {
    const int b = it & 1;
    // buffer b was last read by the MMAs of slab it-2
    if (it >= 2 && !g_wait(g_smem(bars + b), (uint32_t)((it - 2) >> 1) & 1u, a.err, a.timeout_ns)) ok = false;
    if (!__syncthreads_and(ok)) break;
    stage(bufA[b], a.A, a.lda, m0, rows_a, it * kGK, a.K, kGM);
    stage(bufB[b], a.B, a.ldb, n0, rows_b, it * kGK, a.K, NT);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = g_smem(bufA[b]), sb = g_smem(bufB[b]);
#pragma unroll
      for (int s = 0; s < kGK / 16; ++s) {
        const uint64_t da = g_desc(sa + (uint32_t)(2 * s * kGM * 16), kGM * 16);
        const uint64_t db = g_desc(sb + (uint32_t)(2 * s * NT * 16), NT * 16);
        const uint32_t acc = (it > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(g_smem(bars + b))
                   : "memory");
    }
  }
  // all MMAs done
  if (tid == 0)
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(g_smem(bars + 2))
                 : "memory");
  const bool done = g_wait(g_smem(bars + 2), 0, a.err, a.timeout_ns);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (__syncthreads_and(done && ok) && nk > 0) {
    // epilogue: warp w holds rows 32w .. 32w+31 of the tile in TMEM lanes 32w..
    const int m = m0 + 32 * warp + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += 16) {
      uint32_t x[16];
      const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
          "tcgen05.wait::ld.sync.aligned;"
          : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7]),
            "=r"(x[8]), "=r"(x[9]), "=r"(x[10]), "=r"(x[11]), "=r"(x[12]), "=r"(x[13]), "=r"(x[14]), "=r"(x[15])
          : "r"(taddr)
          : "memory");
      if (m < a.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c0 + j;
          if (n >= a.N) break;
          float v = __uint_as_float(x[j]);
          if (a.bias) v += a.bias[n];
          if (a.act == 1) v = fmaxf(v, 0.0f);
          if (a.ref && !(__bfloat162float(a.ref[(size_t)m * a.ldc + n]) > 0.0f)) v = 0.0f;
          if (a.out_f32) a.out_f32[(size_t)m * a.ldc + n] = v;
          if (a.out_bf16) a.out_bf16[(size_t)m * a.ldc + n] = __float2bfloat16_rn(v);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

template <int NT>
size_t gemm_smem() {
  return 2 * (size_t)(kGM + NT) * kGK * 2 + 64;
}

}  // namespace
}  // namespace dpt

using namespace dpt;

extern "C" int drift_pt_gemm_bf16(const DriftPtGemm* g, int32_t* error_flag, void* stream) {
  clear_error();
  if (!g || !g->A || !g->B || (!g->out_f32 && !g->out_bf16)) return set_error(DRIFT_PT_EINVAL, "gemm: null argument");
  if (g->M < 1 || g->N < 1 || g->K < 1) return set_error(DRIFT_PT_EINVAL, "gemm: empty shape");
  if (g->K % 8 || g->lda % 8 || g->ldb % 8 || g->lda < g->K || g->ldb < g->K || g->ldc < g->N)
    return set_error(DRIFT_PT_EINVAL, "gemm: K, lda and ldb must be multiples of 8 with lda, ldb >= K and ldc >= N");
  if ((reinterpret_cast<uintptr_t>(g->A) | reinterpret_cast<uintptr_t>(g->B)) & 15)
    return set_error(DRIFT_PT_EINVAL, "gemm: A and B must be 16-byte aligned");
  if (g->act != 0 && g->act != 1) return set_error(DRIFT_PT_EINVAL, "gemm: act must be 0 (none) or 1 (relu)");
  GemmArgs a;
  std::memset(&a, 0, sizeof a);
  a.M = g->M;
  a.N = g->N;
  a.K = g->K;
  a.lda = g->lda;
  a.ldb = g->ldb;
  a.ldc = g->ldc;
  a.act = g->act;
  a.A = static_cast<const __nv_bfloat16*>(g->A);
  a.B = static_cast<const __nv_bfloat16*>(g->B);
  a.bias = g->bias;
  a.ref = static_cast<const __nv_bfloat16*>(g->relu_ref);
  a.out_f32 = g->out_f32;
  a.out_bf16 = static_cast<__nv_bfloat16*>(g->out_bf16);
  a.err = error_flag;
  a.timeout_ns = 2000000000LL;
  const bool wide = g->N > 64;
  const void* fn = wide ? (const void*)gemm_bf16_kernel<128> : (const void*)gemm_bf16_kernel<64>;
  const size_t smem = wide ? gemm_smem<128>() : gemm_smem<64>();
  int per_sm = 0;
  int rc = prepare_kernel(fn, kGThreads, smem, &per_sm);
  if (rc) return rc;
  const int nt = wide ? 128 : 64;
  dim3 grid((g->M + kGM - 1) / kGM, (g->N + nt - 1) / nt);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (wide)
    gemm_bf16_kernel<128><<<grid, kGThreads, smem, st>>>(a);
  else
    gemm_bf16_kernel<64><<<grid, kGThreads, smem, st>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(DRIFT_PT_ECUDA, "gemm launch: %s", cudaGetErrorString(e));
  return DRIFT_PT_OK;
}
