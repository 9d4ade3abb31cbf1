// dpt_common.cuh - definitions shared by the host code and the sm_100a kernels of the PT engine.
//
// Everything here is part of the *definition* of the Markov chain the engine runs, so it is written
// once for host and device and must give bit-identical results on both:
//   * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
//     SC'11), the counter-based generator every uniform is drawn from;
//   * the counter layout that names each uniform (which attempt / swap / initial spin it feeds);
//   * exp(x) for x <= 0 in double and in float, written from the mathematics (Cody-Waite range
//     reduction x = n ln2 + r, Taylor series of e^r in Horner form with fused multiply-adds,
//     exact scaling by 2^n). Only explicitly rounded operations are used, so host and device agree
//     to the last bit and the CPU oracle can reproduce every accept/reject decision.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define DPT_HD __host__ __device__ __forceinline__
#else
#define DPT_HD static inline
#endif

#if !defined(__CUDA_ARCH__)
#include <math.h>
#include <string.h>
#endif

namespace dpt {

// ---------------------------------------------------------------------------------------------
// Philox4x32-10
// ---------------------------------------------------------------------------------------------
struct U4 {
  uint32_t x, y, z, w;
};

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;  // multiplier applied to counter word 0
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;  // multiplier applied to counter word 2
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;  // Weyl increment of key word 0 (golden ratio)
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;  // Weyl increment of key word 1 (sqrt 3 - 1)

// one widening multiply: on the device a single 32x32->64 multiply-add gives both halves
DPT_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  lo = (uint32_t)p;
  hi = (uint32_t)(p >> 32);
}

// Ten rounds; the key is bumped between rounds (the bump after the last round is never used).
DPT_HD U4 philox(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(kPhiloxM0, c.x, hi0, lo0);
    mulhilo32(kPhiloxM1, c.z, hi1, lo1);
    U4 o;
    o.x = hi1 ^ c.y ^ k0;
    o.y = lo1;
    o.z = hi0 ^ c.w ^ k1;
    o.w = lo0;
    c = o;
    k0 += kPhiloxW0;
    k1 += kPhiloxW1;
  }
  return c;
}

// ---------------------------------------------------------------------------------------------
// Counter layout. Key = (seed & 0xffffffff, seed >> 32). Counter word 3 = (tag << 24) | instance.
//   kTagSweep : ctr = (p >> 3, t, slot, .)  -> the 8 16-bit "primary" halves of the output feed
//               positions p & ~7 .. p | 7 in sweep t: half (p & 1) of word ((p >> 1) & 3).
//   kTagSecond: ctr = (p, t, slot, .)       -> low 16 bits of word 0 are the "secondary" half.
//               The 32-bit uniform of attempt (p, t, slot) is (primary << 16) | secondary; the
//               secondary is only evaluated when primary == thr >> 16 (probability 2^-16).
//   kTagInit  : ctr = (p >> 2, 0, slot, .)  -> bit 31 of word (p & 3) set => initial spin -1.
//   kTagSwap  : ctr = (r, round lo, round hi, .) -> words 0,1 form a 53-bit uniform for the
//               exchange of rungs r, r+1 in that round.
// ---------------------------------------------------------------------------------------------
//   kTagMsSweep: multispin lattices (32 replicas per word), ctr = (q, t, (w << 8) | (p >> 2), .),
//               word (p & 3) is random bit-plane p (p = 0 most significant) of the 32 uniforms
//               u_b = sum_p bit_b(plane_p) 2^(31-p) of site q (colour-split index), word w.
//   kTagMsInit : ctr = (q, 0, w, .) word 0 = the initial bits of site q in word w (1 = spin -1).
//   kTagSkSweep: dense couplings, ctr = (((i >> 7) << 5) | (i & 31), t, slot, .), word ((i >> 5) & 3)
//               is the uniform of spin i in sweep t (one Philox call covers spins i, i+32, i+64,
//               i+96 of a 128-spin tile).
constexpr uint32_t kTagSweep = 1u, kTagSecond = 2u, kTagInit = 3u, kTagSwap = 4u, kTagMsSweep = 5u,
                   kTagMsInit = 6u, kTagSkSweep = 7u;
constexpr uint32_t kMaxInstance = (1u << 24) - 1u;

DPT_HD uint32_t ctr3(uint32_t tag, uint32_t instance) { return (tag << 24) | (instance & kMaxInstance); }

DPT_HD double uniform53(uint32_t a, uint32_t b) {
  // (a >> 5) * 2^26 + (b >> 6): 53 random bits, scaled to [0, 1); exact in double.
  uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * 0x1.0p-53;
}

// ---------------------------------------------------------------------------------------------
// Explicitly rounded arithmetic (never contracted by the compiler).
// ---------------------------------------------------------------------------------------------
DPT_HD double d_mul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  volatile double r = a * b;
  return r;
#endif
}
DPT_HD double d_add(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  volatile double r = a + b;
  return r;
#endif
}
DPT_HD double d_sub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  volatile double r = a - b;
  return r;
#endif
}
DPT_HD double d_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
  return __fma_rn(a, b, c);
#else
  return fma(a, b, c);
#endif
}
DPT_HD double d_rint(double a) { return rint(a); }
DPT_HD float f_mul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  volatile float r = a * b;
  return r;
#endif
}
DPT_HD float f_add(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  volatile float r = a + b;
  return r;
#endif
}
DPT_HD float f_sub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  volatile float r = a - b;
  return r;
#endif
}
DPT_HD float f_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
DPT_HD float f_div(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdiv_rn(a, b);
#else
  volatile float r = a / b;
  return r;
#endif
}
DPT_HD float f_rint(float a) { return rintf(a); }
DPT_HD double bits_to_double(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double d;
  memcpy(&d, &u, sizeof d);
  return d;
#endif
}
DPT_HD float bits_to_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, sizeof f);
  return f;
#endif
}
// float -> int64, round to nearest even (the default rounding mode on the host).
DPT_HD long long f_to_ll_rn(float a) {
#if defined(__CUDA_ARCH__)
  return __float2ll_rn(a);
#else
  return llrintf(a);
#endif
}
// float in [0, 2^32] -> uint32, truncating, saturating at 2^32 - 1.
DPT_HD uint32_t f_to_u32_sat(float a) {
  if (a >= 4294967296.0f) return 0xFFFFFFFFu;
#if defined(__CUDA_ARCH__)
  return __float2uint_rz(a);
#else
  return (uint32_t)a;
#endif
}

// ---------------------------------------------------------------------------------------------
// exp(x) for x <= 0, double. x = n ln2 + r with |r| <= ln2/2; ln2 is split so n * hi is exact.
// e^r = sum_{k<=13} r^k / k! (truncation error < 2^-57 relative on |r| <= 0.3466).
// ---------------------------------------------------------------------------------------------
DPT_HD double exp_neg_d(double x) {
  if (!(x <= 0.0)) return 1.0;
  if (x < -708.0) return 0.0;
  const double kInvLn2 = 0x1.71547652b82fep+0;
  const double kLn2Hi = 0x1.62e4200000000p-1;  // ln 2 with the low 32 mantissa bits cleared
  const double kLn2Lo = 0x1.fdf473de6af28p-22;  // ln 2 - kLn2Hi
  double n = d_rint(d_mul(x, kInvLn2));
  double r = d_fma(-n, kLn2Hi, x);
  r = d_fma(-n, kLn2Lo, r);
  double p = 0x1.6124613a86d09p-33;           // 1/13!
  p = d_fma(p, r, 0x1.1eed8eff8d898p-29);     // 1/12!
  p = d_fma(p, r, 0x1.ae64567f544e4p-26);     // 1/11!
  p = d_fma(p, r, 0x1.27e4fb7789f5cp-22);     // 1/10!
  p = d_fma(p, r, 0x1.71de3a556c734p-19);     // 1/9!
  p = d_fma(p, r, 0x1.a01a01a01a01ap-16);     // 1/8!
  p = d_fma(p, r, 0x1.a01a01a01a01ap-13);     // 1/7!
  p = d_fma(p, r, 0x1.6c16c16c16c17p-10);     // 1/6!
  p = d_fma(p, r, 0x1.1111111111111p-7);      // 1/5!
  p = d_fma(p, r, 0x1.5555555555555p-5);      // 1/4!
  p = d_fma(p, r, 0x1.5555555555555p-3);      // 1/3!
  p = d_fma(p, r, 0.5);
  p = d_fma(p, r, 1.0);
  p = d_fma(p, r, 1.0);
  int ni = (int)n;  // in [-1022, 0]
  double scale = bits_to_double((uint64_t)(ni + 1023) << 52);
  return d_mul(p, scale);
}

// exp(x) for x <= 0, float; degree-7 Taylor series on |r| <= 0.347 (error < 2^-28 relative).
DPT_HD float exp_neg_f(float x) {
  if (!(x <= 0.0f)) return 1.0f;
  if (x < -87.0f) return 0.0f;
  const float kInvLn2 = 0x1.715476p+0f;
  const float kLn2Hi = 0x1.62ep-1f;      // ln 2 with the low 12 mantissa bits cleared
  const float kLn2Lo = 0x1.0bfbe8p-15f;  // ln 2 - kLn2Hi
  float n = f_rint(f_mul(x, kInvLn2));
  float r = f_fma(-n, kLn2Hi, x);
  r = f_fma(-n, kLn2Lo, r);
  float p = 0x1.a01a02p-13f;         // 1/7!
  p = f_fma(p, r, 0x1.6c16c2p-10f);  // 1/6!
  p = f_fma(p, r, 0x1.111112p-7f);   // 1/5!
  p = f_fma(p, r, 0x1.555556p-5f);   // 1/4!
  p = f_fma(p, r, 0x1.555556p-3f);   // 1/3!
  p = f_fma(p, r, 0.5f);
  p = f_fma(p, r, 1.0f);
  p = f_fma(p, r, 1.0f);
  int ni = (int)n;  // in [-126, 0]
  float scale = bits_to_float((uint32_t)(ni + 127) << 23);
  return f_mul(p, scale);
}

// Metropolis threshold for the float-coupling path: accept an attempt with energy change
// dE = 2x > 0 at inverse temperature beta iff u32 < thr, thr = trunc(exp(-beta * 2x) * 2^32).
// neg2beta is -2 * (float)beta (exact), so the product is rounded exactly once.
DPT_HD uint32_t threshold_f(float neg2beta, float x) {
  float e = exp_neg_f(f_mul(neg2beta, x));
  return f_to_u32_sat(f_mul(e, 4294967296.0f));
}

// Integer-coupling path: thr[x-1] for x = s_i (sum_j J_ij s_j + h_i) = dE/2 in 1..F.
DPT_HD uint32_t threshold_int(double beta, int x) {
  double e = exp_neg_d(d_mul(-2.0 * beta, (double)x));
  double v = d_mul(e, 4294967296.0);
  if (v >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)v;  // truncation = floor for v >= 0
}

// ---------------------------------------------------------------------------------------------
// -ln(u) for u in [2^-24, 1), float. u = m 2^e with m in (sqrt(2)/2, sqrt(2)]; with
// z = (m - 1) / (m + 1), ln m = 2 atanh z = 2 z (1 + z^2/3 + z^4/5 + z^6/7 + z^8/9)
// (|z| <= 0.1716, truncation < 2^-28 relative); ln u = e ln2 + ln m.
// ---------------------------------------------------------------------------------------------
DPT_HD float neg_log_unit_f(float u) {
  uint32_t bits;
#if defined(__CUDA_ARCH__)
  bits = __float_as_uint(u);
#else
  memcpy(&bits, &u, sizeof bits);
#endif
  int e = (int)(bits >> 23) - 127;
  uint32_t mb = (bits & 0x007FFFFFu) | 0x3F800000u;
  if (mb > 0x3FB504F3u) {  // m > sqrt(2): halve it
    mb -= 0x00800000u;
    e += 1;
  }
  const float m = bits_to_float(mb);
  const float z = f_div(f_sub(m, 1.0f), f_add(m, 1.0f));
  const float w = f_mul(z, z);
  float p = f_fma(w, 0x1.c71c72p-4f, 0x1.24924ap-3f);  // 1/9, 1/7
  p = f_fma(w, p, 0x1.99999ap-3f);                     // 1/5
  p = f_fma(w, p, 0x1.555556p-2f);                     // 1/3
  p = f_fma(w, p, 1.0f);
  const float lnm = f_mul(f_add(z, z), p);
  const float r = -f_fma((float)e, 0x1.62e430p-1f, lnm);  // ln 2 rounded to float
  return r > 0.0f ? r : 0.0f;
}

// Dense-coupling acceptance. Spin i with integer local field F (couplings and field in units of
// 2^-shift) is flipped iff s_i F <= D, D = floor(-ln(u) * c), c = 2^shift / (2 beta) rounded to
// float, u = (2 (word >> 9) + 1) 2^-24. That is dE = 2 s_i F 2^-shift <= -ln(u) / beta, i.e.
// u <= exp(-beta dE): the Metropolis rule, with the transcendental taken off the spin-to-spin
// dependency chain (D depends only on the uniform and the rung).
DPT_HD int32_t sk_threshold(uint32_t word, float c) {
  const float u = f_mul((float)(2u * (word >> 9) + 1u), 0x1.0p-24f);
  const float v = f_mul(neg_log_unit_f(u), c);
  if (v >= 2147483648.0f) return 2147483647;
#if defined(__CUDA_ARCH__)
  return __float2int_rz(v);
#else
  return (int32_t)v;
#endif
}

// Fixed-point scale of the energy accumulators: the integer path stores E exactly (scale 1); the
// float path stores round(E * 2^32) in int64, so sums of accepted dE are associative and every
// decomposition of the work gives the same bits.
constexpr double kFloatEnergyScale = 0x1.0p-32;
constexpr float kFloatEnergyQuant = 4294967296.0f;

}  // namespace dpt
