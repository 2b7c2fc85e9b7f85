/*
 * Deterministic single-precision exp and log for the training path.
 *
 * The tile binning test, the forward pass's early-stop index and the
 * fixed-point gradient sums are integers decided by float arithmetic that
 * includes exp() and log() (train_types.glsl:58,92; train_forward.comp:84-85;
 * train_backward.glsl:122-123,134). GLSL leaves those functions' last bits to
 * the implementation, and a GPU's hardware approximation differs from a host
 * libm in the last ulp, which would make such integers differ between the GPU
 * and a CPU check. These two functions are built only from IEEE-754
 * operations that round the same way on the GPU and on a host CPU (add, mul,
 * fused multiply-add with explicit fmaf, exact bit manipulation), so a kernel
 * and a CPU restatement that both call them agree bit for bit.
 *
 * Methods (published, restated here from the mathematics):
 *   splat_expf: Cody and Waite's argument reduction (Cody & Waite, Software
 *     Manual for the Elementary Functions, 1980): x = n ln2 + r with ln2 split
 *     into a short high part and a low part, |r| <= ln2/2, then e^r by its
 *     degree-7 Taylor polynomial in Horner form, then 2^n through the exponent
 *     field. n is found with the 1.5 * 2^23 rounding constant, which rounds to
 *     nearest even exactly like rintf for |t| < 2^22.
 *   splat_logf: y = m 2^e with m in [2/3, 4/3) taken from the bit pattern, then
 *     log(m) = 2 atanh(s), s = (m - 1) / (m + 1), |s| <= 1/7, by the odd series
 *     2 (s + s^3/3 + s^5/5 + s^7/7 + s^9/9), and e ln2 added with ln2 split in
 *     two as above.
 * Accuracy against a double-precision libm is checked by the tests (a few
 * ulp); determinism, not the last ulp, is their purpose.
 *
 * Domain: splat_expf clamps x to [-86, 88] (results below e^-86 are not
 * needed: every caller compares them with 1/255 or multiplies them into a
 * transmittance below 1e-4) and returns NaN for NaN. splat_logf expects a
 * positive normal float.
 * Compile device code that uses them without FMA contraction being relevant:
 * every rounding here is explicit.
 */
#ifndef SPLAT_DETMATH_H
#define SPLAT_DETMATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define SPLAT_HD __host__ __device__ __forceinline__
#else
#define SPLAT_HD static inline
#endif

SPLAT_HD int32_t splat_float_bits(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_int(f);
#else
  int32_t i;
  memcpy(&i, &f, sizeof i);
  return i;
#endif
}

SPLAT_HD float splat_bits_float(int32_t i) {
#if defined(__CUDA_ARCH__)
  return __int_as_float(i);
#else
  float f;
  memcpy(&f, &i, sizeof f);
  return f;
#endif
}

SPLAT_HD float splat_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}

SPLAT_HD float splat_mul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}

SPLAT_HD float splat_add(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}

SPLAT_HD float splat_sub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}

/* Clamp that keeps a NaN a NaN (fminf/fmaxf would drop it), so that a NaN
 * parameter stays NaN through exp() and is culled as in the reference. */
SPLAT_HD float splat_clamp_nan(float x, float lo, float hi) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(x), "f"(lo));
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(r), "f"(hi));
  return r;
#else
  return x != x ? x : fminf(fmaxf(x, lo), hi);
#endif
}

SPLAT_HD float splat_expf(float x) {
  x = splat_clamp_nan(x, -86.0f, 88.0f);
  const float kRound = 12582912.0f; /* 1.5 * 2^23 */
  const float j = splat_add(splat_mul(x, 1.44269502f), kRound); /* log2(e) */
  const float n = splat_sub(j, kRound);
  float r = splat_fma(n, -0.693145752f, x);   /* ln2, high part: 0x3f317200, n * it is exact */
  r = splat_fma(n, -1.42860677e-06f, r);      /* ln2, low part */
  float p = 1.98412698e-04f;                  /* 1/5040 */
  p = splat_fma(p, r, 1.38888889e-03f);       /* 1/720 */
  p = splat_fma(p, r, 8.33333377e-03f);       /* 1/120 */
  p = splat_fma(p, r, 4.16666679e-02f);       /* 1/24 */
  p = splat_fma(p, r, 1.66666672e-01f);       /* 1/6 */
  p = splat_fma(p, r, 0.5f);
  p = splat_fma(p, r, 1.0f);
  p = splat_fma(p, r, 1.0f);
  /* The low bits of j hold n (two's complement); shifting them into the
   * exponent field multiplies by 2^n. p is in [0.70, 1.42] and n in
   * [-124, 127], so the result stays a normal float. */
  return splat_bits_float(splat_float_bits(p) + (int32_t)((uint32_t)splat_float_bits(j) << 23));
}

SPLAT_HD float splat_logf(float y) {
  const int32_t bits = splat_float_bits(y);
  const int32_t e = (bits - 0x3f2aaaab) >> 23; /* 0x3f2aaaab: 2/3 */
  const float m = splat_bits_float(bits - (int32_t)((uint32_t)e << 23));
  const float num = splat_sub(m, 1.0f);      /* exact: m in [2/3, 4/3) */
  const float den = splat_add(m, 1.0f);
#if defined(__CUDA_ARCH__)
  const float s = __fdiv_rn(num, den);
#else
  const float s = num / den;
#endif
  const float s2 = splat_mul(s, s);
  float p = 0.111111112f;                     /* 1/9 */
  p = splat_fma(p, s2, 0.142857149f);         /* 1/7 */
  p = splat_fma(p, s2, 0.200000003f);         /* 1/5 */
  p = splat_fma(p, s2, 0.333333343f);         /* 1/3 */
  /* 2 s (1 + s2 p) = 2 s + 2 s s2 p */
  const float s3 = splat_mul(s, s2);
  const float logm = splat_fma(splat_mul(2.0f, s3), p, splat_mul(2.0f, s));
  const float ef = (float)e;
  return splat_fma(ef, 0.693145752f, splat_fma(ef, 1.42860677e-06f, logm));
}

#endif /* SPLAT_DETMATH_H */
