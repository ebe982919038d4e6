/*
 * pyro_math.h — the arithmetic contract of one spin update.
 *
 * Every Monte Carlo update in this engine is a pure function of
 *   (its spin, its neighbours' spins, the couplings, beta, the cone width,
 *    Philox4x32-10(seed; site, replica, sweep, purpose)).
 * The functions below are written with IEEE-754 basic operations only
 * (add, mul, explicit fmaf, correctly rounded divide and sqrt) so that the
 * CUDA kernels and the C++ host oracle produce bit-identical results.
 * Kernels that include this file are compiled with --fmad=false and the host
 * side with -ffp-contract=off, so no compiler-chosen contraction changes the
 * rounding; every fused multiply-add below is spelled out with fmaf.
 *
 * Elementary functions are our own, from textbook methods:
 *   exp   : Cody & Waite (1980) range reduction x = k ln2 + r, |r| <= ln2/2,
 *           Taylor series of e^r to degree 7, scaling by 2^k.
 *   sincospi: reduction of a to the nearest quarter turn, Taylor series of
 *           sin(pi r), cos(pi r) for |r| <= 1/4, quadrant rotation.
 *   log   : m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1))
 *           by its odd power series.
 * Coefficients are the Taylor coefficients (1/n!, pi^n/n!, 1/(2k+1))
 * rounded to float.
 *
 * Philox4x32-10 follows Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11 (multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
 * increments 0x9E3779B9 / 0xBB67AE85, 10 rounds).
 *
 * Reference correspondence (taillefu/cudacode):
 *   sphere sampling cos(theta)=2u-1, phi=2 pi u   Math.cu:120-130
 *   Metropolis rule u < min(1, exp(-beta dE))     Math.cu:968-986
 *   over-relaxation S -> 2(S.h)h/|h|^2 - S         Math.cu:220-242
 *   cone proposal cos(theta)=1-(1-c0)u            Math.cu:244-281
 *     (the frame about the axis is built with the branch-free orthonormal
 *      basis of Duff et al., JCGT 6(1) 2017, instead of a Householder map)
 */
#ifndef PYRO_MATH_H
#define PYRO_MATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define PYRO_HD __host__ __device__ __forceinline__
#else
#define PYRO_HD static inline
#include <math.h>
#include <string.h>
#endif

/* Philox counter word 3 ("purpose") values: one stream per use. */
#define PYRO_PURPOSE_INIT 0x1u       /* random initial spins            */
#define PYRO_PURPOSE_METRO 0x2u      /* cone Metropolis proposal/accept */
#define PYRO_PURPOSE_SWAP 0x3u       /* replica-exchange acceptance     */
/* learned move: +0, +1 proposals and test, +8 training batches, +9 initial weights */
#define PYRO_PURPOSE_TET 0x10u

typedef struct { float x, y, z; } pyro_vec3;

PYRO_HD float pyro_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

PYRO_HD uint32_t pyro_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}

/* Philox4x32-10: c = counter (4 words), k = key (2 words); result in out. */
PYRO_HD void pyro_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                         uint32_t k0, uint32_t k1, uint32_t out[4]) {
#if defined(__CUDACC__)
#pragma unroll
#endif
  for (int round = 0; round < 10; ++round) {
    /* each 32x32 -> 64-bit product once, both halves from it */
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
    const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* Uniform float in [0, 1) with 24 random bits. */
PYRO_HD float pyro_uniform(uint32_t r) { return (float)(r >> 8) * 5.9604644775390625e-8f; }

/* Uniform double in [0, 1) with 53 random bits from two words. */
PYRO_HD double pyro_uniform53(uint32_t a, uint32_t b) {
  const uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
  return (double)m * 1.1102230246251565404236316680908203125e-16;
}

/* e^x for x <= 0; returns 0 below -87 (below that the result would be
 * subnormal; the Metropolis test compares it with u >= 2^-24 or u == 0). */
PYRO_HD float pyro_expf(float x) {
  if (x < -87.0f) return 0.0f;
  if (x > 88.0f) x = 88.0f;
  const float kf = rintf(x * 1.44269502162933349609375f);   /* 1/ln 2 */
  float r = fmaf(-kf, 0.693145751953125f, x);               /* ln2 hi */
  r = fmaf(-kf, 1.428606765330187e-06f, r);                 /* ln2 lo */
  float p = 1.98412701138295233249664306640625e-4f;         /* 1/7!   */
  p = fmaf(p, r, 1.3888889225199818611145019531250e-3f);    /* 1/6!   */
  p = fmaf(p, r, 8.3333337679505348205566406250000e-3f);    /* 1/5!   */
  p = fmaf(p, r, 4.1666667908430099487304687500000e-2f);    /* 1/4!   */
  p = fmaf(p, r, 1.6666667163372039794921875000000e-1f);    /* 1/3!   */
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  const int k = (int)kf;
  const float scale = pyro_u2f((uint32_t)(k + 127) << 23);  /* 2^k, k >= -126 */
  return p * scale;
}

/* Natural log for x > 0 (finite, normal). */
PYRO_HD float pyro_logf(float x) {
  uint32_t u = pyro_f2u(x);
  int e = (int)((u >> 23) & 0xffu) - 127;
  float m = pyro_u2f((u & 0x007fffffu) | 0x3f800000u);      /* [1, 2) */
  if (m > 1.41421353816986083984375f) {                     /* sqrt(2) */
    m = m * 0.5f;
    e += 1;
  }
  const float t = (m - 1.0f) / (m + 1.0f);
  const float t2 = t * t;
  float p = 0.0909090936183929443359375f;                   /* 1/11 */
  p = fmaf(p, t2, 0.111111111938953399658203125f);          /* 1/9  */
  p = fmaf(p, t2, 0.142857149243354797363281250f);          /* 1/7  */
  p = fmaf(p, t2, 0.200000002980232238769531250f);          /* 1/5  */
  p = fmaf(p, t2, 0.333333343267440795898437500f);          /* 1/3  */
  p = p * t2;
  const float lm = fmaf(2.0f * t, p, 2.0f * t);
  return fmaf((float)e, 0.693145751953125f, fmaf((float)e, 1.428606765330187e-06f, lm));
}

/* sin(pi a), cos(pi a) for finite a (used with a in [0, 2)). */
PYRO_HD void pyro_sincospif(float a, float* s_out, float* c_out) {
  const float j = rintf(a * 2.0f);
  const float r = fmaf(j, -0.5f, a);                        /* exact, |r| <= 1/4 */
  const float r2 = r * r;
  /* sin(pi r) = r (pi - pi^3/3! r^2 + pi^5/5! r^4 - ...) */
  float sp = -7.37043097615242004394531250e-3f;
  sp = fmaf(sp, r2, 8.21458846330642700195312500e-2f);
  sp = fmaf(sp, r2, -5.99264502525329589843750000e-1f);
  sp = fmaf(sp, r2, 2.55016398429870605468750000f);
  sp = fmaf(sp, r2, -5.16771268844604492187500000f);
  sp = fmaf(sp, r2, 3.14159274101257324218750000f);
  const float s = sp * r;
  /* cos(pi r) = 1 - pi^2/2! r^2 + pi^4/4! r^4 - ... */
  float cp = -2.58068908005952835083007812e-2f;
  cp = fmaf(cp, r2, 2.35330626368522644042968750e-1f);
  cp = fmaf(cp, r2, -1.33526277542114257812500000f);
  cp = fmaf(cp, r2, 4.05871200561523437500000000f);
  cp = fmaf(cp, r2, -4.93480205535888671875000000f);
  const float c = fmaf(cp, r2, 1.0f);
  const int q = ((int)j) & 3;
  float so = s, co = c;
  if (q == 1) { so = c; co = -s; }
  else if (q == 2) { so = -s; co = -c; }
  else if (q == 3) { so = -c; co = s; }
  *s_out = so;
  *c_out = co;
}

/* Uniform unit vector from two uniforms: cos(theta) = 2 u1 - 1, phi = 2 pi u2. */
PYRO_HD pyro_vec3 pyro_sphere_point(float u1, float u2) {
  const float ct = fmaf(2.0f, u1, -1.0f);
  const float st = sqrtf(fmaxf(0.0f, fmaf(-ct, ct, 1.0f)));
  float sp, cp;
  pyro_sincospif(2.0f * u2, &sp, &cp);
  pyro_vec3 v;
  v.x = st * cp;
  v.y = st * sp;
  v.z = ct;
  return v;
}

/* Vector at polar angle acos(ct) (sin = st) and azimuth (cp, sp) about the
 * unit axis n, using the orthonormal frame of Duff et al. 2017. */
PYRO_HD pyro_vec3 pyro_about_axis(pyro_vec3 n, float ct, float st, float cp, float sp) {
  const float sgn = copysignf(1.0f, n.z);
  const float a = -1.0f / (sgn + n.z);
  const float b = n.x * n.y * a;
  const float e1x = fmaf(sgn * n.x * n.x, a, 1.0f);
  const float e1y = sgn * b;
  const float e1z = -sgn * n.x;
  const float e2x = b;
  const float e2y = fmaf(n.y * n.y, a, sgn);
  const float e2z = -n.y;
  const float c1 = st * cp, c2 = st * sp;
  pyro_vec3 o;
  o.x = fmaf(ct, n.x, fmaf(c2, e2x, c1 * e1x));
  o.y = fmaf(ct, n.y, fmaf(c2, e2y, c1 * e1y));
  o.z = fmaf(ct, n.z, fmaf(c2, e2z, c1 * e1z));
  return o;
}

/* Proposal uniform in the cap of half-angle acos(cosmax) about s. */
PYRO_HD pyro_vec3 pyro_cone_proposal(pyro_vec3 s, float cosmax, float u1, float u2) {
  const float ct = fmaf(-(1.0f - cosmax), u1, 1.0f);
  const float st = sqrtf(fmaxf(0.0f, fmaf(-ct, ct, 1.0f)));
  float sp, cp;
  pyro_sincospif(2.0f * u2, &sp, &cp);
  return pyro_about_axis(s, ct, st, cp, sp);
}

/* h + M v for one bond of the anisotropic exchange, M the row-major 3x3
 * bond matrix: each component one chain of fused multiply-adds over the
 * columns in order. The local field of a site is the sum of these over its
 * six nearest neighbours in canonical order, minus its Zeeman field. */
PYRO_HD pyro_vec3 pyro_matvec_add(pyro_vec3 h, const float* m, float vx, float vy, float vz) {
  pyro_vec3 o;
  o.x = fmaf(m[2], vz, fmaf(m[1], vy, fmaf(m[0], vx, h.x)));
  o.y = fmaf(m[5], vz, fmaf(m[4], vy, fmaf(m[3], vx, h.y)));
  o.z = fmaf(m[8], vz, fmaf(m[7], vy, fmaf(m[6], vx, h.z)));
  return o;
}

/* Energy change of replacing s by t in local field h (E_i = s . h). */
PYRO_HD float pyro_delta_e(pyro_vec3 h, pyro_vec3 s, pyro_vec3 t) {
  const float dx = t.x - s.x, dy = t.y - s.y, dz = t.z - s.z;
  return fmaf(h.z, dz, fmaf(h.y, dy, h.x * dx));
}

/* Metropolis acceptance: dE <= 0, or u < exp(-beta dE). */
PYRO_HD int pyro_metropolis_accept(float dE, float beta, float u) {
  if (dE <= 0.0f) return 1;
  return u < pyro_expf(-(beta * dE));
}

/* Microcanonical over-relaxation: reflection of s about h (|h| > 0). */
PYRO_HD pyro_vec3 pyro_overrelax(pyro_vec3 s, pyro_vec3 h) {
  const float hh = fmaf(h.z, h.z, fmaf(h.y, h.y, h.x * h.x));
  if (!(hh > 0.0f)) return s;
  const float sh = fmaf(s.z, h.z, fmaf(s.y, h.y, s.x * h.x));
  const float k = (2.0f * sh) / hh;
  pyro_vec3 o;
  o.x = fmaf(k, h.x, -s.x);
  o.y = fmaf(k, h.y, -s.y);
  o.z = fmaf(k, h.z, -s.z);
  return o;
}

/* Rescale to unit length. */
PYRO_HD pyro_vec3 pyro_renormalise(pyro_vec3 s) {
  const float n2 = fmaf(s.z, s.z, fmaf(s.y, s.y, s.x * s.x));
  const float inv = 1.0f / sqrtf(n2);
  pyro_vec3 o;
  o.x = s.x * inv;
  o.y = s.y * inv;
  o.z = s.z * inv;
  return o;
}

/* Double-precision e^x for the replica-exchange test (x <= 0):
 * Cody-Waite reduction with a two-part ln 2, Taylor series to degree 13. */
PYRO_HD double pyro_exp64(double x) {
  if (x < -700.0) return 0.0;
  if (x > 700.0) x = 700.0;
  const double kf = rint(x * 1.4426950408889634074);
  double r = fma(-kf, 6.93147180369123816490e-01, x);     /* ln2 hi (33 bits) */
  r = fma(-kf, 1.90821492927058770002e-10, r);            /* ln2 lo */
  double p = 1.0 / 6227020800.0;                          /* 1/13! */
  p = fma(p, r, 1.0 / 479001600.0);
  p = fma(p, r, 1.0 / 39916800.0);
  p = fma(p, r, 1.0 / 3628800.0);
  p = fma(p, r, 1.0 / 362880.0);
  p = fma(p, r, 1.0 / 40320.0);
  p = fma(p, r, 1.0 / 5040.0);
  p = fma(p, r, 1.0 / 720.0);
  p = fma(p, r, 1.0 / 120.0);
  p = fma(p, r, 1.0 / 24.0);
  p = fma(p, r, 1.0 / 6.0);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  const long long k = (long long)kf;
  uint64_t bits = (uint64_t)(k + 1023) << 52;
  double scale;
#if defined(__CUDA_ARCH__)
  scale = __longlong_as_double((long long)bits);
#else
  memcpy(&scale, &bits, 8);
#endif
  return p * scale;
}

/* Replica exchange between two temperature slots: accept with
 * min(1, exp((beta_a - beta_b) (E_a - E_b))), MonteCarlo.cu:122-169. */
PYRO_HD int pyro_swap_accept(double beta_a, double beta_b, double e_a, double e_b, double u) {
  const double x = (beta_a - beta_b) * (e_a - e_b);
  if (x >= 0.0) return 1;
  return u < pyro_exp64(x);
}

#endif /* PYRO_MATH_H */
