/*
 * cbm_rng.h — counter-based random stream shared by the host and the device.
 *
 * Every random number of the per-step path (Euler–Maruyama increments, the
 * division direction, the death draw) is a pure function of
 *     (seed, step, agent, stream, community, sub)
 * so the CUDA kernels, a CPU checker and a Julia caller that re-implements
 * this header all see the same numbers: the noise is "generated once and fed
 * to both" by construction.  It replaces the reference's global `randn()` /
 * `rand()` calls (src/random.jl:8-22, src/integrators.jl:718-724), whose
 * values are not reproducible across platforms.
 *
 * Generator: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11).  Normals: Box–Muller, with log and
 * sin/cos evaluated by the series written out below (atanh series for the
 * logarithm, Taylor series for sin/cos on [-pi/4, pi/4]) using only +,-,*,/
 * so that the bits do not depend on a platform's libm.  On the device every
 * operation goes through the round-to-nearest intrinsics, which the compiler
 * never contracts into FMAs; on the host compile with -ffp-contract=off.
 *
 * This is a C++ / CUDA header (it has overloads and templates).
 *
 * Counter layout of one Philox block:
 *     c0 = agent index (0-based, index before that step's compaction)
 *     c1 = step & 0xffffffff
 *     c2 = ((step >> 32) & 0xffff) | (stream << 16)
 *     c3 = (community << 8) | sub
 *     key = (seed & 0xffffffff, seed >> 32)
 */
#ifndef CBM_RNG_H
#define CBM_RNG_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define CBM_HD __host__ __device__ __forceinline__
#else
#define CBM_HD inline
#endif

#define CBM_STREAM_NOISE 0u    /* EM increments of the position variables */
#define CBM_STREAM_DIVISION 1u /* normal(0,1) x dims for the division axis */
#define CBM_STREAM_DEATH 2u    /* uniform(0,1) for the death branch */
#define CBM_STREAM_USER 3u     /* cbm_rng_fill and tests */
#define CBM_STREAM_NOISE_FINAL 4u /* EulerHeun: the fresh draw of its final update */
#define CBM_STREAM_ROD_TORQUE 5u  /* rods2dGrowth: uniform(-.1, .1) torque kick at division */
#define CBM_STREAM_ROD_TARGET 6u  /* rods2dGrowth: lTarget of the first daughter (+1: second) */

/* ---- exactly rounded primitives that are never fused ------------------- */
#if defined(__CUDA_ARCH__)
CBM_HD double cbm_rn_add(double a, double b) { return __dadd_rn(a, b); }
CBM_HD double cbm_rn_sub(double a, double b) { return __dsub_rn(a, b); }
CBM_HD double cbm_rn_mul(double a, double b) { return __dmul_rn(a, b); }
CBM_HD double cbm_rn_div(double a, double b) { return __ddiv_rn(a, b); }
CBM_HD double cbm_rn_sqrt(double a) { return __dsqrt_rn(a); }
CBM_HD float cbm_rn_add(float a, float b) { return __fadd_rn(a, b); }
CBM_HD float cbm_rn_sub(float a, float b) { return __fsub_rn(a, b); }
CBM_HD float cbm_rn_mul(float a, float b) { return __fmul_rn(a, b); }
CBM_HD float cbm_rn_div(float a, float b) { return __fdiv_rn(a, b); }
CBM_HD float cbm_rn_sqrt(float a) { return __fsqrt_rn(a); }
CBM_HD uint32_t cbm_mulhi32(uint32_t a, uint32_t b) { return __umulhi(a, b); }
CBM_HD uint64_t cbm_f64_bits(double x) { return (uint64_t)__double_as_longlong(x); }
CBM_HD double cbm_bits_f64(uint64_t b) { return __longlong_as_double((long long)b); }
CBM_HD uint32_t cbm_f32_bits(float x) { return (uint32_t)__float_as_uint(x); }
CBM_HD float cbm_bits_f32(uint32_t b) { return __uint_as_float(b); }
#else
#include <math.h>
CBM_HD double cbm_rn_add(double a, double b) { return a + b; }
CBM_HD double cbm_rn_sub(double a, double b) { return a - b; }
CBM_HD double cbm_rn_mul(double a, double b) { return a * b; }
CBM_HD double cbm_rn_div(double a, double b) { return a / b; }
CBM_HD double cbm_rn_sqrt(double a) { return sqrt(a); }
CBM_HD float cbm_rn_add(float a, float b) { return a + b; }
CBM_HD float cbm_rn_sub(float a, float b) { return a - b; }
CBM_HD float cbm_rn_mul(float a, float b) { return a * b; }
CBM_HD float cbm_rn_div(float a, float b) { return a / b; }
CBM_HD float cbm_rn_sqrt(float a) { return sqrtf(a); }
CBM_HD uint32_t cbm_mulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }
CBM_HD uint64_t cbm_f64_bits(double x) { uint64_t b; memcpy(&b, &x, 8); return b; }
CBM_HD double cbm_bits_f64(uint64_t b) { double x; memcpy(&x, &b, 8); return x; }
CBM_HD uint32_t cbm_f32_bits(float x) { uint32_t b; memcpy(&b, &x, 4); return b; }
CBM_HD float cbm_bits_f32(uint32_t b) { float x; memcpy(&x, &b, 4); return x; }
#endif

/* ---- Philox4x32-10 ------------------------------------------------------ */
typedef struct { uint32_t v[4]; } cbm_u32x4;

CBM_HD cbm_u32x4 cbm_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                   uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = cbm_mulhi32(M0, c0), lo0 = M0 * c0;
    uint32_t hi1 = cbm_mulhi32(M1, c2), lo1 = M1 * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += W0; k1 += W1;
  }
  cbm_u32x4 out;
  out.v[0] = c0; out.v[1] = c1; out.v[2] = c2; out.v[3] = c3;
  return out;
}

CBM_HD cbm_u32x4 cbm_rng_block(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                               uint32_t community, uint32_t sub) {
  uint64_t s = (uint64_t)step;
  return cbm_philox4x32_10(agent, (uint32_t)(s & 0xffffffffu),
                           (uint32_t)((s >> 32) & 0xffffu) | (stream << 16),
                           (community << 8) | (sub & 0xffu), (uint32_t)(seed & 0xffffffffu),
                           (uint32_t)(seed >> 32));
}

/* uniform [0,1) with 53 (resp. 24) random bits: exact integer arithmetic */
CBM_HD double cbm_u01_f64(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}
CBM_HD float cbm_u01_f32(uint32_t a) { return (float)(a >> 8) * (1.0f / 16777216.0f); }

/* ---- natural logarithm of x in (0, 2^1023], own series ------------------
 * x = m 2^e with m in (sqrt(1/2), sqrt(2)];  log m = 2 atanh(s),
 * s = (m-1)/(m+1), |s| <= 0.1716, atanh s = s (1 + s^2/3 + s^4/5 + ...). */
CBM_HD double cbm_log_f64(double x) {
  uint64_t b = cbm_f64_bits(x);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  double m = cbm_bits_f64((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
  if (m > 1.4142135623730951) { m = cbm_rn_mul(m, 0.5); e += 1; }
  double s = cbm_rn_div(cbm_rn_sub(m, 1.0), cbm_rn_add(m, 1.0));
  double z = cbm_rn_mul(s, s);
  double p = 0.047619047619047616;                       /* 1/21 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.05263157894736842);  /* 1/19 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.058823529411764705); /* 1/17 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.06666666666666667);  /* 1/15 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.07692307692307693);  /* 1/13 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.09090909090909091);  /* 1/11 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.1111111111111111);   /* 1/9 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.14285714285714285);  /* 1/7 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.2);                  /* 1/5 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.3333333333333333);   /* 1/3 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 1.0);
  double logm = cbm_rn_mul(cbm_rn_add(s, s), p);
  return cbm_rn_add(cbm_rn_mul((double)e, 0.6931471805599453), logm);
}

CBM_HD float cbm_log_f32(float x) {
  uint32_t b = cbm_f32_bits(x);
  int e = (int)((b >> 23) & 0xff) - 127;
  float m = cbm_bits_f32((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356f) { m = cbm_rn_mul(m, 0.5f); e += 1; }
  float s = cbm_rn_div(cbm_rn_sub(m, 1.0f), cbm_rn_add(m, 1.0f));
  float z = cbm_rn_mul(s, s);
  float p = 0.09090909f;                           /* 1/11 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.11111111f);   /* 1/9 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.14285715f);   /* 1/7 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.2f);          /* 1/5 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 0.33333334f);   /* 1/3 */
  p = cbm_rn_add(cbm_rn_mul(p, z), 1.0f);
  float logm = cbm_rn_mul(cbm_rn_add(s, s), p);
  return cbm_rn_add(cbm_rn_mul((float)e, 0.6931472f), logm);
}

/* ---- cos and sin of 2*pi*w for w in [0,1), own Taylor series ------------
 * 4w = n + r with integer n and |r| <= 1/2, theta = r pi/2 in [-pi/4, pi/4],
 * then rotate by n quarter turns. */
CBM_HD void cbm_cossin_turns_f64(double w, double* c, double* s) {
  double w4 = cbm_rn_mul(w, 4.0);
  int n = (int)cbm_rn_add(w4, 0.5);
  double th = cbm_rn_mul(cbm_rn_sub(w4, (double)n), 1.5707963267948966);
  double z = cbm_rn_mul(th, th);
  double ps = 2.8114572543455206e-15;
  ps = cbm_rn_add(cbm_rn_mul(ps, z), -7.647163731819816e-13);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), 1.6059043836821613e-10);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), -2.505210838544172e-08);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), 2.7557319223985893e-06);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), -0.0001984126984126984);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), 0.008333333333333333);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), -0.16666666666666666);
  double sn = cbm_rn_add(th, cbm_rn_mul(cbm_rn_mul(th, z), ps));
  double pc = -1.5619206968586225e-16;
  pc = cbm_rn_add(cbm_rn_mul(pc, z), 4.779477332387385e-14);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -1.1470745597729725e-11);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), 2.08767569878681e-09);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -2.755731922398589e-07);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), 2.48015873015873e-05);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -0.001388888888888889);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), 0.041666666666666664);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -0.5);
  double cs = cbm_rn_add(1.0, cbm_rn_mul(z, pc));
  switch (n & 3) {
    case 0: *c = cs; *s = sn; break;
    case 1: *c = -sn; *s = cs; break;
    case 2: *c = -cs; *s = -sn; break;
    default: *c = sn; *s = -cs; break;
  }
}

CBM_HD void cbm_cossin_turns_f32(float w, float* c, float* s) {
  float w4 = cbm_rn_mul(w, 4.0f);
  int n = (int)cbm_rn_add(w4, 0.5f);
  float th = cbm_rn_mul(cbm_rn_sub(w4, (float)n), 1.57079637f);
  float z = cbm_rn_mul(th, th);
  float ps = -2.5052108e-08f;
  ps = cbm_rn_add(cbm_rn_mul(ps, z), 2.7557319e-06f);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), -0.0001984127f);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), 0.008333334f);
  ps = cbm_rn_add(cbm_rn_mul(ps, z), -0.16666667f);
  float sn = cbm_rn_add(th, cbm_rn_mul(cbm_rn_mul(th, z), ps));
  float pc = 2.0876756e-09f;
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -2.755732e-07f);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), 2.4801588e-05f);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -0.0013888889f);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), 0.041666668f);
  pc = cbm_rn_add(cbm_rn_mul(pc, z), -0.5f);
  float cs = cbm_rn_add(1.0f, cbm_rn_mul(z, pc));
  switch (n & 3) {
    case 0: *c = cs; *s = sn; break;
    case 1: *c = -sn; *s = cs; break;
    case 2: *c = -cs; *s = -sn; break;
    default: *c = sn; *s = -cs; break;
  }
}

/* ---- Box–Muller pairs --------------------------------------------------- */
CBM_HD void cbm_box_muller_f64(double u1, double u2, double* z0, double* z1) {
  double r = cbm_rn_sqrt(cbm_rn_mul(-2.0, cbm_log_f64(cbm_rn_sub(1.0, u1))));
  double c, s;
  cbm_cossin_turns_f64(u2, &c, &s);
  *z0 = cbm_rn_mul(r, c);
  *z1 = cbm_rn_mul(r, s);
}

CBM_HD void cbm_box_muller_f32(float u1, float u2, float* z0, float* z1) {
  float r = cbm_rn_sqrt(cbm_rn_mul(-2.0f, cbm_log_f32(cbm_rn_sub(1.0f, u1))));
  float c, s;
  cbm_cossin_turns_f32(u2, &c, &s);
  *z0 = cbm_rn_mul(r, c);
  *z1 = cbm_rn_mul(r, s);
}

/* Up to 4 standard normals for one (step, agent, stream).  Double: two
 * Philox blocks (sub 0, 1), each giving one Box–Muller pair.  Float: one
 * block giving two pairs. */
CBM_HD void cbm_normals_f64(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                            uint32_t community, int count, double* out) {
  for (int k = 0; 2 * k < count; ++k) {
    cbm_u32x4 r = cbm_rng_block(seed, step, agent, stream, community, (uint32_t)k);
    double z0, z1;
    cbm_box_muller_f64(cbm_u01_f64(r.v[0], r.v[1]), cbm_u01_f64(r.v[2], r.v[3]), &z0, &z1);
    out[2 * k] = z0;
    if (2 * k + 1 < count) out[2 * k + 1] = z1;
  }
}

CBM_HD void cbm_normals_f32(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                            uint32_t community, int count, float* out) {
  cbm_u32x4 r = cbm_rng_block(seed, step, agent, stream, community, 0u);
  float z[4];
  cbm_box_muller_f32(cbm_u01_f32(r.v[0]), cbm_u01_f32(r.v[1]), &z[0], &z[1]);
  if (count > 2) cbm_box_muller_f32(cbm_u01_f32(r.v[2]), cbm_u01_f32(r.v[3]), &z[2], &z[3]);
  for (int k = 0; k < count && k < 4; ++k) out[k] = z[k];
}

CBM_HD double cbm_uniform_f64(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                              uint32_t community) {
  cbm_u32x4 r = cbm_rng_block(seed, step, agent, stream, community, 0u);
  return cbm_u01_f64(r.v[0], r.v[1]);
}

CBM_HD float cbm_uniform_f32(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                             uint32_t community) {
  cbm_u32x4 r = cbm_rng_block(seed, step, agent, stream, community, 0u);
  return cbm_u01_f32(r.v[0]);
}

/* Typed front ends used by templated code. */
CBM_HD void cbm_normals(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                        uint32_t community, int count, double* out) {
  cbm_normals_f64(seed, step, agent, stream, community, count, out);
}
CBM_HD void cbm_normals(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                        uint32_t community, int count, float* out) {
  cbm_normals_f32(seed, step, agent, stream, community, count, out);
}
template <typename T>
CBM_HD T cbm_uniform(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                     uint32_t community);
template <>
CBM_HD double cbm_uniform<double>(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                                  uint32_t community) {
  return cbm_uniform_f64(seed, step, agent, stream, community);
}
template <>
CBM_HD float cbm_uniform<float>(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                                uint32_t community) {
  return cbm_uniform_f32(seed, step, agent, stream, community);
}

#endif /* CBM_RNG_H */
