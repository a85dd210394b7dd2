/*
 * cube_codec.h -- CUBE's compressed particle codec, written once and compiled
 * identically for the host (C/C++, -ffp-contract=off) and the device (nvcc).
 *
 * Particle positions are stored as 1- or 2-byte fixed-point offsets inside the
 * coarse cell and velocities as 1- or 2-byte arctan-compressed residuals
 * relative to the coarse-cell mean velocity (CUBE_v2.0/work/main/parameters.f90:8-19,
 * :111-116).  The arithmetic below follows the reference expressions operation
 * by operation, including their mixed FP32/FP64 promotions:
 *
 *   position  pm.f90:87, update_particle.f90:68
 *       (int(xp+ishift,izipx)+rshift)*x_resolution  == (uint(xp)+0.5)*2^-(8*izipx)
 *   decode    pm.f90:145, update_particle.f90:69
 *       tan((pi*real(vp))/real(nvbin-1)) / (sqrt(pi/2)/(sigma_vi*vrel_boost))
 *       -> FP32 argument, FP32 tan, FP64 divide (vrel_boost is real(8))
 *   encode    pm.f90:154, update_particle.f90:119
 *       nint(real(nvbin-1)*atan(sqrt(pi/2)/(sigma*vrel_boost)*vreal)/pi)
 *       -> FP64 atan, Fortran NINT (ties away from zero)
 *
 * The FP32 tangent only ever sees nvbin distinct arguments, so the library
 * tabulates it once on the host with the C library's tanf (the function the
 * reference's tan(real) resolves to) and the device reads the table: decode is
 * bit-identical on host and device by construction.  The FP64 arctangent sees
 * arbitrary arguments, so it is the project function cube_atan() below,
 * evaluated with explicit fma on both sides:
 *   - reduction |x|>1 : atan(x) = pi/2 - atan(1/x)
 *   - reduction |x|>tan(pi/12) : atan(x) = pi/6 + atan((sqrt(3)x-1)/(x+sqrt(3)))
 *     (the classical argument reduction of Hart et al., "Computer
 *     Approximations", 1968, sec. 6.5)
 *   - Maclaurin series  atan(t) = sum (-1)^n t^(2n+1)/(2n+1), |t| <= 0.268,
 *     truncated after the t^29 term (remainder < 2e-18 relative).
 */
#ifndef CUBE_CODEC_H
#define CUBE_CODEC_H

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define CUBE_HD __host__ __device__ __forceinline__
#else
#define CUBE_HD static inline
#endif

/* ---- IEEE operations that must not be contracted into FMAs ---------------- */
CUBE_HD double cube_dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
CUBE_HD double cube_dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
CUBE_HD double cube_dsub(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
CUBE_HD double cube_ddiv(double a, double b) {
#if defined(__CUDA_ARCH__)
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
CUBE_HD double cube_dfma(double a, double b, double c) { return fma(a, b, c); }
CUBE_HD float cube_fmul(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fmul_rn(a, b);
#else
  return a * b;
#endif
}
CUBE_HD float cube_fadd(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fadd_rn(a, b);
#else
  return a + b;
#endif
}
CUBE_HD float cube_fsub(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fsub_rn(a, b);
#else
  return a - b;
#endif
}
CUBE_HD float cube_fdiv(float a, float b) {
#if defined(__CUDA_ARCH__)
  return __fdiv_rn(a, b);
#else
  return a / b;
#endif
}

/* Fortran NINT for doubles: nearest integer, halfway cases away from zero. */
CUBE_HD int64_t cube_nint(double x) { return (int64_t)round(x); }

/* ---- arctangent (FP64), project-written ------------------------------------ */
#define CUBE_PIO2_HI 1.5707963267948966     /* double nearest pi/2 */
#define CUBE_PIO2_LO 6.123233995736766e-17  /* pi/2 - CUBE_PIO2_HI */
#define CUBE_PIO6_HI 0.5235987755982989     /* double nearest pi/6 */
#define CUBE_PIO6_LO -5.360408832255455e-17 /* pi/6 - CUBE_PIO6_HI */
#define CUBE_SQRT3 1.7320508075688772  /* double nearest sqrt(3) */
#define CUBE_TANPIO12 0.26794919243112270 /* tan(pi/12) = 2 - sqrt(3) */

CUBE_HD double cube_atan(double x) {
  const double ax = fabs(x);
  double t = ax;
  const int recip = ax > 1.0;
  if (recip) t = cube_ddiv(1.0, ax);  /* atan(x) = pi/2 - atan(1/x) */
  const int shift = t > CUBE_TANPIO12;
  if (shift) {                         /* atan(t) = pi/6 + atan((sqrt3 t - 1)/(t + sqrt3)) */
    const double num = cube_dfma(CUBE_SQRT3, t, -1.0);
    const double den = cube_dadd(t, CUBE_SQRT3);
    t = cube_ddiv(num, den);
  }
  /* Maclaurin series, Horner form in t^2: c_n = (-1)^n/(2n+1), n = 0..14 */
  const double t2 = cube_dmul(t, t);
  double p = -1.0 / 29.0;
  p = cube_dfma(p, t2, 1.0 / 27.0);
  p = cube_dfma(p, t2, -1.0 / 25.0);
  p = cube_dfma(p, t2, 1.0 / 23.0);
  p = cube_dfma(p, t2, -1.0 / 21.0);
  p = cube_dfma(p, t2, 1.0 / 19.0);
  p = cube_dfma(p, t2, -1.0 / 17.0);
  p = cube_dfma(p, t2, 1.0 / 15.0);
  p = cube_dfma(p, t2, -1.0 / 13.0);
  p = cube_dfma(p, t2, 1.0 / 11.0);
  p = cube_dfma(p, t2, -1.0 / 9.0);
  p = cube_dfma(p, t2, 1.0 / 7.0);
  p = cube_dfma(p, t2, -1.0 / 5.0);
  p = cube_dfma(p, t2, 1.0 / 3.0);
  p = cube_dmul(p, t2);                 /* t^2 * (1/3 - t^2/5 + ...) */
  const double s = cube_dfma(-t, p, t); /* t - t^3/3 + ... */
  /* atan of the value after the reciprocal; constants split hi + lo */
  const double r = shift ? cube_dadd(CUBE_PIO6_HI, cube_dadd(s, CUBE_PIO6_LO)) : s;
  const double res = recip ? cube_dadd(cube_dsub(CUBE_PIO2_HI, r), CUBE_PIO2_LO) : r;
  return (x < 0.0) ? -res : res;
}

/* ---- codec constants -------------------------------------------------------- */
typedef struct cube_codec {
  float pi_f;          /* pi=4*atan(1.) in FP32 (parameters.f90:67) */
  float sqrt_pio2_f;   /* sqrt(pi/2) in FP32 */
  float nvbin_m1_f;    /* real(nvbin-1) */
  int32_t izipx, izipv;
  double vrel_boost;   /* 2.5, real(8) (parameters.f90:116) */
  double x_resolution; /* 2^-(8*izipx) */
} cube_codec;

/* sqrt(pi/2)/(sigma*vrel_boost), the FP64 factor shared by decode and encode */
CUBE_HD double cube_vcoef(const cube_codec* c, float sigma) {
  return cube_ddiv((double)c->sqrt_pio2_f, cube_dmul((double)sigma, c->vrel_boost));
}

/* FP32 tangent argument of a velocity code: (pi*real(vp))/real(nvbin-1) */
CUBE_HD float cube_varg(const cube_codec* c, int code) {
  return cube_fdiv(cube_fmul(c->pi_f, (float)code), c->nvbin_m1_f);
}

/* decode: tan_of_code / coef (FP64) */
CUBE_HD double cube_vdecode(float tan_of_code, double coef) {
  return cube_ddiv((double)tan_of_code, coef);
}

/* encode: nint(real(nvbin-1)*atan(coef*v)/pi); the result fits the code width
 * because |atan| < pi/2 and pi_f > pi. */
CUBE_HD int32_t cube_vencode(const cube_codec* c, double v, double coef) {
  const double at = cube_atan(cube_dmul(coef, v));
  const double q = cube_ddiv(cube_dmul((double)c->nvbin_m1_f, at), (double)c->pi_f);
  return (int32_t)cube_nint(q);
}

/* in-cell fraction of a stored position code, (uint(xp)+0.5)*x_resolution (FP64,
 * exact) */
CUBE_HD double cube_xfrac(int32_t code, int izipx) {
  const uint32_t mask = (izipx == 1) ? 0xFFu : 0xFFFFu;
  const uint32_t u = ((uint32_t)code) & mask;
  const double xres = (izipx == 1) ? (1.0 / 256.0) : (1.0 / 65536.0);
  return ((double)u + 0.5) * xres;
}

/* wrap an integer to the signed code width (Fortran integer(1)/integer(2) store) */
CUBE_HD int32_t cube_wrap_code(int64_t v, int izip) {
  if (izip == 1) return (int32_t)(int8_t)(uint8_t)(v & 0xFF);
  return (int32_t)(int16_t)(uint16_t)(v & 0xFFFF);
}

#endif /* CUBE_CODEC_H */
