/*
 * oracle_nu.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle of the parity tests).
 *
 * Literal CPU restatement of CUBE's fluid neutrinos, in the reference's own
 * data layout: every fluid is fld(5, 1-ncb:nc+ncb, ...)^3 with halo cells,
 * component fastest, refreshed by a periodic copy (one image).
 *
 *   dfld_setup / f0          hydrodf.f90:53-84, :225-230
 *   dfld_evolve              hydrodf.f90:86-109 (NEUTRINO_IC: ai = 1/(1+z_i_nu))
 *   dfld_gravity             hydrodf.f90:111-132
 *   dfld_density             hydrodf.f90:209-222
 *   hg_setup                 hydrogr.f90:39-90 (q_EQN_OF_STATE)
 *   hg_timestep / evolve     hydrogr.f90:92-132
 *   hg_gravity (CIC, gc=1)   hydrogr.f90:136-238
 *   hg_buffer                hydrogr.f90:240-284 (one image: periodic copy)
 *   hg_density (CIC, gc=1)   hydrogr.f90:312-346
 *   h3_timestep / h3_evolve  hydro3d.f90:10-108
 *   h_evolve / h_riemann     hydro1d.f90:113-225 (HIGH_RES_X, q_EQN_OF_STATE,
 *                            no HIGH_RES_T, no P_SEMILINEAR)
 *
 * FP32 (h_fpp = REAL32) throughout, every expression evaluated left to right
 * as the Fortran source writes it; the file is compiled with
 * -ffp-contract=off so no product is fused into an add.
 */
#ifndef ORACLE_NU_H
#define ORACLE_NU_H

#include <math.h>
#include <algorithm>
#include <vector>

namespace orcnu {

// hydrodf.f90:8-28, hydro1d.f90:14-18
const float kBetaEV = 5966.34f;
const float kSol = 2.998e5f;
const float kGLv[3] = {0.41577456f, 2.29428036f, 6.28994508f};
const float kGLw[3] = {0.71109301f, 0.27851773f, 0.01038926f};
const float kCfl = 0.71f;
const float kLim = 1.5f;

struct Hydro {                 // hydrogr.f90:18-35
  int nc = 0, ncb = 0, ext = 0;
  float g = 0, cs2 = 0, dx = 0, dv = 0;
  std::vector<float> fld;      // fld(5, 1-ncb:nc+ncb, ...)^3, component fastest
  size_t at(int c, int i, int j, int k) const {  // c = 1..5, i,j,k = 1-ncb..nc+ncb
    return ((((size_t)(k - 1 + ncb) * ext + (size_t)(j - 1 + ncb)) * ext + (size_t)(i - 1 + ncb)) * 5) + (c - 1);
  }
  float& f(int c, int i, int j, int k) { return fld[at(c, i, j, k)]; }
  float f(int c, int i, int j, int k) const { return fld[at(c, i, j, k)]; }
};

struct Dfld {                  // hydrodf.f90:34-49
  float beta = 0;
  Hydro h[3];
  float dwgts[3] = {0, 0, 0};
};

inline float f0(float v) { return (v * v) / (expf(v) + 1.f); }  // hydrodf.f90:225-230

// hg_setup (hydrogr.f90:39-90), called with cs present and iso present
inline void hg_setup(Hydro& h, int nc, float g, float cs, int hg_nf, int hg_nfb, float hg_dv) {
  h.nc = nc;
  h.dx = (1.f * (float)hg_nf) / (float)nc;
  h.dv = hg_dv;
  h.ncb = std::max(2, 1 + (int)floorf((float)hg_nfb / h.dx));
  h.ext = nc + 2 * h.ncb;
  h.g = g;
  const float t = cs * h.dv;
  h.cs2 = std::max(1e-6f, t * t);
  h.fld.assign((size_t)5 * h.ext * h.ext * h.ext, 0.f);
  for (size_t q = 0; q < (size_t)h.ext * h.ext * h.ext; ++q) {
    h.fld[5 * q + 0] = 1.f;
    h.fld[5 * q + 4] = (h.cs2 * 1.f) / (h.g - 1.f);  // q_EQN_OF_STATE form
  }
}

// dfld_setup (hydrodf.f90:53-84); nc_n are the three fluid meshes
inline void dfld_setup(Dfld& d, float g, float m, const int nc_n[3], int hg_nf, int hg_nfb, float hg_dv) {
  d.beta = kBetaEV * m;
  for (int n = 0; n < 3; ++n) {
    const float v = (kGLv[n] / d.beta) * kSol;
    hg_setup(d.h[n], nc_n[n], g, v, hg_nf, hg_nfb, hg_dv);
    d.dwgts[n] = (kGLw[n] * f0(kGLv[n])) * expf(kGLv[n]);
  }
  const float s = (d.dwgts[0] + d.dwgts[1]) + d.dwgts[2];
  for (int n = 0; n < 3; ++n) d.dwgts[n] = d.dwgts[n] / s;
}

// hg_buffer (hydrogr.f90:240-284) for one image: x, then y, then z halos
inline void hg_buffer(Hydro& h) {
  const int nc = h.nc, ncb = h.ncb, lo = 1 - ncb, hi = nc + ncb;
  for (int k = lo; k <= hi; ++k)
    for (int j = lo; j <= hi; ++j)
      for (int i = 1; i <= ncb; ++i)
        for (int c = 1; c <= 5; ++c) {
          h.f(c, i - ncb, j, k) = h.f(c, nc - ncb + i, j, k);
        }
  for (int k = lo; k <= hi; ++k)
    for (int j = lo; j <= hi; ++j)
      for (int i = 1; i <= ncb; ++i)
        for (int c = 1; c <= 5; ++c) h.f(c, nc + i, j, k) = h.f(c, i, j, k);
  for (int k = lo; k <= hi; ++k)
    for (int j = 1; j <= ncb; ++j)
      for (int i = lo; i <= hi; ++i)
        for (int c = 1; c <= 5; ++c) h.f(c, i, j - ncb, k) = h.f(c, i, nc - ncb + j, k);
  for (int k = lo; k <= hi; ++k)
    for (int j = 1; j <= ncb; ++j)
      for (int i = lo; i <= hi; ++i)
        for (int c = 1; c <= 5; ++c) h.f(c, i, nc + j, k) = h.f(c, i, j, k);
  for (int k = 1; k <= ncb; ++k)
    for (int j = lo; j <= hi; ++j)
      for (int i = lo; i <= hi; ++i)
        for (int c = 1; c <= 5; ++c) h.f(c, i, j, k - ncb) = h.f(c, i, j, nc - ncb + k);
  for (int k = 1; k <= ncb; ++k)
    for (int j = lo; j <= hi; ++j)
      for (int i = lo; i <= hi; ++i)
        for (int c = 1; c <= 5; ++c) h.f(c, i, j, nc + k) = h.f(c, i, j, k);
}

// ---- hydro1d on one pencil p[5][n] (components 1..5 as rows) --------------
typedef std::vector<float> Row;

inline float sgn1(float a) { return copysignf(1.f, a); }  // Fortran sign(1.,a)

inline float minmod(float a, float b, float c) {  // hydro1d.f90:216-225
  const float sa = sgn1(a), sb = sgn1(b), sc = sgn1(c);
  return ((0.25f * fabsf(sa + sb)) * (sa + sc)) * std::min(std::min(fabsf(a), fabsf(b)), fabsf(c));
}

inline int cs_(int i, int s, int n) { return ((i + s) % n + n) % n; }  // cshift index

inline Row left_biased(const Row& u) {  // hydro1d.f90:185-198
  const int n = (int)u.size();
  Row l(n);
  for (int i = 0; i < n; ++i) {
    const float um = u[cs_(i, -1, n)], up = u[cs_(i, 1, n)];
    l[i] = u[i] + 0.5f * minmod(kLim * (u[i] - um), 0.5f * (up - um), kLim * (up - u[i]));
  }
  return l;
}

inline Row right_biased(const Row& u) {  // hydro1d.f90:200-213
  const int n = (int)u.size();
  Row r(n);
  for (int i = 0; i < n; ++i) {
    const float up = u[cs_(i, 1, n)], upp = u[cs_(i, 2, n)];
    r[i] = up - 0.5f * minmod(kLim * (up - u[i]), 0.5f * (upp - u[i]), kLim * (upp - up));
  }
  return r;
}

struct State { Row c[5]; };  // c[0..4] = components 1..5 of a pencil

inline Row kinetic(const State& h) {  // 0.5*sum(h(2:4,:)**2,1)/h(1,:)
  const int n = (int)h.c[0].size();
  Row k(n);
  for (int i = 0; i < n; ++i) {
    const float s = (h.c[1][i] * h.c[1][i] + h.c[2][i] * h.c[2][i]) + h.c[3][i] * h.c[3][i];
    k[i] = (0.5f * s) / h.c[0][i];
  }
  return k;
}

inline Row pressure(const State& h, float g) {  // max(0,(E-K)*(g-1))
  const Row k = kinetic(h);
  Row p(k.size());
  for (size_t i = 0; i < k.size(); ++i) p[i] = std::max(0.f, (h.c[4][i] - k[i]) * (g - 1.f));
  return p;
}

inline Row velocity(const State& h, int d) {  // h(d)/h(1), d = 2..4
  Row v(h.c[0].size());
  for (size_t i = 0; i < v.size(); ++i) v[i] = h.c[d - 1][i] / h.c[0][i];
  return v;
}

inline Row soundspd(const State& h, float g) {  // q_EQN_OF_STATE: sqrt(p/rho)
  const Row p = pressure(h, g);
  Row s(p.size());
  for (size_t i = 0; i < s.size(); ++i) s[i] = sqrtf(p[i] / h.c[0][i]);
  return s;
}

inline State flux(const State& h, float g) {  // hydro1d.f90:168-182
  const int n = (int)h.c[0].size();
  const Row p = pressure(h, g), v2 = velocity(h, 2), v3 = velocity(h, 3), v4 = velocity(h, 4);
  State f;
  for (int d = 0; d < 5; ++d) f.c[d].resize(n);
  for (int i = 0; i < n; ++i) {
    const float m = h.c[1][i];
    f.c[0][i] = m;
    f.c[1][i] = m * v2[i] + p[i];
    f.c[2][i] = m * v3[i];
    f.c[3][i] = m * v4[i];
    f.c[4][i] = h.c[4][i] * v2[i];  // q_EQN_OF_STATE
  }
  return f;
}

// h_riemann (hydro1d.f90:130-165): returns -f + cshift(f,-1)
inline State riemann(const State& h, float g) {
  const int n = (int)h.c[0].size();
  const Row p = pressure(h, g), v2 = velocity(h, 2), v3 = velocity(h, 3), v4 = velocity(h, 4);
  State hl, hr;
  hl.c[0] = left_biased(h.c[0]);
  hr.c[0] = right_biased(h.c[0]);
  const Row lv2 = left_biased(v2), lv3 = left_biased(v3), lv4 = left_biased(v4), lp = left_biased(p);
  const Row rv2 = right_biased(v2), rv3 = right_biased(v3), rv4 = right_biased(v4), rp = right_biased(p);
  for (int d = 1; d < 5; ++d) { hl.c[d].resize(n); hr.c[d].resize(n); }
  for (int i = 0; i < n; ++i) {
    hl.c[1][i] = hl.c[0][i] * lv2[i];
    hl.c[2][i] = hl.c[0][i] * lv3[i];
    hl.c[3][i] = hl.c[0][i] * lv4[i];
    hr.c[1][i] = hr.c[0][i] * rv2[i];
    hr.c[2][i] = hr.c[0][i] * rv3[i];
    hr.c[3][i] = hr.c[0][i] * rv4[i];
  }
  const Row kl = kinetic(hl), kr = kinetic(hr);
  for (int i = 0; i < n; ++i) {
    hl.c[4][i] = lp[i] / (g - 1.f) + kl[i];
    hr.c[4][i] = rp[i] / (g - 1.f) + kr[i];
  }
  const State fl = flux(hl, g), fr = flux(hr, g);
  const Row vl = velocity(hl, 2), vr = velocity(hr, 2), sl = soundspd(hl, g), sr = soundspd(hr, g);
  State f, out;
  for (int d = 0; d < 5; ++d) { f.c[d].resize(n); out.c[d].resize(n); }
  for (int i = 0; i < n; ++i) {
    const float ap = std::max(std::max(0.f, vl[i] + sl[i]), vr[i] + sr[i]);
    const float am = std::max(std::max(0.f, -vl[i] + sl[i]), -vr[i] + sr[i]);
    for (int d = 0; d < 5; ++d)
      f.c[d][i] = ((ap * fl.c[d][i] + am * fr.c[d][i]) - (ap * am) * (hr.c[d][i] - hl.c[d][i])) / (ap + am);
  }
  for (int d = 0; d < 5; ++d)
    for (int i = 0; i < n; ++i) out.c[d][i] = -f.c[d][i] + f.c[d][cs_(i, -1, n)];
  return out;
}

inline void h_evolve(State& h, float g, float dt, float dx) {  // hydro1d.f90:113-127
  const State r = riemann(h, g);
  const int n = (int)h.c[0].size();
  for (int d = 0; d < 5; ++d)
    for (int i = 0; i < n; ++i) h.c[d][i] = h.c[d][i] + (dt * r.c[d][i]) / dx;
}

// h3_evolve_xyz (hydro3d.f90:52-108): pencils of the whole extended array; the
// y and z sweeps swap momentum component 2 with 3 or 4 around the 1-D solver
inline void h3_evolve_xyz(Hydro& h, float dt, int xyz) {
  const int e = h.ext, lo = 1 - h.ncb, hi = h.nc + h.ncb;
  if (e <= 7) return;
  const int sw = (xyz == 1) ? 1 : (xyz == 2 ? 2 : 3);  // component index (0-based) placed in slot 1
  State p;
  for (int d = 0; d < 5; ++d) p.c[d].resize(e);
  auto pos = [xyz](int s, int a, int b, int& i, int& j, int& k) {
    if (xyz == 1) { i = s; j = a; k = b; }
    else if (xyz == 2) { i = a; j = s; k = b; }
    else { i = a; j = b; k = s; }
  };
  for (int b = lo; b <= hi; ++b)
    for (int a = lo; a <= hi; ++a) {
      int i, j, k;
      for (int s = lo; s <= hi; ++s) {
        pos(s, a, b, i, j, k);
        for (int d = 0; d < 5; ++d) {
          const int src = (d == 1) ? sw : (d == sw ? 1 : d);
          p.c[d][s - lo] = h.f(src + 1, i, j, k);
        }
      }
      h_evolve(p, h.g, dt, h.dx);
      for (int s = lo; s <= hi; ++s) {
        pos(s, a, b, i, j, k);
        for (int d = 0; d < 5; ++d) {
          const int dst = (d == 1) ? sw : (d == sw ? 1 : d);
          h.f(dst + 1, i, j, k) = p.c[d][s - lo];
        }
      }
    }
}

// h3_timestep (hydro3d.f90:10-31) with h_timestep (hydro1d.f90:98-110) per x-pencil
inline float h3_timestep(const Hydro& h) {
  const int e = h.ext, lo = 1 - h.ncb, hi = h.nc + h.ncb;
  float dt = 1e9f;
  State p;
  for (int d = 0; d < 5; ++d) p.c[d].resize(e);
  for (int k = lo; k <= hi; ++k)
    for (int j = lo; j <= hi; ++j) {
      for (int i = lo; i <= hi; ++i)
        for (int d = 0; d < 5; ++d) p.c[d][i - lo] = h.f(d + 1, i, j, k);
      float v2 = 0.f, v3 = 0.f, v4 = 0.f, smax = 0.f;
      const Row a = velocity(p, 2), b = velocity(p, 3), c = velocity(p, 4), s = soundspd(p, h.g);
      for (int i = 0; i < e; ++i) {
        v2 = (i == 0) ? fabsf(a[i]) : std::max(v2, fabsf(a[i]));
        v3 = (i == 0) ? fabsf(b[i]) : std::max(v3, fabsf(b[i]));
        v4 = (i == 0) ? fabsf(c[i]) : std::max(v4, fabsf(c[i]));
        smax = (i == 0) ? s[i] : std::max(smax, s[i]);
      }
      const float v = std::max(std::max(std::max(0.f, v2), v3), v4);
      const float dtn = (kCfl * h.dx) / (v + smax);
      dt = std::min(dt, dtn);
    }
  if (dt == 1e9f) dt = 1.f;
  return dt;
}

// hg_evolve (hydrogr.f90:110-132)
inline void hg_evolve(Hydro& h, float dt, float& dtg, int dir) {
  hg_buffer(h);
  if (dir > 0) {
    h3_evolve_xyz(h, dt, 1); h3_evolve_xyz(h, dt, 2); h3_evolve_xyz(h, dt, 3);
  } else {
    h3_evolve_xyz(h, dt, 3); h3_evolve_xyz(h, dt, 2); h3_evolve_xyz(h, dt, 1);
  }
  hg_buffer(h);
  dtg = std::min(dtg, h3_timestep(h));
}

// turn-on scale factor: with NEUTRINO_IC (hydrodf.f90:1,14-15) ai_min = ai_max,
// so min(ai_kms*cs2, ai_max) clamped below by ai_min is ai_max = 1/(1+z_i_nu)
inline float dfld_ai(float z_i_nu) { return 1.f / (1.f + z_i_nu); }

inline void dfld_evolve(Dfld& d, float dt, float& dtg, int dir, float a, float z_i_nu) {
  for (int n = 0; n < 3; ++n)
    if (a >= dfld_ai(z_i_nu)) hg_evolve(d.h[n], dt, dtg, dir);
}

// hg_density, gc=1 (hydrogr.f90:312-346)
inline float hg_density(const Hydro& h, const float x[3]) {
  int i1[3], i2[3];
  float d1[3], d2[3];
  for (int e = 0; e < 3; ++e) {
    const float xx = x[e] / h.dx - 0.5f;
    i1[e] = 1 + (int)floorf(xx);
    i2[e] = 1 + i1[e];
    d1[e] = (float)i1[e] - xx;
    d2[e] = 1.f - d1[e];
  }
  float d = h.f(1, i1[0], i1[1], i1[2]) * d1[0] * d1[1] * d1[2];
  d = d + h.f(1, i2[0], i1[1], i1[2]) * d2[0] * d1[1] * d1[2];
  d = d + h.f(1, i1[0], i2[1], i1[2]) * d1[0] * d2[1] * d1[2];
  d = d + h.f(1, i2[0], i2[1], i1[2]) * d2[0] * d2[1] * d1[2];
  d = d + h.f(1, i1[0], i1[1], i2[2]) * d1[0] * d1[1] * d2[2];
  d = d + h.f(1, i2[0], i1[1], i2[2]) * d2[0] * d1[1] * d2[2];
  d = d + h.f(1, i1[0], i2[1], i2[2]) * d1[0] * d2[1] * d2[2];
  d = d + h.f(1, i2[0], i2[1], i2[2]) * d2[0] * d2[1] * d2[2];
  return d;
}

inline float dfld_density(const Dfld& d, const float x[3]) {  // hydrodf.f90:209-222
  float den = 0.f;
  for (int n = 0; n < 3; ++n) den = den + d.dwgts[n] * hg_density(d.h[n], x);
  return den;
}

// hg_gravity, gc=1 (hydrogr.f90:136-238): acc is real(8), accr real(h_fpp)
inline void hg_gravity(Hydro& h, const float x[3], const double acc[3]) {
  const float dx3 = (h.dx * h.dx) * h.dx;
  float ar[3];
  for (int e = 0; e < 3; ++e) ar[e] = (float)(acc[e] / (double)dx3);
  int i1[3], i2[3];
  float d1[3], d2[3];
  for (int e = 0; e < 3; ++e) {
    const float xx = x[e] / h.dx - 0.5f;
    i1[e] = 1 + (int)floorf(xx);
    i2[e] = 1 + i1[e];
    d1[e] = (float)i1[e] - xx;
    d2[e] = 1.f - d1[e];
  }
  // corner order 111,211,121,221,112,212,122,222
  const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  for (int c = 0; c < 8; ++c) {
    const int i = ox[c] ? i2[0] : i1[0], j = oy[c] ? i2[1] : i1[1], k = oz[c] ? i2[2] : i1[2];
    const float dV = ((ox[c] ? d2[0] : d1[0]) * (oy[c] ? d2[1] : d1[1])) * (oz[c] ? d2[2] : d1[2]);
    const float rho = h.f(1, i, j, k);
    const float s1 = (h.f(2, i, j, k) * ar[0] + h.f(3, i, j, k) * ar[1]) + h.f(4, i, j, k) * ar[2];
    const float s2 = ((ar[0] * ar[0]) * rho + (ar[1] * ar[1]) * rho) + (ar[2] * ar[2]) * rho;
    const float dE = s1 + 0.5f * s2;
    h.f(5, i, j, k) = h.f(5, i, j, k) + dV * dE;
    for (int e = 0; e < 3; ++e) h.f(2 + e, i, j, k) = h.f(2 + e, i, j, k) + dV * (ar[e] * rho);
  }
}

inline void dfld_gravity(Dfld& d, const float x[3], const double acc[3], float a, float z_i_nu) {
  for (int n = 0; n < 3; ++n)
    if (a >= dfld_ai(z_i_nu)) hg_gravity(d.h[n], x, acc);
}

}  // namespace orcnu

#endif
