/*
 * cube_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of CUBE's particle-mesh step, used as the checker of the
 * CUDA library's parity tests and as the timed CPU baseline.  Nothing in the
 * product links or calls this file.  It follows the reference Fortran
 * (CUBE_v2.0/work/main/) routine by routine, in the reference's own data layout:
 * per-tile extended arrays with ncb buffer cells, particles duplicated into the
 * buffers, the nlayer interleaved loop orders, per-tile fine meshes of nfe^3
 * with an nfb buffer and one FFT per tile.
 *
 *   spine_image        variables.f90:148-218
 *   buffer_grid/x/v    buffer_grid.f90:16-192, buffer_particle.f90:21-343
 *                      (one image, periodic: every halo cell holds a copy of the
 *                      periodic physical cell, in the same particle order)
 *   update_xp          update_particle.f90:13-259
 *   particle_mesh      pm.f90:2-451 (fine per tile, then coarse)
 *   ext_pp_force       ext_pp_force.f90:9-160
 *   kernel_f/kernel_c  kernel_f.f90:2-43, kernel_c.f90:2-134 (FP64 here)
 *   halofind           halofind.f90:18-598 (global periodic box, namespace hf)
 *
 * Precision: FP32 where the reference is FP32 (rho_f, force_f, vfield, ...),
 * FP64 where it is real(8).  The FFTs run in FP64 (FFTW single precision is
 * not available; see oracle_fft.h), which makes this an FP64-FFT oracle.
 *
 * Two choices replace reference behaviour that is not deterministic:
 *   - the velocity statistics of update_xp (update_particle.f90:174-226) are an
 *     OpenMP reduction in the reference; here the per-particle terms, in the new
 *     storage order, and the per-cell terms are each summed by a fixed pairwise
 *     tree (cube_tree_sum below), the same order the GPU uses;
 *   - the fine deposit has two modes: the reference's FP32 accumulation in its
 *     (layer,k,j,i,l) order, and a 64-bit fixed-point accumulation (weights
 *     scaled by 2^32) whose result is order-independent.
 */
#include <stdint.h>
#include <string.h>
#include <math.h>
#include <algorithm>
#include <complex>
#include <string>
#include <vector>

#include "../include/cube_gpu.h"
#include "../cube_nufluid_b200/csrc/cube_codec.h"
#include "oracle_fft.h"
#include "oracle_nu.h"

namespace {

typedef std::complex<double> cd;

struct Orc {
  cube_params P;
  int nc, nnt, nt, ncell, ncb, nte, nf, nft, nfe, nfb, nfc;
  int izipx, izipv;
  cube_codec codec;
  std::vector<float> tan_table;  // tanf of each velocity code, index code+nvbin/2
  int libm_codec = 0;            // 1: velocity codec on the C library's atan (orc_enc)
  // timing sample (CPU-baseline leg): when set, the step routines run the tile
  // loops of the marked tiles only, leave the particle state as it was, skip the
  // global coarse Poisson solve (timed apart by orc_coarse_poisson) and the
  // whole-mesh diagnostic copies
  std::vector<char> tmask;
  int nvbin;
  // compact physical state (checkpoint layout)
  int64_t np;
  std::vector<int32_t> xp, vp;  // [np][3] as wrapped codes
  std::vector<int32_t> pid;
  std::vector<int32_t> rhoc;    // [tile][nt^3]
  std::vector<float> vfield;    // [cell][3]
  // Green's functions
  std::vector<double> kern_f;   // [3][nfe][nfe][nfe/2+1] imaginary parts
  std::vector<double> kern_c;   // [3][nc][nc][nc/2+1]
  std::vector<float> fk_table, ck_table;
  // diagnostics of the last particle_mesh
  std::vector<float> rho_f_global;    // [nf^3] central regions of the tile meshes
  std::vector<uint64_t> rho_q_global; // [nf^3] fixed-point mode: node sums without the mass (scale 2^32)
  std::vector<float> force_f_global;  // [3][nf^3]
  std::vector<float> r3;              // [nc^3]
  std::vector<float> force_c;         // [3][nc^3]
  // fluid neutrinos (one species, hydrodf.f90 type dfld)
  bool nu_on = false;
  orcnu::Dfld nu;
  std::string err;
};

inline bool tile_on(const Orc& o, int tx, int ty, int tz) {
  return o.tmask.empty() || o.tmask[((size_t)tz * o.nnt + ty) * o.nnt + tx];
}

inline int64_t cell_id(const Orc& o, int tx, int ty, int tz, int lx, int ly, int lz) {
  return ((((int64_t)tz * o.nnt + ty) * o.nnt + tx) * o.nt + lz) * (int64_t)o.nt * o.nt +
         (int64_t)ly * o.nt + lx;
}

inline float tanf_code(const Orc& o, int code) { return o.tan_table[code + o.nvbin / 2]; }

/* Velocity encode nint(real(nvbin-1)*atan(sqrt(pi/2)/(sigma*vrel_boost)*vreal)/pi)
 * (pm.f90:154, update_particle.f90:119).  By default the library's own codec
 * (cube_codec.h: the project arctangent).  With libm_codec the oracle evaluates it
 * by itself with the C library's atan (what gfortran's atan(real(8)) calls) and
 * Fortran NINT (halfway cases away from zero), so the library's codec is checked
 * against an evaluation that shares none of its code. */
inline int32_t orc_enc(const Orc& o, double v, double coef) {
  if (!o.libm_codec) return cube_vencode(&o.codec, v, coef);
  const double q = ((double)o.codec.nvbin_m1_f * atan(coef * v)) / (double)o.codec.pi_f;
  return (int32_t)llround(q);
}

/* ------------------------------------------------------------------------- */
/* Extended tile view: the reference's rhoc/vfield/xp after buffer_grid +    */
/* buffer_x + buffer_v, built in closed form for one image (periodic copies). */
struct ExtTile {
  int tx, ty, tz;
  std::vector<int32_t> rho;      // rhoc(1-ncb:nt+ncb)^3, x fastest
  std::vector<float> vf;         // vfield(3, ...)
  std::vector<int64_t> idx_b_r;  // idx_b_r(1-ncb:nt+ncb,1-ncb:nt+ncb) within this tile's array
  std::vector<int64_t> src;      // compact index of each extended particle slot
  std::vector<int64_t> cstart;   // start offset of each extended cell inside src
};

void build_ext(const Orc& o, const std::vector<int64_t>& cell_start, int tx, int ty, int tz,
               ExtTile& e) {
  const int nte = o.nte, lo = 1 - o.ncb;
  e.tx = tx; e.ty = ty; e.tz = tz;
  e.rho.assign((size_t)nte * nte * nte, 0);
  e.vf.assign((size_t)3 * nte * nte * nte, 0.f);
  e.idx_b_r.assign((size_t)nte * nte, 0);
  e.cstart.assign((size_t)nte * nte * nte + 1, 0);
  e.src.clear();
  int64_t n = 0;
  for (int k = lo; k <= o.nt + o.ncb; ++k)
    for (int j = lo; j <= o.nt + o.ncb; ++j) {
      for (int i = lo; i <= o.nt + o.ncb; ++i) {
        const int gx = ((tx * o.nt + i - 1) % o.nc + o.nc) % o.nc;
        const int gy = ((ty * o.nt + j - 1) % o.nc + o.nc) % o.nc;
        const int gz = ((tz * o.nt + k - 1) % o.nc + o.nc) % o.nc;
        const int64_t c = cell_id(o, gx / o.nt, gy / o.nt, gz / o.nt, gx % o.nt, gy % o.nt, gz % o.nt);
        const size_t q = ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo);
        const int32_t cnt = o.rhoc[c];
        e.rho[q] = cnt;
        for (int d = 0; d < 3; ++d) e.vf[3 * q + d] = o.vfield[3 * c + d];
        e.cstart[q] = n;
        for (int l = 0; l < cnt; ++l) e.src.push_back(cell_start[c] + l);
        n += cnt;
      }
      e.idx_b_r[(size_t)(k - lo) * nte + (j - lo)] = n;
    }
  e.cstart[(size_t)nte * nte * nte] = n;
}

std::vector<int64_t> compact_cell_start(const Orc& o) {
  const int64_t ncells = (int64_t)o.nc * o.nc * o.nc;
  std::vector<int64_t> cs(ncells + 1, 0);
  for (int64_t c = 0; c < ncells; ++c) cs[c + 1] = cs[c] + o.rhoc[c];
  return cs;
}

/* ------------------------------------------------------------------------- */
/* Deterministic sum: fixed pairwise tree over blocks of 1024 (the GPU order). */
double cube_tree_sum(std::vector<double> a) {
  if (a.empty()) return 0.0;
  while (a.size() > 1) {
    const size_t nb = (a.size() + 1023) / 1024;
    std::vector<double> out(nb);
    for (size_t b = 0; b < nb; ++b) {
      double loc[1024];
      for (int i = 0; i < 1024; ++i) {
        const size_t q = b * 1024 + i;
        loc[i] = q < a.size() ? a[q] : 0.0;
      }
      for (int s = 512; s >= 1; s >>= 1)
        for (int i = 0; i < s; ++i) loc[i] = cube_dadd(loc[i], loc[i + s]);
      out[b] = loc[0];
    }
    a.swap(out);
  }
  return a[0];
}

/* ------------------------------------------------------------------------- */
/* update_xp (update_particle.f90:13-259)                                     */
int update_xp(Orc& o, cube_scalars* s) {
  const int nt = o.nt, ncb = o.ncb;
  const int lo2 = 1 - 2 * ncb, n2 = nt + 4 * ncb;  // rhoce(1-2ncb:nt+2ncb)
  s->dt_mid = (s->dt_old + s->dt) / 2;
  const float dt_mid = s->dt_mid;
  // nlayer=2*ceiling(dt_mid*sim%vz_max/ncell)+1 : float product, int8 division -> real
  const int nlayer = 2 * (int)ceilf(cube_fdiv(cube_fmul(dt_mid, s->vz_max), (float)o.ncell)) + 1;
  s->nlayer = nlayer;
  const double coef = cube_vcoef(&o.codec, s->sigma_vi);
  const std::vector<int64_t> cs = compact_cell_start(o);
  const int64_t ncells = (int64_t)o.nc * o.nc * o.nc;
  std::vector<int32_t> nx, nv, npid;
  std::vector<int32_t> nrho(ncells, 0);
  std::vector<float> nvf((size_t)3 * ncells, 0.f);
  nx.reserve(o.np * 3); nv.reserve(o.np * 3); npid.reserve(o.np);
  int64_t np_prev = 0;
  int rc = CUBE_OK;
  ExtTile e;
  for (int tz = 0; tz < o.nnt; ++tz)
    for (int ty = 0; ty < o.nnt; ++ty)
      for (int tx = 0; tx < o.nnt; ++tx) {
        if (!tile_on(o, tx, ty, tz)) continue;
        build_ext(o, cs, tx, ty, tz, e);
        const int nte = o.nte, lo = 1 - ncb;
        std::vector<int32_t> rhoce((size_t)n2 * n2 * n2, 0), rholocal((size_t)n2 * n2 * n2, 0);
        std::vector<float> vfn((size_t)3 * n2 * n2 * n2, 0.f);
        auto q2 = [&](int i, int j, int k) { return ((size_t)(k - lo2) * n2 + (j - lo2)) * n2 + (i - lo2); };
        // vfield_new(:,1-ncb:nt+ncb,...)=vfield*weight_v
        for (int k = lo; k <= nt + ncb; ++k)
          for (int j = lo; j <= nt + ncb; ++j)
            for (int i = lo; i <= nt + ncb; ++i) {
              const size_t qe = ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo);
              for (int d = 0; d < 3; ++d)
                vfn[3 * q2(i, j, k) + d] = (float)cube_dmul((double)e.vf[3 * qe + d], 0.1);
            }
        struct Hit { int ig[3]; double v[3]; };
        auto drift = [&](size_t qe, int i, int j, int k, int64_t ip, Hit& h) {
          const int ijk[3] = {i, j, k};
          for (int d = 0; d < 3; ++d) {
            const double xq = cube_dadd((double)ijk[d] - 1.0, cube_xfrac(o.xp[3 * ip + d], o.izipx));
            double v = cube_vdecode(tanf_code(o, o.vp[3 * ip + d]), coef);
            v = cube_dadd(v, (double)e.vf[3 * qe + d]);
            const double dx = cube_ddiv(cube_dmul((double)dt_mid, v), (double)o.ncell);
            h.ig[d] = (int)ceil(cube_dadd(xq, dx));
            h.v[d] = v;
          }
        };
        // density loop (update_particle.f90:57-80)
        for (int il = 0; il < nlayer; ++il)
          for (int k = lo + il; k <= nt + ncb; k += nlayer)
            for (int j = lo; j <= nt + ncb; ++j)
              for (int i = lo; i <= nt + ncb; ++i) {
                const size_t qe = ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo);
                for (int64_t l = 0; l < e.rho[qe]; ++l) {
                  const int64_t ip = e.src[e.cstart[qe] + l];
                  Hit h;
                  drift(qe, i, j, k, ip, h);
                  for (int d = 0; d < 3; ++d)
                    if (h.ig[d] < lo2 || h.ig[d] > nt + 2 * ncb) { o.err = "particle left the extended tile"; return CUBE_ERR_MOVE; }
                  const size_t q = q2(h.ig[0], h.ig[1], h.ig[2]);
                  rhoce[q] += 1;
                  for (int d = 0; d < 3; ++d) vfn[3 * q + d] = (float)cube_dadd((double)vfn[3 * q + d], h.v[d]);
                }
              }
        for (size_t q = 0; q < rhoce.size(); ++q)
          for (int d = 0; d < 3; ++d)
            vfn[3 * q + d] = (float)cube_ddiv((double)vfn[3 * q + d], cube_dadd((double)rhoce[q], 0.1));
        // spine_tile (variables.f90:103-146): cumulative index over (y,z) rows
        std::vector<int64_t> idx_ex_r((size_t)n2 * n2);
        int64_t nsum = 0;
        for (int k = lo2; k <= nt + 2 * ncb; ++k)
          for (int j = lo2; j <= nt + 2 * ncb; ++j) {
            for (int i = lo2; i <= nt + 2 * ncb; ++i) nsum += rhoce[q2(i, j, k)];
            idx_ex_r[(size_t)(k - lo2) * n2 + (j - lo2)] = nsum;
          }
        const int64_t ntot = nsum;
        std::vector<int32_t> xn((size_t)3 * ntot), vn((size_t)3 * ntot), pn(ntot);
        // xvnew loop (update_particle.f90:99-128)
        for (int il = 0; il < nlayer; ++il)
          for (int k = lo + il; k <= nt + ncb; k += nlayer)
            for (int j = lo; j <= nt + ncb; ++j)
              for (int i = lo; i <= nt + ncb; ++i) {
                const size_t qe = ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo);
                for (int64_t l = 0; l < e.rho[qe]; ++l) {
                  const int64_t ip = e.src[e.cstart[qe] + l];
                  Hit h;
                  drift(qe, i, j, k, ip, h);
                  const size_t q = q2(h.ig[0], h.ig[1], h.ig[2]);
                  rholocal[q] += 1;
                  int64_t right = 0;
                  for (int ii = h.ig[0]; ii <= nt + 2 * ncb; ++ii) right += rhoce[q2(ii, h.ig[1], h.ig[2])];
                  const int64_t idx = idx_ex_r[(size_t)(h.ig[2] - lo2) * n2 + (h.ig[1] - lo2)] - right + rholocal[q];
                  for (int d = 0; d < 3; ++d) {
                    const double step = cube_ddiv(cube_dmul((double)dt_mid, h.v[d]),
                                                  cube_dmul(o.codec.x_resolution, (double)o.ncell));
                    const int64_t nv_ = cube_nint(step);
                    xn[3 * (idx - 1) + d] = cube_wrap_code((int64_t)o.xp[3 * ip + d] + (int32_t)nv_, o.izipx);
                    const double vr = cube_dsub(h.v[d], (double)vfn[3 * q + d]);
                    vn[3 * (idx - 1) + d] = cube_wrap_code(orc_enc(o, vr, coef), o.izipv);
                  }
                  pn[idx - 1] = o.pid.empty() ? 0 : o.pid[ip];
                }
              }
        // keep physical particles, tile-major compact order (update_particle.f90:134-149)
        for (int k = 1; k <= nt; ++k)
          for (int j = 1; j <= nt; ++j)
            for (int i = 1; i <= nt; ++i) {
              const size_t q = q2(i, j, k);
              int64_t right = 0;
              for (int ii = i; ii <= nt + 2 * ncb; ++ii) right += rhoce[q2(ii, j, k)];
              const int64_t first = idx_ex_r[(size_t)(k - lo2) * n2 + (j - lo2)] - right;  // zero-based start
              const int64_t c = cell_id(o, tx, ty, tz, i - 1, j - 1, k - 1);
              nrho[c] = rhoce[q];
              for (int d = 0; d < 3; ++d) nvf[3 * c + d] = vfn[3 * q + d];
              for (int64_t l = 0; l < rhoce[q]; ++l) {
                for (int d = 0; d < 3; ++d) {
                  nx.push_back(xn[3 * (first + l) + d]);
                  nv.push_back(vn[3 * (first + l) + d]);
                }
                npid.push_back(pn[first + l]);
              }
              np_prev += rhoce[q];
            }
      }
  if (!o.tmask.empty()) return rc;  // timing sample: the state stays as it was
  o.xp.swap(nx); o.vp.swap(nv);
  if (!o.pid.empty()) o.pid.swap(npid);
  o.rhoc.swap(nrho); o.vfield.swap(nvf);
  o.np = np_prev;
  s->nplocal = np_prev;
  // velocity statistics (update_particle.f90:171-226) in the fixed order: the
  // per-cell |vfield|^2 and the per-particle |v_res|^2, |v|^2 in the new storage
  // order, each list summed by the fixed pairwise tree
  std::vector<int64_t> cs2 = compact_cell_start(o);
  std::vector<double> sc(ncells), sr(o.np), ss(o.np);
  for (int64_t c = 0; c < ncells; ++c) {
    const float* vf = &o.vfield[3 * c];
    float f2 = cube_fadd(cube_fadd(cube_fmul(vf[0], vf[0]), cube_fmul(vf[1], vf[1])), cube_fmul(vf[2], vf[2]));
    sc[c] = (double)f2;
    for (int64_t ip = cs2[c]; ip < cs2[c + 1]; ++ip) {
      double v[3], w[3];
      for (int d = 0; d < 3; ++d) {
        v[d] = cube_vdecode(tanf_code(o, o.vp[3 * ip + d]), coef);
        w[d] = cube_dadd(v[d], (double)vf[d]);
      }
      sr[ip] = cube_dadd(cube_dadd(cube_dmul(v[0], v[0]), cube_dmul(v[1], v[1])), cube_dmul(v[2], v[2]));
      ss[ip] = cube_dadd(cube_dadd(cube_dmul(w[0], w[0]), cube_dmul(w[1], w[1])), cube_dmul(w[2], w[2]));
    }
  }
  const double sum_c = cube_tree_sum(sc), sum_r = cube_tree_sum(sr), sum_s = cube_tree_sum(ss);
  const double npg = (double)(s->npglobal > 0 ? s->npglobal : o.np);
  s->std_vsim = sqrt(sum_s / npg);
  s->std_vsim_c = sqrt(sum_c / (double)ncells);
  s->std_vsim_res = sqrt(sum_r / npg);
  s->sigma_vi_new = (float)(s->std_vsim_res / (double)sqrtf(3.f));
  return rc;
}

/* ------------------------------------------------------------------------- */
/* kernel_f (kernel_f.f90:14-37) on the nfe grid, FP64                        */
void kernel_f(Orc& o) {
  const int nfe = o.nfe, nfc = o.nfc, nh = nfe / 2 + 1;
  o.kern_f.assign((size_t)3 * nfe * nfe * nh, 0.0);
  std::vector<double> r((size_t)nfe * nfe * nfe);
  std::vector<cd> h;
  for (int d = 0; d < 3; ++d) {
    std::fill(r.begin(), r.end(), 0.0);
    auto at = [&](int i, int j, int k) -> double& { return r[((size_t)(k - 1) * nfe + (j - 1)) * nfe + (i - 1)]; };
    for (int k = 1; k <= nfc; ++k)
      for (int j = 1; j <= nfc; ++j)
        for (int i = 1; i <= nfc; ++i)
          at(i, j, k) = (double)o.fk_table[(((size_t)d * nfc + (k - 1)) * nfc + (j - 1)) * nfc + (i - 1)];
    if (o.P.ext_pp_force)
      for (int k = 1; k <= o.P.pp_range + 1; ++k)
        for (int j = 1; j <= o.P.pp_range + 1; ++j)
          for (int i = 1; i <= o.P.pp_range + 1; ++i) at(i, j, k) = 0;
    const double mf[3] = {d == 0 ? -1.0 : 1.0, d == 1 ? -1.0 : 1.0, d == 2 ? -1.0 : 1.0};
    for (int k = 1; k <= nfe; ++k)
      for (int j = 1; j <= nfe; ++j)
        for (int m = 0; m < nfc - 1; ++m) at(nfe - nfc + 2 + m, j, k) = mf[0] * at(nfc - m, j, k);
    for (int k = 1; k <= nfe; ++k)
      for (int m = 0; m < nfc - 1; ++m)
        for (int i = 1; i <= nfe; ++i) at(i, nfe - nfc + 2 + m, k) = mf[1] * at(i, nfc - m, k);
    for (int m = 0; m < nfc - 1; ++m)
      for (int j = 1; j <= nfe; ++j)
        for (int i = 1; i <= nfe; ++i) at(i, j, nfe - nfc + 2 + m) = mf[2] * at(i, j, nfc - m);
    orc::rfft3_forward(r.data(), h, nfe);
    for (size_t q = 0; q < h.size(); ++q) o.kern_f[(size_t)d * h.size() + q] = h[q].imag();
  }
}

/* kernel_c (kernel_c.f90:1-134) with LRCKCORR, one image, FP64 */
void kernel_c(Orc& o) {
  const int nc = o.nc, nh = nc / 2 + 1, ncell = o.ncell;
  const double pi = 3.14159265358979323846;
  std::vector<double> ck((size_t)3 * nc * nc * nc), direct((size_t)3 * nc * nc * nc);
  auto ckat = [&](std::vector<double>& a, int d, int i, int j, int k) -> double& {
    return a[(((size_t)d * nc + (k - 1)) * nc + (j - 1)) * nc + (i - 1)];
  };
  for (int k = 1; k <= nc; ++k)
    for (int j = 1; j <= nc; ++j)
      for (int i = 1; i <= nc; ++i) {
        const int g[3] = {i, j, k};
        double rx[3];
        for (int d = 0; d < 3; ++d) rx[d] = (double)ncell * (double)(((g[d] + nc / 2 - 1) % nc) - nc / 2);
        const double r = sqrt(rx[0] * rx[0] + rx[1] * rx[1] + rx[2] * rx[2]);
        for (int d = 0; d < 3; ++d) {
          const double v = (r == 0) ? 0.0 : -rx[d] / (r * r * r);
          ckat(ck, d, i, j, k) = v;
          ckat(direct, d, i, j, k) = v;
        }
      }
  // ck_table(3,4,4,4): component fastest
  auto tab = [&](int d, int i, int j, int k) -> double {
    return (double)o.ck_table[(((size_t)(k - 1) * 4 + (j - 1)) * 4 + (i - 1)) * 3 + d];
  };
  // octants (kernel_c.f90:43-72): each dimension is either offsets 0..3 (index 1..4)
  // or offsets -3..-1 (index nc-2..nc, from table index 4..2), odd in the component's own dimension
  for (int oct = 0; oct < 8; ++oct) {
    const bool fx = oct & 1, fy = oct & 2, fz = oct & 4;
    for (int k = 1; k <= (fz ? 3 : 4); ++k)
      for (int j = 1; j <= (fy ? 3 : 4); ++j)
        for (int i = 1; i <= (fx ? 3 : 4); ++i) {
          const int ti = fx ? 5 - i : i, tj = fy ? 5 - j : j, tk = fz ? 5 - k : k;  // 4:2:-1 -> 4,3,2
          const int ci = fx ? nc - 3 + i : i, cj = fy ? nc - 3 + j : j, ck_ = fz ? nc - 3 + k : k;
          for (int d = 0; d < 3; ++d) {
            double sgn = 1.0;
            if ((d == 0 && fx) || (d == 1 && fy) || (d == 2 && fz)) sgn = -1.0;
            ckat(ck, d, ci, cj, ck_) = sgn * tab(d, ti, tj, tk);
          }
        }
  }
  o.kern_c.assign((size_t)3 * nc * nc * nh, 0.0);
  std::vector<cd> hc, hd;
  for (int d = 0; d < 3; ++d) {
    orc::rfft3_forward(&ck[(size_t)d * nc * nc * nc], hc, nc);
    orc::rfft3_forward(&direct[(size_t)d * nc * nc * nc], hd, nc);
    for (int k = 0; k < nc; ++k)
      for (int j = 0; j < nc; ++j)
        for (int i = 0; i < nh; ++i) {
          const size_t q = ((size_t)k * nc + j) * nh + i;
          const int kg = k + 1, jg = j + 1, ig = i + 1;
          const int kx[3] = {((ig + nc / 2 - 1) % nc) - nc / 2, ((jg + nc / 2 - 1) % nc) - nc / 2,
                             ((kg + nc / 2 - 1) % nc) - nc / 2};
          const double kr = sqrt((double)kx[0] * kx[0] + (double)kx[1] * kx[1] + (double)kx[2] * kx[2]);
          double ks[3], ks2 = 0;
          for (int e = 0; e < 3; ++e) { ks[e] = 2 * sin(pi * kx[e] / (double)nc); ks2 += ks[e] * ks[e]; }
          double v = hc[q].imag();
          // the component is odd in its own dimension: zero on the Nyquist plane
          // (FP64 round-off there would otherwise enter the |k|<=8 rescaling when nc=16)
          if (kx[d] == -nc / 2) v = 0.0;
          else if (!(kr > 8.0 || kx[d] == 0))
            v = v * 0.25 * pi * ks[d] / ks2 / hd[q].imag();
          o.kern_c[(size_t)d * nc * nc * nh + q] = v;
        }
  }
}

/* ------------------------------------------------------------------------- */
/* particle_mesh (pm.f90:2-451); neutrino terms enter through the fluid module */
/* dt constraints (pm.f90:427-443), FP32 like the reference */
void dt_constraints(const Orc& o, cube_scalars* s) {
  const float pi_f = o.codec.pi_f;
  const float GG = cube_fdiv(cube_fdiv(1.0f, 6.0f), pi_f);  /* variables.f90:22 */
  float v = cube_fdiv(1.5f, s->a);
  v = cube_fmul(v, o.P.box);
  v = cube_fmul(v, o.P.h0);
  v = cube_fmul(v, 100.f);
  v = cube_fmul(v, sqrtf(o.P.omega_m));
  s->vsim2phys = cube_fdiv(v, (float)o.nf);
  s->dt_fine = sqrtf(cube_fdiv(1.0f, cube_fmul(cube_fmul(sqrtf(s->f2_max_fine), s->a_mid), GG)));
  s->dt_coarse = sqrtf(cube_fdiv((float)o.ncell, cube_fmul(cube_fmul(sqrtf(s->f2_max_coarse), s->a_mid), GG)));
  const float vm = std::max(s->vmax[0], std::max(s->vmax[1], s->vmax[2]));
  s->dt_vmax = cube_fdiv(cube_fmul(o.P.vbuf, 20.f), vm);
  s->vz_max = s->vmax[2];
  // vmax_nu is zeroed at pm.f90:40 and never raised by the fluid: dt_vmax_nu = +Inf
  if (o.nu_on) s->dt_vmax_nu = cube_fdiv(cube_fmul(o.P.vbuf, 20.f), 0.f);
}

struct KickIn {
  const std::vector<float>* fine_force;    // optional external [3][nf^3]
  const std::vector<float>* coarse_force;  // optional external [3][nc^3]
};

int particle_mesh(Orc& o, cube_scalars* s, int deposit_mode, const KickIn* ext) {
  const int nt = o.nt, ncb = o.ncb, ncell = o.ncell, nfe = o.nfe, nfb = o.nfb, nft = o.nft;
  const int nh = nfe / 2 + 1, nf = o.nf, nc = o.nc;
  const float mass = s->mass_p_cdm;
  const float a_mid = s->a_mid, dt = s->dt;
  const float pi_f = o.codec.pi_f;
  double vmax[3] = {0, 0, 0};
  float f2_max_fine = 0.f;
  double testrhof = 0, testrhoc = 0;
  const std::vector<int64_t> cs = compact_cell_start(o);
  const bool sample = !o.tmask.empty();
  if (!sample) o.rho_f_global.assign((size_t)nf * nf * nf, 0.f);
  if (deposit_mode == 1) o.rho_q_global.assign((size_t)nf * nf * nf, 0);
  const double unit_f = (double)mass * (1.0 / 4294967296.0);  // exact
  if (!sample) o.force_f_global.assign((size_t)3 * nf * nf * nf, 0.f);
  const double coef_old = cube_vcoef(&o.codec, s->sigma_vi);
  const double coef_new = cube_vcoef(&o.codec, s->sigma_vi_new);
  std::vector<float> rho_f((size_t)nfe * nfe * nfe);
  std::vector<int64_t> rho_q;
  std::vector<float> force_f((size_t)3 * (nft + 2) * (nft + 2) * (nft + 2));
  std::vector<cd> spec, prod;
  std::vector<double> rr((size_t)nfe * nfe * nfe);
  ExtTile e;
  const int lo = 1 - ncb, nte = o.nte;
  auto ptempx = [&](int ijk, int32_t code) -> float {  // ncell*(i-1)+ncell*frac, FP64 -> real
    return (float)cube_dadd((double)ncell * (double)(ijk - 1), cube_dmul((double)ncell, cube_xfrac(code, o.izipx)));
  };
  for (int tz = 0; tz < o.nnt; ++tz)
    for (int ty = 0; ty < o.nnt; ++ty)
      for (int tx = 0; tx < o.nnt; ++tx) {
        if (!tile_on(o, tx, ty, tz)) continue;
        build_ext(o, cs, tx, ty, tz, e);
        auto eq = [&](int i, int j, int k) { return ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo); };
        std::fill(rho_f.begin(), rho_f.end(), 0.f);
        if (deposit_mode == 1) rho_q.assign(rho_f.size(), 0);
        auto fat = [&](int i, int j, int k) -> size_t { return ((size_t)(k - 1) * nfe + (j - 1)) * nfe + (i - 1); };
        // neutrino density into the fine mesh (pm.f90:55-74), before the particles
        std::vector<float> nu_t;
        if (o.nu_on) {
          nu_t.assign(rho_f.size(), 0.f);
          if (1.f / a_mid - 1.f > o.P.z_i_nu) {
            for (size_t q = 0; q < nu_t.size(); ++q) nu_t[q] = 0.f + o.P.f_neu;
          } else {
#pragma omp parallel for schedule(static)
            for (int k = 1; k <= nfe; ++k)
              for (int j = 1; j <= nfe; ++j)
                for (int i = 1; i <= nfe; ++i) {
                  const float x[3] = {(float)(tx * nt * ncell + i - nfb) - 0.5f, (float)(ty * nt * ncell + j - nfb) - 0.5f,
                                      (float)(tz * nt * ncell + k - nfb) - 0.5f};
                  nu_t[fat(i, j, k)] = 0.f + orcnu::dfld_density(o.nu, x) * o.P.f_neu;
                }
          }
          if (deposit_mode == 0) rho_f = nu_t;
        }
        // fine_cic_mass (pm.f90:76-107): three layers of k-planes, each layer's planes
        // are CIC-disjoint, so the threads of a layer never touch the same node
        for (int il = 0; il < 3; ++il)
#pragma omp parallel for schedule(static, 2)
          for (int k = 2 - ncb + il; k <= nt + ncb - 1; k += 3)
            for (int j = 2 - ncb; j <= nt + ncb - 1; ++j)
              for (int i = 2 - ncb; i <= nt + ncb - 1; ++i) {
                const size_t qe = eq(i, j, k);
                for (int64_t l = 0; l < e.rho[qe]; ++l) {
                  const int64_t ip = e.src[e.cstart[qe] + l];
                  const int ijk[3] = {i, j, k};
                  int i1[3], i2[3];
                  float dx1[3], dx2[3];
                  for (int d = 0; d < 3; ++d) {
                    const float tx_ = ptempx(ijk[d], o.xp[3 * ip + d]);
                    const int f = (int)floorf(tx_) + 1;
                    dx1[d] = cube_fsub((float)f, tx_);
                    dx2[d] = cube_fsub(1.f, dx1[d]);
                    i1[d] = f + nfb; i2[d] = f + 1 + nfb;
                  }
                  const int cx[8][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,1},{0,1,1},{1,0,1},{1,1,0},{1,1,1}};
                  for (int c8 = 0; c8 < 8; ++c8) {
                    const float wx = cx[c8][0] ? dx2[0] : dx1[0];
                    const float wy = cx[c8][1] ? dx2[1] : dx1[1];
                    const float wz = cx[c8][2] ? dx2[2] : dx1[2];
                    const size_t q = fat(cx[c8][0] ? i2[0] : i1[0], cx[c8][1] ? i2[1] : i1[1], cx[c8][2] ? i2[2] : i1[2]);
                    // fixed point: the weight without the mass, q = RN(w 2^32); the
                    // mass is applied once per node
                    if (deposit_mode == 1)
                      rho_q[q] += (int64_t)llrint((double)cube_fmul(cube_fmul(wx, wy), wz) * 4294967296.0);
                    else rho_f[q] = cube_fadd(rho_f[q], cube_fmul(cube_fmul(cube_fmul(wx, wy), wz), mass));
                  }
                }
              }
        if (deposit_mode == 1)
          for (size_t q = 0; q < rho_f.size(); ++q) {
            rho_f[q] = (float)((double)rho_q[q] * unit_f);
            if (o.nu_on) rho_f[q] = cube_fadd(rho_f[q], nu_t[q]);
          }
        for (int k = nfb + 1; k <= nft + nfb; ++k)
          for (int j = nfb + 1; j <= nft + nfb; ++j)
            for (int i = nfb + 1; i <= nft + nfb; ++i) {
              testrhof += (double)rho_f[fat(i, j, k)];
              const size_t g = ((size_t)(tz * nft + k - nfb - 1) * nf + (ty * nft + j - nfb - 1)) * nf + (tx * nft + i - nfb - 1);
              if (!sample) o.rho_f_global[g] = rho_f[fat(i, j, k)];
              if (deposit_mode == 1) o.rho_q_global[g] = (uint64_t)rho_q[fat(i, j, k)];
            }
        // fine force (pm.f90:112-126)
        const int nfo = nft + 2;  // force_f(3, nfb:nfe-nfb+1)
        if (ext && ext->fine_force) {
          for (int k = 0; k < nfo; ++k)
            for (int j = 0; j < nfo; ++j)
              for (int i = 0; i < nfo; ++i) {
                const int gx = ((tx * nft + i - 1) % nf + nf) % nf, gy = ((ty * nft + j - 1) % nf + nf) % nf,
                          gz = ((tz * nft + k - 1) % nf + nf) % nf;
                for (int d = 0; d < 3; ++d)
                  force_f[(((size_t)k * nfo + j) * nfo + i) * 3 + d] =
                      (*ext->fine_force)[(size_t)d * nf * nf * nf + ((size_t)gz * nf + gy) * nf + gx];
              }
        } else {
          for (size_t q = 0; q < rr.size(); ++q) rr[q] = (double)rho_f[q];
          orc::rfft3_forward(rr.data(), spec, nfe);
          prod.resize(spec.size());
          for (int d = 0; d < 3; ++d) {
            for (size_t q = 0; q < spec.size(); ++q) {
              const double kv = o.kern_f[(size_t)d * spec.size() + q];
              prod[q] = cd(-spec[q].imag() * kv, spec[q].real() * kv);
            }
            orc::rfft3_backward(prod, rr.data(), nfe);
            const double norm = (double)nfe * nfe * nfe;
            for (int k = 0; k < nfo; ++k)
              for (int j = 0; j < nfo; ++j)
                for (int i = 0; i < nfo; ++i)
                  force_f[(((size_t)k * nfo + j) * nfo + i) * 3 + d] =
                      (float)(rr[fat(nfb + i, nfb + j, nfb + k)] / norm);
          }
          (void)nh;
        }
        for (int k = 0; k < nfo; ++k)
          for (int j = 0; j < nfo; ++j)
            for (int i = 0; i < nfo; ++i) {
              const float* f = &force_f[(((size_t)k * nfo + j) * nfo + i) * 3];
              const float f2 = cube_fadd(cube_fadd(cube_fmul(f[0], f[0]), cube_fmul(f[1], f[1])), cube_fmul(f[2], f[2]));
              f2_max_fine = std::max(f2_max_fine, f2);
              if (!sample && i >= 1 && i <= nft && j >= 1 && j <= nft && k >= 1 && k <= nft) {
                const size_t g = ((size_t)(tz * nft + k - 1) * nf + (ty * nft + j - 1)) * nf + (tx * nft + i - 1);
                for (int d = 0; d < 3; ++d) o.force_f_global[(size_t)d * nf * nf * nf + g] = f[d];
              }
            }
        // fine velocity (pm.f90:131-155)
        const float kfac_a = a_mid, kfac_dt = dt;
#pragma omp parallel for schedule(static, 2)
        for (int k = 1; k <= nt; ++k)
          for (int j = 1; j <= nt; ++j)
            for (int i = 1; i <= nt; ++i) {
              const size_t qe = eq(i, j, k);
              for (int64_t l = 0; l < e.rho[qe]; ++l) {
                const int64_t ip = e.src[e.cstart[qe] + l];
                const int ijk[3] = {i, j, k};
                int i1[3];
                float dx1[3], dx2[3];
                for (int d = 0; d < 3; ++d) {
                  const float tx_ = ptempx(ijk[d], o.xp[3 * ip + d]);
                  const int f = (int)floorf(tx_) + 1;
                  dx1[d] = cube_fsub((float)f, tx_);
                  dx2[d] = cube_fsub(1.f, dx1[d]);
                  i1[d] = f + nfb;  // index into force_f(nfb:...) -> offset i1-nfb
                }
                const int cx[8][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,1},{0,1,1},{1,0,1},{1,1,0},{1,1,1}};
                for (int d = 0; d < 3; ++d) {
                  double v = cube_vdecode(tanf_code(o, o.vp[3 * ip + d]), coef_old);
                  for (int c8 = 0; c8 < 8; ++c8) {
                    const int fi = i1[0] + cx[c8][0] - nfb, fj = i1[1] + cx[c8][1] - nfb, fk = i1[2] + cx[c8][2] - nfb;
                    const float fv = force_f[(((size_t)fk * nfo + fj) * nfo + fi) * 3 + d];
                    float t = cube_fmul(fv, kfac_a);
                    t = cube_fmul(t, kfac_dt);
                    t = cube_fdiv(t, 6.f);
                    t = cube_fdiv(t, pi_f);
                    t = cube_fmul(t, cx[c8][0] ? dx2[0] : dx1[0]);
                    t = cube_fmul(t, cx[c8][1] ? dx2[1] : dx1[1]);
                    t = cube_fmul(t, cx[c8][2] ? dx2[2] : dx1[2]);
                    v = cube_dadd(v, (double)t);
                  }
                  o.vp[3 * ip + d] = cube_wrap_code(orc_enc(o, v, coef_new), o.izipv);
                }
              }
            }
        // neutrino gravity from the fine force (pm.f90:157-171), sequential in the
        // reference's (k,j,i,kk,jj,ii) order: the scatter is order-dependent
        if (o.nu_on)
          for (int k = 1; k <= nt; ++k)
            for (int j = 1; j <= nt; ++j)
              for (int i = 1; i <= nt; ++i)
                for (int kk = 1; kk <= ncell; ++kk)
                  for (int jj = 1; jj <= ncell; ++jj)
                    for (int ii = 1; ii <= ncell; ++ii) {
                      const int m[3] = {ncell * (i - 1) + ii, ncell * (j - 1) + jj, ncell * (k - 1) + kk};
                      // idx1 = floor(tempx)+1+nfb -> force_f offset m+1 from rho index nfb
                      const float* f = &force_f[(((size_t)(m[2] + 1) * nfo + (m[1] + 1)) * nfo + (m[0] + 1)) * 3];
                      double acc[3];
                      for (int d = 0; d < 3; ++d)
                        acc[d] = (double)cube_fdiv(cube_fdiv(cube_fmul(cube_fmul(f[d], a_mid), dt), 6.f), pi_f);
                      const int tt[3] = {tx, ty, tz};
                      float x[3];
                      for (int d = 0; d < 3; ++d) x[d] = (float)(tt[d] * nt * ncell + m[d]) - 0.5f;
                      orcnu::dfld_gravity(o.nu, x, acc, a_mid, o.P.z_i_nu);
                    }
      }
  s->f2_max_fine = f2_max_fine;
  s->sigma_vi = s->sigma_vi_new;
  // coarse_cic_mass (pm.f90:192-278)
  o.r3.assign((size_t)nc * nc * nc, 0.f);
  std::vector<uint64_t> r3nu;  // fixed-point mode: coarse neutrino sums (mass units, 2^32)
  if (deposit_mode == 1) r3nu.assign((size_t)nc * nc * nc, 0);
  for (int tz = 0; tz < o.nnt; ++tz)
    for (int ty = 0; ty < o.nnt; ++ty)
      for (int tx = 0; tx < o.nnt; ++tx) {
        if (!tile_on(o, tx, ty, tz)) continue;
        build_ext(o, cs, tx, ty, tz, e);
        auto eq = [&](int i, int j, int k) { return ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo); };
        const int n3 = nt + 4;  // r3t(-1:nt+2)
        std::vector<float> r3t((size_t)n3 * n3 * n3, 0.f);
        std::vector<int64_t> r3q;
        if (deposit_mode == 1) r3q.assign(r3t.size(), 0);
        auto tat = [&](int i, int j, int k) { return ((size_t)(k + 1) * n3 + (j + 1)) * n3 + (i + 1); };
        // neutrino density into the coarse mesh (pm.f90:198-242), buffer cells included
        auto r3add = [&](size_t q, float w) {
          if (deposit_mode == 1) r3q[q] += (int64_t)llrint((double)w * 4294967296.0);
          else r3t[q] = cube_fadd(r3t[q], w);
        };
        if (o.nu_on) {
          if (1.f / a_mid - 1.f > o.P.z_i_nu) {
            const float hom = o.P.f_neu * (float)(ncell * ncell * ncell);
            for (size_t q = 0; q < r3t.size(); ++q) r3add(q, hom);
          } else {
            for (int k = 0; k <= nt + 1; ++k)
              for (int j = 0; j <= nt + 1; ++j)
                for (int i = 0; i <= nt + 1; ++i)
                  for (int kk = 1; kk <= ncell; ++kk)
                    for (int jj = 1; jj <= ncell; ++jj)
                      for (int ii = 1; ii <= ncell; ++ii) {
                        const int ijk[3] = {i, j, k}, sub[3] = {ii, jj, kk}, tt[3] = {tx, ty, tz};
                        float x[3], c1[3], c2[3];
                        int i1[3];
                        for (int d = 0; d < 3; ++d) {
                          x[d] = (float)(tt[d] * nt * ncell + (ijk[d] - 1) * ncell + sub[d]) - 0.5f;
                          float xc = ((float)((ijk[d] - 1) * ncell + sub[d]) - 0.5f) / (float)ncell;
                          xc = xc - 0.5f;
                          i1[d] = 1 + (int)floorf(xc);
                          c1[d] = (float)i1[d] - xc;
                          c2[d] = 1.f - c1[d];
                        }
                        const float rho_nu = orcnu::dfld_density(o.nu, x) * o.P.f_neu;
                        const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1},
                                  oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                        for (int c8 = 0; c8 < 8; ++c8) {
                          const float w = cube_fmul(cube_fmul(cube_fmul(rho_nu, ox[c8] ? c2[0] : c1[0]), oy[c8] ? c2[1] : c1[1]),
                                                    oz[c8] ? c2[2] : c1[2]);
                          r3add(tat(i1[0] + ox[c8], i1[1] + oy[c8], i1[2] + oz[c8]), w);
                        }
                      }
          }
        }
        // reference order (mode 0) only: the fixed-point mode restricts the fine sums below
        for (int il = 0; il < 3 && deposit_mode == 0; ++il)
#pragma omp parallel for schedule(static, 2)
          for (int k = 0 + il; k <= nt + 1; k += 3)
            for (int j = 0; j <= nt + 1; ++j)
              for (int i = 0; i <= nt + 1; ++i) {
                const size_t qe = eq(i, j, k);
                for (int64_t l = 0; l < e.rho[qe]; ++l) {
                  const int64_t ip = e.src[e.cstart[qe] + l];
                  const int ijk[3] = {i, j, k};
                  int i1[3];
                  float dx1[3], dx2[3];
                  for (int d = 0; d < 3; ++d) {
                    const float t_ = (float)cube_dsub(cube_dadd((double)(ijk[d] - 1), cube_xfrac(o.xp[3 * ip + d], o.izipx)), 0.5);
                    i1[d] = (int)floorf(t_) + 1;
                    dx1[d] = cube_fsub((float)i1[d], t_);
                    dx2[d] = cube_fsub(1.f, dx1[d]);
                  }
                  const int cx[8][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,1},{0,1,1},{1,0,1},{1,1,0},{1,1,1}};
                  for (int c8 = 0; c8 < 8; ++c8) {
                    const float wx = cx[c8][0] ? dx2[0] : dx1[0];
                    const float wy = cx[c8][1] ? dx2[1] : dx1[1];
                    const float wz = cx[c8][2] ? dx2[2] : dx1[2];
                    const float w = cube_fmul(cube_fmul(cube_fmul(wx, wy), wz), mass);
                    const size_t q = tat(i1[0] + cx[c8][0], i1[1] + cx[c8][1], i1[2] + cx[c8][2]);
                    r3t[q] = cube_fadd(r3t[q], w);
                  }
                }
              }
        for (int k = 1; k <= nt; ++k)
          for (int j = 1; j <= nt; ++j)
            for (int i = 1; i <= nt; ++i) {
              const size_t g = ((size_t)(tz * nt + k - 1) * nc + (ty * nt + j - 1)) * nc + (tx * nt + i - 1);
              if (deposit_mode == 1) r3nu[g] = (uint64_t)r3q[tat(i, j, k)];  // neutrinos only
              else o.r3[g] = r3t[tat(i, j, k)];
            }
      }
  if (deposit_mode == 1) {
    // the coarse CIC of the particles is the fine node sums restricted with the
    // weights (4 - |d|)/4, |d| <= 3, per dimension (coarse node J is centred on fine
    // node 4J+2), exact in 64-bit integers at scale 2^38; the neutrinos' coarse
    // sums (mass units, scale 2^32) are added when the node is written
    const double unit_c = (double)mass * (1.0 / (64.0 * 4294967296.0));  // exact
#pragma omp parallel for schedule(static)
    for (int J2 = 0; J2 < nc; ++J2)
      for (int J1 = 0; J1 < nc; ++J1)
        for (int J0 = 0; J0 < nc; ++J0) {
          uint64_t acc = 0;
          for (int d2 = -3; d2 <= 3; ++d2) {
            const int n2 = ((4 * J2 + 2 + d2) % nf + nf) % nf;
            for (int d1 = -3; d1 <= 3; ++d1) {
              const int n1 = ((4 * J1 + 2 + d1) % nf + nf) % nf;
              for (int d0 = -3; d0 <= 3; ++d0) {
                const int n0 = ((4 * J0 + 2 + d0) % nf + nf) % nf;
                const uint64_t t = (uint64_t)((4 - std::abs(d0)) * (4 - std::abs(d1)) * (4 - std::abs(d2)));
                acc += t * o.rho_q_global[((size_t)n2 * nf + n1) * nf + n0];
              }
            }
          }
          const size_t g = ((size_t)J2 * nc + J1) * nc + J0;
          o.r3[g] = (float)((double)acc * unit_c + (double)r3nu[g] * (1.0 / 4294967296.0));
        }
  }
  for (size_t q = 0; q < o.r3.size(); ++q) testrhoc += (double)o.r3[q];
  // coarse force (pm.f90:288-300), pencil_fft on one image = 3-D r2c/c2r
  o.force_c.assign((size_t)3 * nc * nc * nc, 0.f);
  if (ext && ext->coarse_force) {
    o.force_c = *ext->coarse_force;
  } else if (!sample) {
    std::vector<double> r((size_t)nc * nc * nc);
    for (size_t q = 0; q < r.size(); ++q) r[q] = (double)o.r3[q];
    std::vector<cd> sp, pr;
    orc::rfft3_forward(r.data(), sp, nc);
    pr.resize(sp.size());
    for (int d = 0; d < 3; ++d) {
      for (size_t q = 0; q < sp.size(); ++q) {
        const double kv = o.kern_c[(size_t)d * sp.size() + q];
        pr[q] = cd(-sp[q].imag() * kv, sp[q].real() * kv);
      }
      orc::rfft3_backward(pr, r.data(), nc);
      const double norm = (double)nc * nc * nc;
      for (size_t q = 0; q < r.size(); ++q) o.force_c[(size_t)d * r.size() + q] = (float)(r[q] / norm);
    }
  }
  float f2c = 0.f;
  for (size_t q = 0; q < (size_t)nc * nc * nc; ++q) {
    const float a = o.force_c[q], b = o.force_c[(size_t)nc * nc * nc + q], c = o.force_c[(size_t)2 * nc * nc * nc + q];
    f2c = std::max(f2c, cube_fadd(cube_fadd(cube_fmul(a, a), cube_fmul(b, b)), cube_fmul(c, c)));
  }
  s->f2_max_coarse = f2c;
  // coarse velocity (pm.f90:335-372)
  const double coef = cube_vcoef(&o.codec, s->sigma_vi);
  double vmx0 = 0, vmx1 = 0, vmx2 = 0;
  for (int tz = 0; tz < o.nnt; ++tz)
    for (int ty = 0; ty < o.nnt; ++ty)
      for (int tx = 0; tx < o.nnt; ++tx)
        if (tile_on(o, tx, ty, tz))
#pragma omp parallel for schedule(static, 2) reduction(max : vmx0, vmx1, vmx2)
        for (int k = 1; k <= nt; ++k)
          for (int j = 1; j <= nt; ++j)
            for (int i = 1; i <= nt; ++i) {
              const int64_t c = cell_id(o, tx, ty, tz, i - 1, j - 1, k - 1);
              const int tt[3] = {tx, ty, tz}, ijk[3] = {i, j, k};
              for (int64_t ip = cs[c]; ip < cs[c + 1]; ++ip) {
                int i1[3];
                float dx1[3], dx2[3];
                for (int d = 0; d < 3; ++d) {
                  const double g = cube_dadd((double)(tt[d] * nt) + (double)(ijk[d] - 1), cube_xfrac(o.xp[3 * ip + d], o.izipx));
                  const float t_ = (float)cube_dsub(g, 0.5);
                  i1[d] = (int)floorf(t_) + 1;
                  dx1[d] = cube_fsub((float)i1[d], t_);
                  dx2[d] = cube_fsub(1.f, dx1[d]);
                }
                const int cx[8][3] = {{0,0,0},{1,0,0},{0,1,0},{0,0,1},{0,1,1},{1,0,1},{1,1,0},{1,1,1}};
                for (int d = 0; d < 3; ++d) {
                  double v = cube_vdecode(tanf_code(o, o.vp[3 * ip + d]), coef);
                  for (int c8 = 0; c8 < 8; ++c8) {
                    // force_c(:,0:nc+1) with periodic halo: node index idx in 0..nc+1
                    const int fi = ((i1[0] + cx[c8][0] - 1) % nc + nc) % nc;
                    const int fj = ((i1[1] + cx[c8][1] - 1) % nc + nc) % nc;
                    const int fk = ((i1[2] + cx[c8][2] - 1) % nc + nc) % nc;
                    const float fv = o.force_c[(size_t)d * nc * nc * nc + ((size_t)fk * nc + fj) * nc + fi];
                    float t = cube_fmul(fv, a_mid);
                    t = cube_fmul(t, dt);
                    t = cube_fdiv(t, 6.f);
                    t = cube_fdiv(t, pi_f);
                    t = cube_fmul(t, cx[c8][0] ? dx2[0] : dx1[0]);
                    t = cube_fmul(t, cx[c8][1] ? dx2[1] : dx1[1]);
                    t = cube_fmul(t, cx[c8][2] ? dx2[2] : dx1[2]);
                    v = cube_dadd(v, (double)t);
                  }
                  const double am = fabs(cube_dadd(v, (double)o.vfield[3 * c + d]));
                  if (d == 0) vmx0 = std::max(vmx0, am);
                  else if (d == 1) vmx1 = std::max(vmx1, am);
                  else vmx2 = std::max(vmx2, am);
                  o.vp[3 * ip + d] = cube_wrap_code(orc_enc(o, v, coef), o.izipv);
                }
              }
            }
  // neutrino gravity from the coarse force (pm.f90:374-422), sequential
  if (o.nu_on)
    for (int k = 0; k <= nc + 1; ++k)
      for (int j = 0; j <= nc + 1; ++j)
        for (int i = 0; i <= nc + 1; ++i)
          for (int kk = 1; kk <= ncell; ++kk)
            for (int jj = 1; jj <= ncell; ++jj)
              for (int ii = 1; ii <= ncell; ++ii) {
                const int m[3] = {(i - 1) * ncell + ii, (j - 1) * ncell + jj, (k - 1) * ncell + kk};
                if (std::min(std::min(m[0], m[1]), m[2]) < -1 || std::max(std::max(m[0], m[1]), m[2]) > nf + 2) continue;
                float x[3], c1[3], c2[3];
                int i1[3];
                for (int d = 0; d < 3; ++d) {
                  x[d] = (float)m[d] - 0.5f;
                  float xc = x[d] / (float)ncell;
                  xc = xc - 0.5f;
                  i1[d] = 1 + (int)floorf(xc);
                  c1[d] = (float)i1[d] - xc;
                  c2[d] = 1.f - c1[d];
                }
                const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1}, oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
                double acc[3] = {0.0, 0.0, 0.0};
                for (int c8 = 0; c8 < 8; ++c8) {
                  // force_c(:,0:nc+1) with its periodic halo
                  const int fi = ((i1[0] + ox[c8] - 1) % nc + nc) % nc, fj = ((i1[1] + oy[c8] - 1) % nc + nc) % nc,
                            fk = ((i1[2] + oz[c8] - 1) % nc + nc) % nc;
                  for (int d = 0; d < 3; ++d) {
                    const float fv = o.force_c[(size_t)d * nc * nc * nc + ((size_t)fk * nc + fj) * nc + fi];
                    float t = cube_fdiv(cube_fdiv(cube_fmul(cube_fmul(fv, a_mid), dt), 6.f), pi_f);
                    t = cube_fmul(t, ox[c8] ? c2[0] : c1[0]);
                    t = cube_fmul(t, oy[c8] ? c2[1] : c1[1]);
                    t = cube_fmul(t, oz[c8] ? c2[2] : c1[2]);
                    acc[d] = cube_dadd(acc[d], (double)t);
                  }
                }
                orcnu::dfld_gravity(o.nu, x, acc, a_mid, o.P.z_i_nu);
              }
  vmax[0] = vmx0; vmax[1] = vmx1; vmax[2] = vmx2;
  for (int d = 0; d < 3; ++d) s->vmax[d] = (float)vmax[d];
  s->testrhof = testrhof;
  s->testrhoc = testrhoc;
  dt_constraints(o, s);
  return CUBE_OK;
}

/* ------------------------------------------------------------------------- */
/* ext_pp_force (ext_pp_force.f90:34-143)                                     */
int ext_pp_force(Orc& o, cube_scalars* s) {
  const int nt = o.nt, ncb = o.ncb, ncell = o.ncell, nft = o.nft, pr = o.P.pp_range;
  const int lo = 1 - ncb, nte = o.nte;
  const double coef = cube_vcoef(&o.codec, s->sigma_vi);
  const std::vector<int64_t> cs = compact_cell_start(o);
  const double rsoft = (double)o.P.rsoft;
  const double mass = (double)s->mass_p_cdm;
  double ftemp = (double)s->f2_max_pp;  // saved local in the reference: never reset between calls
  int64_t itest1 = 0, npairs = 0;
  ExtTile e;
  const int nfl = nft + 2 * ncell;  // hoc(1-ncell:nft+ncell)
  std::vector<int64_t> hoc((size_t)nfl * nfl * nfl);
  std::vector<int64_t> ll;
  for (int tz = 0; tz < o.nnt; ++tz)
    for (int ty = 0; ty < o.nnt; ++ty)
      for (int tx = 0; tx < o.nnt; ++tx) {
        if (!tile_on(o, tx, ty, tz)) continue;
        build_ext(o, cs, tx, ty, tz, e);
        auto eq = [&](int i, int j, int k) { return ((size_t)(k - lo) * nte + (j - lo)) * nte + (i - lo); };
        auto hq = [&](int i, int j, int k) { return ((size_t)(k + ncell - 1) * nfl + (j + ncell - 1)) * nfl + (i + ncell - 1); };
        std::fill(hoc.begin(), hoc.end(), -1);
        ll.assign(e.src.size(), -1);
        // linked list (ext_pp_force.f90:51-73): LIFO per fine cell
        for (int igz = 0; igz <= nt + 1; ++igz)
          for (int igy = 0; igy <= nt + 1; ++igy)
            for (int igx = 0; igx <= nt + 1; ++igx) {
              const size_t qe = eq(igx, igy, igz);
              const int g[3] = {igx, igy, igz};
              for (int64_t l = 0; l < e.rho[qe]; ++l) {
                const int64_t slot = e.cstart[qe] + l;
                const int64_t ip = e.src[slot];
                int iv[3];
                for (int d = 0; d < 3; ++d) {
                  const double xv = cube_dadd((double)ncell * (double)(g[d] - 1), cube_dmul((double)ncell, cube_xfrac(o.xp[3 * ip + d], o.izipx)));
                  iv[d] = (int)floor(xv) + 1;
                }
                const size_t h = hq(iv[0], iv[1], iv[2]);
                ll[slot] = hoc[h];
                hoc[h] = slot;
              }
            }
        auto xvec = [&](int fi, int32_t code) -> double {
          const int cidx = (int)floorf(cube_fdiv((float)(fi - 1), 4.f));
          return cube_dadd((double)ncell * (double)cidx, cube_dmul((double)ncell, cube_xfrac(code, o.izipx)));
        };
#pragma omp parallel for schedule(static, 2) reduction(+ : itest1, npairs) reduction(max : ftemp)
        for (int igz = 1; igz <= nft; ++igz)
          for (int igy = 1; igy <= nft; ++igy)
            for (int igx = 1; igx <= nft; ++igx) {
              int64_t s1 = hoc[hq(igx, igy, igz)];
              while (s1 >= 0) {
                ++itest1;
                const int64_t ip1 = e.src[s1];
                double x1[3], v[3], ft[3] = {0, 0, 0};
                const int g1[3] = {igx, igy, igz};
                for (int d = 0; d < 3; ++d) {
                  x1[d] = xvec(g1[d], o.xp[3 * ip1 + d]);
                  v[d] = cube_vdecode(tanf_code(o, o.vp[3 * ip1 + d]), coef);
                }
                for (int kk = igz - pr; kk <= igz + pr; ++kk)
                  for (int jj = igy - pr; jj <= igy + pr; ++jj)
                    for (int ii = igx - pr; ii <= igx + pr; ++ii) {
                      int64_t s2 = hoc[hq(ii, jj, kk)];
                      const int g2[3] = {ii, jj, kk};
                      while (s2 >= 0) {
                        ++npairs;
                        const int64_t ip2 = e.src[s2];
                        double x21[3];
                        for (int d = 0; d < 3; ++d) x21[d] = cube_dsub(xvec(g2[d], o.xp[3 * ip2 + d]), x1[d]);
                        double rmag = sqrt(cube_dadd(cube_dadd(cube_dmul(x21[0], x21[0]), cube_dmul(x21[1], x21[1])), cube_dmul(x21[2], x21[2])));
                        if (rmag == 0) rmag = 1.0;
                        const double rc = cube_ddiv(rmag, (double)o.P.nf_cutoff);
                        const double rc2 = cube_dmul(rc, rc);
                        const double rc3 = cube_dmul(rc2, rc);
                        const double rc5 = cube_dmul(cube_dmul(rc2, rc2), rc);
                        const double pcut = cube_dadd(cube_dsub(1.0, cube_dmul(1.75, rc3)), cube_dmul(0.75, rc5));
                        const double r3 = cube_dmul(cube_dmul(rmag, rmag), rmag);
                        for (int d = 0; d < 3; ++d) {
                          double fp = cube_dmul(cube_dmul(mass, cube_ddiv(x21[d], r3)), pcut);
                          if (!(rmag > rsoft)) fp = cube_dmul(fp, 0.0);
                          ft[d] = cube_dadd(ft[d], fp);
                        }
                        s2 = ll[s2];
                      }
                    }
                for (int d = 0; d < 3; ++d) {
                  double k = cube_dmul(ft[d], (double)s->a_mid);
                  k = cube_dmul(k, (double)s->dt);
                  k = cube_ddiv(k, 6.0);
                  k = cube_ddiv(k, (double)o.codec.pi_f);
                  v[d] = cube_dadd(v[d], k);
                }
                // vp(:,ip1) is written at the physical slot; buffer copies are refreshed by buffer_v
                for (int d = 0; d < 3; ++d)
                  o.vp[3 * ip1 + d] = cube_wrap_code(orc_enc(o, v[d], coef), o.izipv);
                const double f2 = cube_dadd(cube_dadd(cube_dmul(ft[0], ft[0]), cube_dmul(ft[1], ft[1])), cube_dmul(ft[2], ft[2]));
                ftemp = std::max(ftemp, (double)(float)f2);
                s1 = ll[s1];
              }
            }
      }
  s->f2_max_pp = (float)ftemp;
  const float pi_f = o.codec.pi_f;
  const float GG = cube_fdiv(cube_fdiv(1.0f, 6.0f), pi_f);
  s->dt_pp = cube_fdiv(cube_fmul(1.0f, sqrtf(1.0f)), cube_fmul(cube_fmul(sqrtf(s->f2_max_pp), s->a_mid), GG));
  s->itest1 = itest1;
  s->npairs = npairs;
  if (o.tmask.empty() && itest1 != o.np) { o.err = "PP did not touch every particle once"; return CUBE_ERR_STATE; }
  return CUBE_OK;
}

/* ------------------------------------------------------------------------- */
/* Run-time halo finder, halofind.f90:18-598, on the global periodic box of   */
/* one image instead of tile by tile (every halo is then found once).  The    */
/* reference's FP32 meshes become 64-bit fixed point (weights * 2^32), ties   */
/* it leaves to its unstable quicksort are broken by index, and the moment    */
/* accumulators start from zero for each halo; see the library's k_halo.cu    */
/* for the list.  Plain sequential loops in the reference's step order.       */
namespace hf {

const double FIX = 4294967296.0;
const int RMAX = 64, NB_MAX = 300, MIN_NP = 100;

struct Cand {
  int64_t node;
  uint64_t acc;
  double mass;
  double pos[3];
  double rp;
};

inline int wrapn(int64_t x, int64_t n) { x %= n; return (int)(x < 0 ? x + n : x); }
inline double pmod(double a, double p) { return a - floor(a / p) * p; }  /* Fortran modulo */
inline double dist3(const double a[3], const double b[3]) {
  const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return sqrt((d0 * d0 + d1 * d1) + d2 * d2);
}
inline double parab(int64_t m, int64_t p, int64_t den) { return (0.5 * (double)(p - m)) / (double)den; }

void cell_xyz(const Orc& o, int64_t c, int g[3]) {
  const int64_t nt3 = (int64_t)o.nt * o.nt * o.nt;
  const int64_t t = c / nt3, r = c % nt3;
  g[0] = (int)(t % o.nnt) * o.nt + (int)(r % o.nt);
  g[1] = (int)((t / o.nnt) % o.nnt) * o.nt + (int)((r / o.nt) % o.nt);
  g[2] = (int)(t / ((int64_t)o.nnt * o.nnt)) * o.nt + (int)(r / ((int64_t)o.nt * o.nt));
}

/* distance-ordered offsets (:68-87) with exact r^2 and a stable order */
struct Off { int dx, dy, dz, r2; };
std::vector<Off> shell_list() {
  std::vector<Off> L;
  for (int i = -RMAX; i <= RMAX; ++i)
    for (int j = -RMAX; j <= RMAX; ++j)
      for (int k = -RMAX; k <= RMAX; ++k) {
        const int r2 = i * i + j * j + k * k;
        if (r2 <= RMAX * RMAX) L.push_back(Off{i, j, k, r2});
      }
  std::stable_sort(L.begin(), L.end(), [](const Off& a, const Off& b) { return a.r2 < b.r2; });
  return L;
}

int halofind(Orc& o, const cube_scalars* s, const cube_halo_args* ha, cube_halo_result* res) {
  const int nf = o.nf, nc = o.nc, ncell = o.ncell;
  const int64_t n3 = (int64_t)nf * nf * nf;
  const double den_odc = ha->den_odc > 0.f ? (double)ha->den_odc : 200.0;
  const double mass = (double)s->mass_p_cdm, unit = mass / FIX, pi = (double)o.codec.pi_f;
  const double coef = cube_vcoef(&o.codec, s->sigma_vi);
  const std::vector<int64_t> cs = compact_cell_start(o);
  const int64_t ncells = (int64_t)nc * nc * nc;
  *res = cube_halo_result{0, 0, 0};
  /* fine mass assignment, CIC at pos - 1/2 (:144-177) */
  std::vector<uint64_t> rhof((size_t)n3, 0);
  for (int64_t c = 0; c < ncells; ++c) {
    int g[3];
    cell_xyz(o, c, g);
    for (int64_t ip = cs[c]; ip < cs[c + 1]; ++ip) {
      int i1[3];
      double w1[3], w2[3];
      for (int d = 0; d < 3; ++d) {
        const double p = 4.0 * ((double)g[d] + cube_xfrac(o.xp[3 * ip + d], o.izipx)) - 0.5;
        const double f = floor(p);
        w1[d] = (f + 1.0) - p;
        w2[d] = 1.0 - w1[d];
        i1[d] = (int)f;
      }
      for (int cc = 0; cc < 8; ++cc) {
        const int ox = cc & 1, oy = (cc >> 1) & 1, oz = cc >> 2;
        const double w = ((ox ? w2[0] : w1[0]) * (oy ? w2[1] : w1[1])) * (oz ? w2[2] : w1[2]);
        const size_t q = ((size_t)wrapn(i1[2] + oz, nf) * nf + wrapn(i1[1] + oy, nf)) * nf + wrapn(i1[0] + ox, nf);
        rhof[q] += (uint64_t)llrint(w * FIX);
      }
    }
  }
  /* density peaks, their mesh mass and parabolic position (:179-208) */
  const std::vector<Off> sl = shell_list();
  std::vector<Cand> cand;
  auto at = [&](int x, int y, int z) { return (int64_t)rhof[((size_t)wrapn(z, nf) * nf + wrapn(y, nf)) * nf + wrapn(x, nf)]; };
  for (int z = 0; z < nf; ++z)
    for (int y = 0; y < nf; ++y)
      for (int x = 0; x < nf; ++x) {
        const uint64_t a0 = rhof[((size_t)z * nf + y) * nf + x];
        if (!((double)a0 * unit > 100.0)) continue;
        bool peak = true;
        for (int dz = -1; dz <= 1; ++dz)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
              if ((uint64_t)at(x + dx, y + dy, z + dz) > a0) peak = false;
        if (!peak) continue;
        uint64_t m = 0;
        for (size_t i = 0; i < sl.size(); ++i) {
          m += (uint64_t)at(x + sl[i].dx, y + sl[i].dy, z + sl[i].dz);
          if (i + 1 < sl.size() && sl[i + 1].r2 == sl[i].r2) continue;
          if (i + 1 >= 19 && (double)m * unit / (double)(i + 1) < den_odc) break;
        }
        const double mm = (double)m * unit;
        if (!(mm > mass * 50.0)) continue;
        Cand h;
        h.node = ((int64_t)z * nf + y) * nf + x;
        h.acc = a0;
        h.mass = mm;
        const int c3[3] = {x, y, z};
        for (int d = 0; d < 3; ++d) {
          const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
          const int64_t am = at(x - e0, y - e1, z - e2), ap = at(x + e0, y + e1, z + e2);
          const int64_t den = 2 * (int64_t)a0 - am - ap;
          h.pos[d] = ((double)c3[d] + 0.5) + (den != 0 ? parab(am, ap, den) : 0.0);
        }
        cand.push_back(h);
      }
  std::sort(cand.begin(), cand.end(), [](const Cand& a, const Cand& b) {
    return a.acc != b.acc ? a.acc > b.acc : a.node < b.node;
  });
  for (Cand& h : cand) h.rp = cbrt(0.75 / pi / den_odc * h.mass);
  res->npeak = (int32_t)cand.size();
  /* halos, densest peak first (:231-513) */
  std::vector<uint8_t> tag((size_t)o.np, 0);
  if (ha->hid && ha->hid_len > 0) std::fill(ha->hid, ha->hid + ha->hid_len, 0);
  const double ng = 1.0 / 3.0, half_ng = 0.5 / 3.0, hnf = (double)(nf / 2);
  const bool use_pid = o.P.use_pid && !o.pid.empty();
  int nhalo = 0;
  int64_t nmem = 0;
  std::vector<double> gx, gv;
  std::vector<int64_t> gip;
  std::vector<uint64_t> grid;
  for (const Cand& h : cand) {
    double hpos[3] = {h.pos[0], h.pos[1], h.pos[2]};
    const double rp = h.rp, rs = fmin(2.0 * rp, (double)((o.ncb - 1) * ncell));
    int clo[3], cn[3], flo[3], nb[3], mx[3];
    for (int d = 0; d < 3; ++d) {
      clo[d] = (int)floor((hpos[d] - rs) / ncell);
      cn[d] = (int)floor((hpos[d] + rs) / ncell) - clo[d] + 1;
      const int rlo = (int)floor((hpos[d] - rp) / ncell), rhi = (int)floor((hpos[d] + rp) / ncell);
      flo[d] = ncell * rlo;
      nb[d] = 3 * ncell * (rhi - rlo + 1);
      mx[d] = std::min(nb[d] + 1, NB_MAX);
      if (nb[d] > NB_MAX) { o.err = "halofind: newbox > newbox_max"; return CUBE_ERR_CAPACITY; }
      if (cn[d] > nc) { o.err = "halofind: search box wraps onto itself"; return CUBE_ERR_PARAM; }
    }
    const int gxn = nb[0] + 3, gyn = nb[1] + 3, gzn = nb[2] + 3;
    grid.assign((size_t)gxn * gyn * gzn, 0);
    gx.clear(); gv.clear(); gip.clear();
    for (int q = 0; q < cn[0] * cn[1] * cn[2]; ++q) {
      const int cu[3] = {clo[0] + q % cn[0], clo[1] + (q / cn[0]) % cn[1], clo[2] + q / (cn[0] * cn[1])};
      const int gw[3] = {wrapn(cu[0], nc), wrapn(cu[1], nc), wrapn(cu[2], nc)};
      const int64_t c = cell_id(o, gw[0] / o.nt, gw[1] / o.nt, gw[2] / o.nt, gw[0] % o.nt, gw[1] % o.nt, gw[2] % o.nt);
      for (int64_t ip = cs[c]; ip < cs[c + 1]; ++ip) {
        if (tag[ip]) continue;
        double x[3];
        for (int d = 0; d < 3; ++d) x[d] = 4.0 * ((double)cu[d] + cube_xfrac(o.xp[3 * ip + d], o.izipx));
        const double r = dist3(x, hpos);
        if (!(r < rs)) continue;
        for (int d = 0; d < 3; ++d) {
          gx.push_back(x[d]);
          gv.push_back(cube_dadd(cube_vdecode(tanf_code(o, o.vp[3 * ip + d]), coef), (double)o.vfield[3 * c + d]));
        }
        gip.push_back(ip);
        if (r < rp) {
          int i1[3];
          double w1[3], w2[3];
          for (int d = 0; d < 3; ++d) {
            const double p = ((x[d] - half_ng) - (double)flo[d]) / ng;
            const double f = floor(p);
            w1[d] = (f + 1.0) - p;
            w2[d] = 1.0 - w1[d];
            i1[d] = (int)f + 1;
          }
          for (int cc = 0; cc < 8; ++cc) {
            const int ox = cc & 1, oy = (cc >> 1) & 1, oz = cc >> 2;
            const int ix = i1[0] + ox, iy = i1[1] + oy, iz = i1[2] + oz;
            if (ix < 0 || iy < 0 || iz < 0 || ix >= gxn || iy >= gyn || iz >= gzn) continue;
            const double w = ((ox ? w2[0] : w1[0]) * (oy ? w2[1] : w1[1])) * (oz ? w2[2] : w1[2]);
            grid[((size_t)iz * gyn + iy) * gxn + ix] += (uint64_t)llrint(w * FIX);
          }
        }
      }
    }
    const int n = (int)gip.size();
    /* refined maximum, maxloc(finegrid(1:newbox_max,...)) (:347) */
    auto g = [&](int a, int b, int c) { return (int64_t)grid[((size_t)c * gyn + b) * gxn + a]; };
    int i0 = 1, j0 = 1, k0 = 1;
    int64_t best = g(1, 1, 1);
    for (int iz = 1; iz <= mx[2]; ++iz)
      for (int iy = 1; iy <= mx[1]; ++iy)
        for (int ix = 1; ix <= mx[0]; ++ix)
          if (g(ix, iy, iz) > best) { best = g(ix, iy, iz); i0 = ix; j0 = iy; k0 = iz; }
    const int64_t g0 = g(i0, j0, k0);
    const int64_t dxn = 2 * g0 - g(i0 - 1, j0, k0) - g(i0 + 1, j0, k0);
    const int64_t dyn = 2 * g0 - g(i0, j0 - 1, k0) - g(i0, j0 + 1, k0);
    const int64_t dzn = 2 * g0 - g(i0, j0, k0 - 1) - g(i0, j0, k0 - 1);  /* as :354-355 */
    if (dxn == 0 || dyn == 0 || dzn == 0) continue;
    const double hr[3] = {(i0 - 0.5) + parab(g(i0 - 1, j0, k0), g(i0 + 1, j0, k0), dxn),
                          (j0 - 0.5) + parab(g(i0, j0 - 1, k0), g(i0, j0 + 1, k0), dyn),
                          (k0 - 0.5) + parab(g(i0, j0, k0 - 1), g(i0, j0, k0 + 1), dzn)};
    for (int d = 0; d < 3; ++d) hpos[d] = (double)flo[d] + ng * hr[d];
    /* sort by radius (:361-369), ties by storage index */
    std::vector<double> key(n);
    std::vector<int> ord(n);
    for (int i = 0; i < n; ++i) {
      key[i] = dist3(&gx[3 * i], hpos);
      ord[i] = i;
    }
    std::sort(ord.begin(), ord.end(), [&](int a, int b) {
      return key[a] != key[b] ? key[a] < key[b] : gip[a] < gip[b];
    });
    /* halo radius (:385-401) */
    const double c43 = 0.75 / pi;
    int iis = 0;
    for (int ii = 2; ii <= n; ++ii) {
      const double r = key[ord[ii - 1]];
      if (c43 * ii * mass / (r * r * r) < den_odc) { iis = ii; break; }
    }
    const int iodc = iis ? iis - 1 : 0;
    if (iodc < MIN_NP) continue;
    /* tag, halo number per PID, member PIDs (:404-405, :450-458) */
    for (int i = 0; i < iodc; ++i) {
      const int64_t ip = gip[ord[i]];
      tag[ip] = 1;
      if (use_pid) {
        const int32_t p = o.pid[ip];
        if (ha->hid && p >= 1 && p <= ha->hid_len) ha->hid[p - 1] = nhalo + 1;
        if (ha->member_pid && nmem + i < ha->member_capacity) ha->member_pid[nmem + i] = p;
      }
    }
    cube_halo H;
    memset(&H, 0, sizeof(H));
    double xm[3] = {0, 0, 0}, vm[3] = {0, 0, 0};
    for (int i = 0; i < iodc; ++i)
      for (int d = 0; d < 3; ++d) {
        xm[d] += gx[3 * ord[i] + d];
        vm[d] += gv[3 * ord[i] + d];
      }
    double xw[3];
    for (int d = 0; d < 3; ++d) {
      xm[d] /= iodc;
      vm[d] /= iodc;
      xw[d] = pmod(xm[d], (double)nf);
    }
    double sxx[3] = {0, 0, 0}, svv = 0, am[3] = {0, 0, 0}, in[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < iodc; ++i) {
      double dx[3], v[3];
      for (int d = 0; d < 3; ++d) {
        dx[d] = gx[3 * ord[i] + d] - xm[d];
        v[d] = gv[3 * ord[i] + d];
        sxx[d] += dx[d] * dx[d];
        svv += (v[d] - vm[d]) * (v[d] - vm[d]);
      }
      am[0] += dx[1] * v[2] - dx[2] * v[1];
      am[1] += dx[2] * v[0] - dx[0] * v[2];
      am[2] += dx[0] * v[1] - dx[1] * v[0];
      in[0] += dx[0] * dx[0]; in[1] += dx[1] * dx[1]; in[2] += dx[2] * dx[2];
      in[3] += dx[0] * dx[1]; in[4] += dx[1] * dx[2]; in[5] += dx[2] * dx[0];
    }
    /* q-space: PID - 1 = iq_x + nf iq_y + nf^2 iq_z, qpos = iq + 1/2 (:460-500) */
    double qm[3] = {0, 0, 0}, iq[6] = {0, 0, 0, 0, 0, 0};
    if (use_pid) {
      const int64_t nfl = nf;
      double dq[3] = {0, 0, 0};
      int64_t nq = 0;
      auto qpos = [&](int64_t qt, double q[3]) {
        const int64_t qz = qt / (nfl * nfl), qy = (qt - qz * nfl * nfl) / nfl, qx = qt % nfl;
        q[0] = qx + 0.5; q[1] = qy + 0.5; q[2] = qz + 0.5;
      };
      for (int i = 0; i < iodc; ++i) {
        const int64_t qt = (int64_t)o.pid[gip[ord[i]]] - 1;
        if (qt < 0) continue;
        double q[3];
        qpos(qt, q);
        for (int d = 0; d < 3; ++d) dq[d] += pmod((q[d] - xw[d]) + hnf, (double)nf) - hnf;
        ++nq;
      }
      if (nq > 0) {
        for (int d = 0; d < 3; ++d) qm[d] = pmod(xw[d] + dq[d] / (double)nq, (double)nf);
        for (int i = 0; i < iodc; ++i) {
          const int64_t qt = (int64_t)o.pid[gip[ord[i]]] - 1;
          if (qt < 0) continue;
          double q[3], e[3];
          qpos(qt, q);
          for (int d = 0; d < 3; ++d) e[d] = pmod(((q[d] + 0.5) - qm[d]) + hnf, (double)nf) - hnf;
          iq[0] += e[0] * e[0]; iq[1] += e[1] * e[1]; iq[2] += e[2] * e[2];
          iq[3] += e[0] * e[1]; iq[4] += e[1] * e[2]; iq[5] += e[2] * e[0];
        }
      }
    }
    for (int d = 0; d < 3; ++d) H.hpos[d] = (float)pmod(hpos[d], (double)nf);
    H.mass_odc = (float)iodc;
    {
      const double r2 = key[ord[iis - 1]], r1 = key[ord[iis - 2]];
      const double den2 = c43 * iis * mass / (r2 * r2 * r2), den1 = c43 * (iis - 1) * mass / (r1 * r1 * r1);
      const double lr2 = log10(r2), lr1 = log10(r1), d2 = log10(den2), d1 = log10(den1), lo = log10(den_odc);
      H.radius_odc = (float)pow(10.0, ((lo - d2) * lr1 + (d1 - lo) * lr2) / (d1 - d2));
    }
    H.v_disp = (float)sqrt(svv / (iodc - 1));
    for (int d = 0; d < 3; ++d) {
      H.x_mean[d] = (float)xw[d];
      H.v_mean[d] = (float)vm[d];
      H.var_x[d] = (float)(sxx[d] / (iodc - 1));
      H.ang_mom[d] = (float)am[d];
      H.q_mean[d] = (float)qm[d];
    }
    const int sym[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};
    for (int k = 0; k < 9; ++k) {
      H.inertia[k] = (float)in[sym[k]];
      H.inertia_q[k] = (float)iq[sym[k]];
    }
    /* redshift-space mean position (:425-430); ng_global = nc in the main code */
    double los[3], ln = 0.0, vlos = 0.0;
    const double cen[3] = {30.0, 370.0, 370.0};
    for (int d = 0; d < 3; ++d) {
      los[d] = xw[d] - cen[d] / 500.0 * (double)nc;
      ln += los[d] * los[d];
    }
    ln = sqrt(ln);
    for (int d = 0; d < 3; ++d) {
      los[d] /= ln;
      vlos += vm[d] * los[d];
    }
    for (int d = 0; d < 3; ++d) {
      const double sx = vlos * los[d] * (double)s->vsim2phys / (double)s->a / (100.0 * (double)o.P.h0) /
                        ((double)o.P.h0 * (double)o.P.box / nf);
      H.s_mean[d] = (float)pmod(xw[d] + sx, (double)nf);
    }
    if (nhalo < ha->capacity) ha->halos[nhalo] = H;
    ++nhalo;
    if (use_pid) nmem += iodc;
  }
  res->nhalo = nhalo;
  res->nmember = nmem;
  if (nhalo > ha->capacity || (ha->member_pid && nmem > ha->member_capacity)) {
    o.err = "halofind: the output arrays are too small";
    return CUBE_ERR_CAPACITY;
  }
  return CUBE_OK;
}

}  // namespace hf

void setup_sizes(Orc& o, const cube_params* p) {
  o.P = *p;
  o.nc = p->nc; o.nnt = p->nnt; o.nt = p->nc / p->nnt; o.ncell = p->ncell; o.ncb = p->ncb;
  o.nte = o.nt + 2 * o.ncb; o.nf = o.nc * o.ncell; o.nft = o.nt * o.ncell;
  o.nfb = o.ncb * o.ncell; o.nfe = o.nft + 2 * o.nfb; o.nfc = p->nf_cutoff;
  o.izipx = p->izipx; o.izipv = p->izipv;
  o.codec.pi_f = 4.0f * atanf(1.0f);
  o.codec.sqrt_pio2_f = sqrtf(o.codec.pi_f / 2.0f);
  o.nvbin = 1 << (8 * p->izipv);
  o.codec.nvbin_m1_f = (float)(o.nvbin - 1);
  o.codec.izipx = p->izipx; o.codec.izipv = p->izipv;
  o.codec.vrel_boost = p->vrel_boost;
  o.codec.x_resolution = (p->izipx == 1) ? 1.0 / 256.0 : 1.0 / 65536.0;
  o.tan_table.resize(o.nvbin);
  // the FP32 argument (pi*real(vp))/real(nvbin-1) and tan(real) of pm.f90:145
  for (int c = -o.nvbin / 2; c < o.nvbin / 2; ++c)
    o.tan_table[c + o.nvbin / 2] = tanf((o.codec.pi_f * (float)c) / o.codec.nvbin_m1_f);
}

}  // namespace

/* ========================================================================= */
/* C interface for the tests (ctypes)                                         */
extern "C" {

void* orc_create(const cube_params* p, const float* fk_table, const float* ck_table, int build_kernels) {
  Orc* o = new Orc();
  setup_sizes(*o, p);
  o->fk_table.assign(fk_table, fk_table + (size_t)3 * p->nf_cutoff * p->nf_cutoff * p->nf_cutoff);
  o->ck_table.assign(ck_table, ck_table + 3 * 64);
  o->np = 0;
  if (build_kernels) { kernel_f(*o); kernel_c(*o); }
  if (p->neutrino) {
    // one species (Nneu=1, parameters.f90:80-93); gamma = 5/3 (main.f90:38)
    o->nu_on = true;
    const int nf = o->nf;
    const int nc_n[3] = {p->nu_nc[0] > 0 ? p->nu_nc[0] : nf / 2, p->nu_nc[1] > 0 ? p->nu_nc[1] : nf / 4,
                         p->nu_nc[2] > 0 ? p->nu_nc[2] : nf / 8};
    const float hg_dv = (float)(2 * nf) / ((300.f * sqrtf(p->omega_m)) * p->box);  // hydrogr.f90:13
    orcnu::dfld_setup(o->nu, 5.f / 3.f, p->m_nu_ev, nc_n, nf, p->ncb * p->ncell, hg_dv);
  }
  return o;
}

/* fluid n (0..2) interior as fld(1:5,1:nc,1:nc,1:nc), component fastest */
int orc_nu_load(void* h, int n, const float* fld) {
  Orc& o = *(Orc*)h;
  if (!o.nu_on || n < 0 || n > 2) return CUBE_ERR_STATE;
  orcnu::Hydro& y = o.nu.h[n];
  size_t q = 0;
  for (int k = 1; k <= y.nc; ++k)
    for (int j = 1; j <= y.nc; ++j)
      for (int i = 1; i <= y.nc; ++i)
        for (int c = 1; c <= 5; ++c) y.f(c, i, j, k) = fld[q++];
  orcnu::hg_buffer(y);
  return CUBE_OK;
}

int orc_nu_store(void* h, int n, float* fld) {
  Orc& o = *(Orc*)h;
  if (!o.nu_on || n < 0 || n > 2) return CUBE_ERR_STATE;
  const orcnu::Hydro& y = o.nu.h[n];
  size_t q = 0;
  for (int k = 1; k <= y.nc; ++k)
    for (int j = 1; j <= y.nc; ++j)
      for (int i = 1; i <= y.nc; ++i)
        for (int c = 1; c <= 5; ++c) fld[q++] = y.f(c, i, j, k);
  return CUBE_OK;
}

/* neu%evolve(dt,dtg,dir,a) (hydrodf.f90:86-109) */
int orc_nu_evolve(void* h, float dt, float* dtg, int dir, float a) {
  Orc& o = *(Orc*)h;
  if (!o.nu_on) return CUBE_ERR_STATE;
  orcnu::dfld_evolve(o.nu, dt, *dtg, dir, a, o.P.z_i_nu);
  return CUBE_OK;
}

/* beta, dwgts[3], then per fluid: nc, ncb, dx, cs2, dv (3 x 5) */
void orc_nu_info(void* h, float* out) {
  const Orc& o = *(Orc*)h;
  out[0] = o.nu.beta;
  for (int n = 0; n < 3; ++n) out[1 + n] = o.nu.dwgts[n];
  for (int n = 0; n < 3; ++n) {
    const orcnu::Hydro& y = o.nu.h[n];
    float* q = out + 4 + 5 * n;
    q[0] = (float)y.nc; q[1] = (float)y.ncb; q[2] = y.dx; q[3] = y.cs2; q[4] = y.dv;
  }
}

void orc_destroy(void* h) { delete (Orc*)h; }

const char* orc_error(void* h) { return ((Orc*)h)->err.c_str(); }

int orc_load_state(void* h, int64_t np, const void* xp, const void* vp, const int32_t* pid,
                   const int32_t* rhoc, const float* vfield) {
  Orc& o = *(Orc*)h;
  const int64_t ncells = (int64_t)o.nc * o.nc * o.nc;
  o.np = np;
  o.xp.resize(3 * np); o.vp.resize(3 * np);
  for (int64_t q = 0; q < 3 * np; ++q) {
    o.xp[q] = o.izipx == 1 ? ((const int8_t*)xp)[q] : ((const int16_t*)xp)[q];
    o.vp[q] = o.izipv == 1 ? ((const int8_t*)vp)[q] : ((const int16_t*)vp)[q];
  }
  if (pid) o.pid.assign(pid, pid + np); else o.pid.clear();
  o.rhoc.assign(rhoc, rhoc + ncells);
  o.vfield.assign(vfield, vfield + 3 * ncells);
  int64_t tot = 0;
  for (int64_t c = 0; c < ncells; ++c) tot += o.rhoc[c];
  if (tot != np) { o.err = "sum(rhoc) != nplocal"; return CUBE_ERR_PARAM; }
  return CUBE_OK;
}

int orc_store_state(void* h, int64_t* np, void* xp, void* vp, int32_t* pid, int32_t* rhoc, float* vfield) {
  Orc& o = *(Orc*)h;
  const int64_t ncells = (int64_t)o.nc * o.nc * o.nc;
  if (np) *np = o.np;
  for (int64_t q = 0; q < 3 * o.np; ++q) {
    if (xp) { if (o.izipx == 1) ((int8_t*)xp)[q] = (int8_t)o.xp[q]; else ((int16_t*)xp)[q] = (int16_t)o.xp[q]; }
    if (vp) { if (o.izipv == 1) ((int8_t*)vp)[q] = (int8_t)o.vp[q]; else ((int16_t*)vp)[q] = (int16_t)o.vp[q]; }
  }
  if (pid && !o.pid.empty()) memcpy(pid, o.pid.data(), sizeof(int32_t) * o.np);
  if (rhoc) memcpy(rhoc, o.rhoc.data(), sizeof(int32_t) * ncells);
  if (vfield) memcpy(vfield, o.vfield.data(), sizeof(float) * 3 * ncells);
  return CUBE_OK;
}

int orc_update_x(void* h, cube_scalars* s) { return update_xp(*(Orc*)h, s); }

int orc_ext_pp_force(void* h, cube_scalars* s) { return ext_pp_force(*(Orc*)h, s); }

/* deposit_mode 0: reference FP32 order; 1: 64-bit fixed point */
int orc_particle_mesh(void* h, cube_scalars* s, int deposit_mode) {
  return particle_mesh(*(Orc*)h, s, deposit_mode, nullptr);
}

/* particle_mesh with externally supplied force meshes ([3][nf^3] and [3][nc^3]) */
int orc_particle_mesh_with_force(void* h, cube_scalars* s, int deposit_mode, const float* fine,
                                 const float* coarse) {
  Orc& o = *(Orc*)h;
  std::vector<float> f(fine, fine + (size_t)3 * o.nf * o.nf * o.nf);
  std::vector<float> c(coarse, coarse + (size_t)3 * o.nc * o.nc * o.nc);
  KickIn k{&f, &c};
  return particle_mesh(o, s, deposit_mode, &k);
}

/* which: 0 rho_f (nf^3), 1 r3 (nc^3), 2 force_f (3 nf^3), 3 force_c (3 nc^3),
 *        4 kern_f (3 nfe nfe (nfe/2+1), double), 5 kern_c (3 nc nc (nc/2+1), double) */
int64_t orc_fetch(void* h, int which, void* out, int64_t cap) {
  Orc& o = *(Orc*)h;
  const void* src = nullptr;
  int64_t n = 0;
  size_t es = 4;
  switch (which) {
    case 0: src = o.rho_f_global.data(); n = o.rho_f_global.size(); break;
    case 1: src = o.r3.data(); n = o.r3.size(); break;
    case 2: src = o.force_f_global.data(); n = o.force_f_global.size(); break;
    case 3: src = o.force_c.data(); n = o.force_c.size(); break;
    case 4: src = o.kern_f.data(); n = o.kern_f.size(); es = 8; break;
    case 5: src = o.kern_c.data(); n = o.kern_c.size(); es = 8; break;
    default: return -1;
  }
  if (n > cap) return -1;
  memcpy(out, src, es * n);
  return n;
}

/* run-time halo finder (halofind.f90:18-598), global periodic box */
int orc_halofind(void* h, const cube_scalars* s, const cube_halo_args* a, cube_halo_result* r) {
  return hf::halofind(*(Orc*)h, s, a, r);
}

/* dt constraints only (pm.f90:427-443) */
void orc_dt_constraints(void* h, cube_scalars* s) { dt_constraints(*(Orc*)h, s); }

/* codec helpers for the tests */
float orc_tanf_code(void* h, int code) { return tanf_code(*(Orc*)h, code); }
/* Timing sample: mask[nnt^3] (tile-major, x fastest) marks the tiles the step
 * routines run; NULL runs every tile again.  See Orc::tmask. */
void orc_set_tile_mask(void* h, const char* mask) {
  Orc& o = *(Orc*)h;
  if (mask) o.tmask.assign(mask, mask + (size_t)o.nnt * o.nnt * o.nnt);
  else o.tmask.clear();
}

/* The global coarse Poisson solve of particle_mesh (pm.f90:288-300: forward FFT of
 * r3, three Green multiplies and inverse FFTs), on whatever r3 holds. */
void orc_coarse_poisson(void* h) {
  Orc& o = *(Orc*)h;
  const int nc = o.nc;
  std::vector<double> r((size_t)nc * nc * nc);
  for (size_t q = 0; q < r.size() && q < o.r3.size(); ++q) r[q] = (double)o.r3[q];
  std::vector<cd> sp, pr;
  orc::rfft3_forward(r.data(), sp, nc);
  pr.resize(sp.size());
  o.force_c.assign((size_t)3 * nc * nc * nc, 0.f);
  for (int d = 0; d < 3; ++d) {
    for (size_t q = 0; q < sp.size(); ++q) {
      const double kv = o.kern_c[(size_t)d * sp.size() + q];
      pr[q] = cd(-sp[q].imag() * kv, sp[q].real() * kv);
    }
    orc::rfft3_backward(pr, r.data(), nc);
    const double norm = (double)nc * nc * nc;
    for (size_t q = 0; q < r.size(); ++q) o.force_c[(size_t)d * r.size() + q] = (float)(r[q] / norm);
  }
}

/* 1: the step's velocity encodes use the C library's atan (orc_enc) */
void orc_set_libm_codec(void* h, int on) { ((Orc*)h)->libm_codec = on ? 1 : 0; }
double orc_atan(double x) { return cube_atan(x); }
int orc_vencode(void* h, double v, float sigma) {
  Orc& o = *(Orc*)h;
  return cube_wrap_code(cube_vencode(&o.codec, v, cube_vcoef(&o.codec, sigma)), o.izipv);
}
double orc_vdecode(void* h, int code, float sigma) {
  Orc& o = *(Orc*)h;
  return cube_vdecode(tanf_code(o, code), cube_vcoef(&o.codec, sigma));
}
/* same encode with the C library's atan instead of the project arctangent */
int orc_vencode_libm(void* h, double v, float sigma) {
  Orc& o = *(Orc*)h;
  const double coef = cube_vcoef(&o.codec, sigma);
  const double q = ((double)o.codec.nvbin_m1_f * atan(coef * v)) / (double)o.codec.pi_f;
  return cube_wrap_code((int64_t)round(q), o.izipv);
}
double orc_tree_sum(const double* a, int64_t n) { return cube_tree_sum(std::vector<double>(a, a + n)); }

}  // extern "C"

extern "C" {
/* forward r2c of an n^3 real array (x fastest) into (n/2+1) x n x n complex (interleaved re,im) */
void orc_rfft3(const double* in, int n, double* out) {
  std::vector<cd> h;
  orc::rfft3_forward(in, h, n);
  memcpy(out, h.data(), sizeof(cd) * h.size());
}
}

/* ------------------------------------------------------------------------- */
/* Division by a constant y with a precomputed reciprocal z = RN(1/y) and one  */
/* FMA correction (Brisebarre, Muller and Raina, "Accelerating correctly       */
/* rounded floating-point division when the divisor is known in advance",     */
/* IEEE Trans. Computers 53(8), 2004):                                          */
/*     q0 = RN(x z),  r = RN(x - q0 y) (fma, exact),  q = RN(q0 + r z) (fma).   */
/* Whether q = RN(x/y) for every x depends on y; this counts the FP32 inputs    */
/* where it differs from IEEE division (NaN/Inf inputs skipped), over all 2^32  */
/* bit patterns, and reports the largest |x| among the failures.                */
extern "C" int64_t orc_check_const_div(float y, float* worst_abs_x) {
  const float z = 1.0f / y;
  int64_t nfail = 0;
  float worst = 0.f;
#pragma omp parallel for reduction(+ : nfail) reduction(max : worst) schedule(static)
  for (int64_t b = 0; b < (1ll << 32); ++b) {
    const uint32_t u = (uint32_t)b;
    float x;
    memcpy(&x, &u, 4);
    if (!std::isfinite(x)) continue;
    const float q0 = x * z;
    const float r = fmaf(-q0, y, x);
    const float q = fmaf(r, z, q0);
    const float ref = x / y;
    if (memcmp(&q, &ref, 4) != 0) {
      ++nfail;
      worst = std::max(worst, fabsf(x));
    }
  }
  *worst_abs_x = worst;
  return nfail;
}
