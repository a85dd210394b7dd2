/*
 * k_pp.cu -- ext_pp_force: particle-particle correction over the fine cells
 * within +-pp_range of each particle's fine cell (ext_pp_force.f90:34-143).
 *
 * The reference builds a head-of-chain linked list per fine cell (LIFO, over
 * the coarse cells 0..nt+1 of a tile) and, for every particle of a physical
 * fine cell, sums m*(dx/r^3)*(1-7/4 rho^3+3/4 rho^5), rho=r/nf_cutoff, zero
 * for r <= rsoft, over the neighbour cells in (k,j,i) order, each chain
 * newest-first.  A fine cell lies inside exactly one coarse cell, so its chain
 * is that coarse cell's particles in reverse storage order, filtered by fine
 * cell.  Per particle the GPU scans the (at most 2^3) coarse cells under the
 * +-pp_range fine window newest-first, keeps the members of the window (from
 * a precomputed fine sub-cell byte per particle), and sorts them stably by
 * window cell, which is exactly the reference's summation order; lists longer
 * than MAXL fall back to walking the window cell by cell.  The pair
 * arithmetic is FP64 as in the reference (xvec* are real(8)), so the kicked
 * codes are bit-identical to the oracle.  One thread per particle.
 */
#include "cube_internal.cuh"

namespace {

constexpr int PCELLS = 64;  // cells of one 4^3 brick

// fine sub-cell of every particle inside its coarse cell: sx + 4 sy + 16 sz,
// s = floor(ncell*frac) (exact: the FP64 position ncell*(i-1)+ncell*frac has no rounding)
template <int ZX>
__global__ void k_pp_subcell(const void* __restrict__ xp_, int64_t cap, int64_t np, uint8_t* __restrict__ sub) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
    int sc = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + i], ZX);
      sc |= ((int)floor(cube_dmul(4.0, fr))) << (2 * d);
    }
    sub[i] = (uint8_t)sc;
  }
}

constexpr int MAXL = 40;  // candidate list of one particle; longer lists take the direct walk

template <int ZX, int ZV>
__global__ void __launch_bounds__(256) k_pp(const void* __restrict__ xp_, void* __restrict__ vp_,
                                            const int64_t* __restrict__ cell_start, int64_t cap, int64_t ncells,
                                            int nc, int nt, int nnt, int pr, int nf_cutoff, double rsoft,
                                            double mass, double a_mid, double dt, double pi_d,
                                            const float* __restrict__ tan_table, int half_nvbin, cube_codec codec,
                                            double coef, const uint8_t* __restrict__ sub,
                                            const int32_t* __restrict__ spill, DevScal* __restrict__ dscal) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  TV* vp = reinterpret_cast<TV*>(vp_);
  // the CTA's cells: a brick listed by k_pp_brick (its 4^3 cells)
  __shared__ int64_t cid[PCELLS], cst[PCELLS];
  __shared__ int cpre[PCELLS + 1];
  const int brick = spill[blockIdx.x];
  const int nb = nc / 4;
  const int bx = brick % nb, by = (brick / nb) % nb, bz = brick / (nb * nb);
  if (threadIdx.x < 32) {
    int run = 0;
    for (int base = 0; base < PCELLS; base += 32) {
      const int q = base + threadIdx.x;
      const int64_t c = cube_cell_of(bx * 4 + q % 4, by * 4 + (q / 4) % 4, bz * 4 + q / 16, nt, nnt);
      cid[q] = c;
      cst[q] = cell_start[c];
      const int cnt = (int)(cell_start[c + 1] - cst[q]);
      int inc = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)threadIdx.x >= o) inc += v;
      }
      cpre[q] = run + inc - cnt;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (threadIdx.x == 0) cpre[PCELLS] = run;
  }
  __syncthreads();
  unsigned long long n1 = 0, npair = 0;
  float f2max = 0.f;
  const int nt3 = nt * nt * nt;
  for (int m = threadIdx.x; m < cpre[PCELLS]; m += blockDim.x) {
    int lo = 0, hi = PCELLS - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cpre[mid] <= m) lo = mid; else hi = mid - 1;
    }
    const int64_t c = cid[lo];
    const int64_t ip = cst[lo] + (m - cpre[lo]);
    const int64_t tile = c / nt3;
    const int rem = (int)(c - tile * nt3);
    const int l[3] = {rem % nt, (rem / nt) % nt, rem / (nt * nt)};
    const int t[3] = {(int)(tile % nnt), (int)((tile / nnt) % nnt), (int)(tile / ((int64_t)nnt * nnt))};
    double x1[3], v[3], ft[3] = {0.0, 0.0, 0.0};
    int g1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX);
      x1[d] = cube_dadd(4.0 * (double)l[d], cube_dmul(4.0, fr));
      g1[d] = (int)floor(x1[d]) + 1;  // fine cell, 1-based, tile-relative
      const int code = (int)vp[(size_t)d * cap + ip];
      v[d] = cube_vdecode(__ldg(&tan_table[code + half_nvbin]), coef);
    }
    ++n1;
    auto pair_force = [&](int64_t jp, const int cf[3]) {
      double x21[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + jp], ZX);
        x21[d] = cube_dsub(cube_dadd(4.0 * (double)cf[d], cube_dmul(4.0, fr)), x1[d]);
      }
      double rmag = sqrt(cube_dadd(cube_dadd(cube_dmul(x21[0], x21[0]), cube_dmul(x21[1], x21[1])),
                                   cube_dmul(x21[2], x21[2])));
      if (rmag == 0.0) rmag = 1.0;
      const double rc = cube_ddiv(rmag, (double)nf_cutoff);
      const double rc2 = cube_dmul(rc, rc);
      const double rc3 = cube_dmul(rc2, rc);
      const double rc5 = cube_dmul(cube_dmul(rc2, rc2), rc);
      const double pcut = cube_dadd(cube_dsub(1.0, cube_dmul(1.75, rc3)), cube_dmul(0.75, rc5));
      const double r3 = cube_dmul(cube_dmul(rmag, rmag), rmag);
      const bool keep = rmag > rsoft;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double fp = cube_dmul(cube_dmul(mass, cube_ddiv(x21[d], r3)), pcut);
        if (!keep) fp = cube_dmul(fp, 0.0);
        ft[d] = cube_dadd(ft[d], fp);
      }
    };
    // coarse cells (T coordinates, 0-based) covering the fine window g1 +- pr
    int clo[3], chi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int a = g1[d] - pr - 1, b = g1[d] + pr - 1;
      clo[d] = a >= 0 ? a / 4 : -((3 - a) / 4);
      chi[d] = b >= 0 ? b / 4 : -((3 - b) / 4);
    }
    const int W = 2 * pr + 1;
    uint8_t lw[MAXL];
    int64_t li[MAXL];
    int8_t lc[MAXL][3];
    int nl = 0;
    bool overflow = false;
    for (int cz = clo[2]; cz <= chi[2] && !overflow; ++cz)
      for (int cy = clo[1]; cy <= chi[1] && !overflow; ++cy)
        for (int cx = clo[0]; cx <= chi[0] && !overflow; ++cx) {
          const int gx = ((t[0] * nt + cx) % nc + nc) % nc, gy = ((t[1] * nt + cy) % nc + nc) % nc,
                    gz = ((t[2] * nt + cz) % nc + nc) % nc;
          const int64_t c2 = cube_cell_of(gx, gy, gz, nt, nnt);
          const int64_t b0 = cell_start[c2], b1 = cell_start[c2 + 1];
          for (int64_t jp = b1 - 1; jp >= b0; --jp) {  // newest-first, as the linked list
            const int sc = sub[jp];
            const int wx = 4 * cx + (sc & 3) + 1 - g1[0] + pr;
            const int wy = 4 * cy + ((sc >> 2) & 3) + 1 - g1[1] + pr;
            const int wz = 4 * cz + (sc >> 4) + 1 - g1[2] + pr;
            if ((unsigned)wx >= (unsigned)W || (unsigned)wy >= (unsigned)W || (unsigned)wz >= (unsigned)W) continue;
            if (nl == MAXL) { overflow = true; break; }
            lw[nl] = (uint8_t)((wz * W + wy) * W + wx);
            li[nl] = jp;
            lc[nl][0] = (int8_t)cx; lc[nl][1] = (int8_t)cy; lc[nl][2] = (int8_t)cz;
            ++nl;
          }
        }
    if (!overflow) {
      // stable insertion sort by window cell: the reference's (k,j,i) cell order,
      // chain order (newest first) kept inside a cell
      for (int i = 1; i < nl; ++i) {
        const uint8_t w = lw[i];
        const int64_t ix = li[i];
        const int8_t c0_ = lc[i][0], c1_ = lc[i][1], c2_ = lc[i][2];
        int j = i - 1;
        while (j >= 0 && lw[j] > w) {
          lw[j + 1] = lw[j]; li[j + 1] = li[j];
          lc[j + 1][0] = lc[j][0]; lc[j + 1][1] = lc[j][1]; lc[j + 1][2] = lc[j][2];
          --j;
        }
        lw[j + 1] = w; li[j + 1] = ix;
        lc[j + 1][0] = c0_; lc[j + 1][1] = c1_; lc[j + 1][2] = c2_;
      }
      npair += nl;
      for (int i = 0; i < nl; ++i) {
        const int cf[3] = {lc[i][0], lc[i][1], lc[i][2]};
        pair_force(li[i], cf);
      }
    } else {
      for (int kk = g1[2] - pr; kk <= g1[2] + pr; ++kk)
        for (int jj = g1[1] - pr; jj <= g1[1] + pr; ++jj)
          for (int ii = g1[0] - pr; ii <= g1[0] + pr; ++ii) {
            const int fc[3] = {ii, jj, kk};
            int cf[3], gg[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              cf[d] = (fc[d] - 1 >= 0) ? (fc[d] - 1) / 4 : -((4 - fc[d]) / 4);  // floor((f-1)/4)
              gg[d] = ((t[d] * nt + cf[d]) % nc + nc) % nc;
            }
            const int want = ((fc[0] - 1 - 4 * cf[0])) | ((fc[1] - 1 - 4 * cf[1]) << 2) | ((fc[2] - 1 - 4 * cf[2]) << 4);
            const int64_t c2 = cube_cell_of(gg[0], gg[1], gg[2], nt, nnt);
            const int64_t b0 = cell_start[c2], b1 = cell_start[c2 + 1];
            for (int64_t jp = b1 - 1; jp >= b0; --jp) {
              if (sub[jp] != want) continue;
              ++npair;
              pair_force(jp, cf);
            }
          }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double k = cube_dmul(ft[d], a_mid);
      k = cube_dmul(k, dt);
      k = cube_ddiv(k, 6.0);
      k = cube_ddiv(k, pi_d);
      v[d] = cube_dadd(v[d], k);
      vp[(size_t)d * cap + ip] = (TV)cube_wrap_code(cube_vencode(&codec, v[d], coef), ZV);
    }
    const double f2 = cube_dadd(cube_dadd(cube_dmul(ft[0], ft[0]), cube_dmul(ft[1], ft[1])), cube_dmul(ft[2], ft[2]));
    f2max = fmaxf(f2max, (float)f2);
  }
  for (int o = 16; o > 0; o >>= 1) {
    n1 += __shfl_xor_sync(0xffffffffu, n1, o);
    npair += __shfl_xor_sync(0xffffffffu, npair, o);
    f2max = fmaxf(f2max, __shfl_xor_sync(0xffffffffu, f2max, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&dscal->itest1, n1);
    atomicAdd(&dscal->npairs, npair);
    atomicMax(&dscal->f2_pp_bits, __float_as_uint(f2max));
  }
}

// FP64 pair term of ext_pp_force.f90:99-107 for a separation x21 (exact in FP64).
// rc = rmag/nf_cutoff is evaluated as rmag*(1/nf_cutoff) only when nf_cutoff is
// a power of two, where both are the same exact scaling.
__device__ __forceinline__ void pp_pair(const double x21[3], double mass, double rsoft, int nf_cutoff,
                                        bool pow2_cut, double inv_cut, double fp[3]) {
  double rmag = sqrt(cube_dadd(cube_dadd(cube_dmul(x21[0], x21[0]), cube_dmul(x21[1], x21[1])),
                               cube_dmul(x21[2], x21[2])));
  if (rmag == 0.0) rmag = 1.0;
  const double rc = pow2_cut ? cube_dmul(rmag, inv_cut) : cube_ddiv(rmag, (double)nf_cutoff);
  const double rc2 = cube_dmul(rc, rc);
  const double rc3 = cube_dmul(rc2, rc);
  const double rc5 = cube_dmul(cube_dmul(rc2, rc2), rc);
  const double pcut = cube_dadd(cube_dsub(1.0, cube_dmul(1.75, rc3)), cube_dmul(0.75, rc5));
  const double r3 = cube_dmul(cube_dmul(rmag, rmag), rmag);
  const bool keep = rmag > rsoft;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double f = cube_dmul(cube_dmul(mass, cube_ddiv(x21[d], r3)), pcut);
    if (!keep) f = cube_dmul(f, 0.0);
    fp[d] = f;
  }
}

// ---------------------------------------------------------------------------
// Brick kernel: one CTA per 4^3-cell brick.  The particles of the brick and of
// its one-cell halo (6^3 cells; pp_range <= 4 fine cells = one coarse cell)
// are staged in shared memory, the reference's per-fine-cell chains are built
// there (one thread per coarse cell inserts its particles in storage order, so
// each chain is newest-first exactly like the linked list of
// ext_pp_force.f90:51-73), and each particle of the brick walks the chains of
// its +-pp_range window.  Positions enter the pair sums as differences of
// ncell*(cell)+ncell*frac, which are exact in FP64 whatever the origin, so
// region-local coordinates give the reference's values.  Bricks holding more
// than PB_CAP particles are listed and done by k_pp_list below.
constexpr int PB = 4;                     // brick edge in coarse cells
constexpr int PR = PB + 2;                // with the halo
constexpr int PRC = PR * PR * PR;         // 216 region cells
constexpr int PF = 4 * PR;                // region edge in fine cells (24)
constexpr int PB_CAP = 4096;              // particles staged per brick

template <int ZX, int ZV>
__global__ void __launch_bounds__(256, 3) k_pp_brick(const void* __restrict__ xp_, void* __restrict__ vp_,
                                                  const int64_t* __restrict__ cell_start, int64_t cap, int nc,
                                                  int nt, int nnt, int pr, int nf_cutoff, double rsoft,
                                                  double mass, double a_mid, double dt, double pi_d,
                                                  const float* __restrict__ tan_table, int half_nvbin,
                                                  cube_codec codec, double coef, int32_t* __restrict__ spill,
                                                  DevScal* __restrict__ dscal) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  TV* vp = reinterpret_cast<TV*>(vp_);
  extern __shared__ unsigned char pbsm[];
  uint16_t* head = reinterpret_cast<uint16_t*>(pbsm);                       // PF^3
  uint16_t* nxt = head + PF * PF * PF;                                      // PB_CAP
  uint16_t* fidx = nxt + PB_CAP;                                            // PB_CAP
  uint16_t* code = fidx + PB_CAP;                                           // 3*PB_CAP, raw position codes
  __shared__ int64_t cst[PRC];
  __shared__ int cpre[PRC + 1];
  __shared__ int tpre[PB * PB * PB + 1];  // prefix of the brick's own cells (targets)
  const int nb = nc / PB;
  const int bx = blockIdx.x % nb, by = (blockIdx.x / nb) % nb, bz = blockIdx.x / (nb * nb);
  const int x0 = bx * PB - 1, y0 = by * PB - 1, z0 = bz * PB - 1;  // region origin (global coarse, unwrapped)
  if (threadIdx.x < 32) {
    int run = 0;
    for (int base = 0; base < PRC; base += 32) {
      const int q = base + threadIdx.x;
      int cnt = 0;
      if (q < PRC) {
        const int cx = q % PR, cy = (q / PR) % PR, cz = q / (PR * PR);
        const int gx = (x0 + cx + nc) % nc, gy = (y0 + cy + nc) % nc, gz = (z0 + cz + nc) % nc;
        const int64_t c = cube_cell_of(gx, gy, gz, nt, nnt);
        cst[q] = cell_start[c];
        cnt = (int)(cell_start[c + 1] - cst[q]);
      }
      int inc = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)threadIdx.x >= o) inc += v;
      }
      if (q < PRC) cpre[q] = run + inc - cnt;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (threadIdx.x == 0) cpre[PRC] = run;
    __syncwarp();
    // the 64 own cells in (z,y,x) order, two per lane
    int c2[2], n2[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = 2 * threadIdx.x + h;
      const int q = (((t >> 4) + 1) * PR + ((t >> 2) & 3) + 1) * PR + (t & 3) + 1;
      c2[h] = q;
      n2[h] = cpre[q + 1] - cpre[q];
    }
    int inc = n2[0] + n2[1];
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, inc, o);
      if ((int)threadIdx.x >= o) inc += v;
    }
    tpre[2 * threadIdx.x] = inc - n2[0] - n2[1];
    tpre[2 * threadIdx.x + 1] = inc - n2[1];
    if (threadIdx.x == 31) tpre[PB * PB * PB] = inc;
    (void)c2;
  }
  __syncthreads();
  const int M = cpre[PRC];
  if (M > PB_CAP) {  // crowded: handled by the list kernel
    if (threadIdx.x == 0) {
      const unsigned long long q = atomicAdd(&dscal->n_big, 1ull);
      spill[q] = blockIdx.x;
    }
    return;
  }
  for (int i = threadIdx.x; i < PF * PF * PF; i += blockDim.x) head[i] = 0xFFFFu;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    int lo = 0, hi = PRC - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cpre[mid] <= m) lo = mid; else hi = mid - 1;
    }
    const int q = lo;
    const int64_t ip = cst[q] + (m - cpre[q]);
    const int cc[3] = {q % PR, (q / PR) % PR, q / (PR * PR)};
    int f[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int cd = (int)xp[(size_t)d * cap + ip];
      code[3 * m + d] = (uint16_t)cd;
      f[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, cube_xfrac(cd, ZX)));
    }
    fidx[m] = (uint16_t)((f[2] * PF + f[1]) * PF + f[0]);
  }
  __syncthreads();
  // chains: the thread of region cell q inserts q's particles in storage order
  for (int q = threadIdx.x; q < PRC; q += blockDim.x)
    for (int m = cpre[q]; m < cpre[q + 1]; ++m) {
      const int f = fidx[m];
      nxt[m] = head[f];
      head[f] = (uint16_t)m;
    }
  __syncthreads();
  unsigned long long n1 = 0, npair = 0;
  float f2max = 0.f;
  // targets: the particles of the brick's own cells (region cells 1..PB), compacted
  const int T = tpre[PB * PB * PB];
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    int lo = 0, hi = PB * PB * PB - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tpre[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int cc[3] = {(lo & 3) + 1, ((lo >> 2) & 3) + 1, (lo >> 4) + 1};
    const int q = (cc[2] * PR + cc[1]) * PR + cc[0];
    const int m = cpre[q] + (t - tpre[lo]);
    const int64_t ip = cst[q] + (m - cpre[q]);
    double x1[3], v[3], ft[3] = {0.0, 0.0, 0.0};
    int g1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fr = cube_xfrac((int32_t)(int16_t)code[3 * m + d], ZX);
      x1[d] = cube_dadd(4.0 * (double)cc[d], cube_dmul(4.0, fr));
      g1[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, fr));
      const int vc = (int)vp[(size_t)d * cap + ip];
      v[d] = cube_vdecode(__ldg(&tan_table[vc + half_nvbin]), coef);
    }
    ++n1;
    const bool pow2_cut = (nf_cutoff & (nf_cutoff - 1)) == 0;
    const double inv_cut = 1.0 / (double)nf_cutoff;
    for (int kk = g1[2] - pr; kk <= g1[2] + pr; ++kk)
      for (int jj = g1[1] - pr; jj <= g1[1] + pr; ++jj)
        for (int ii = g1[0] - pr; ii <= g1[0] + pr; ++ii) {
          int m2 = head[(kk * PF + jj) * PF + ii];
          const int cf[3] = {ii >> 2, jj >> 2, kk >> 2};
          while (m2 != 0xFFFF) {
            ++npair;
            double x21[3], fp[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const double fr = cube_xfrac((int32_t)(int16_t)code[3 * m2 + d], ZX);
              x21[d] = cube_dsub(cube_dadd(4.0 * (double)cf[d], cube_dmul(4.0, fr)), x1[d]);
            }
            pp_pair(x21, mass, rsoft, nf_cutoff, pow2_cut, inv_cut, fp);
#pragma unroll
            for (int d = 0; d < 3; ++d) ft[d] = cube_dadd(ft[d], fp[d]);
            m2 = nxt[m2];
          }
        }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double k = cube_dmul(ft[d], a_mid);
      k = cube_dmul(k, dt);
      k = cube_ddiv(k, 6.0);
      k = cube_ddiv(k, pi_d);
      v[d] = cube_dadd(v[d], k);
      vp[(size_t)d * cap + ip] = (TV)cube_wrap_code(cube_vencode(&codec, v[d], coef), ZV);
    }
    const double f2 = cube_dadd(cube_dadd(cube_dmul(ft[0], ft[0]), cube_dmul(ft[1], ft[1])), cube_dmul(ft[2], ft[2]));
    f2max = fmaxf(f2max, (float)f2);
  }
  for (int o = 16; o > 0; o >>= 1) {
    n1 += __shfl_xor_sync(0xffffffffu, n1, o);
    npair += __shfl_xor_sync(0xffffffffu, npair, o);
    f2max = fmaxf(f2max, __shfl_xor_sync(0xffffffffu, f2max, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&dscal->itest1, n1);
    atomicAdd(&dscal->npairs, npair);
    atomicMax(&dscal->f2_pp_bits, __float_as_uint(f2max));
  }
}

template <int ZX, int ZV>
int launch_pp(cube_ctx* ctx, const cube_scalars* io) {
  const double coef = cube_vcoef(&ctx->codec, io->sigma_vi);
  if (ctx->nc % PB) {
    ctx->err = "nc must be a multiple of 4 for the PP bricks";
    return CUBE_ERR_PARAM;
  }
  int32_t* spill = ctx->big_list;  // re-bin scratch, free outside update_x
  const int nbricks = (ctx->nc / PB) * (ctx->nc / PB) * (ctx->nc / PB);
  const size_t smem = sizeof(uint16_t) * ((size_t)PF * PF * PF + 5 * (size_t)PB_CAP);
  CUBE_CUDA_TRY(ctx, cudaFuncSetAttribute(k_pp_brick<ZX, ZV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_pp_brick<ZX, ZV><<<nbricks, 256, smem, ctx->stream>>>(
      ctx->xp, ctx->vp, ctx->cell_start, ctx->cap, ctx->nc, ctx->nt, ctx->nnt, ctx->P.pp_range, ctx->P.nf_cutoff,
      (double)ctx->P.rsoft, (double)io->mass_p_cdm, (double)io->a_mid, (double)io->dt, (double)ctx->codec.pi_f,
      ctx->tan_table, ctx->nvbin / 2, ctx->codec, coef, spill, ctx->dscal);
  CUBE_LAUNCH_CHECK(ctx);
  unsigned long long nspill = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&nspill, &ctx->dscal->n_big, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (nspill) {
    uint8_t* sub = reinterpret_cast<uint8_t*>(ctx->tkey);  // re-bin scratch, free outside update_x
    k_pp_subcell<ZX><<<1184, 256, 0, ctx->stream>>>(ctx->xp, ctx->cap, ctx->np, sub);
    CUBE_LAUNCH_CHECK(ctx);
    k_pp<ZX, ZV><<<(unsigned)nspill, 256, 0, ctx->stream>>>(
        ctx->xp, ctx->vp, ctx->cell_start, ctx->cap, ctx->ncells, ctx->nc, ctx->nt, ctx->nnt, ctx->P.pp_range,
        ctx->P.nf_cutoff, (double)ctx->P.rsoft, (double)io->mass_p_cdm, (double)io->a_mid, (double)io->dt,
        (double)ctx->codec.pi_f, ctx->tan_table, ctx->nvbin / 2, ctx->codec, coef, sub, spill, ctx->dscal);
    CUBE_LAUNCH_CHECK(ctx);
  }
  return CUBE_OK;
}

}  // namespace

int cube_pp(cube_ctx* ctx, cube_scalars* io) {
  if (ctx->P.pp_range < 0 || ctx->P.pp_range > 4) {
    ctx->err = "pp_range must be in 0..4";
    return CUBE_ERR_PARAM;
  }
  if (ctx->izipx == 1 && ctx->izipv == 1) return launch_pp<1, 1>(ctx, io);
  if (ctx->izipx == 1 && ctx->izipv == 2) return launch_pp<1, 2>(ctx, io);
  if (ctx->izipx == 2 && ctx->izipv == 1) return launch_pp<2, 1>(ctx, io);
  return launch_pp<2, 2>(ctx, io);
}
