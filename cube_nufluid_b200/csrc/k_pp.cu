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
 * cell.  The GPU walks the coarse cells directly in that order, with the
 * pair arithmetic in FP64 as in the reference (xvec* are real(8)), so the
 * kicked codes are bit-identical to the oracle.  One thread per particle.
 */
#include "cube_internal.cuh"

namespace {

constexpr int PCELLS = 64;

template <int ZX, int ZV>
__global__ void __launch_bounds__(256) k_pp(const void* __restrict__ xp_, void* __restrict__ vp_,
                                            const int64_t* __restrict__ cell_start, int64_t cap, int64_t ncells,
                                            int nc, int nt, int nnt, int pr, int nf_cutoff, double rsoft,
                                            double mass, double a_mid, double dt, double pi_d,
                                            const float* __restrict__ tan_table, int half_nvbin, cube_codec codec,
                                            double coef, DevScal* __restrict__ dscal) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  TV* vp = reinterpret_cast<TV*>(vp_);
  __shared__ int64_t cs[PCELLS + 1];
  const int64_t c0 = (int64_t)blockIdx.x * PCELLS;
  const int ncl = (int)min((int64_t)PCELLS, ncells - c0);
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = cell_start[c0 + i];
  __syncthreads();
  unsigned long long n1 = 0, npair = 0;
  float f2max = 0.f;
  const int nt3 = nt * nt * nt;
  for (int64_t ip = cs[0] + threadIdx.x; ip < cs[ncl]; ip += blockDim.x) {
    int lo = 0, hi = ncl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cs[mid] <= ip) lo = mid; else hi = mid - 1;
    }
    const int64_t c = c0 + lo;
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
          const int64_t c2 = cube_cell_of(gg[0], gg[1], gg[2], nt, nnt);
          const int64_t b0 = cell_start[c2], b1 = cell_start[c2 + 1];
          for (int64_t jp = b1 - 1; jp >= b0; --jp) {
            double x2[3];
            bool inside = true;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + jp], ZX);
              x2[d] = cube_dadd(4.0 * (double)cf[d], cube_dmul(4.0, fr));
              if ((int)floor(x2[d]) + 1 != fc[d]) inside = false;
            }
            if (!inside) continue;
            ++npair;
            double x21[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) x21[d] = cube_dsub(x2[d], x1[d]);
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
  const int64_t blocks = (ctx->ncells + PCELLS - 1) / PCELLS;
  const double coef = cube_vcoef(&ctx->codec, io->sigma_vi);
  k_pp<ZX, ZV><<<(unsigned)blocks, 256, 0, ctx->stream>>>(
      ctx->xp, ctx->vp, ctx->cell_start, ctx->cap, ctx->ncells, ctx->nc, ctx->nt, ctx->nnt, ctx->P.pp_range,
      ctx->P.nf_cutoff, (double)ctx->P.rsoft, (double)io->mass_p_cdm, (double)io->a_mid, (double)io->dt,
      (double)ctx->codec.pi_f, ctx->tan_table, ctx->nvbin / 2, ctx->codec, coef, ctx->dscal);
  CUBE_LAUNCH_CHECK(ctx);
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
