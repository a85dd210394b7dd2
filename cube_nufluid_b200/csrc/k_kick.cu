/*
 * k_kick.cu -- force interpolation and kick of particle_mesh, fine then
 * coarse, fused into one pass over the particles (pm.f90:131-155, :335-372).
 *
 * Per particle and component the arithmetic is the reference's, in its
 * order: decode with sigma_vi, add the eight fine CIC terms
 * force*a_mid*dt/6/pi*dx*dy*dz (FP32 products, FP64 accumulation; the first four
 * factors are the same for every particle reading a node, so the Green multiply of
 * the Poisson solve has applied them to the mesh already), encode
 * with sigma_vi_new; decode that code again with sigma_vi_new, add the
 * eight coarse terms, record |v+vfield| for vmax, encode.  The intermediate
 * quantisation between the two kicks is kept, so the result is bit-identical
 * to running the reference's two loops one after the other; the codes are
 * read and written once.
 *
 * A CTA takes a contiguous range of cells (tile-major order), so the
 * particles it touches are contiguous and the force nodes they read are
 * neighbours in the mesh (served from L1/L2).
 */
#include "cube_internal.cuh"

namespace {

constexpr int KCELLS = 64;  // cells per work item at most (cube_cell_items)

// One thread per particle: the node indices and CIC weights of a particle are
// shared by its three components, which then run their chains (decode, eight
// fine terms, encode, decode, eight coarse terms, encode) one after the other.
// The position arithmetic is FP32: the reference forms the position in FP64
// from exact terms (integer cell, code fraction) and rounds it to FP32 once,
// and the same single rounding of the same exact sum is what the FP32 add gives.
// Decodes read the per-step tables of tan(code)/coef (bit-identical to the
// per-particle FP64 division).  (Staging each 4^3-cell brick's force nodes in
// shared memory first was measured twice as slow: at ~500 particles per brick
// the copies of 17^3 x 3 nodes outweigh the gathers they replace, which hit L1/L2.)
// IT: the index type of a node within one force component, uint32_t when every
// component has fewer than 2^32 elements (one wide multiply-add per gather), else size_t
template <int ZX, int ZV, typename IT>
__global__ void __launch_bounds__(256, 4) k_kick(const void* __restrict__ xp_, void* __restrict__ vp_,
                                              const int64_t* __restrict__ cell_start, const float* __restrict__ vfield,
                                              int64_t cap, int64_t ncells, int nc, int nt, int nnt,
                                              const float* __restrict__ ff, size_t fcomp, int frp, size_t fplane,
                                              const float* __restrict__ fc, size_t ccomp, int crp, size_t cplane,
                                              const double* __restrict__ dec_old, const double* __restrict__ dec_new,
                                              int half_nvbin, cube_codec codec, double coef_new, VencTab tab,
                                              DevScal* __restrict__ dscal, const int64_t* __restrict__ items,
                                              int64_t items_max) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  TV* vp = reinterpret_cast<TV*>(vp_);
  __shared__ int64_t cs[KCELLS + 1];
  __shared__ int cl[KCELLS][3], ctb[KCELLS][3];  // per cell: local coords, tile base
  __shared__ unsigned int vmx_s[3];
  int64_t c0, p0, p1;
  int ncl;
  if (!cube_cell_item(items, ncells, items_max, dscal, c0, ncl, p0, p1)) return;
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = cell_start[c0 + i];
  if (threadIdx.x < ncl) cube_cell_coords(c0 + threadIdx.x, nt, nnt, cl[threadIdx.x], ctb[threadIdx.x]);
  if (threadIdx.x < 3) vmx_s[threadIdx.x] = 0u;
  __syncthreads();
  const int nf = 4 * nc;
  const int npb = (int)(p1 - p0);
  const float xres = ZX == 1 ? 0.00390625f : 1.52587890625e-05f;  // 2^-8, 2^-16
  // reference corner order: 111,211,121,112,122,212,221,222
  const int ox[8] = {0, 1, 0, 0, 0, 1, 1, 1}, oy[8] = {0, 0, 1, 0, 1, 0, 1, 1}, oz[8] = {0, 0, 0, 1, 1, 1, 0, 1};
  float vm[3] = {0.f, 0.f, 0.f};  // per-thread |v+vfield| maxima (non-negative)
  for (int i = threadIdx.x; i < npb; i += blockDim.x) {
    const int64_t ip = p0 + i;
    int lo = 0, hi = ncl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cs[mid] <= ip) lo = mid; else hi = mid - 1;
    }
    const int64_t c = c0 + lo;
    int fi[3][2], gi[3][2];
    float dx1[3], dx2[3], cx1[3], cx2[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int l = cl[lo][e], tb = ctb[lo][e];
      const uint32_t u = (uint32_t)(int32_t)xp[(size_t)e * cap + ip] & (ZX == 1 ? 0xFFu : 0xFFFFu);
      const float fr = __fmul_rn((float)u + 0.5f, xres);                  // exact
      const float tf = __fadd_rn(4.f * (float)l, __fmul_rn(4.f, fr));   // RN(4l + 4 fr)
      const float f = floorf(tf) + 1.f;
      dx1[e] = cube_fsub(f, tf);
      dx2[e] = cube_fsub(1.f, dx1[e]);
      const int n1 = 4 * tb + (int)f - 1;  // global fine node of idx1 (0-based), <= nf
      fi[e][0] = cube_wrap(n1, nf);
      fi[e][1] = cube_wrap(n1 + 1, nf);
      const float tc = __fadd_rn((float)(tb + l) - 0.5f, fr);            // RN(cell + fr - 1/2)
      const float ci = floorf(tc) + 1.f;
      cx1[e] = cube_fsub(ci, tc);
      cx2[e] = cube_fsub(1.f, cx1[e]);
      const int m1 = (int)ci - 1;  // global coarse node of idx1, may be -1
      gi[e][0] = cube_wrap(m1, nc);
      gi[e][1] = cube_wrap(m1 + 1, nc);
    }
    // the eight fine and eight coarse node indices, shared by the three components
    IT fo[8], go[8];
    {
      const IT fz[2] = {(IT)fi[2][0] * (IT)fplane, (IT)fi[2][1] * (IT)fplane};
      const IT gz[2] = {(IT)gi[2][0] * (IT)cplane, (IT)gi[2][1] * (IT)cplane};
      const int fy[2] = {fi[1][0] * frp, fi[1][1] * frp}, gy[2] = {gi[1][0] * crp, gi[1][1] * crp};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        fo[k] = fz[oz[k]] + (IT)(fy[oy[k]] + fi[0][ox[k]]);
        go[k] = gz[oz[k]] + (IT)(gy[oy[k]] + gi[0][ox[k]]);
      }
    }
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
      const float* F = ff + d * fcomp;
      const float* G = fc + d * ccomp;
      const int code = (int)vp[(size_t)d * cap + ip];
      float fv[8], gv[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        fv[k] = __ldg(&F[fo[k]]);
        gv[k] = __ldg(&G[go[k]]);
      }
      const float vf = __ldg(&vfield[(size_t)d * ncells + c]);
      double v = __ldg(&dec_old[code + half_nvbin]);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float q = fv[k];  // force*a_mid*dt/6/pi of the node, applied by the Green multiply
        q = cube_fmul(q, ox[k] ? dx2[0] : dx1[0]);
        q = cube_fmul(q, oy[k] ? dx2[1] : dx1[1]);
        q = cube_fmul(q, oz[k] ? dx2[2] : dx1[2]);
        v = cube_dadd(v, (double)q);
      }
      const int code1 = cube_wrap_code(cube_vencode_step(&codec, tab, v, coef_new), ZV);
      v = __ldg(&dec_new[code1 + half_nvbin]);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float q = gv[k];
        q = cube_fmul(q, ox[k] ? cx2[0] : cx1[0]);
        q = cube_fmul(q, oy[k] ? cx2[1] : cx1[1]);
        q = cube_fmul(q, oz[k] ? cx2[2] : cx1[2]);
        v = cube_dadd(v, (double)q);
      }
      const float am = (float)fabs(cube_dadd(v, (double)vf));
      vm[0] = (d == 0) ? fmaxf(vm[0], am) : vm[0];
      vm[1] = (d == 1) ? fmaxf(vm[1], am) : vm[1];
      vm[2] = (d == 2) ? fmaxf(vm[2], am) : vm[2];
      vp[(size_t)d * cap + ip] = (TV)cube_wrap_code(cube_vencode_step(&codec, tab, v, coef_new), ZV);
    }
  }
  // every thread reaches here: warp maxima, then one shared atomic per warp and component
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const unsigned int w = __reduce_max_sync(0xffffffffu, __float_as_uint(vm[e]));
    if ((threadIdx.x & 31) == 0 && w) atomicMax(&vmx_s[e], w);
  }
  __syncthreads();
  if (threadIdx.x < 3) atomicMax(&dscal->vmax_bits[threadIdx.x], vmx_s[threadIdx.x]);
}

// The kick of the FP64 Poisson mode: the same per-particle steps on FP64 force
// meshes (kick increments formed in FP64 by the Green multiply), with the CIC
// weights and the products force*dx*dy*dz in FP64 (the positions are exact in
// FP64).  The velocity codec, its tables and the intermediate quantisation are the
// FP32 path's, so the two runs differ only in the mesh arithmetic.
template <int ZX, int ZV>
__global__ void __launch_bounds__(256, 3) k_kick64(const void* __restrict__ xp_, void* __restrict__ vp_,
                                                const int64_t* __restrict__ cell_start, const float* __restrict__ vfield,
                                                int64_t cap, int64_t ncells, int nc, int nt, int nnt,
                                                const double* __restrict__ ff, size_t fcomp, int frp, size_t fplane,
                                                const double* __restrict__ fc, size_t ccomp, int crp, size_t cplane,
                                                const double* __restrict__ dec_old, const double* __restrict__ dec_new,
                                                int half_nvbin, cube_codec codec, double coef_new, VencTab tab,
                                                DevScal* __restrict__ dscal, const int64_t* __restrict__ items,
                                                int64_t items_max) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  TV* vp = reinterpret_cast<TV*>(vp_);
  __shared__ int64_t cs[KCELLS + 1];
  __shared__ int cl[KCELLS][3], ctb[KCELLS][3];
  __shared__ unsigned int vmx_s[3];
  int64_t c0, p0, p1;
  int ncl;
  if (!cube_cell_item(items, ncells, items_max, dscal, c0, ncl, p0, p1)) return;
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = cell_start[c0 + i];
  if (threadIdx.x < ncl) cube_cell_coords(c0 + threadIdx.x, nt, nnt, cl[threadIdx.x], ctb[threadIdx.x]);
  if (threadIdx.x < 3) vmx_s[threadIdx.x] = 0u;
  __syncthreads();
  const int nf = 4 * nc;
  const int npb = (int)(p1 - p0);
  const int ox[8] = {0, 1, 0, 0, 0, 1, 1, 1}, oy[8] = {0, 0, 1, 0, 1, 0, 1, 1}, oz[8] = {0, 0, 0, 1, 1, 1, 0, 1};
  float vm[3] = {0.f, 0.f, 0.f};
  for (int i = threadIdx.x; i < npb; i += blockDim.x) {
    const int64_t ip = p0 + i;
    int lo = 0, hi = ncl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cs[mid] <= ip) lo = mid; else hi = mid - 1;
    }
    const int64_t c = c0 + lo;
    int fi[3][2], gi[3][2];
    double dx1[3], dx2[3], cx1[3], cx2[3];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int l = cl[lo][e], tb = ctb[lo][e];
      const double fr = cube_xfrac((int32_t)xp[(size_t)e * cap + ip], ZX);
      const double tf = 4.0 * (double)l + 4.0 * fr;  // exact
      const double f = floor(tf) + 1.0;
      dx1[e] = f - tf;
      dx2[e] = 1.0 - dx1[e];
      const int n1 = 4 * tb + (int)f - 1;
      fi[e][0] = cube_wrap(n1, nf);
      fi[e][1] = cube_wrap(n1 + 1, nf);
      const double tc = ((double)(tb + l) - 0.5) + fr;  // exact
      const double ci = floor(tc) + 1.0;
      cx1[e] = ci - tc;
      cx2[e] = 1.0 - cx1[e];
      const int m1 = (int)ci - 1;
      gi[e][0] = cube_wrap(m1, nc);
      gi[e][1] = cube_wrap(m1 + 1, nc);
    }
    const size_t fz[2] = {(size_t)fi[2][0] * fplane, (size_t)fi[2][1] * fplane};
    const size_t gz[2] = {(size_t)gi[2][0] * cplane, (size_t)gi[2][1] * cplane};
    const int fy[2] = {fi[1][0] * frp, fi[1][1] * frp}, gy[2] = {gi[1][0] * crp, gi[1][1] * crp};
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
      const double* F = ff + d * fcomp;
      const double* G = fc + d * ccomp;
      const int code = (int)vp[(size_t)d * cap + ip];
      const float vf = __ldg(&vfield[(size_t)d * ncells + c]);
      double v = __ldg(&dec_old[code + half_nvbin]);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double q = __ldg(&F[fz[oz[k]] + (size_t)(fy[oy[k]] + fi[0][ox[k]])]);
        v += ((q * (ox[k] ? dx2[0] : dx1[0])) * (oy[k] ? dx2[1] : dx1[1])) * (oz[k] ? dx2[2] : dx1[2]);
      }
      const int code1 = cube_wrap_code(cube_vencode_step(&codec, tab, v, coef_new), ZV);
      v = __ldg(&dec_new[code1 + half_nvbin]);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double q = __ldg(&G[gz[oz[k]] + (size_t)(gy[oy[k]] + gi[0][ox[k]])]);
        v += ((q * (ox[k] ? cx2[0] : cx1[0])) * (oy[k] ? cx2[1] : cx1[1])) * (oz[k] ? cx2[2] : cx1[2]);
      }
      const float am = (float)fabs(v + (double)vf);
      vm[d] = fmaxf(vm[d], am);
      vp[(size_t)d * cap + ip] = (TV)cube_wrap_code(cube_vencode_step(&codec, tab, v, coef_new), ZV);
    }
  }
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const unsigned int w = __reduce_max_sync(0xffffffffu, __float_as_uint(vm[e]));
    if ((threadIdx.x & 31) == 0 && w) atomicMax(&vmx_s[e], w);
  }
  __syncthreads();
  if (threadIdx.x < 3) atomicMax(&dscal->vmax_bits[threadIdx.x], vmx_s[threadIdx.x]);
}

template <int ZX, int ZV>
int launch_kick(cube_ctx* ctx, const cube_scalars* io) {
  // work items of at most 64 cells and 4096 particles, so that the blocks over
  // crowded cells take no longer than the others
  int64_t blocks = 0;
  if (int irc = cube_cell_items(ctx, ctx->cell_start, &blocks)) return irc;
  const double coef_old = cube_vcoef(&ctx->codec, io->sigma_vi);
  const double coef_new = cube_vcoef(&ctx->codec, io->sigma_vi_new);
  int rc;
  const double* dec_old = cube_vdec_table(ctx, coef_old, &rc);
  if (rc) return rc;
  const double* dec_new = cube_vdec_table(ctx, coef_new, &rc);
  if (rc) return rc;
  MeshLevel& F = ctx->fine;
  MeshLevel& Cc = ctx->coarse;
  if (F.fp64) {
    k_kick64<ZX, ZV><<<(unsigned)blocks, 256, 0, ctx->stream>>>(
        ctx->xp, ctx->vp, ctx->cell_start, ctx->vfield, ctx->cap, ctx->ncells, ctx->nc, ctx->nt, ctx->nnt,
        reinterpret_cast<const double*>(F.force), (size_t)F.n * F.plane, F.rp, F.plane,
        reinterpret_cast<const double*>(Cc.force), (size_t)Cc.n * Cc.plane, Cc.rp, Cc.plane, dec_old, dec_new,
        ctx->nvbin / 2, ctx->codec, coef_new, cube_venc_tab(ctx), ctx->dscal, ctx->rebin_items,
        cube_rebin_items_max(ctx->ncells, ctx->cap));
    CUBE_LAUNCH_CHECK(ctx);
    return CUBE_OK;
  }
  auto kk = (size_t)F.n * F.plane < (size_t(1) << 32) ? k_kick<ZX, ZV, uint32_t> : k_kick<ZX, ZV, size_t>;
  kk<<<(unsigned)blocks, 256, 0, ctx->stream>>>(
      ctx->xp, ctx->vp, ctx->cell_start, ctx->vfield, ctx->cap, ctx->ncells, ctx->nc, ctx->nt, ctx->nnt, F.force,
      (size_t)F.n * F.plane, F.rp, F.plane, Cc.force, (size_t)Cc.n * Cc.plane, Cc.rp, Cc.plane, dec_old, dec_new,
      ctx->nvbin / 2, ctx->codec, coef_new, cube_venc_tab(ctx), ctx->dscal, ctx->rebin_items,
      cube_rebin_items_max(ctx->ncells, ctx->cap));
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

}  // namespace

int cube_kick(cube_ctx* ctx, cube_scalars* io) {
  if (ctx->izipx == 1 && ctx->izipv == 1) return launch_kick<1, 1>(ctx, io);
  if (ctx->izipx == 1 && ctx->izipv == 2) return launch_kick<1, 2>(ctx, io);
  if (ctx->izipx == 2 && ctx->izipv == 1) return launch_kick<2, 1>(ctx, io);
  return launch_kick<2, 2>(ctx, io);
}
