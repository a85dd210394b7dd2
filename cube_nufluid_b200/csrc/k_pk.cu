/*
 * k_pk.cu -- power spectrum of the resident state on the fine mesh, the
 * analysis CUBE's utilities run on a checkpoint (cicpower.f90:84-255 with
 * powerspectrum.f90:27-137, built with FFTFINE: ng = nf):
 *
 *   - CIC of the particles with unit mass on ng^3 nodes centred in the fine
 *     cells: pos = (global coarse position)*ng/nc - 1/2 (cicpower.f90:104-107);
 *   - delta_c = rho/mean(rho) - 1 (:150-163); with fluid neutrinos,
 *     delta_nu = sum_k w_k rho_k((n+1/2)) - 1 at fine node n (:199-214);
 *   - forward r2c of both, modes binned by nint(|k|) (linear_kbin, the
 *     reference's default) or 4 per octave from 0.95 (its alternative), with the
 *     CIC window sinc^4 divided out, Delta^2 = |c|^2 4 pi k^3 (:58-92);
 *   - per bin: count, mean k, the two auto powers, the cross power, the two
 *     kernels, r, b and the reconstruction line (:124-135).
 *
 * The deposit is the library's 64-bit fixed point (order-independent); the bin
 * sums are FP64 (the reference's are FP32), added per CTA in shared memory and
 * then across CTAs with FP64 atomics, so a bin can differ between runs in the
 * last bits of its FP64 sum.  Scratch: the fine density and force meshes, which
 * are free outside cube_particle_mesh.
 */
#include "cube_internal.cuh"

namespace {

constexpr int PKCELLS = 64;
constexpr double FIX = 4294967296.0;

template <int ZX>
__global__ void __launch_bounds__(256) k_pk_deposit(const void* __restrict__ xp_, const int64_t* __restrict__ cell_start,
                                                   int64_t cap, int64_t ncells, int nt, int nnt, int nc, int ng,
                                                   unsigned long long* __restrict__ acc) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  __shared__ int64_t cs[PKCELLS + 1];
  __shared__ int cg[PKCELLS][3];  // global coarse cell of each cell of the CTA
  const int64_t c0 = (int64_t)blockIdx.x * PKCELLS;
  const int ncl = (int)min((int64_t)PKCELLS, ncells - c0);
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = cell_start[c0 + i];
  if (threadIdx.x < ncl) {
    int l[3], tb[3];
    cube_cell_coords(c0 + threadIdx.x, nt, nnt, l, tb);
    for (int d = 0; d < 3; ++d) cg[threadIdx.x][d] = tb[d] + l[d];
  }
  __syncthreads();
  const float scale = (float)ng, cnc = (float)nc;
  for (int64_t ip = cs[0] + threadIdx.x; ip < cs[ncl]; ip += blockDim.x) {
    int lo = 0, hi = ncl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cs[mid] <= ip) lo = mid; else hi = mid - 1;
    }
    int i0[3];
    float w1[3], w2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      // pos1 = nt*(it-1)+(i-1)+frac (FP64 -> real(4)), then pos1*real(ng)/real(nc) - 0.5
      float p = (float)cube_dadd((double)cg[lo][d], cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX));
      p = cube_fsub(cube_fdiv(cube_fmul(p, scale), cnc), 0.5f);
      const float f = floorf(p);
      w1[d] = cube_fsub(f + 1.f, p);  // dx1 = idx1 - pos1, idx1 = floor(pos1)+1
      w2[d] = cube_fsub(1.f, w1[d]);
      i0[d] = (int)f;  // 0-based node of idx1 (may be -1: the buffer sync folds it back)
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const float w = cube_fmul(cube_fmul(ox ? w2[0] : w1[0], oy ? w2[1] : w1[1]), oz ? w2[2] : w1[2]);
      const int gx = cube_wrap(i0[0] + ox, ng), gy = cube_wrap(i0[1] + oy, ng), gz = cube_wrap(i0[2] + oz, ng);
      atomicAdd(&acc[((size_t)gz * ng + gy) * ng + gx], (unsigned long long)__double2ll_rn((double)w * FIX));
    }
  }
}

// delta_c = rho/(sum/ng^3) - 1 into the pitched mesh
__global__ void k_pk_delta(const unsigned long long* __restrict__ acc, int ng, double mean, float* __restrict__ out,
                           int rp) {
  const int64_t tot = (int64_t)ng * ng * ng;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % ng);
    const int64_t row = i / ng;
    const float rho = (float)((double)acc[i] * (1.0 / FIX));  // rho_c is real(4)
    out[row * rp + x] = (float)((double)rho / mean - 1.0);
  }
}

struct Rho3 {
  const float* r[3];
  int n[3];
  float dx[3], w[3];
};

// delta_nu = dfld_density(n + 1/2) - 1 at fine node n (cicpower.f90:201-214)
__global__ void k_pk_delta_nu(Rho3 F, int ng, float* __restrict__ out, int rp) {
  const int64_t tot = (int64_t)ng * ng * ng;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % ng);
    const int64_t row = i / ng;
    const int y = (int)(row % ng), z = (int)(row / ng);
    const int q[3] = {x, y, z};
    float den = 0.f;
    for (int k = 0; k < 3; ++k) {
      const int n = F.n[k];
      int i0[3], i1[3];
      float d1[3], d2[3];
      for (int e = 0; e < 3; ++e) {
        const float xx = cube_fsub(cube_fmul(cube_fadd((float)q[e], 0.5f), 1.f / F.dx[k]), 0.5f);
        const int lo = (int)floorf(xx);
        d1[e] = cube_fsub((float)(lo + 1), xx);
        d2[e] = cube_fsub(1.f, d1[e]);
        i0[e] = cube_wrap(lo, n);
        i1[e] = cube_wrap(lo + 1, n);
      }
      float d = 0.f;
      for (int c = 0; c < 8; ++c) {
        const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
        const float f = __ldg(&F.r[k][((size_t)(oz ? i1[2] : i0[2]) * n + (oy ? i1[1] : i0[1])) * n + (ox ? i1[0] : i0[0])]);
        const float t = cube_fmul(cube_fmul(cube_fmul(f, ox ? d2[0] : d1[0]), oy ? d2[1] : d1[1]), oz ? d2[2] : d1[2]);
        d = (c == 0) ? t : cube_fadd(d, t);
      }
      den = cube_fadd(den, cube_fmul(F.w[k], d));
    }
    out[row * rp + x] = (float)((double)den - 1.0);
  }
}

// bins: [0] count, [1] sum k, [2] amp11, [3] amp22, [4] amp12, [5] 1/sinc^2, [6] 1/sinc^4
constexpr int NQ = 7;

__global__ void __launch_bounds__(256) k_pk_bin(const float2* __restrict__ c1, const float2* __restrict__ c2, int has2,
                                               int ng, int cp, int kx_major, int nbin, int logbins, float norm,
                                               double* __restrict__ gbins) {
  extern __shared__ double sb[];  // NQ * (nbin + 1)
  for (int i = threadIdx.x; i < NQ * (nbin + 1); i += blockDim.x) sb[i] = 0.0;
  __syncthreads();
  const int nyq = ng / 2, nh = nyq + 1;
  const float pi_f = 4.f * atanf(1.f);
  const int64_t tot = (int64_t)ng * ng * nh;
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < tot; m += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(m % nh);
    const int64_t jk = m / nh;
    const int j = (int)(jk % ng), k = (int)(jk / ng);
    // 1-based ig, jg, kg of the reference; skip the zero mode and the redundant
    // half of the kx = 0 and kx = nyquist planes (powerspectrum.f90:64-66)
    const int ig = i + 1, jg = j + 1, kg = k + 1;
    if (ig == 1 && jg == 1 && kg == 1) continue;
    if ((ig == 1 || ig == nyq + 1) && jg > nyq + 1) continue;
    if ((ig == 1 || ig == nyq + 1) && (jg == 1 || jg == nyq + 1) && kg > nyq + 1) continue;
    const float kx = (float)((ig + nyq - 1) % ng - nyq), ky = (float)((jg + nyq - 1) % ng - nyq),
                kz = (float)((kg + nyq - 1) % ng - nyq);
    const float kr = sqrtf(kx * kx + ky * ky + kz * kz);
    auto snc = [&](float kk) { return kk == 0.f ? 1.f : sinf(pi_f * kk / (float)ng) / (pi_f * kk / (float)ng); };
    const float sinc = snc(kx) * snc(ky) * snc(kz);
    int ib;
    if (logbins) {
      const float rb = 4.f / logf(2.f) * logf(kr / 0.95f);
      ib = rb < 1.f ? (int)ceilf(rb) : (int)floorf(rb);
    } else {
      ib = (int)roundf(kr);  // Fortran nint: halves away from zero
    }
    if (ib < 0 || ib > nbin) continue;
    // spectrum layout: [kz][ky][kx] at row pitch cp, or [kx][ky][kz] dense (kx_major)
    const size_t o = kx_major ? ((size_t)i * ng + j) * ng + k : (size_t)k * ng * cp + (size_t)j * cp + i;
    const float2 a = c1[o];
    const float ax = a.x * norm, ay = a.y * norm;
    // real(c*conjg(c))/(sinc**4.0)*4*pi*kr**3, left to right
    const float s4 = powf(sinc, 4.f);
    const float k3 = (kr * kr) * kr;
    auto amp = [&](float re) { return (((re / s4) * 4.f) * pi_f) * k3; };
    const float p11 = amp(ax * ax + ay * ay);
    float p22 = 0.f, p12 = 0.f;
    if (has2) {
      const float2 b = c2[o];
      const float bx = b.x * norm, by = b.y * norm;
      p22 = amp(bx * bx + by * by);
      p12 = amp(ax * bx + ay * by);
    }
    double* B = sb + ib;
    atomicAdd(&B[0 * (nbin + 1)], 1.0);
    atomicAdd(&B[1 * (nbin + 1)], (double)kr);
    atomicAdd(&B[2 * (nbin + 1)], (double)p11);
    atomicAdd(&B[3 * (nbin + 1)], (double)p22);
    atomicAdd(&B[4 * (nbin + 1)], (double)p12);
    atomicAdd(&B[5 * (nbin + 1)], 1.0 / ((double)sinc * sinc));
    atomicAdd(&B[6 * (nbin + 1)], 1.0 / (double)s4);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < NQ * (nbin + 1); i += blockDim.x)
    if (sb[i] != 0.0) atomicAdd(&gbins[i], sb[i]);
}

}  // namespace

// number of bins of powerspectrum.f90:11-16 for a mesh of ng per side
int cube_pk_nbin(int ng, int logbins) {
  const float nyq = (float)(ng / 2);
  if (logbins) return (int)floorf(4.f * logf(nyq * sqrtf(3.f) / 0.95f) / logf(2.f));
  return (int)lrintf(nyq * sqrtf(3.f));
}

int cube_power_spectrum_dev(cube_ctx* ctx, int logbins, std::vector<double>& bins, int* nbin_out) {
  MeshLevel& L = ctx->fine;
  const int ng = L.n;
  const int nbin = cube_pk_nbin(ng, logbins);
  *nbin_out = nbin;
  const int64_t n3 = (int64_t)ng * ng * ng;
  // scratch: int64 accumulator over force components 0-1, delta_c in rho, delta_nu in component 2
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(L.force);
  float* dnu = L.force + 2 * (size_t)ng * L.plane;
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(acc, 0, 8 * (size_t)n3, ctx->stream));
  const int64_t blocks = (ctx->ncells + PKCELLS - 1) / PKCELLS;
  if (ctx->izipx == 1)
    k_pk_deposit<1><<<(unsigned)blocks, 256, 0, ctx->stream>>>(ctx->xp, ctx->cell_start, ctx->cap, ctx->ncells,
                                                              ctx->nt, ctx->nnt, ctx->nc, ng, acc);
  else
    k_pk_deposit<2><<<(unsigned)blocks, 256, 0, ctx->stream>>>(ctx->xp, ctx->cell_start, ctx->cap, ctx->ncells,
                                                              ctx->nt, ctx->nnt, ctx->nc, ng, acc);
  CUBE_LAUNCH_CHECK(ctx);
  // mean density: every particle deposits its unit mass (to the fixed point's rounding)
  const double mean = (double)ctx->np / (double)n3;
  const int g = ctx->num_sms * 8;
  k_pk_delta<<<g, 256, 0, ctx->stream>>>(acc, ng, mean, L.rho, L.rp);
  CUBE_LAUNCH_CHECK(ctx);
  const int has2 = ctx->nu.on ? 1 : 0;
  if (has2) {
    Rho3 R;
    for (int k = 0; k < 3; ++k) {
      R.r[k] = ctx->nu.fl[k].a[0];
      R.n[k] = ctx->nu.fl[k].n;
      R.dx[k] = ctx->nu.fl[k].dx;
      R.w[k] = ctx->nu.dwgts[k];
    }
    k_pk_delta_nu<<<g, 256, 0, ctx->stream>>>(R, ng, dnu, L.rp);
    CUBE_LAUNCH_CHECK(ctx);
  }
  int kxm = 0, kxm2 = 0;
  int rc = cube_fft_forward3(ctx, L, L.rho, &kxm);
  if (rc) return rc;
  if (has2 && (rc = cube_fft_forward3(ctx, L, dnu, &kxm2))) return rc;
  double* gb = ctx->pk_bins;  // NQ * (nbin_max + 1), allocated by cube_create
  const size_t nb = (size_t)NQ * (nbin + 1);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(gb, 0, 8 * nb, ctx->stream));
  const size_t smem = 8 * nb;
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_pk_bin, smem));
  const float norm = (float)(1.0 / ((double)ng * ng * ng));
  k_pk_bin<<<ctx->num_sms * 2, 256, smem, ctx->stream>>>(reinterpret_cast<const float2*>(L.rho),
                                                        reinterpret_cast<const float2*>(dnu), has2, ng, L.cp, kxm, nbin,
                                                        logbins, norm, gb);
  CUBE_LAUNCH_CHECK(ctx);
  bins.assign(nb, 0.0);
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(bins.data(), gb, 8 * nb, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return CUBE_OK;
}
