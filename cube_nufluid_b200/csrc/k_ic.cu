/*
 * k_ic.cu -- Zel'dovich initial conditions generated on the device, the state a
 * CUBE run starts from (initial_conditions.f90:268-900 produces it on the host
 * and writes checkpoint files; here it lands directly in the context).
 *
 *   noise      Philox4x32-10 (Salmon et al. 2011) uniforms, word i of the grid =
 *              output word i mod 4 of counter (i div 4, 0, 0) with the seed as key,
 *              (w >> 8) * 2^-24, through the reference's Box-Muller pairing along x
 *              (initial_conditions.f90:320-336); the host generator in ic.py draws
 *              the same uniforms;
 *   displacement psi_d = IFFT( i k_d / k^2 * amp(k) * FFT(noise) ) on the particle
 *              grid (npd = np_nc*nc per side), amp^2 = Delta^2(k)/(4 pi) (npd/k)^3 with
 *              the Eisenstein-Hu no-wiggle transfer, sigma8 normalisation and growth
 *              passed in by the host; evaluated with the library's Poisson passes and
 *              a "Green" octant K_d = amp k_d / k^2 (odd in k_d, zero on its Nyquist
 *              plane);
 *   particles  lattice q = i/np_nc + 1/(2 ncell) (coarse units), x = q + psi/np_nc,
 *              v = psi/np_nc * ncell * vf; sorted by tile-major cell, in lattice
 *              order inside a cell; PID = 1 + the fine-mesh index of the lattice
 *              point, iq = (ncell/np_nc)*lattice index per dimension (:834-836); per cell the mean
 *              velocity (vfield), the residuals' dispersion sigma_vi, and the codes
 *              (initial_conditions.f90:797-838).
 */
#include "cube_internal.cuh"

namespace {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// one thread per pair of x-neighbours: Box-Muller of (u_even, u_odd) into the mesh
__global__ void k_ic_noise(float* __restrict__ rho, int n, int rp, uint32_t k0, uint32_t k1, float pi_f) {
  const int64_t pairs = (int64_t)n * n * n / 2;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < pairs; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = 2 * p;  // even word of the pair, same Philox block
    uint32_t c[4] = {(uint32_t)(i >> 2), (uint32_t)((uint64_t)(i >> 2) >> 32), 0u, 0u};
    philox4x32_10(c, k0, k1);
    const bool w = (i & 3) != 0;  // 0 or 2
    const uint32_t w0 = w ? c[2] : c[0], w1 = w ? c[3] : c[1];
    const float u0 = (float)(w0 >> 8) * 0x1p-24f, u1 = (float)(w1 >> 8) * 0x1p-24f;
    const float theta = (2.f * pi_f) * u0;
    const float r = sqrtf(-2.f * logf(1.f - u1));
    float sn, cs;
    sincosf(theta, &sn, &cs);
    const int x = (int)(i % n);
    const int64_t row = i / n;
    rho[row * rp + x] = r * cs;
    rho[row * rp + x + 1] = r * sn;
  }
}

struct IcSpec {
  double norm_d2, n_s, h, eh_s, eh_alpha, eh_omh, eh_theta2;
  double box, amplitude;
  int npd;
};

__device__ double eh_nowiggle(double k_hmpc, const IcSpec& S) {
  const double k_mpc = k_hmpc * S.h;
  const double x = 0.43 * k_mpc * S.eh_s;
  const double gamma = S.eh_omh * (S.eh_alpha + (1.0 - S.eh_alpha) / (1.0 + x * x * x * x));
  const double q = k_hmpc * S.eh_theta2 / gamma;
  const double l0 = log(2.0 * 2.718281828459045 + 1.8 * q);
  const double c0 = 14.2 + 731.0 / (1.0 + 62.5 * q);
  return l0 / (l0 + c0 * q * q);
}

// Zel'dovich "Green" octant [d][ky][kx][kz] (kz fastest), (n/2+1)^3 per component,
// with 1/n^3 folded in like the force kernels
__global__ void k_ic_kernel(float* __restrict__ kern, IcSpec S) {
  const int n = S.npd, nh = n / 2, kp = nh + 1;
  const int64_t tot = (int64_t)kp * kp * kp;
  const float kgrid = (float)(2.0 * 3.14159265358979323846 / n);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int kz = (int)(i % kp);
    const int64_t r = i / kp;
    const int kx = (int)(r % kp), ky = (int)(r / kp);
    const float kr2 = (float)kx * kx + (float)ky * ky + (float)kz * kz;
    const float kr = sqrtf(fmaxf(kr2, 1.f));
    const double kphys = 2.0 * 3.14159265358979323846 * (double)kr / S.box;
    const double t = eh_nowiggle(kphys, S);
    const float d2 = (float)(S.norm_d2 * t * t * pow(kphys, 3.0 + S.n_s));
    const float nk = (float)n / kr;
    const float amp = sqrtf(d2 / (float)(4.0 * 3.14159265358979323846) * nk) * nk * (float)S.amplitude;
    const float inv = kr2 > 0.f ? 1.f / (kgrid * kgrid * kr2) : 0.f;
    const float norm = 1.f / ((float)n * (float)n * (float)n);
    const int kd[3] = {kx, ky, kz};
    for (int d = 0; d < 3; ++d) {
      float v = (kd[d] == nh) ? 0.f : kgrid * (float)kd[d] * inv * amp * norm;
      kern[(size_t)d * tot + ((size_t)ky * kp + kx) * kp + kz] = v;
    }
  }
}

struct PartArgs {
  const float* psi;   // three displacement meshes, component stride cstride, pitch rp
  size_t cstride;
  int rp, npd, np_nc, ncell, nc, nt, nnt;
  double vf;
};

// lattice point -> cell (tile-major) and counts
__global__ void k_ic_cells(PartArgs A, int32_t* __restrict__ cell, int32_t* __restrict__ cnt) {
  const int n = A.npd;
  const int64_t tot = (int64_t)n * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int q[3] = {(int)(i % n), (int)((i / n) % n), (int)(i / ((int64_t)n * n))};
    const size_t o = ((size_t)q[2] * n + q[1]) * A.rp + q[0];
    int g[3];
    for (int d = 0; d < 3; ++d) {
      const double psi = (double)A.psi[d * A.cstride + o];
      double x = (double)q[d] / A.np_nc + 0.5 / A.ncell + psi / A.np_nc;
      x = fmod(x, (double)A.nc);
      if (x < 0.0) x += (double)A.nc;
      int gg = (int)ceil(x) - 1;  // ic.pack: ceil(x) - 1 mod nc
      gg = cube_wrap(gg, A.nc);
      g[d] = gg;
    }
    const int32_t c = (int32_t)cube_cell_of(g[0], g[1], g[2], A.nt, A.nnt);
    cell[i] = c;
    atomicAdd(&cnt[c], 1);
  }
}

__global__ void k_ic_place(const int32_t* __restrict__ cell, const int64_t* __restrict__ start,
                           int32_t* __restrict__ cursor, int32_t* __restrict__ perm, int64_t tot) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = cell[i];
    perm[start[c] + atomicAdd(&cursor[c], 1)] = (int32_t)i;
  }
}

__device__ __forceinline__ void lattice_state(const PartArgs& A, int64_t i, double x[3], double v[3]) {
  const int n = A.npd;
  const int q[3] = {(int)(i % n), (int)((i / n) % n), (int)(i / ((int64_t)n * n))};
  const size_t o = ((size_t)q[2] * n + q[1]) * A.rp + q[0];
  for (int d = 0; d < 3; ++d) {
    const double dsp = (double)A.psi[d * A.cstride + o] / A.np_nc;
    double xx = (double)q[d] / A.np_nc + 0.5 / A.ncell + dsp;
    xx = fmod(xx, (double)A.nc);
    if (xx < 0.0) xx += (double)A.nc;
    x[d] = xx;
    v[d] = dsp * (A.ncell * A.vf);
  }
}

// per cell: lattice order inside the cell (insertion sort; larger cells were
// sorted by k_ic_sort_big), mean velocity (FP64 in order), residual |v|^2 sum
__global__ void k_ic_cellsum(PartArgs A, const int64_t* __restrict__ start, int32_t* __restrict__ perm,
                             float* __restrict__ vfield, double* __restrict__ res2, int64_t ncells) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = start[c], e = start[c + 1];
    if (e - b <= 64)
      for (int64_t s = b + 1; s < e; ++s) {  // ascending lattice index
        const int32_t key = perm[s];
        int64_t t = s - 1;
        while (t >= b && perm[t] > key) { perm[t + 1] = perm[t]; --t; }
        perm[t + 1] = key;
      }
    double sv[3] = {0.0, 0.0, 0.0};
    for (int64_t s = b; s < e; ++s) {
      double x[3], v[3];
      lattice_state(A, perm[s], x, v);
      for (int d = 0; d < 3; ++d) sv[d] += v[d];
    }
    const double nn = (double)(e - b > 0 ? e - b : 1);
    float vf[3];
    for (int d = 0; d < 3; ++d) {
      vf[d] = (float)(sv[d] / nn);
      vfield[(size_t)d * ncells + c] = vf[d];
    }
    double r2 = 0.0;
    for (int64_t s = b; s < e; ++s) {
      double x[3], v[3];
      lattice_state(A, perm[s], x, v);
      for (int d = 0; d < 3; ++d) {
        const double r = v[d] - (double)vf[d];
        r2 += r * r;
      }
    }
    res2[c] = r2;
  }
}

// cells above 64 particles: bitonic sort of the lattice indices in shared memory (<= 4096)
__global__ void k_ic_sort_big(const int64_t* __restrict__ start, int32_t* __restrict__ perm, int64_t ncells,
                              DevScal* __restrict__ dscal) {
  __shared__ int32_t buf[4096];
  for (int64_t c = blockIdx.x; c < ncells; c += gridDim.x) {
    const int64_t b = start[c], e = start[c + 1];
    const int m = (int)(e - b);
    if (m <= 64) continue;
    if (m > 4096) {
      if (threadIdx.x == 0) cube_dev_error(dscal, CUBE_ERR_CELL, (int)c);
      continue;
    }
    int p2 = 1;
    while (p2 < m) p2 <<= 1;
    for (int i = threadIdx.x; i < p2; i += blockDim.x) buf[i] = i < m ? perm[b + i] : 0x7FFFFFFF;
    __syncthreads();
    for (int k = 2; k <= p2; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < p2; i += blockDim.x) {
          const int l = i ^ j;
          if (l > i) {
            const bool up = (i & k) == 0;
            if ((buf[i] > buf[l]) == up) { const int32_t t = buf[i]; buf[i] = buf[l]; buf[l] = t; }
          }
        }
        __syncthreads();
      }
    for (int i = threadIdx.x; i < m; i += blockDim.x) perm[b + i] = buf[i];
    __syncthreads();
  }
}

// per slot: position and velocity codes, PID, and |v| maxima
template <int ZX, int ZV>
__global__ void k_ic_emit(PartArgs A, const int32_t* __restrict__ perm, const int32_t* __restrict__ slot_cell,
                          const float* __restrict__ vfield, int64_t ncells, int64_t np, int64_t cap,
                          cube_codec codec, double coef, void* __restrict__ xp_, void* __restrict__ vp_,
                          int32_t* __restrict__ pid, unsigned int* __restrict__ vmax_bits) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  TX* xp = reinterpret_cast<TX*>(xp_);
  TV* vp = reinterpret_cast<TV*>(vp_);
  const double xres = ZX == 1 ? 1.0 / 256.0 : 1.0 / 65536.0;
  const int64_t mask = ZX == 1 ? 0xFF : 0xFFFF;
  float vm[3] = {0.f, 0.f, 0.f};
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < np; s += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = perm[s];
    const int64_t c = slot_cell[i];
    double x[3], v[3];
    lattice_state(A, i, x, v);
    for (int d = 0; d < 3; ++d) {
      const int64_t xc = (int64_t)floor(x[d] / xres) & mask;
      xp[(size_t)d * cap + s] = (TX)cube_wrap_code(xc, ZX);
      const double r = v[d] - (double)vfield[(size_t)d * ncells + c];
      vp[(size_t)d * cap + s] = (TV)cube_wrap_code(cube_vencode(&codec, r, coef), ZV);
      vm[d] = fmaxf(vm[d], (float)fabs(v[d]));
    }
    {
      const int64_t n = A.npd, nf = (int64_t)A.nc * A.ncell, st = A.ncell / A.np_nc;
      pid[s] = (int32_t)(st * (i % n) + nf * (st * ((i / n) % n)) + nf * nf * (st * (i / (n * n))) + 1);
    }
  }
  for (int d = 0; d < 3; ++d) {
    float m = vm[d];
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&vmax_bits[d], __float_as_uint(m));
  }
}

// cell counts from the starts
__global__ void k_ic_counts(const int64_t* __restrict__ start, int32_t* __restrict__ rhoc, int64_t ncells) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncells; c += (int64_t)gridDim.x * blockDim.x)
    rhoc[c] = (int32_t)(start[c + 1] - start[c]);
}

}  // namespace

// temporaries of one cube_make_ic call, freed on every return path
struct IcScratch {
  float* kern = nullptr;
  float2* tw = nullptr;
  float2* tw2 = nullptr;
  double2* twd = nullptr;
  ~IcScratch() {
    if (kern) cudaFree(kern);
    if (tw) cudaFree(tw);
    if (tw2) cudaFree(tw2);
    if (twd) cudaFree(twd);
  }
};

int cube_make_ic_dev(cube_ctx* ctx, const cube_ic_params* icp, cube_scalars* io) {
  const int np_nc = icp->np_nc;
  const int npd = np_nc * ctx->nc;
  const int64_t np = (int64_t)npd * npd * npd;
  if (np_nc < 1 || np_nc > ctx->ncell || npd % 2) {
    ctx->err = "initial conditions: need 1 <= np_nc <= ncell and np_nc*nc even";
    return CUBE_ERR_PARAM;
  }
  if (np > ctx->cap || np >= (1ll << 31)) {
    ctx->err = "initial conditions: np_nc^3 nc^3 particles exceed the context capacity";
    return CUBE_ERR_CAPACITY;
  }
  if ((int64_t)ctx->nf * ctx->nf * ctx->nf >= (1ll << 31)) {
    ctx->err = "initial conditions: PIDs are fine-mesh indices + 1 and need nf^3 < 2^31";
    return CUBE_ERR_PARAM;
  }
  // the particle grid borrows the fine mesh's arrays (free outside particle_mesh);
  // npd <= nf, so it fits with its own pitch
  MeshLevel M{};  // an FP32 level (fp64 = 0, no FP64 Green table)
  M.n = npd;
  M.rp = npd + 32;
  M.cp = M.rp / 2;
  M.plane = (size_t)npd * M.rp;
  M.rho = ctx->fine.rho;
  M.force = ctx->fine.force;
  M.ext = ctx->fine.ext;
  M.kern_octant = 1;
  M.kern_pitch = npd / 2 + 1;
  IcScratch tmp;
  int rc = cube_fft_plan(ctx, M.plan, npd);
  tmp.tw = M.plan.tw;
  tmp.tw2 = M.plan.tw2;
  tmp.twd = M.plan.twd;
  if (rc) return rc;
  const size_t ksz = (size_t)M.kern_pitch * M.kern_pitch * M.kern_pitch;
  CUBE_CUDA_TRY(ctx, cudaMalloc((void**)&tmp.kern, sizeof(float) * 3 * ksz));
  M.kern = tmp.kern;
  const int g = ctx->num_sms * 8;
  const uint64_t seed = (uint64_t)icp->seed;
  k_ic_noise<<<g, 256, 0, ctx->stream>>>(M.rho, npd, M.rp, (uint32_t)seed, (uint32_t)(seed >> 32), ctx->codec.pi_f);
  CUBE_LAUNCH_CHECK(ctx);
  IcSpec S = {icp->norm_d2, icp->n_s,      icp->h,          icp->eh_s, icp->eh_alpha, icp->eh_omh,
              icp->eh_theta2, (double)ctx->P.box, icp->amplitude, npd};
  k_ic_kernel<<<g, 256, 0, ctx->stream>>>(M.kern, S);
  CUBE_LAUNCH_CHECK(ctx);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  const KickScale none = {0.f, 0.f, 1.f, 0, 1.f, 1.f};
  if ((rc = cube_fft_poisson(ctx, M, &ctx->dscal->f2_coarse_bits, none))) return rc;
  // cells, counting sort, lattice order inside each cell, per-cell sums
  PartArgs A = {M.force, (size_t)npd * M.plane, M.rp, npd, np_nc, ctx->ncell, ctx->nc, ctx->nt, ctx->nnt, icp->vf};
  int32_t* cell = ctx->tcell;  // cell of each lattice point
  int32_t* perm = ctx->perm;   // slot -> lattice index
  const int64_t nce = ctx->ncells;
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->rhoc, 0, 4 * nce, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->cursor, 0, 4 * nce, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  k_ic_cells<<<g, 256, 0, ctx->stream>>>(A, cell, ctx->rhoc);
  CUBE_LAUNCH_CHECK(ctx);
  if ((rc = cube_exclusive_scan(ctx, ctx->rhoc, nce, ctx->cell_start))) return rc;
  k_ic_place<<<g, 256, 0, ctx->stream>>>(cell, ctx->cell_start, ctx->cursor, perm, np);
  CUBE_LAUNCH_CHECK(ctx);
  k_ic_sort_big<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(ctx->cell_start, perm, nce, ctx->dscal);
  CUBE_LAUNCH_CHECK(ctx);
  double* res2 = ctx->cell_stats;
  k_ic_cellsum<<<g, 256, 0, ctx->stream>>>(A, ctx->cell_start, perm, ctx->vfield, res2, nce);
  CUBE_LAUNCH_CHECK(ctx);
  double r2sum = 0.0;
  if ((rc = cube_tree_sum_dev(ctx, res2, nce, &r2sum))) return rc;
  // sigma_vi = float32(sqrt(mean over particles of |v - vfield|^2) / sqrt(3))
  const float sigma = (float)(sqrt(r2sum / (double)np) / sqrt(3.0));
  const double coef = cube_vcoef(&ctx->codec, sigma);
  unsigned int* vmb = ctx->dscal->vmax_bits;
#define IC_EMIT(ZX, ZV)                                                                                           \
  k_ic_emit<ZX, ZV><<<g, 256, 0, ctx->stream>>>(A, perm, cell, ctx->vfield, nce, np, ctx->cap, ctx->codec, coef, \
                                                ctx->xp, ctx->vp, ctx->pid, vmb)
  if (ctx->izipx == 1 && ctx->izipv == 1) IC_EMIT(1, 1);
  else if (ctx->izipx == 1) IC_EMIT(1, 2);
  else if (ctx->izipv == 1) IC_EMIT(2, 1);
  else IC_EMIT(2, 2);
#undef IC_EMIT
  CUBE_LAUNCH_CHECK(ctx);
  DevScal hs;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&hs, ctx->dscal, sizeof(DevScal), cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (hs.err) {
    ctx->err = "initial conditions: a coarse cell holds more than 4096 particles";
    ctx->state_loaded = 0;
    return hs.err;
  }
  ctx->np = np;
  ctx->state_loaded = 1;
  ctx->cells_le32 = 0;
  float vmax[3];
  for (int d = 0; d < 3; ++d) memcpy(&vmax[d], &hs.vmax_bits[d], 4);
  // the scalar block of a freshly read IC (particle_initialization.f90:37-39)
  const double a = icp->a;
  io->a = (float)a;
  io->sigma_vi = io->sigma_vi_new = sigma;
  io->mass_p_cdm = (float)(icp->f_cdm * (double)ctx->nf * ctx->nf * ctx->nf / (double)np);
  io->vz_max = vmax[2];
  for (int d = 0; d < 3; ++d) io->vmax[d] = vmax[d];
  io->dt = io->dt_old = 0.f;
  io->dt_fine = io->dt_coarse = io->dt_pp = io->dt_vmax_nu = 1000.f;
  io->dt_vmax = (float)(0.9 * 20.0 / std::max((double)std::max(vmax[0], std::max(vmax[1], vmax[2])), 1e-30));
  io->dt_neu = 1000.f;
  io->nplocal = io->npglobal = np;
  return CUBE_OK;
}
