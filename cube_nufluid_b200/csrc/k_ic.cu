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
 *   potential  the reference's method (initial_conditions.f90:449-523,776-836): on the
 *              fine mesh (nf = ncell*nc per side) phi = K' * delta_L, K = -4 pi/khat^2
 *              with the discrete Laplacian khat^2 = sum (2 sin(pi m/nf))^2, corrected
 *              in real space to the exact -1/r within 8 cells (-2.5 at r = 0) and
 *              shifted by -(phi8 + 1/8) beyond; the correction is the transform of a
 *              stencil of 8-cell radius, built from the kernel's own transform (two
 *              forward FFTs of the library); delta_L = amp(k) FFT(noise), amp^2 =
 *              Delta^2(k)/(4 pi) (nf/k)^3 with the Eisenstein-Hu no-wiggle transfer,
 *              sigma8 normalisation and growth passed in by the host;
 *   displacement psi_d = -(phi(i+1) - phi(i-1))/(8 pi) along d at each particle's fine
 *              node: in k space the multiplier -i sin(2 pi m_d/nf) K'/(4 pi), odd in its
 *              own wavenumber, so the library's Poisson passes evaluate it as a "Green"
 *              octant (zero on the own-dimension Nyquist plane);
 *   particles  lattice q = i/np_nc + 1/(2 ncell) (coarse units), the centre of fine cell
 *              (ncell/np_nc) i, x = q + psi/ncell, v = psi * vf; sorted by tile-major cell, in lattice
 *              order inside a cell; PID = 1 + the fine-mesh index of the lattice
 *              point, iq = (ncell/np_nc)*lattice index per dimension (:834-836); per cell the mean
 *              velocity (vfield), the residuals' dispersion sigma_vi, and the codes
 *              (initial_conditions.f90:797-838).
 */
#include "cube_internal.cuh"

#include <cmath>
#include <cstdlib>
#include <vector>

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
  int n;              // the fine mesh per side
  double psi_scale;   // np_nc / ncell: the packer's lattice units per fine cell
  const float2* W;    // transform of the kernel correction stencil (null: none)
  int kx_major, cp;   // its layout: [kx][ky][kz] dense, or [kz][ky][kx] at row pitch cp
};

constexpr int EWALD_R = 8;  // radius (cells) of the exact -1/r near field

// the discrete-Laplacian potential kernel -4 pi/khat^2 at integer wavenumbers (0 at k = 0)
__device__ __forceinline__ double ic_laplace_kernel(int mx, int my, int mz, int n) {
  const double pin = 3.14159265358979323846 / (double)n;
  const double sx = 2.0 * sin(pin * mx), sy = 2.0 * sin(pin * my), sz = 2.0 * sin(pin * mz);
  const double kr = sx * sx + sy * sy + sz * sz;
  return kr > 0.0 ? -4.0 * 3.14159265358979323846 / kr : 0.0;
}

// the kernel at every wavenumber of the mesh (index = wavenumber mod n), as a real field
__global__ void k_ic_kfill(float* __restrict__ mesh, int n, int rp) {
  const int64_t tot = (int64_t)n * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((int64_t)n * n));
    mesh[((size_t)z * n + y) * rp + x] = (float)ic_laplace_kernel(x, y, z, n);
  }
}

// element (kx, ky, kz) of a forward 3-D transform left by cube_fft_forward3
__device__ __forceinline__ float2 ic_spec(const float2* S, int kx, int ky, int kz, int n, int kx_major, int cp) {
  return kx_major ? S[((size_t)kx * n + ky) * n + kz] : S[((size_t)kz * n + ky) * cp + kx];
}

// the real-space kernel K_r(r) = Re FFT(K)(r) / n^3 (K is real and even) for r in [0, 8]^3
__global__ void k_ic_kreal(const float2* __restrict__ S, int n, int kx_major, int cp, double* __restrict__ out) {
  constexpr int R1 = EWALD_R + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R1 * R1 * R1) return;
  const int rx = i % R1, ry = (i / R1) % R1, rz = i / (R1 * R1);
  out[i] = (double)ic_spec(S, rx, ry, rz, n, kx_major, cp).x / ((double)n * n * n);
}

// the correction stencil w(r) (2R+1)^3 into the zeroed mesh at r mod n
__global__ void k_ic_wfill(float* __restrict__ mesh, int n, int rp, const float* __restrict__ w) {
  constexpr int D = 2 * EWALD_R + 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= D * D * D) return;
  const float v = w[i];
  if (v == 0.f) return;
  const int x = (i % D - EWALD_R + n) % n, y = ((i / D) % D - EWALD_R + n) % n, z = (i / (D * D) - EWALD_R + n) % n;
  mesh[((size_t)z * n + y) * rp + x] = v;
}

__device__ double eh_nowiggle(double k_hmpc, const IcSpec& S) {
  const double k_mpc = k_hmpc * S.h;
  const double x = 0.43 * k_mpc * S.eh_s;
  const double gamma = S.eh_omh * (S.eh_alpha + (1.0 - S.eh_alpha) / (1.0 + x * x * x * x));
  const double q = k_hmpc * S.eh_theta2 / gamma;
  const double l0 = log(2.0 * 2.718281828459045 + 1.8 * q);
  const double c0 = 14.2 + 731.0 / (1.0 + 62.5 * q);
  return l0 / (l0 + c0 * q * q);
}

// the displacement "Green" octant [d][ky][kx][kz] (kz fastest), (n/2+1)^3 per
// component: -sin(2 pi k_d/n)/(4 pi) K'(k) amp(k) (np_nc/ncell) / n^3, K' = K + Re W,
// zero on the own-dimension Nyquist plane
__global__ void k_ic_kernel(float* __restrict__ kern, IcSpec S) {
  const int n = S.n, nh = n / 2, kp = nh + 1;
  const int64_t tot = (int64_t)kp * kp * kp;
  const double twopi = 2.0 * 3.14159265358979323846;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int kz = (int)(i % kp);
    const int64_t r = i / kp;
    const int kx = (int)(r % kp), ky = (int)(r / kp);
    const float kr2 = (float)kx * kx + (float)ky * ky + (float)kz * kz;
    const float kr = sqrtf(fmaxf(kr2, 1.f));
    const double kphys = twopi * (double)kr / S.box;
    const double t = eh_nowiggle(kphys, S);
    const float d2 = (float)(S.norm_d2 * t * t * pow(kphys, 3.0 + S.n_s));
    const float nk = (float)n / kr;
    const float amp = sqrtf(d2 / (float)(4.0 * 3.14159265358979323846) * nk) * nk * (float)S.amplitude;
    double kc = ic_laplace_kernel(kx, ky, kz, n);
    if (S.W && (kx | ky | kz)) kc += (double)ic_spec(S.W, kx, ky, kz, n, S.kx_major, S.cp).x;
    const float kcf = (float)kc;
    const float norm = 1.f / ((float)n * (float)n * (float)n);
    const int kd[3] = {kx, ky, kz};
    for (int d = 0; d < 3; ++d) {
      const float g = (kd[d] == nh) ? 0.f : (float)(-sin(twopi * kd[d] / n) / (4.0 * 3.14159265358979323846));
      kern[(size_t)d * tot + ((size_t)ky * kp + kx) * kp + kz] = g * kcf * amp * (float)S.psi_scale * norm;
    }
  }
}

struct PartArgs {
  const float* psi;   // three displacement meshes (fine mesh nf^3), component stride cstride, pitch rp
  size_t cstride;
  int rp, npd, np_nc, ncell, nc, nt, nnt;
  double vf;
  int nf, st;         // fine mesh per side; fine cells between lattice points (ncell/np_nc)
};

// lattice point -> cell (tile-major) and counts
__global__ void k_ic_cells(PartArgs A, int32_t* __restrict__ cell, int32_t* __restrict__ cnt) {
  const int n = A.npd;
  const int64_t tot = (int64_t)n * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int q[3] = {(int)(i % n), (int)((i / n) % n), (int)(i / ((int64_t)n * n))};
    const size_t o = ((size_t)(A.st * q[2]) * A.nf + A.st * q[1]) * A.rp + A.st * q[0];
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
  const size_t o = ((size_t)(A.st * q[2]) * A.nf + A.st * q[1]) * A.rp + A.st * q[0];
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
  double* kr = nullptr;
  float* w = nullptr;
  ~IcScratch() {
    if (kern) cudaFree(kern);
    if (kr) cudaFree(kr);
    if (w) cudaFree(w);
  }
};

int cube_make_ic_dev(cube_ctx* ctx, const cube_ic_params* icp, cube_scalars* io) {
  const int np_nc = icp->np_nc;
  const int npd = np_nc * ctx->nc;
  const int64_t np = (int64_t)npd * npd * npd;
  if (np_nc < 1 || np_nc > ctx->ncell || ctx->ncell % np_nc) {
    ctx->err = "initial conditions: need np_nc to divide ncell";
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
  // everything runs on the fine mesh's arrays (free outside particle_mesh), with its
  // own Green table set aside for a displacement table of the same octant layout
  MeshLevel& F = ctx->fine;
  const int n = F.n;
  MeshLevel M = F;
  M.kern_octant = 1;
  M.kern_pitch = n / 2 + 1;
  M.kernd = nullptr;
  IcScratch tmp;
  const size_t ksz = (size_t)M.kern_pitch * M.kern_pitch * M.kern_pitch;
  CUBE_CUDA_TRY(ctx, cudaMalloc((void**)&tmp.kern, sizeof(float) * 3 * ksz));
  M.kern = tmp.kern;
  const int g = ctx->num_sms * 8;
  int rc;
  IcSpec S = {icp->norm_d2, icp->n_s, icp->h, icp->eh_s, icp->eh_alpha, icp->eh_omh, icp->eh_theta2,
              (double)ctx->P.box, icp->amplitude, n, (double)np_nc / (double)ctx->ncell, nullptr, 0, F.cp};
  if (n >= 2 * EWALD_R + 2) {
    // the kernel correction: K_r(r) for r in [0, 8]^3 from the forward transform of K,
    // the stencil w(r) = exact(r) - K_r(r) + phi8 + 1/8 within r <= 8, its transform W
    constexpr int R1 = EWALD_R + 1, D = 2 * EWALD_R + 1;
    int kxm = 0;
    k_ic_kfill<<<g, 256, 0, ctx->stream>>>(F.rho, n, F.rp);
    CUBE_LAUNCH_CHECK(ctx);
    if ((rc = cube_fft_forward3(ctx, F, F.rho, &kxm))) return rc;
    CUBE_CUDA_TRY(ctx, cudaMalloc((void**)&tmp.kr, sizeof(double) * R1 * R1 * R1));
    CUBE_CUDA_TRY(ctx, cudaMalloc((void**)&tmp.w, sizeof(float) * D * D * D));
    k_ic_kreal<<<(R1 * R1 * R1 + 255) / 256, 256, 0, ctx->stream>>>(reinterpret_cast<const float2*>(F.rho), n, kxm,
                                                                    F.cp, tmp.kr);
    CUBE_LAUNCH_CHECK(ctx);
    std::vector<double> kr(R1 * R1 * R1);
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(kr.data(), tmp.kr, sizeof(double) * kr.size(), cudaMemcpyDeviceToHost,
                                       ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    auto K_r = [&](int x, int y, int z) { return kr[((size_t)std::abs(z) * R1 + std::abs(y)) * R1 + std::abs(x)]; };
    const double phi8 = (K_r(EWALD_R, 0, 0) + K_r(0, EWALD_R, 0) + K_r(0, 0, EWALD_R)) / 3.0;
    std::vector<float> w((size_t)D * D * D, 0.f);
    for (int z = -EWALD_R; z <= EWALD_R; ++z)
      for (int y = -EWALD_R; y <= EWALD_R; ++y)
        for (int x = -EWALD_R; x <= EWALD_R; ++x) {
          const double d = std::sqrt((double)(x * x + y * y + z * z));
          if (d > EWALD_R) continue;
          const double exact = d > 0.0 ? -1.0 / d : -2.5;
          w[((size_t)(z + EWALD_R) * D + (y + EWALD_R)) * D + (x + EWALD_R)] =
              (float)(exact - K_r(x, y, z) + phi8 + 1.0 / EWALD_R);
        }
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(tmp.w, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaMemsetAsync(F.rho, 0, sizeof(float) * (size_t)n * F.plane, ctx->stream));
    k_ic_wfill<<<(D * D * D + 255) / 256, 256, 0, ctx->stream>>>(F.rho, n, F.rp, tmp.w);
    CUBE_LAUNCH_CHECK(ctx);
    if ((rc = cube_fft_forward3(ctx, F, F.rho, &kxm))) return rc;
    S.W = reinterpret_cast<const float2*>(F.rho);
    S.kx_major = kxm;
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));  // the host stencil buffer stays alive until here
  }
  k_ic_kernel<<<g, 256, 0, ctx->stream>>>(M.kern, S);
  CUBE_LAUNCH_CHECK(ctx);
  const uint64_t seed = (uint64_t)icp->seed;
  k_ic_noise<<<g, 256, 0, ctx->stream>>>(M.rho, n, M.rp, (uint32_t)seed, (uint32_t)(seed >> 32), ctx->codec.pi_f);
  CUBE_LAUNCH_CHECK(ctx);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  const KickScale none = {0.f, 0.f, 1.f, 0, 1.f, 1.f};
  if ((rc = cube_fft_poisson(ctx, M, &ctx->dscal->f2_coarse_bits, none))) return rc;
  // cells, counting sort, lattice order inside each cell, per-cell sums
  PartArgs A = {M.force, (size_t)n * M.plane, M.rp, npd,     np_nc, ctx->ncell, ctx->nc, ctx->nt,
                ctx->nnt, icp->vf, n,           ctx->ncell / np_nc};
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
