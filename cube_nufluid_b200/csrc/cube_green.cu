/*
 * cube_green.cu -- Green's functions of the two PM levels, built once in FP64.
 *
 * Fine level (kernel_f.f90:14-37): the 16^3 force table T_d is mirrored into
 * all octants, odd in the component's own dimension and even in the others
 * (mfactor), the PP core |offset| <= pp_range is zeroed when PP is on, and the
 * multiplier is the imaginary part of its Fourier transform.  On the periodic
 * nf^3 mesh that transform is a separable sum over the table,
 *   Im K_d(k) = sum_a T_d(a) * S_d(k_d, a_d) * C(k_e, a_e) * C(k_f, a_f),
 *   S(k,a) = -2 sin(2 pi k a/nf) (a > 0),  C(k,0) = 1,  C(k,a) = 2 cos(2 pi k a/nf),
 * evaluated on the device in FP64 in three passes (x, y, z) over the octant
 * 0 <= kx,ky,kz <= nf/2 and stored as FP32 divided by nf^3, layout
 * [d][ky][kx][kz] (kz fastest, the order in which the z pass reads it).
 *
 * Coarse level (kernel_c.f90:16-117, LRCKCORR on): ck = -r/r^3 on the periodic
 * coarse mesh (fine-cell units), the 4^3 corner replaced by the matching table
 * in the eight octants, transformed; for |k| <= 8 the multiplier is rescaled
 * by 0.25 pi sin-k_d/|sin-k|^2 / Im FFT(-r/r^3).  Built on the host in FP64
 * with a mixed-radix FFT, stored as the same octant layout divided by nc^3.
 */
#include "cube_internal.cuh"

#include <cmath>
#include <complex>
#include <thread>

namespace {

__device__ __forceinline__ double fac(int k, int a, int n, bool odd) {
  if (a == 0) return odd ? 0.0 : 1.0;
  const long long m = ((long long)k * a) % n;
  double s, c;
  sincospi(2.0 * (double)m / (double)n, &s, &c);
  return odd ? -2.0 * s : 2.0 * c;
}

// S1[d][kx][az][ay] = sum_ax T_d(ax,ay,az) F_x(kx,ax)
__global__ void k_green_x(const float* __restrict__ fk, int nfc, int n, int d, int pp_zero, double* __restrict__ s1) {
  const int kp = n / 2 + 1;
  const int64_t tot = (int64_t)kp * nfc * nfc;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
    const int ay = q % nfc, az = (q / nfc) % nfc, kx = (int)(q / ((int64_t)nfc * nfc));
    double acc = 0.0;
    for (int ax = 0; ax < nfc; ++ax) {
      double t = (double)fk[(((size_t)d * nfc + az) * nfc + ay) * nfc + ax];
      if (pp_zero >= 0 && ax <= pp_zero && ay <= pp_zero && az <= pp_zero) t = 0.0;
      acc += t * fac(kx, ax, n, d == 0);
    }
    s1[q] = acc;
  }
}

// S2[kx][ky][az] = sum_ay S1[kx][az][ay] F_y(ky,ay)
__global__ void k_green_y(const double* __restrict__ s1, int nfc, int n, int d, double* __restrict__ s2) {
  const int kp = n / 2 + 1;
  const int64_t tot = (int64_t)kp * kp * nfc;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
    const int az = q % nfc, ky = (q / nfc) % kp, kx = (int)(q / ((int64_t)nfc * kp));
    double acc = 0.0;
    for (int ay = 0; ay < nfc; ++ay) acc += s1[((size_t)kx * nfc + az) * nfc + ay] * fac(ky, ay, n, d == 1);
    s2[q] = acc;
  }
}

// K[ky][kx][kz] = sum_az S2[kx][ky][az] F_z(kz,az) / n^3
__global__ void k_green_z(const double* __restrict__ s2, int nfc, int n, int d, float* __restrict__ kern,
                          double* __restrict__ kernd) {
  const int kp = n / 2 + 1;
  const int64_t tot = (int64_t)kp * kp * kp;
  const double inv = 1.0 / ((double)n * n * n);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < tot; q += (int64_t)gridDim.x * blockDim.x) {
    // octant layout [ky][kx][kz], kz fastest (the z pass reads columns along kz)
    const int kz = q % kp, kx = (q / kp) % kp, ky = (int)(q / ((int64_t)kp * kp));
    double acc = 0.0;
    for (int az = 0; az < nfc; ++az) acc += s2[((size_t)kx * kp + ky) * nfc + az] * fac(kz, az, n, d == 2);
    kern[(size_t)d * tot + q] = (float)(acc * inv);
    if (kernd) kernd[(size_t)d * tot + q] = acc * inv;  // FP64 Poisson mode
  }
}

// ---- host FP64 FFT (mixed radix 2/3/5 plus generic), for the coarse kernel --
typedef std::complex<double> cd;

struct HostDft {
  int n;
  std::vector<cd> w;  // exp(-2 pi i j/n)
  std::vector<int> fac;
  explicit HostDft(int n_) : n(n_), w(n_) {
    for (int j = 0; j < n; ++j) {
      const long double a = -2.0L * 3.14159265358979323846264338327950288L * j / n;
      w[j] = cd((double)cosl(a), (double)sinl(a));
    }
    int m = n;
    for (int p = 2; p * p <= m; ++p)
      while (m % p == 0) { fac.push_back(p); m /= p; }
    if (m > 1) fac.push_back(m);
  }
  // Stockham passes, out-of-place ping-pong; result in x
  void run(cd* x, cd* y) const {
    int T = 1;
    cd* a = x;
    cd* b = y;
    for (size_t st = 0; st < fac.size(); ++st) {
      const int p = fac[st];
      const int nb = n / p;
      const int tstep = n / (p * T);
      cd v[64];
      for (int i = 0; i < nb; ++i) {
        const int k = i % T;
        for (int r = 0; r < p; ++r) v[r] = a[i + r * nb] * w[(size_t)r * k * tstep];
        const int j0 = (i - k) * p + k;
        for (int s = 0; s < p; ++s) {
          cd acc(0, 0);
          for (int r = 0; r < p; ++r) acc += v[r] * w[((size_t)r * s * (n / p)) % n];
          b[j0 + s * T] = acc;
        }
      }
      std::swap(a, b);
      T *= p;
    }
    if (a != x)
      for (int i = 0; i < n; ++i) x[i] = a[i];
  }
};

// forward complex 3-D transform of c[(k*n+j)*n+i], threaded over lines
void host_fft3(std::vector<cd>& c, int n) {
  HostDft D(n);
  const unsigned nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  for (int axis = 0; axis < 3; ++axis) {
    auto work = [&](unsigned tid) {
      std::vector<cd> line(n), tmp(n);
      for (long r = tid; r < (long)n * n; r += nth) {
        const int p = r % n, q = r / n;
        for (int i = 0; i < n; ++i) {
          size_t idx = axis == 0 ? ((size_t)q * n + p) * n + i
                     : axis == 1 ? ((size_t)q * n + i) * n + p
                                 : ((size_t)i * n + q) * n + p;
          line[i] = c[idx];
        }
        D.run(line.data(), tmp.data());
        for (int i = 0; i < n; ++i) {
          size_t idx = axis == 0 ? ((size_t)q * n + p) * n + i
                     : axis == 1 ? ((size_t)q * n + i) * n + p
                                 : ((size_t)i * n + q) * n + p;
          c[idx] = line[i];
        }
      }
    };
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nth; ++t) th.emplace_back(work, t);
    for (auto& t : th) t.join();
  }
}

}  // namespace

int cube_build_green(cube_ctx* ctx, const float* fk_table, const float* ck_table) {
  // ---- fine ----
  {
    const int n = ctx->fine.n, nfc = ctx->P.nf_cutoff, kp = n / 2 + 1;
    float* dfk = nullptr;
    double *s1 = nullptr, *s2 = nullptr;
    const size_t nfk = (size_t)3 * nfc * nfc * nfc;
    CUBE_CUDA_TRY(ctx, cudaMalloc(&dfk, sizeof(float) * nfk));
    CUBE_CUDA_TRY(ctx, cudaMalloc(&s1, sizeof(double) * (size_t)kp * nfc * nfc));
    CUBE_CUDA_TRY(ctx, cudaMalloc(&s2, sizeof(double) * (size_t)kp * kp * nfc));
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dfk, fk_table, sizeof(float) * nfk, cudaMemcpyHostToDevice, ctx->stream));
    const int ppz = ctx->P.ext_pp_force ? ctx->P.pp_range : -1;
    for (int d = 0; d < 3; ++d) {
      k_green_x<<<1184, 256, 0, ctx->stream>>>(dfk, nfc, n, d, ppz, s1);
      CUBE_LAUNCH_CHECK(ctx);
      k_green_y<<<1184, 256, 0, ctx->stream>>>(s1, nfc, n, d, s2);
      CUBE_LAUNCH_CHECK(ctx);
      k_green_z<<<4736, 256, 0, ctx->stream>>>(s2, nfc, n, d, ctx->fine.kern, ctx->fine.kernd);
      CUBE_LAUNCH_CHECK(ctx);
    }
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(dfk);
    cudaFree(s1);
    cudaFree(s2);
  }
  // ---- coarse ----
  {
    const int nc = ctx->nc, ncell = ctx->ncell, kp = nc / 2 + 1;
    const size_t n3 = (size_t)nc * nc * nc;
    const double pi = 3.14159265358979323846;
    std::vector<float> oct((size_t)3 * kp * kp * kp);
    std::vector<double> octd(ctx->coarse.kernd ? oct.size() : 0);
    std::vector<cd> z(n3);
    auto off = [&](int g) { return ((g + nc / 2) % nc) - nc / 2; };  // 0-based index -> signed offset
    for (int d = 0; d < 3; ++d) {
      for (int k = 0; k < nc; ++k)
        for (int j = 0; j < nc; ++j)
          for (int i = 0; i < nc; ++i) {
            const double rx[3] = {(double)ncell * off(i), (double)ncell * off(j), (double)ncell * off(k)};
            const double r = std::sqrt(rx[0] * rx[0] + rx[1] * rx[1] + rx[2] * rx[2]);
            const double direct = r == 0 ? 0.0 : -rx[d] / (r * r * r);
            double corr = direct;
            const int oi = off(i), oj = off(j), ok = off(k);
            if (std::abs(oi) <= 3 && std::abs(oj) <= 3 && std::abs(ok) <= 3) {
              // kernel_c.f90:43-72: table index |offset|+1, odd in the component's dimension
              const int ti = std::abs(oi), tj = std::abs(oj), tk = std::abs(ok);
              double v = (double)ck_table[(((size_t)tk * 4 + tj) * 4 + ti) * 3 + d];
              const int od = d == 0 ? oi : d == 1 ? oj : ok;
              if (od < 0) v = -v;
              corr = v;
            }
            z[((size_t)k * nc + j) * nc + i] = cd(corr, direct);
          }
      host_fft3(z, nc);
      for (int kz = 0; kz < kp; ++kz)
        for (int ky = 0; ky < kp; ++ky)
          for (int kx = 0; kx < kp; ++kx) {
            const cd Z = z[((size_t)kz * nc + ky) * nc + kx];
            const cd Zm = std::conj(z[((size_t)((nc - kz) % nc) * nc + (nc - ky) % nc) * nc + (nc - kx) % nc]);
            const cd C = 0.5 * (Z + Zm);                    // transform of the corrected kernel
            const cd D = cd(0, -0.5) * (Z - Zm);            // transform of -r/r^3
            const int kk[3] = {kx, ky, kz};  // folded indices are the signed wavenumbers here
            const double kr = std::sqrt((double)kx * kx + (double)ky * ky + (double)kz * kz);
            double ks[3], ks2 = 0;
            for (int e = 0; e < 3; ++e) { ks[e] = 2 * std::sin(pi * kk[e] / (double)nc); ks2 += ks[e] * ks[e]; }
            double v = C.imag();
            if (kk[d] == nc / 2) v = 0.0;  // odd in k_d: exactly zero on the Nyquist plane
            else if (!(kr > 8.0 || kk[d] == 0)) v = v * 0.25 * pi * ks[d] / ks2 / D.imag();
            oct[(size_t)d * kp * kp * kp + ((size_t)ky * kp + kx) * kp + kz] = (float)(v / (double)n3);
            if (!octd.empty()) octd[(size_t)d * kp * kp * kp + ((size_t)ky * kp + kx) * kp + kz] = v / (double)n3;
          }
    }
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->coarse.kern, oct.data(), sizeof(float) * oct.size(), cudaMemcpyHostToDevice,
                                       ctx->stream));
    if (!octd.empty())
      CUBE_CUDA_TRY(ctx, cudaMemcpy(ctx->coarse.kernd, octd.data(), sizeof(double) * octd.size(), cudaMemcpyHostToDevice));
  }
  return CUBE_OK;
}
