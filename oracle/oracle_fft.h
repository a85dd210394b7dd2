/*
 * oracle_fft.h -- TEST INFRASTRUCTURE ONLY (the CPU oracle of the parity tests).
 *
 * Mixed-radix complex DFT for any length (Stockham autosort passes, radix =
 * prime factors of n, a plain DFT inside each butterfly, twiddles computed in
 * long double) and 3-D real transforms built on it, threaded over lines with
 * OpenMP.  This stands in for FFTW 3.x (single precision in the reference:
 * sfftw_plan_dft_r2c_3d / c2r_3d, CUBE_v2.0/work/main/cubefft.f90:25-26,
 * pencil_fft.f90:178-189), which is not vendored with the reference.  Sign
 * conventions follow FFTW: the forward transform uses exp(-2 pi i jk/N), the
 * backward transform exp(+2 pi i jk/N), both unnormalised.  The results are
 * checked against numpy's FFT in the CPU tests.
 */
#ifndef ORACLE_FFT_H
#define ORACLE_FFT_H

#include <cmath>
#include <complex>
#include <vector>

namespace orc {

template <typename R>
struct Dft1 {
  int n;
  int sign;
  std::vector<std::complex<R>> w;  // w[j] = exp(sign*2 pi i j/n)
  std::vector<int> fac;
  Dft1(int n_, int sign_) : n(n_), sign(sign_), w(n_) {
    for (int j = 0; j < n; ++j) {
      long double ang = (long double)sign * 2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
      w[j] = std::complex<R>((R)cosl(ang), (R)sinl(ang));
    }
    int m = n;
    for (int p = 2; p * p <= m; ++p)
      while (m % p == 0) { fac.push_back(p); m /= p; }
    if (m > 1) fac.push_back(m);
  }
  // in place on x with scratch y (both length n)
  void run(std::complex<R>* x, std::complex<R>* y) const {
    int T = 1;
    std::complex<R>* a = x;
    std::complex<R>* b = y;
    std::complex<R> v[64];
    for (size_t st = 0; st < fac.size(); ++st) {
      const int p = fac[st];
      const int nb = n / p;
      const int tstep = n / (p * T);
      for (int i = 0; i < nb; ++i) {
        const int k = i % T;
        for (int r = 0; r < p; ++r) v[r] = a[i + r * nb] * w[(size_t)r * k * tstep];
        const int j0 = (i - k) * p + k;
        for (int s = 0; s < p; ++s) {
          std::complex<R> acc(0, 0);
          for (int r = 0; r < p; ++r) acc += v[r] * w[((size_t)r * s * nb) % n];
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

// In-place 3-D complex transform of c[(k*ny + j)*nx + i] along all three axes.
template <typename R>
void cfft3(std::vector<std::complex<R>>& c, int nx, int ny, int nz, int sign) {
  {
    Dft1<R> d(nx, sign);
#pragma omp parallel
    {
      std::vector<std::complex<R>> line(nx), tmp(nx);
#pragma omp for schedule(static)
      for (long r = 0; r < (long)ny * nz; ++r) {
        for (int i = 0; i < nx; ++i) line[i] = c[r * nx + i];
        d.run(line.data(), tmp.data());
        for (int i = 0; i < nx; ++i) c[r * nx + i] = line[i];
      }
    }
  }
  {
    Dft1<R> d(ny, sign);
#pragma omp parallel
    {
      std::vector<std::complex<R>> line(ny), tmp(ny);
#pragma omp for schedule(static)
      for (long r = 0; r < (long)nz * nx; ++r) {
        const long k = r / nx, i = r % nx;
        for (int j = 0; j < ny; ++j) line[j] = c[((long)k * ny + j) * nx + i];
        d.run(line.data(), tmp.data());
        for (int j = 0; j < ny; ++j) c[((long)k * ny + j) * nx + i] = line[j];
      }
    }
  }
  {
    Dft1<R> d(nz, sign);
#pragma omp parallel
    {
      std::vector<std::complex<R>> line(nz), tmp(nz);
#pragma omp for schedule(static)
      for (long r = 0; r < (long)ny * nx; ++r) {
        const long j = r / nx, i = r % nx;
        for (int k = 0; k < nz; ++k) line[k] = c[((long)k * ny + j) * nx + i];
        d.run(line.data(), tmp.data());
        for (int k = 0; k < nz; ++k) c[((long)k * ny + j) * nx + i] = line[k];
      }
    }
  }
}

// Real-to-complex forward transform of r[(k*n+j)*n+i] (n^3) into the half
// spectrum h[(k*n + j)*(n/2+1) + i] (FFTW r2c layout).
template <typename R>
void rfft3_forward(const R* r, std::vector<std::complex<R>>& h, int n) {
  std::vector<std::complex<R>> c((size_t)n * n * n);
  for (size_t q = 0; q < c.size(); ++q) c[q] = std::complex<R>(r[q], 0);
  cfft3(c, n, n, n, -1);
  const int nh = n / 2 + 1;
  h.assign((size_t)nh * n * n, std::complex<R>(0, 0));
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < nh; ++i) h[((size_t)k * n + j) * nh + i] = c[((size_t)k * n + j) * n + i];
}

// Complex-to-real backward transform of a Hermitian half spectrum (FFTW c2r
// semantics: the imaginary parts of self-conjugate bins are ignored).
template <typename R>
void rfft3_backward(const std::vector<std::complex<R>>& h, R* r, int n) {
  const int nh = n / 2 + 1;
  std::vector<std::complex<R>> c((size_t)n * n * n);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        std::complex<R> v;
        if (i < nh) {
          v = h[((size_t)k * n + j) * nh + i];
        } else {
          const int ii = n - i, jj = (n - j) % n, kk = (n - k) % n;
          v = std::conj(h[((size_t)kk * n + jj) * nh + ii]);
        }
        c[((size_t)k * n + j) * n + i] = v;
      }
  cfft3(c, n, n, n, +1);
  for (size_t q = 0; q < c.size(); ++q) r[q] = c[q].real();
}

}  // namespace orc

#endif
