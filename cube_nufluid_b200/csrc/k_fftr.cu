/*
 * k_fftr.cu -- register-resident FFT passes for power-of-two meshes and three
 * times a power of two.
 *
 * A length N = R*T transform runs on a group of T threads (T <= 32, inside
 * one warp): with n = t + T*q and k = k1 + R*k2,
 *   X[k1 + R*k2] = sum_t W_N^{t k1} W_T^{t k2} sum_q x[t + T q] W_R^{q k1}
 * so each thread does one R-point DFT in registers (over q), multiplies by
 * W_N^{t k1} (a table laid out [k1][t], so a warp's loads are contiguous), the
 * group exchanges once through shared memory (padded so neither side of the
 * transpose has bank conflicts), and each thread does
 * R/T T-point DFTs in registers (over t).  Only __syncwarp is needed inside a
 * transform.  Sizes: 1024 = 32*32, 512 = 32*16, 256 = 16*16, 128 = 16*8,
 * 64 = 8*8, 32 = 8*4, and with a radix-3 first stage 768 = 48*16, 384 = 48*8,
 * 192 = 24*8, 96 = 24*4; other sizes use the shared-memory Stockham passes of
 * k_fft.cu.
 *
 * Passes of the Poisson solve (the layouts are listed above k_xr2c_t):
 *   x r2c    : 8 rows of a z-plane per CTA, packed in pairs as complex rows
 *   y        : 8 rows per CTA, output transposed so that z is innermost
 *   z+Green  : forward along z, the spectrum kept in registers, then for each
 *              component d: x i*K_d into the inverse FFT, output transposed
 *   y^-1     : per component, output transposed back to x innermost
 *   x c2r    : the three force components of RB row pairs in place, max f^2
 * The forward 3-D transform of the power spectrum is x r2c, y and an in-place
 * pass along z.
 */
#include "cube_internal.cuh"

#include <algorithm>
#include <utility>

namespace {

// cos(pi*k/16), k = 0..8
__device__ constexpr float kC16[9] = {1.0f,
                                      0.98078528040323044913f,
                                      0.92387953251128675613f,
                                      0.83146961230254523708f,
                                      0.70710678118654752440f,
                                      0.55557023301960222474f,
                                      0.38268343236508977173f,
                                      0.19509032201612826785f,
                                      0.0f};

__device__ constexpr float cos16(int j) {  // cos(pi j / 16), any integer j
  return (j & 31) <= 8    ? kC16[j & 31]
         : (j & 31) <= 16 ? -kC16[16 - (j & 31)]
         : (j & 31) <= 24 ? -kC16[(j & 31) - 16]
                          : kC16[32 - (j & 31)];
}
__device__ constexpr float sin16(int j) { return cos16(8 - j); }

// cos(2 pi j/48), j = 0..47 (twiddles of the radix-3 in-register DFTs)
__device__ constexpr float kC48[48] = {
    1.00000000000000000000e+00f,
    9.91444861373810382155e-01f,
    9.65925826289068312214e-01f,
    9.23879532511286738483e-01f,
    8.66025403784438707611e-01f,
    7.93353340291235165083e-01f,
    7.07106781186547572737e-01f,
    6.08761429008720655887e-01f,
    5.00000000000000111022e-01f,
    3.82683432365089837290e-01f,
    2.58819045102520739476e-01f,
    1.30526192220051712178e-01f,
    6.12323399573676603587e-17f,
    -1.30526192220051601156e-01f,
    -2.58819045102520628454e-01f,
    -3.82683432365089504223e-01f,
    -4.99999999999999777955e-01f,
    -6.08761429008720655887e-01f,
    -7.07106781186547461715e-01f,
    -7.93353340291235054060e-01f,
    -8.66025403784438707611e-01f,
    -9.23879532511286738483e-01f,
    -9.65925826289068201191e-01f,
    -9.91444861373810382155e-01f,
    -1.00000000000000000000e+00f,
    -9.91444861373810382155e-01f,
    -9.65925826289068312214e-01f,
    -9.23879532511286849505e-01f,
    -8.66025403784438818633e-01f,
    -7.93353340291235165083e-01f,
    -7.07106781186547905804e-01f,
    -6.08761429008720877931e-01f,
    -5.00000000000000444089e-01f,
    -3.82683432365089504223e-01f,
    -2.58819045102520628454e-01f,
    -1.30526192220051628912e-01f,
    -1.83697019872102968750e-16f,
    1.30526192220051268089e-01f,
    2.58819045102520295387e-01f,
    3.82683432365089171157e-01f,
    5.00000000000000111022e-01f,
    6.08761429008719878730e-01f,
    7.07106781186547350693e-01f,
    7.93353340291234943038e-01f,
    8.66025403784438374544e-01f,
    9.23879532511286849505e-01f,
    9.65925826289068090169e-01f,
    9.91444861373810382155e-01f};
__device__ constexpr float cos48(int j) { return kC48[((j % 48) + 48) % 48]; }  // cos(2 pi j/48)
__device__ constexpr float sin48(int j) { return cos48(j - 12); }                // sin(2 pi j/48)

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__host__ __device__ constexpr int bitrev(int L, int i) {
  int r = 0;
  for (int b = 1; b < L; b <<= 1) {
    r = (r << 1) | (i & 1);
    i >>= 1;
  }
  return r;
}

template <int L, int I>
struct BitRev {
  static constexpr int value = bitrev(L, I);
};

// bit-reversal permutation with every index fixed at compile time (keeps v in registers)
template <int L, int... I>
__device__ __forceinline__ void bitrev_perm(float2* v, std::integer_sequence<int, I...>) {
  const float2 t[L] = {v[BitRev<L, I>::value]...};
  ((v[I] = t[I]), ...);
}

// one radix-2 butterfly stage of span LEN (twiddles are compile-time constants)
template <int L, int SIGN, int LEN>
__device__ __forceinline__ void dft_stage(float2* v) {
#pragma unroll
  for (int i = 0; i < L; i += LEN) {
#pragma unroll
    for (int j = 0; j < LEN / 2; ++j) {
      const int e = j * (32 / LEN);  // exponent in units of 2 pi/32
      float2 b = v[i + j + LEN / 2];
      if (e == 0) {
      } else if (e == 8) {  // w = SIGN * i
        b = make_float2(-SIGN * b.y, SIGN * b.x);
      } else {
        const float2 w = make_float2(cos16(e), SIGN * sin16(e));
        b = cmul(b, w);
      }
      const float2 a = v[i + j];
      v[i + j] = make_float2(a.x + b.x, a.y + b.y);
      v[i + j + LEN / 2] = make_float2(a.x - b.x, a.y - b.y);
    }
  }
  if constexpr (LEN < L) dft_stage<L, SIGN, 2 * LEN>(v);
}

template <int L, int SIGN>
__device__ __forceinline__ void dft_reg(float2* v);

// in-register DFT of length L = 3*M (M a power of two, L dividing 48): the three
// decimated sequences v[3m + r] by M-point DFTs, twiddled by W_L^{r k} and joined
// by a 3-point DFT, X[k + M q] = sum_r W_L^{r k} Y_r[k] W_3^{r q}
template <int L, int SIGN>
__device__ __forceinline__ void dft_reg3(float2* v) {
  constexpr int M = L / 3, S = 48 / L;  // angle 2 pi j/L = 2 pi (S j)/48
  float2 y[3][M];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
#pragma unroll
    for (int m = 0; m < M; ++m) y[r][m] = v[3 * m + r];
    dft_reg<M, SIGN>(y[r]);
  }
  const float c3 = -0.5f, s3 = SIGN * 0.86602540378443864676f;  // W_3 = exp(SIGN 2 pi i/3)
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const float2 z0 = y[0][k];
    const float2 z1 = k == 0 ? y[1][k] : cmul(y[1][k], make_float2(cos48(S * k), SIGN * sin48(S * k)));
    const float2 z2 = k == 0 ? y[2][k] : cmul(y[2][k], make_float2(cos48(2 * S * k), SIGN * sin48(2 * S * k)));
    const float2 a = make_float2(z1.x + z2.x, z1.y + z2.y), b = make_float2(z1.x - z2.x, z1.y - z2.y);
    v[k] = make_float2(z0.x + a.x, z0.y + a.y);
    // z0 + W3 z1 + W3^2 z2 = z0 + c3 (z1 + z2) + i s3 (z1 - z2), and its conjugate-twiddle partner
    const float2 m0 = make_float2(z0.x + c3 * a.x, z0.y + c3 * a.y), m1 = make_float2(-s3 * b.y, s3 * b.x);
    v[k + M] = make_float2(m0.x + m1.x, m0.y + m1.y);
    v[k + 2 * M] = make_float2(m0.x - m1.x, m0.y - m1.y);
  }
}

// in-register DFT of length L on v[0..L-1], natural order out; SIGN = -1 forward
// (exp(-2 pi i jk/L)), +1 inverse.  Powers of two <= 32 by decimation in time,
// 24 and 48 by dft_reg3.
template <int L, int SIGN>
__device__ __forceinline__ void dft_reg(float2* v) {
  if constexpr (L % 3 == 0) {
    dft_reg3<L, SIGN>(v);
  } else {
    bitrev_perm<L>(v, std::make_integer_sequence<int, L>{});
    if constexpr (L > 1) dft_stage<L, SIGN, 2>(v);
  }
}

// sequence element n at s[n*ES]; ROW layout has ES = 1 and a padded exchange,
// COL layout has ES = pitch of the interleaved columns and a swizzled exchange
template <int R, int T, bool ROW>
__device__ __forceinline__ int xidx(int k1, int t, int es) {
  if (ROW) return k1 * (T + 1) + t;
  return (k1 * T + ((t + k1) & (T - 1))) * es;
}

// stage 1 (R-point DFT + twiddle) from registers v, exchange, stage 2; result
// in natural order in s.  The T threads of the group call it together.
template <int N, int R, int T, int SIGN, bool ROW>
__device__ __forceinline__ void fft_from_regs(float2* v, float2* s, int es, int t, const float2* __restrict__ tw) {
  dft_reg<R, SIGN>(v);
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) {
    float2 w = __ldg(&tw[k1 * T + t]);  // = exp(-2 pi i ((t k1) mod N)/N)
    if (SIGN > 0) w.y = -w.y;
    v[k1] = cmul(v[k1], w);
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < R; ++k1) s[xidx<R, T, ROW>(k1, t, es)] = v[k1];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < R / T; ++m)
#pragma unroll
    for (int tt = 0; tt < T; ++tt) v[m * T + tt] = s[xidx<R, T, ROW>(t + T * m, tt, es)];
  __syncwarp();
#pragma unroll
  for (int m = 0; m < R / T; ++m) dft_reg<T, SIGN>(v + m * T);
#pragma unroll
  for (int m = 0; m < R / T; ++m)
#pragma unroll
    for (int k2 = 0; k2 < T; ++k2) s[(t + T * m + R * k2) * (ROW ? 1 : es)] = v[m * T + k2];
  __syncwarp();
}

// ---------------------------------------------------------------------------
// Transposed-layout passes.  Every transform runs along contiguous memory: a
// group of T threads loads its row straight into registers (coalesced), and the
// pass writes its output with the next transform's dimension innermost (through
// the natural-order result in shared memory, read across the CTA's 8 rows).
// Per complex point that is two shared-memory round trips (the in-warp exchange
// and the transpose) instead of three, and no global->shared copy.  Layouts of
// a level with n = N, H = N/2 + 1, cp = complex row pitch:
//   S1 [z][kx][y]  after x r2c           (in L.ext)
//   S2 [kx][ky][z] after y forward       (in L.rho)
//   S3 [z][kx][ky] after z+Green+z^-1    (components 0,1,2 in force 1, force 2, L.ext)
//   S4 [z][y][kx]  after y^-1, pitch cp  (components 0,1,2 in force 0, 1, 2)
// then x c2r in place gives the real force meshes.  (Same transforms, bit for bit,
// as in-place column passes over the [z][y][kx] spectrum, which moved the same
// bytes at 3 TB/s: their global->shared copies and column-wise shared accesses
// saturated the L1 data path.)

// group stride in float2 for RT rows per CTA: >= N + R + 8 and == 16/RT (mod 16),
// so that reading one column across the RT rows (two rows per thread) is free of
// bank conflicts
template <int N, int R, int RT>
constexpr int cs_row() {
  return ((N + R + 8 + 15) / 16) * 16 + 16 / RT;
}

// x r2c of 8 rows (4 packed complex transforms) of one z-plane -> S1
template <int N, int R, int T>
__global__ void __launch_bounds__(4 * T) k_xr2c_t(const float* __restrict__ rho, int rp, float2* __restrict__ out,
                                                  const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int CS = cs_row<N, R, 4>();
  constexpr int H = N / 2 + 1;
  constexpr int YB = N / 8;
  const int z = blockIdx.x / YB, y0 = (blockIdx.x - z * YB) * 8;
  const int g = threadIdx.x / T, t = threadIdx.x - g * T;
  const float* ra = rho + ((size_t)z * N + y0 + 2 * g) * rp;
  const float* rb = ra + rp;
  float2 v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = make_float2(__ldg(&ra[t + T * q]), __ldg(&rb[t + T * q]));
  fft_from_regs<N, R, T, -1, true>(v, sm + g * CS, 1, t, tw);
  __syncthreads();
  float2* o = out + (size_t)z * H * N + y0;
  for (int i = threadIdx.x; i < 4 * H; i += 4 * T) {
    const int k = i >> 2, p = i & 3;
    const float2 Zk = sm[p * CS + k];
    const float2 Zm = sm[p * CS + (k ? N - k : 0)];
    const float2 A = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    const float2 B = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
    *reinterpret_cast<float4*>(o + (size_t)k * N + 2 * p) = make_float4(A.x, A.y, B.x, B.y);
  }
}

// natural-order results of the CTA's RT rows (group stride CS) -> out + B0 + k*B1 + r,
// two rows per thread (16-byte stores), rows r >= nrows skipped
template <int N, int NT, int RT, int CS>
__device__ __forceinline__ void store_transposed(const float2* sm, float2* __restrict__ out, size_t B0, size_t B1,
                                                 int nrows) {
  constexpr int HP = RT / 2;  // row pairs
  for (int i = threadIdx.x; i < HP * N; i += NT) {
    const int k = i / HP, r = 2 * (i % HP);
    const float2 a = sm[r * CS + k], b = sm[(r + 1) * CS + k];
    float2* o = out + B0 + (size_t)k * B1 + r;
    if (r + 1 < nrows) *reinterpret_cast<float4*>(o) = make_float4(a.x, a.y, b.x, b.y);
    else if (r < nrows) *o = a;
  }
}

// one transform along rows of 8 consecutive row indices, transposed output:
//   MODE 0  y forward : S1 rows (z, kx), CTA = (kx, 8 z)  -> S2 [kx][ky][z]
//   MODE 1  y inverse : S3 rows (z, kx), CTA = (z, 8 kx)  -> S4 [z][y][kx] (pitch cp)
template <int N, int R, int T, int SIGN, int MODE>
__global__ void __launch_bounds__(8 * T) k_row_t(const float2* __restrict__ in, float2* __restrict__ out, int cp,
                                                 const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int CS = cs_row<N, R, 8>();
  constexpr int H = N / 2 + 1;
  const int g = threadIdx.x / T, t = threadIdx.x - g * T;
  size_t row, B0, B1;
  int nrows = 8;
  if (MODE == 0) {
    constexpr int ZB = N / 8;
    const int kx = blockIdx.x / ZB, z0 = (blockIdx.x - kx * ZB) * 8;
    row = ((size_t)(z0 + g) * H + kx) * N;
    B0 = (size_t)kx * N * N + z0;
    B1 = N;
  } else {
    constexpr int KB = (H + 7) / 8;
    const int z = blockIdx.x / KB, kx0 = (blockIdx.x - z * KB) * 8;
    nrows = min(8, H - kx0);
    row = ((size_t)z * H + min(kx0 + g, H - 1)) * N;
    B0 = (size_t)z * N * cp + kx0;
    B1 = cp;
  }
  float2 v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = __ldg(&in[row + t + T * q]);
  fft_from_regs<N, R, T, SIGN, true>(v, sm + g * CS, 1, t, tw);
  __syncthreads();
  store_transposed<N, 8 * T, 8, CS>(sm, out, B0, B1, nrows);
}

// z forward, Green multiply, z inverse on S2 rows (kx, ky), CTA = (kx, 8 ky);
// the three components go out transposed to S3 in o0, o1, o2.  The forward
// spectrum stays in registers (255 of them: one CTA per SM; staging the Green rows
// in shared memory, or keeping the spectrum there with the inverse exchanges in a
// second buffer so that three 128-thread CTAs fit an SM, measured slower: 23.3 ms
// against 21.7 ms for the 1024^3 solve).
template <int N, int R, int T>
__global__ void __launch_bounds__(8 * T) k_zgreen_t(const float2* __restrict__ in, float2* __restrict__ o0,
                                                    float2* __restrict__ o1, float2* __restrict__ o2,
                                                    const float2* __restrict__ tw, const float* __restrict__ kern,
                                                    int kp, float ksc) {
  extern __shared__ float2 sm[];
  constexpr int CS = cs_row<N, R, 8>();
  constexpr int H = N / 2 + 1;
  constexpr int nh = N / 2;
  constexpr int YB = N / 8;
  const int kx = blockIdx.x / YB, ky0 = (blockIdx.x - kx * YB) * 8;
  const int g = threadIdx.x / T, t = threadIdx.x - g * T;
  const int ky = ky0 + g;
  const size_t ksz = (size_t)kp * kp * kp;
  const float2* bi = in + ((size_t)kx * N + ky) * N;
  float2 v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = __ldg(&bi[t + T * q]);
  float2* s = sm + g * CS;
  fft_from_regs<N, R, T, -1, true>(v, s, 1, t, tw);
  float2 keep[R];
#pragma unroll
  for (int q = 0; q < R; ++q) keep[q] = s[t + T * q];
  const int fy = ky <= nh ? ky : N - ky;
  const float sy = ky <= nh ? 1.f : -1.f;
  const size_t B0 = (size_t)kx * N + ky0, B1 = (size_t)H * N;
#pragma unroll 1
  for (int d = 0; d < 3; ++d) {
    const float* K = kern + d * ksz + ((size_t)fy * kp + kx) * kp;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int kz = t + T * q;
      const int fz = kz <= nh ? kz : N - kz;
      float kv = __ldg(&K[fz]) * ksc;
      if (d == 1) kv *= sy;
      if (d == 2 && kz > nh) kv = -kv;
      v[q] = make_float2(-keep[q].y * kv, keep[q].x * kv);
    }
    __syncwarp();
    fft_from_regs<N, R, T, 1, true>(v, s, 1, t, tw);
    __syncthreads();
    store_transposed<N, 8 * T, 8, CS>(sm, d == 0 ? o0 : (d == 1 ? o1 : o2), B0, B1, 8);
    __syncthreads();
  }
}

// in-place transform of 8 contiguous rows of length N (the z pass of the forward
// 3-D transform on S2)
template <int N, int R, int T, int SIGN>
__global__ void __launch_bounds__(8 * T) k_row_inplace(float2* __restrict__ data, long long nrows,
                                                       const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  constexpr int CS = cs_row<N, R, 8>();
  const int g = threadIdx.x / T, t = threadIdx.x - g * T;
  const long long row = min((long long)blockIdx.x * 8 + g, nrows - 1);
  float2* b = data + (size_t)row * N;
  float2 v[R];
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = b[t + T * q];
  float2* s = sm + g * CS;
  fft_from_regs<N, R, T, SIGN, true>(v, s, 1, t, tw);
  if ((long long)blockIdx.x * 8 + g < nrows) {
#pragma unroll
    for (int q = 0; q < R; ++q) b[t + T * q] = s[t + T * q];
  }
}

// x c2r of the three force components (S4 rows of RB row pairs, in place) with
// max f^2, as k_xc2r3 but loading the half spectra straight into registers
template <int N, int R, int T, int RB>
__global__ void __launch_bounds__(3 * T * RB, 4) k_xc2r3_t(float* __restrict__ data, size_t comp_stride, int rp,
                                                        int npairs, const float2* __restrict__ tw,
                                                        unsigned int* __restrict__ f2_bits) {
  extern __shared__ float2 sm[];
  constexpr int CS = N + R + 8;
  constexpr int NT = 3 * T * RB;
  constexpr int nh = N / 2;
  const int pair0 = blockIdx.x * RB;
  const int cp = rp / 2;
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  {
    const int c = g / RB, q = g - c * RB;
    const int pr = min(pair0 + q, npairs - 1);
    const float2* A = reinterpret_cast<const float2*>(data + c * comp_stride) + (size_t)(2 * pr) * cp;
    const float2* B = A + cp;
    // Z[n] = A[n] + i B[n] for n <= N/2 and conj(A[N-n]) + i conj(B[N-n]) above; the
    // imaginary parts of A, B at n = 0 and N/2 are dropped.  n < N/2 exactly when
    // k < R/2 (n = N/2 is t = 0, k = R/2), so every load is unconditional.
    float2 a[R], b[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int n = t + T * k;
      const int m = (k < R / 2) ? n : N - n;
      a[k] = __ldg(&A[m]);
      b[k] = __ldg(&B[m]);
    }
    float2 v[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int n = t + T * k;
      if (n == 0 || n == nh) v[k] = make_float2(a[k].x, b[k].x);
      else if (k < R / 2) v[k] = make_float2(a[k].x - b[k].y, a[k].y + b[k].x);
      else v[k] = make_float2(a[k].x + b[k].y, b[k].x - a[k].y);
    }
    fft_from_regs<N, R, T, 1, true>(v, sm + g * CS, 1, t, tw);
  }
  __syncthreads();
  // two nodes per thread: one 16-byte shared load and two 8-byte stores per component
  float f2max = 0.f;
  for (int i = threadIdx.x; i < RB * (N / 2); i += NT) {
    const int q = i / (N / 2), j = 2 * (i - q * (N / 2));
    if (pair0 + q >= npairs) continue;
    const size_t ra = (size_t)(2 * (pair0 + q)) * rp;
    float fa[3][2], fb[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float4 z = *reinterpret_cast<const float4*>(&sm[(c * RB + q) * CS + j]);
      float* base = data + c * comp_stride;
      *reinterpret_cast<float2*>(&base[ra + j]) = make_float2(z.x, z.z);
      *reinterpret_cast<float2*>(&base[ra + rp + j]) = make_float2(z.y, z.w);
      fa[c][0] = z.x; fa[c][1] = z.z;
      fb[c][0] = z.y; fb[c][1] = z.w;
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const float a2 = __fadd_rn(__fadd_rn(__fmul_rn(fa[0][e], fa[0][e]), __fmul_rn(fa[1][e], fa[1][e])),
                                 __fmul_rn(fa[2][e], fa[2][e]));
      const float b2 = __fadd_rn(__fadd_rn(__fmul_rn(fb[0][e], fb[0][e]), __fmul_rn(fb[1][e], fb[1][e])),
                                 __fmul_rn(fb[2][e], fb[2][e]));
      f2max = fmaxf(f2max, fmaxf(a2, b2));
    }
  }
  for (int o = 16; o > 0; o >>= 1) f2max = fmaxf(f2max, __shfl_xor_sync(0xffffffffu, f2max, o));
  if ((threadIdx.x & 31) == 0) atomicMax(f2_bits, __float_as_uint(f2max));
}


template <int N, int R, int T>
int run_poisson_t(cube_ctx* ctx, MeshLevel& L, unsigned int* f2_bits, KickScale ks) {
  constexpr int H = N / 2 + 1;
  constexpr int RB3 = (T >= 32) ? 2 : (T >= 16 ? 4 : 8);
  const float2* tw = L.plan.tw2;
  const size_t cstride = (size_t)N * L.plane;  // floats per force component
  float* F[3] = {L.force, L.force + cstride, L.force + 2 * cstride};
  const size_t sm1 = sizeof(float2) * 4 * cs_row<N, R, 4>();
  const size_t sm8 = sizeof(float2) * 8 * cs_row<N, R, 8>();
  const size_t sm3 = sizeof(float2) * 3 * RB3 * (N + R + 8);
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_xr2c_t<N, R, T>, sm1));
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_row_t<N, R, T, -1, 0>, sm8));
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_row_t<N, R, T, 1, 1>, sm8));

  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_xc2r3_t<N, R, T, RB3>, sm3));
  float2* ext = reinterpret_cast<float2*>(L.ext);
  float2* rho = reinterpret_cast<float2*>(L.rho);
  // x r2c: rho -> S1 (ext)
  k_xr2c_t<N, R, T><<<N * (N / 8), 4 * T, sm1, ctx->stream>>>(L.rho, L.rp, ext, tw);
  CUBE_LAUNCH_CHECK(ctx);
  // y forward: S1 -> S2 (rho)
  k_row_t<N, R, T, -1, 0><<<H * (N / 8), 8 * T, sm8, ctx->stream>>>(ext, rho, L.cp, tw);
  CUBE_LAUNCH_CHECK(ctx);
  // z forward, Green, z inverse: S2 -> S3 of components 0, 1, 2 in force 1, force 2, ext
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_zgreen_t<N, R, T>, sm8));
  k_zgreen_t<N, R, T><<<H * (N / 8), 8 * T, sm8, ctx->stream>>>(
      rho, reinterpret_cast<float2*>(F[1]), reinterpret_cast<float2*>(F[2]), ext, tw, L.kern, L.kern_pitch,
      cube_kick_scalar(ks));
  CUBE_LAUNCH_CHECK(ctx);
  // y inverse, component by component into the freed buffers: S3 -> S4 in force 0, 1, 2
  const float2* s3[3] = {reinterpret_cast<float2*>(F[1]), reinterpret_cast<float2*>(F[2]), ext};
  for (int d = 0; d < 3; ++d) {
    k_row_t<N, R, T, 1, 1><<<N * ((H + 7) / 8), 8 * T, sm8, ctx->stream>>>(s3[d], reinterpret_cast<float2*>(F[d]),
                                                                           L.cp, tw);
    CUBE_LAUNCH_CHECK(ctx);
  }
  // x c2r of the three components in place, max f^2
  const int npairs = N * N / 2;
  k_xc2r3_t<N, R, T, RB3><<<(npairs + RB3 - 1) / RB3, 3 * T * RB3, sm3, ctx->stream>>>(L.force, cstride, L.rp,
                                                                                       npairs, tw, f2_bits);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

// forward 3-D r2c: x (data -> ext), y (ext -> data), z in place; the spectrum ends
// in data as [kx][ky][kz], dense rows of N
template <int N, int R, int T>
int run_forward3_t(cube_ctx* ctx, MeshLevel& L, float* data) {
  constexpr int H = N / 2 + 1;
  const float2* tw = L.plan.tw2;
  const size_t sm1 = sizeof(float2) * 4 * cs_row<N, R, 4>();
  const size_t sm8 = sizeof(float2) * 8 * cs_row<N, R, 8>();
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_xr2c_t<N, R, T>, sm1));
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_row_t<N, R, T, -1, 0>, sm8));
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_row_inplace<N, R, T, -1>, sm8));
  float2* ext = reinterpret_cast<float2*>(L.ext);
  float2* d2 = reinterpret_cast<float2*>(data);
  k_xr2c_t<N, R, T><<<N * (N / 8), 4 * T, sm1, ctx->stream>>>(data, L.rp, ext, tw);
  CUBE_LAUNCH_CHECK(ctx);
  k_row_t<N, R, T, -1, 0><<<H * (N / 8), 8 * T, sm8, ctx->stream>>>(ext, d2, L.cp, tw);
  CUBE_LAUNCH_CHECK(ctx);
  const long long nrows = (long long)H * N;
  k_row_inplace<N, R, T, -1><<<(unsigned)((nrows + 7) / 8), 8 * T, sm8, ctx->stream>>>(d2, nrows, tw);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

}  // namespace

int cube_fft_forward3_fast(cube_ctx* ctx, MeshLevel& L, float* data, int* rc, int* kx_major) {
  *kx_major = 1;
  switch (L.n) {
#define CUBE_F3(n, r, t) \
  case n: *rc = run_forward3_t<n, r, t>(ctx, L, data); return 1;
    CUBE_F3(1024, 32, 32)
    CUBE_F3(512, 32, 16)
    CUBE_F3(256, 16, 16)
    CUBE_F3(128, 16, 8)
    CUBE_F3(64, 8, 8)
    CUBE_F3(32, 8, 4)
    CUBE_F3(768, 48, 16)
    CUBE_F3(384, 48, 8)
    CUBE_F3(192, 24, 8)
    CUBE_F3(96, 24, 4)
#undef CUBE_F3
    default: return 0;
  }
}

// returns 1 if handled by a register-resident path
int cube_fft_poisson_fast(cube_ctx* ctx, MeshLevel& L, unsigned int* f2_bits, KickScale ks, int* rc) {
  switch (L.n) {
#define CUBE_PS(n, r, t) \
  case n: *rc = run_poisson_t<n, r, t>(ctx, L, f2_bits, ks); return 1;
    CUBE_PS(1024, 32, 32)
    CUBE_PS(512, 32, 16)
    CUBE_PS(256, 16, 16)
    CUBE_PS(128, 16, 8)
    CUBE_PS(64, 8, 8)
    CUBE_PS(32, 8, 4)
    CUBE_PS(768, 48, 16)
    CUBE_PS(384, 48, 8)
    CUBE_PS(192, 24, 8)
    CUBE_PS(96, 24, 4)
#undef CUBE_PS
    default: return 0;
  }
}
