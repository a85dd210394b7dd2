/*
 * k_fft.cu -- 3-D real FFT Poisson solve of one mesh level (fine or coarse).
 *
 * Replaces the reference's FFTW calls of the PM step: the fine r2c + 3x
 * (x i*kern_f, c2r) of pm.f90:112-125 and the coarse pencil_fft_forward +
 * 3x (x i*kern_c, pencil_fft_backward) of pm.f90:288-300.  On one GPU the
 * fine level is one periodic nf^3 transform: the fine kernel has a support of
 * +-(nf_cutoff-1) fine cells, smaller than the nfb=24 buffer of the
 * reference's per-tile meshes, so the per-tile circular convolutions and the
 * periodic one agree cell for cell in exact arithmetic (checked against the
 * per-tile oracle in the tests).
 *
 * Passes over HBM (each a Stockham mixed-radix FFT in shared memory):
 *   X  : r2c along x, two real rows packed into one complex transform
 *   Y  : complex along y, TK consecutive kx columns per CTA
 *   Z  : complex along z, then per force component d: x i*K_d(k), inverse
 *        along z, store  (one read, three writes)
 *   Y^-1 x3, X^-1 (c2r) x3 with the max of f^2 fused (pm.f90:126,328)
 * The half spectrum lives in place in the real arrays (row pitch rp floats,
 * complex pitch cp = rp/2).  Normalisation 1/n^3 is folded into K.
 */
#include "cube_internal.cuh"

#include <cmath>

namespace {

// complex arithmetic on float2 (the FP32 meshes) or double2 (the FP64 Poisson mode)
template <typename C> struct CT;
template <> struct CT<float2> { typedef float R; };
template <> struct CT<double2> { typedef double R; };
__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
template <typename C2>
__device__ __forceinline__ C2 cmulf(C2 a, C2 b) {
  return mk2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C2>
__device__ __forceinline__ C2 caddf(C2 a, C2 b) { return mk2(a.x + b.x, a.y + b.y); }
template <typename C2>
__device__ __forceinline__ C2 csubf(C2 a, C2 b) { return mk2(a.x - b.x, a.y - b.y); }
// multiply by sign*i
template <typename C2>
__device__ __forceinline__ C2 mul_si(C2 a, typename CT<C2>::R s) { return mk2(-s * a.y, s * a.x); }

template <int P, typename C2>
__device__ __forceinline__ void dft(C2* v, typename CT<C2>::R s) {
  typedef typename CT<C2>::R R;
  if (P == 2) {
    const C2 a = v[0], b = v[1];
    v[0] = caddf(a, b);
    v[1] = csubf(a, b);
  } else if (P == 4) {
    const C2 t0 = caddf(v[0], v[2]), t1 = csubf(v[0], v[2]);
    const C2 t2 = caddf(v[1], v[3]), t3 = mul_si(csubf(v[1], v[3]), s);
    v[0] = caddf(t0, t2);
    v[2] = csubf(t0, t2);
    v[1] = caddf(t1, t3);
    v[3] = csubf(t1, t3);
  } else if (P == 3) {
    const R c = (R)-0.5, sn = (R)0.86602540378443864676;
    const C2 sm = caddf(v[1], v[2]), df = csubf(v[1], v[2]);
    const C2 m = mk2(v[0].x + c * sm.x, v[0].y + c * sm.y);
    const C2 r = mul_si(mk2(sn * df.x, sn * df.y), s);
    v[0] = caddf(v[0], sm);
    v[1] = caddf(m, r);
    v[2] = csubf(m, r);
  } else if (P == 5) {
    // X_k = sum_r v_r w^{rk}, w = exp(s 2 pi i/5)
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
    const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
    const C2 a1 = caddf(v[1], v[4]), b1 = csubf(v[1], v[4]);
    const C2 a2 = caddf(v[2], v[3]), b2 = csubf(v[2], v[3]);
    const C2 m1 = mk2(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const C2 m2 = mk2(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const C2 n1 = mul_si(mk2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), s);
    const C2 n2 = mul_si(mk2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), s);
    v[0] = caddf(v[0], caddf(a1, a2));
    v[1] = caddf(m1, n1);
    v[4] = csubf(m1, n1);
    v[2] = caddf(m2, n2);
    v[3] = csubf(m2, n2);
  }
}

// One Stockham stage on nseq sequences of length n stored at buf[s*ss + j*js].
// Reads are staged in registers so the stage runs in place.
template <int P, int MAXIT, typename C2>
__device__ __forceinline__ void fft_stage(C2* buf, int n, int nseq, int ss, int js, int T,
                                          const C2* __restrict__ tw, typename CT<C2>::R sgn, bool seq_fast) {
  const int nb = n / P;
  const int total = nb * nseq;
  const int nthr = blockDim.x;
  C2 v[MAXIT][P];
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int t = threadIdx.x + it * nthr;
    if (t < total) {
      int s, i;
      if (seq_fast) { s = t % nseq; i = t / nseq; } else { i = t % nb; s = t / nb; }
#pragma unroll
      for (int r = 0; r < P; ++r) v[it][r] = buf[s * ss + (i + r * nb) * js];
    }
  }
  __syncthreads();
  const int tstep = n / (P * T);
#pragma unroll
  for (int it = 0; it < MAXIT; ++it) {
    const int t = threadIdx.x + it * nthr;
    if (t < total) {
      int s, i;
      if (seq_fast) { s = t % nseq; i = t / nseq; } else { i = t % nb; s = t / nb; }
      const int k = i % T;
#pragma unroll
      for (int r = 1; r < P; ++r) {
        C2 w = __ldg(&tw[r * k * tstep]);
        w.y *= -sgn;  // table holds exp(-2 pi i j/n); sgn=-1 forward, +1 inverse
        v[it][r] = cmulf(v[it][r], w);
      }
      dft<P>(v[it], sgn);
      const int j0 = (i - k) * P + k;
#pragma unroll
      for (int r = 0; r < P; ++r) buf[s * ss + (j0 + r * T) * js] = v[it][r];
    }
  }
  __syncthreads();
}

// the plan's twiddle table of the complex type
__device__ __forceinline__ const float2* plan_tw(const FftPlan& pl, float2*) { return pl.tw; }
__device__ __forceinline__ const double2* plan_tw(const FftPlan& pl, double2*) { return pl.twd; }

template <int MAXIT, typename C2>
__device__ void fft_smem(C2* buf, int n, int nseq, int ss, int js, const FftPlan& pl, typename CT<C2>::R sgn,
                         bool seq_fast) {
  const C2* tw = plan_tw(pl, buf);
  int T = 1;
  for (int st = 0; st < pl.nst; ++st) {
    const int p = pl.radix[st];
    if (p == 4) fft_stage<4, MAXIT>(buf, n, nseq, ss, js, T, tw, sgn, seq_fast);
    else if (p == 2) fft_stage<2, MAXIT * 2>(buf, n, nseq, ss, js, T, tw, sgn, seq_fast);
    else if (p == 3) fft_stage<3, MAXIT * 2>(buf, n, nseq, ss, js, T, tw, sgn, seq_fast);
    else if (p == 5) fft_stage<5, MAXIT>(buf, n, nseq, ss, js, T, tw, sgn, seq_fast);
    T *= p;
  }
}

__device__ __forceinline__ void atomic_max_pos(unsigned int* addr, float v) {
  atomicMax(addr, __float_as_uint(v));  // v >= 0: IEEE order equals unsigned order
}

// f^2 of the three components at one node: FP32 in the reference's order, or FP64
// (the FP64 mode), reported as the FP32 value of the maximum
__device__ __forceinline__ float f2_of(const float f[3]) {
  return __fadd_rn(__fadd_rn(__fmul_rn(f[0], f[0]), __fmul_rn(f[1], f[1])), __fmul_rn(f[2], f[2]));
}
__device__ __forceinline__ float f2_of(const double f[3]) { return (float)(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]); }

// ---------------------------------------------------------------------------
// X pass: r2c (inverse=0) or c2r (inverse=1) along contiguous rows.
// Rows r = z*n + y at data + r*rp.  A CTA takes RPB row pairs; for the c2r of
// the force (ncomp=3) it takes the same rows of the three components and
// reduces max(fx^2+fy^2+fz^2).
template <int MAXIT, typename C2>
__global__ void k_fft_x(typename CT<C2>::R* __restrict__ data, size_t comp_stride, int ncomp, int n, int rp,
                        int npairs, int rpb, FftPlan pl, int inverse, unsigned int* f2_bits) {
  typedef typename CT<C2>::R R;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C2* sm = reinterpret_cast<C2*>(sm_raw);
  const int ss = n + 1;  // odd pitch spreads rows over banks
  const int pair0 = blockIdx.x * rpb;
  const int np_blk = min(rpb, npairs - pair0);
  const int cp = rp / 2;
  for (int c = 0; c < ncomp; ++c) {
    R* base = data + c * comp_stride;
    C2* buf = sm + (size_t)c * rpb * ss;
    if (!inverse) {
      for (int t = threadIdx.x; t < np_blk * n; t += blockDim.x) {
        const int q = t / n, j = t - q * n;
        const size_t ra = (size_t)(2 * (pair0 + q)) * rp;
        buf[q * ss + j] = mk2(base[ra + j], base[ra + rp + j]);
      }
    } else {
      const C2* cb = reinterpret_cast<const C2*>(base);
      const int nh = n / 2;
      for (int t = threadIdx.x; t < np_blk * n; t += blockDim.x) {
        const int q = t / n, k = t - q * n;
        const size_t ra = (size_t)(2 * (pair0 + q)) * cp;
        C2 z;
        if (k == 0 || k == nh) {
          const C2 A = cb[ra + k], B = cb[ra + cp + k];
          z = mk2(A.x, B.x);
        } else if (k < nh) {
          const C2 A = cb[ra + k], B = cb[ra + cp + k];
          z = mk2(A.x - B.y, A.y + B.x);
        } else {
          const C2 A = cb[ra + (n - k)], B = cb[ra + cp + (n - k)];
          z = mk2(A.x + B.y, B.x - A.y);
        }
        buf[q * ss + k] = z;
      }
    }
  }
  __syncthreads();
  for (int c = 0; c < ncomp; ++c)
    fft_smem<MAXIT>(sm + (size_t)c * rpb * ss, n, np_blk, ss, 1, pl, inverse ? (R)1 : (R)-1, false);
  if (!inverse) {
    R* base = data;
    C2* cb = reinterpret_cast<C2*>(base);
    const int nh = n / 2;
    const R half = (R)0.5;
    for (int t = threadIdx.x; t < np_blk * (nh + 1); t += blockDim.x) {
      const int q = t / (nh + 1), k = t - q * (nh + 1);
      const C2 Zk = sm[q * ss + k];
      const C2 Zm = sm[q * ss + ((n - k) % n)];
      const C2 Zc = mk2(Zm.x, -Zm.y);
      const C2 A = mk2(half * (Zk.x + Zc.x), half * (Zk.y + Zc.y));
      const C2 D = csubf(Zk, Zc);
      const C2 B = mk2(half * D.y, -half * D.x);
      const size_t ra = (size_t)(2 * (pair0 + q)) * cp;
      cb[ra + k] = A;
      cb[ra + cp + k] = B;
    }
  } else {
    float f2max = 0.f;
    for (int t = threadIdx.x; t < np_blk * n; t += blockDim.x) {
      const int q = t / n, j = t - q * n;
      const size_t ra = (size_t)(2 * (pair0 + q)) * rp;
      R fa[3], fb[3];
      for (int c = 0; c < ncomp; ++c) {
        const C2 z = sm[(size_t)c * rpb * ss + q * ss + j];
        R* base = data + c * comp_stride;
        base[ra + j] = z.x;
        base[ra + rp + j] = z.y;
        fa[c] = z.x;
        fb[c] = z.y;
      }
      if (ncomp == 3 && f2_bits) f2max = fmaxf(f2max, fmaxf(f2_of(fa), f2_of(fb)));
    }
    if (ncomp == 3 && f2_bits) {
      for (int o = 16; o > 0; o >>= 1) f2max = fmaxf(f2max, __shfl_xor_sync(0xffffffffu, f2max, o));
      if ((threadIdx.x & 31) == 0) atomic_max_pos(f2_bits, f2max);
    }
  }
}

// ---------------------------------------------------------------------------
// Column pass along y (other = z) or z (other = y): TK consecutive kx columns.
template <int MAXIT, typename C2>
__global__ void k_fft_col(C2* __restrict__ base, size_t comp_stride, int n, int ncol, int tk,
                          long long jstride, long long ostride, FftPlan pl, typename CT<C2>::R sgn) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C2* sm = reinterpret_cast<C2*>(sm_raw);
  const int kx0 = blockIdx.x * tk;
  const int nk = min(tk, ncol - kx0);
  C2* b = base + blockIdx.z * comp_stride + (size_t)blockIdx.y * ostride + kx0;
  for (int t = threadIdx.x; t < n * tk; t += blockDim.x) {
    const int j = t / tk, c = t - j * tk;
    sm[j * tk + c] = (c < nk) ? b[(size_t)j * jstride + c] : mk2((typename CT<C2>::R)0, (typename CT<C2>::R)0);
  }
  __syncthreads();
  fft_smem<MAXIT>(sm, n, tk, 1, tk, pl, sgn, true);
  for (int t = threadIdx.x; t < n * tk; t += blockDim.x) {
    const int j = t / tk, c = t - j * tk;
    if (c < nk) b[(size_t)j * jstride + c] = sm[j * tk + c];
  }
}

// Fused z pass: forward along z, then for each component d multiply by i*K_d
// (octant table, odd in k_d, even in the others) and transform back.
template <int MAXIT, typename C2>
__global__ void k_fft_z_green(const C2* __restrict__ in, C2* __restrict__ out0, size_t comp_stride,
                              int n, int ncol, int tk, long long jstride, long long ostride, FftPlan pl,
                              const typename CT<C2>::R* __restrict__ kern, int kp, typename CT<C2>::R ksc) {
  typedef typename CT<C2>::R R;
  extern __shared__ __align__(16) unsigned char sm_raw[];
  C2* A = reinterpret_cast<C2*>(sm_raw);
  C2* B = A + (size_t)n * tk;
  const int kx0 = blockIdx.x * tk;
  const int nk = min(tk, ncol - kx0);
  const int ky = blockIdx.y;
  const C2* bi = in + (size_t)ky * ostride + kx0;
  for (int t = threadIdx.x; t < n * tk; t += blockDim.x) {
    const int j = t / tk, c = t - j * tk;
    A[j * tk + c] = (c < nk) ? bi[(size_t)j * jstride + c] : mk2((R)0, (R)0);
  }
  __syncthreads();
  fft_smem<MAXIT>(A, n, tk, 1, tk, pl, (R)-1, true);
  const int nh = n / 2;
  const int fy = ky <= nh ? ky : n - ky;
  const R sy = ky <= nh ? (R)1 : (R)-1;
  const size_t ksz = (size_t)kp * kp * kp;
  for (int d = 0; d < 3; ++d) {
    const R* K = kern + d * ksz;
    for (int t = threadIdx.x; t < n * tk; t += blockDim.x) {
      const int kz = t / tk, c = t - kz * tk;
      const int kx = kx0 + c;
      R kv = 0;
      if (c < nk) {
        const int fz = kz <= nh ? kz : n - kz;
        kv = __ldg(&K[((size_t)fy * kp + kx) * kp + fz]);
        if (d == 1) kv *= sy;
        if (d == 2 && kz > nh) kv = -kv;
        kv *= ksc;
      }
      const C2 a = A[kz * tk + c];
      B[kz * tk + c] = mk2(-a.y * kv, a.x * kv);
    }
    __syncthreads();
    fft_smem<MAXIT>(B, n, tk, 1, tk, pl, (R)1, true);
    C2* bo = out0 + d * comp_stride + (size_t)ky * ostride + kx0;
    for (int t = threadIdx.x; t < n * tk; t += blockDim.x) {
      const int j = t / tk, c = t - j * tk;
      if (c < nk) bo[(size_t)j * jstride + c] = B[j * tk + c];
    }
    __syncthreads();
  }
}

int pick_threads(int butterflies4, int maxit) {
  int t = (butterflies4 + maxit - 1) / maxit;
  t = ((t + 31) / 32) * 32;
  return t < 64 ? 64 : (t > 1024 ? 1024 : t);
}

}  // namespace

// ---------------------------------------------------------------------------
int cube_fft_plan(cube_ctx* ctx, FftPlan& p, int n) {
  p.n = n;
  p.nst = 0;
  p.tw = p.tw2 = nullptr;
  p.twd = nullptr;
  int m = n;
  while (m % 4 == 0) { p.radix[p.nst++] = 4; m /= 4; }
  while (m % 2 == 0) { p.radix[p.nst++] = 2; m /= 2; }
  while (m % 3 == 0) { p.radix[p.nst++] = 3; m /= 3; }
  while (m % 5 == 0) { p.radix[p.nst++] = 5; m /= 5; }
  if (m != 1 || p.nst > CUBE_MAX_RADIX_STAGES) {
    ctx->err = "mesh size must factor into 2, 3 and 5";
    return CUBE_ERR_PARAM;
  }
  std::vector<float2> tw(n);
  for (int j = 0; j < n; ++j) {
    const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
    tw[j] = make_float2((float)cosl(ang), (float)sinl(ang));
  }
  CUBE_CUDA_TRY(ctx, cudaMalloc(&p.tw, sizeof(float2) * n));
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(p.tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, ctx->stream));
  {  // the same table in FP64 for the FP64 Poisson mode
    std::vector<double2> twd(n);
    for (int j = 0; j < n; ++j) {
      const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
      twd[j] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    CUBE_CUDA_TRY(ctx, cudaMalloc(&p.twd, sizeof(double2) * n));
    CUBE_CUDA_TRY(ctx, cudaMemcpy(p.twd, twd.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
  }
  int R, T;
  if (cube_fast_rt(n, &R, &T)) {
    // the twiddles thread t of a register transform multiplies its k1-th value by,
    // laid out so that a warp's loads are contiguous
    std::vector<float2> tw2((size_t)R * T);
    for (int k1 = 0; k1 < R; ++k1)
      for (int t = 0; t < T; ++t) tw2[(size_t)k1 * T + t] = tw[(t * k1) % n];
    CUBE_CUDA_TRY(ctx, cudaMalloc(&p.tw2, sizeof(float2) * R * T));
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(p.tw2, tw2.data(), sizeof(float2) * R * T, cudaMemcpyHostToDevice, ctx->stream));
  }
  return CUBE_OK;
}

#define MAXIT_X 8
#define MAXIT_C 8

namespace {

// butterflies per thread and stage: half in FP64, whose values take twice the registers
template <typename C2>
constexpr int maxit_x() { return sizeof(C2) == 16 ? MAXIT_X / 2 : MAXIT_X; }
template <typename C2>
constexpr int maxit_c() { return sizeof(C2) == 16 ? MAXIT_C / 2 : MAXIT_C; }

template <typename C2>
int r2c_x_t(cube_ctx* ctx, MeshLevel& L, typename CT<C2>::R* data, int inverse, int ncomp, unsigned int* f2_bits) {
  const int n = L.n;
  const int npairs = n * n / 2;
  const int rpb = ncomp == 3 ? 1 : 2;
  const int ss = n + 1;
  const size_t smem = sizeof(C2) * (size_t)ncomp * rpb * ss;
  constexpr int MX = maxit_x<C2>();
  const int thr = pick_threads(rpb * n / 2, MX);
  const int blocks = (npairs + rpb - 1) / rpb;
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_fft_x<MX, C2>, smem));
  k_fft_x<MX, C2><<<blocks, thr, smem, ctx->stream>>>(data, (size_t)n * L.plane, ncomp, n, L.rp, npairs, rpb,
                                                           L.plan, inverse, f2_bits);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

// kx columns per CTA of the column passes: 8 or 16 in FP32, half of it in FP64
template <typename C2>
int col_tk(int n) {
  const int tk = n >= 512 ? 8 : 16;
  return sizeof(C2) == 16 ? tk / 2 : tk;
}

template <typename C2>
int col_pass_t(cube_ctx* ctx, MeshLevel& L, typename CT<C2>::R* data, int ncomp, int along_z,
               typename CT<C2>::R sgn) {
  const int n = L.n;
  const int ncol = n / 2 + 1;
  const int tk = col_tk<C2>(n);
  const size_t smem = sizeof(C2) * (size_t)n * tk;
  constexpr int MC = maxit_c<C2>();
  const int thr = pick_threads(tk * n / 4, MC);
  dim3 grid((ncol + tk - 1) / tk, n, ncomp);
  const long long cp = L.cp;
  const long long jstride = along_z ? (long long)n * cp : cp;
  const long long ostride = along_z ? cp : (long long)n * cp;
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_fft_col<MC, C2>, smem));
  k_fft_col<MC, C2><<<grid, thr, smem, ctx->stream>>>(reinterpret_cast<C2*>(data), (size_t)n * L.plane / 2, n,
                                                           ncol, tk, jstride, ostride, L.plan, sgn);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

// r2c, y, z + Green + z^-1 (three outputs), y^-1 x3, c2r x3 with max f^2
template <typename C2>
int poisson_t(cube_ctx* ctx, MeshLevel& L, typename CT<C2>::R* rho, typename CT<C2>::R* force,
              const typename CT<C2>::R* kern, typename CT<C2>::R ksc, unsigned int* f2_bits) {
  typedef typename CT<C2>::R R;
  const int n = L.n;
  int rc;
  if ((rc = r2c_x_t<C2>(ctx, L, rho, 0, 1, nullptr))) return rc;
  if ((rc = col_pass_t<C2>(ctx, L, rho, 1, 0, (R)-1))) return rc;
  {
    const int ncol = n / 2 + 1;
    const int tk = col_tk<C2>(n);
    const size_t smem = 2 * sizeof(C2) * (size_t)n * tk;
    constexpr int MC = maxit_c<C2>();
    const int thr = pick_threads(tk * n / 4, MC);
    dim3 grid((ncol + tk - 1) / tk, n, 1);
    const long long cp = L.cp;
    CUBE_CUDA_TRY(ctx, cube_smem_limit(k_fft_z_green<MC, C2>, smem));
    k_fft_z_green<MC, C2><<<grid, thr, smem, ctx->stream>>>(
        reinterpret_cast<const C2*>(rho), reinterpret_cast<C2*>(force), (size_t)n * L.plane / 2, n, ncol, tk,
        (long long)n * cp, cp, L.plan, kern, L.kern_pitch, ksc);
    CUBE_LAUNCH_CHECK(ctx);
  }
  if ((rc = col_pass_t<C2>(ctx, L, force, 3, 0, (R)1))) return rc;
  return r2c_x_t<C2>(ctx, L, force, 1, 3, f2_bits);
}

}  // namespace

int cube_fft_r2c_x(cube_ctx* ctx, MeshLevel& L, float* data, int inverse, int ncomp, unsigned int* f2_bits) {
  return r2c_x_t<float2>(ctx, L, data, inverse, ncomp, f2_bits);
}

static int col_pass(cube_ctx* ctx, MeshLevel& L, float* data, int ncomp, int along_z, float sgn) {
  return col_pass_t<float2>(ctx, L, data, ncomp, along_z, sgn);
}

__global__ void k_force_scale(float* __restrict__ f, int n, int rp, KickScale ks) {
  const int64_t tot = 3ll * n * n * n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % n);
    const int64_t row = i / n;  // (c*n + z)*n + y
    float* p = f + row * rp + x;
    *p = cube_kick_scale(*p, ks);
  }
}

int cube_force_scale(cube_ctx* ctx, MeshLevel& L, KickScale ks) {
  k_force_scale<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(L.force, L.n, L.rp, ks);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

int cube_fft_poisson(cube_ctx* ctx, MeshLevel& L, unsigned int* f2_bits, KickScale ks) {
  int rc;
  if (L.fp64)  // FP64 mode: kick scalar ((a_mid*dt)/6)/pi in FP64 with the reference's pi
    return poisson_t<double2>(ctx, L, reinterpret_cast<double*>(L.rho), reinterpret_cast<double*>(L.force), L.kernd,
                              (((double)ks.a_mid * (double)ks.dt) / 6.0) / (double)ks.pi_f, f2_bits);
  if (!ctx->P.stockham_only && cube_fft_poisson_fast(ctx, L, f2_bits, ks, &rc)) return rc;
  return poisson_t<float2>(ctx, L, L.rho, L.force, L.kern, cube_kick_scalar(ks), f2_bits);
}

// forward 3-D r2c in place (x, y, z), unnormalised
int cube_fft_forward3(cube_ctx* ctx, MeshLevel& L, float* data, int* kx_major) {
  int rc;
  if (!ctx->P.stockham_only && cube_fft_forward3_fast(ctx, L, data, &rc, kx_major)) return rc;
  *kx_major = 0;
  if ((rc = cube_fft_r2c_x(ctx, L, data, 0, 1, nullptr))) return rc;
  if ((rc = col_pass(ctx, L, data, 1, 0, -1.f))) return rc;
  return col_pass(ctx, L, data, 1, 1, -1.f);
}
