/*
 * k_reduce.cu -- deterministic reductions and the cell-count prefix scan.
 *
 * cube_tree_sum_dev: the sum of n doubles as a fixed pairwise tree over
 * blocks of 1024 (pad with zeros; loc[i] += loc[i+s] for s = 512..1), then
 * the same tree over the block sums, until one value is left.  The CPU
 * oracle uses the identical tree, so sums such as the velocity statistics of
 * update_x (update_particle.f90:174-226) agree to the last bit.
 *
 * cube_exclusive_scan: int32 cell counts -> int64 cell starts (n+1 entries),
 * the role of spine_tile / spine_image (variables.f90:103-218).
 */
#include "cube_internal.cuh"

namespace {

__global__ void k_tree_block(const double* __restrict__ in, int64_t n, double* __restrict__ out) {
  __shared__ double loc[1024];
  const int i = threadIdx.x;  // 512 threads
  const int64_t b = blockIdx.x;
  const int64_t q0 = b * 1024 + i, q1 = q0 + 512;
  const double a0 = q0 < n ? in[q0] : 0.0;
  const double a1 = q1 < n ? in[q1] : 0.0;
  loc[i] = __dadd_rn(a0, a1);  // s = 512
  __syncthreads();
  for (int s = 256; s >= 32; s >>= 1) {
    if (i < s) loc[i] = __dadd_rn(loc[i], loc[i + s]);
    __syncthreads();
  }
  if (i < 32) {
    double v = loc[i];
    for (int s = 16; s >= 1; s >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, v, s);
      if (i < s) v = __dadd_rn(v, o);
    }
    if (i == 0) out[b] = v;
  }
}

// The first level of the tree over the per-particle velocity statistics of update_x
// (update_particle.f90:174-226) with the terms formed here: for slot q of the new
// storage order, vr = tan(code)/coef of its new residual code and vs = vr + vfield of
// its new cell, r2 = (vr_x^2 + vr_y^2) + vr_z^2 and s2 likewise from vs; the two
// block sums follow the tree of k_tree_block exactly, so the totals are the ones a
// stored list of terms would give.  One element's terms: (vr_x^2 + vr_y^2) + vr_z^2 and
// the same from vs (0 past the end)
template <int ZV>
__device__ __forceinline__ void stats_terms(const typename CodeT<ZV>::T* __restrict__ vp, int64_t cap,
                                            const int32_t* __restrict__ slot_cell, const float* __restrict__ vfield,
                                            int64_t ncells, const double* __restrict__ dec, int half_nvbin, int64_t n,
                                            int64_t q, double& r2, double& s2) {
  r2 = 0.0;
  s2 = 0.0;
  if (q >= n) return;
  const int64_t c = slot_cell[q];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double vr = __ldg(&dec[(int)vp[(size_t)d * cap + q] + half_nvbin]);
    const double vs = __dadd_rn(vr, (double)__ldg(&vfield[(size_t)d * ncells + c]));
    r2 = __dadd_rn(r2, __dmul_rn(vr, vr));
    s2 = __dadd_rn(s2, __dmul_rn(vs, vs));
  }
}

// One warp per 1024-block of the tree, the same additions in the same order as
// k_tree_block: lane l holds elements l + 32k, so the shared-memory stages of stride
// 512 .. 32 (loc[i] += loc[i + s] for i < s) are register pairs (k, k + s/32), and the
// last five stages are the same shuffles.  Elements k and k + 16 are formed together
// and added at once (the stride-512 stage), so 16 partial sums per quantity are held.
template <int ZV>
__global__ void __launch_bounds__(256) k_stats_first(const void* __restrict__ vp_, int64_t cap,
                                                     const int32_t* __restrict__ slot_cell,
                                                     const float* __restrict__ vfield, int64_t ncells,
                                                     const double* __restrict__ dec, int half_nvbin, int64_t n,
                                                     int64_t nblocks, double* __restrict__ out_r,
                                                     double* __restrict__ out_s) {
  typedef typename CodeT<ZV>::T TV;
  const TV* vp = reinterpret_cast<const TV*>(vp_);
  const int lane = threadIdx.x & 31;
  const int64_t b = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (b >= nblocks) return;  // the whole warp
  const int64_t base = b * 1024 + lane;
  double R[16], S[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    double r0, s0, r1, s1;
    stats_terms<ZV>(vp, cap, slot_cell, vfield, ncells, dec, half_nvbin, n, base + 32 * k, r0, s0);
    stats_terms<ZV>(vp, cap, slot_cell, vfield, ncells, dec, half_nvbin, n, base + 32 * (k + 16), r1, s1);
    R[k] = __dadd_rn(r0, r1);  // stride 512
    S[k] = __dadd_rn(s0, s1);
  }
#pragma unroll
  for (int h = 8; h >= 1; h >>= 1)  // strides 256, 128, 64, 32
#pragma unroll
    for (int k = 0; k < h; ++k) {
      R[k] = __dadd_rn(R[k], R[k + h]);
      S[k] = __dadd_rn(S[k], S[k + h]);
    }
  double v = R[0], w = S[0];
  for (int s = 16; s >= 1; s >>= 1) {
    const double o = __shfl_down_sync(0xffffffffu, v, s);
    const double p = __shfl_down_sync(0xffffffffu, w, s);
    if (lane < s) {
      v = __dadd_rn(v, o);
      w = __dadd_rn(w, p);
    }
  }
  if (lane == 0) {
    out_r[b] = v;
    out_s[b] = w;
  }
}

constexpr int SCAN_PER_THREAD = 8;
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_BLOCK = SCAN_PER_THREAD * SCAN_THREADS;

__global__ void k_scan_sums(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ bsum) {
  __shared__ int64_t ws[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x * SCAN_PER_THREAD;
  int64_t s = 0;
  for (int k = 0; k < SCAN_PER_THREAD; ++k)
    if (base + k < n) s += in[base + k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
    bsum[blockIdx.x] = t;
  }
}

// exclusive scan of nb values in place by one block
__global__ void k_scan_top(int64_t* __restrict__ v, int64_t nb) {
  __shared__ int64_t carry;
  __shared__ int64_t ws[32];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nb; base += blockDim.x) {
    const int64_t q = base + threadIdx.x;
    const int64_t x = q < nb ? v[q] : 0;
    int64_t inc = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if ((threadIdx.x & 31) >= o) inc += y;
    }
    if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = inc;
    __syncthreads();
    if (threadIdx.x < 32) {
      const int nw = blockDim.x >> 5;
      int64_t w = threadIdx.x < nw ? ws[threadIdx.x] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
        if ((int)threadIdx.x >= o) w += y;
      }
      ws[threadIdx.x] = w;  // inclusive warp totals
    }
    __syncthreads();
    const int wi = threadIdx.x >> 5;
    const int64_t before = (wi ? ws[wi - 1] : 0) + carry;
    if (q < nb) v[q] = before + inc - x;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = before + inc;
    __syncthreads();
  }
}

__global__ void k_scan_apply(const int32_t* __restrict__ in, int64_t n, const int64_t* __restrict__ boff,
                             int64_t* __restrict__ out) {
  __shared__ int64_t ws[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x * SCAN_PER_THREAD;
  int64_t vals[SCAN_PER_THREAD];
  int64_t s = 0;
  for (int k = 0; k < SCAN_PER_THREAD; ++k) {
    vals[k] = (base + k < n) ? in[base + k] : 0;
    s += vals[k];
  }
  int64_t inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if ((threadIdx.x & 31) >= o) inc += y;
  }
  if ((threadIdx.x & 31) == 31) ws[threadIdx.x >> 5] = inc;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int nw = blockDim.x >> 5;
    int64_t w = threadIdx.x < nw ? ws[threadIdx.x] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
      if ((int)threadIdx.x >= o) w += y;
    }
    ws[threadIdx.x] = w;
  }
  __syncthreads();
  const int wi = threadIdx.x >> 5;
  int64_t run = boff[blockIdx.x] + (wi ? ws[wi - 1] : 0) + inc - s;
  for (int k = 0; k < SCAN_PER_THREAD; ++k) {
    if (base + k < n) out[base + k] = run;
    run += vals[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = boff[blockIdx.x] + ws[(blockDim.x >> 5) - 1];
}

}  // namespace

// the velocity statistics sums of update_x in the new layout (see k_stats_first)
int cube_stats_sums(cube_ctx* ctx, const int32_t* slot_cell, const double* dec, double* sum_r, double* sum_s) {
  const int64_t n = ctx->np;
  if (n == 0) { *sum_r = *sum_s = 0.0; return CUBE_OK; }
  const int64_t nb = (n + 1023) / 1024;
  // block sums in the per-slot arrays, free after the re-bin
  double* br = ctx->slot_s2;
  double* bs = ctx->slot_s2 + nb;
  const unsigned grid = (unsigned)((nb + 7) / 8);  // a warp per 1024-block
  if (ctx->izipv == 1)
    k_stats_first<1><<<grid, 256, 0, ctx->stream>>>(ctx->vp, ctx->cap, slot_cell, ctx->vfield, ctx->ncells, dec,
                                                    ctx->nvbin / 2, n, nb, br, bs);
  else
    k_stats_first<2><<<grid, 256, 0, ctx->stream>>>(ctx->vp, ctx->cap, slot_cell, ctx->vfield, ctx->ncells, dec,
                                                    ctx->nvbin / 2, n, nb, br, bs);
  CUBE_LAUNCH_CHECK(ctx);
  int rc = cube_tree_sum_dev(ctx, br, nb, sum_r);
  if (rc) return rc;
  return cube_tree_sum_dev(ctx, bs, nb, sum_s);
}

int cube_tree_sum_dev(cube_ctx* ctx, const double* in, int64_t n, double* out_host) {
  double* a = ctx->red_tmp + 4;  // first slots hold the deposit mass totals
  const double* src = in;
  int64_t m = n;
  int flip = 0;
  double* bufs[2] = {a, a + (n + 1023) / 1024 + 8};
  if (m == 0) { *out_host = 0.0; return CUBE_OK; }
  while (true) {
    const int64_t nb = (m + 1023) / 1024;
    double* dst = bufs[flip];
    k_tree_block<<<(unsigned)nb, 512, 0, ctx->stream>>>(src, m, dst);
    CUBE_LAUNCH_CHECK(ctx);
    src = dst;
    m = nb;
    flip ^= 1;
    if (m == 1) break;
  }
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(out_host, src, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return CUBE_OK;
}

int cube_exclusive_scan(cube_ctx* ctx, const int32_t* in, int64_t n, int64_t* out) {
  const int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  int64_t* bs = ctx->scan_tmp;
  k_scan_sums<<<(unsigned)nb, SCAN_THREADS, 0, ctx->stream>>>(in, n, bs);
  CUBE_LAUNCH_CHECK(ctx);
  k_scan_top<<<1, 1024, 0, ctx->stream>>>(bs, nb);
  CUBE_LAUNCH_CHECK(ctx);
  k_scan_apply<<<(unsigned)nb, SCAN_THREADS, 0, ctx->stream>>>(in, n, bs, out);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

namespace {
// decode of every code, and one bit per code: the step's encode returns the code
// itself for its decoded velocity (nvbin is a multiple of 256, so every warp is full)
__global__ void k_vdec_build(const float* __restrict__ tan_table, double coef, double* __restrict__ out, int nvbin,
                             cube_codec codec, VencTab tab) {
  uint32_t* fix = reinterpret_cast<uint32_t*>(out + nvbin);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nvbin; c += gridDim.x * blockDim.x) {
    const double v = cube_vdecode(tan_table[c], coef);
    out[c] = v;
    const int code = c - nvbin / 2;
    const bool same = cube_wrap_code(cube_vencode_step(&codec, tab, v, coef), codec.izipv) == code;
    const uint32_t bits = __ballot_sync(0xffffffffu, same);
    if ((threadIdx.x & 31) == 0) fix[c >> 5] = bits;
  }
}
}  // namespace

// decode table for coef: the velocity decode tan(pi*code/(nvbin-1))/coef of every
// code, computed by the same FP32 table and FP64 division as a per-particle decode,
// so a lookup is bit-identical to it; followed by the bits of cube_vfixed
const double* cube_vdec_table(cube_ctx* ctx, double coef, int* rc) {
  *rc = CUBE_OK;
  for (int i = 0; i < 2; ++i)
    if (ctx->vdec[i] && ctx->vdec_coef[i] == coef) return ctx->vdec[i];
  const int i = ctx->vdec_next;
  ctx->vdec_next ^= 1;
  if (!ctx->vdec[i] && cudaMalloc((void**)&ctx->vdec[i], sizeof(double) * ctx->nvbin + sizeof(uint32_t) * (ctx->nvbin / 32)) !=
                           cudaSuccess) {
    ctx->err = "cudaMalloc of the velocity decode table failed";
    *rc = CUBE_ERR_CUDA;
    return nullptr;
  }
  k_vdec_build<<<(ctx->nvbin + 255) / 256, 256, 0, ctx->stream>>>(ctx->tan_table, coef, ctx->vdec[i], ctx->nvbin,
                                                                  ctx->codec, cube_venc_tab(ctx));
  ctx->launches++;
  if (cudaGetLastError() != cudaSuccess) {
    ctx->err = "velocity decode table launch failed";
    *rc = CUBE_ERR_CUDA;
    return nullptr;
  }
  ctx->vdec_coef[i] = coef;
  return ctx->vdec[i];
}

namespace {
// velocities spread over the code range: v = tan(pi*(code + off)/(nvbin-1))/coef with
// off in (-1, 1) drawn from a hash of the index, so that many land near the
// rounding boundaries code +- 1/2 (within 1.3e-8 of a boundary, the fallback's 1e-9
// band in q included, and within 3.3e-5); the step's encode against cube_vencode
__global__ void k_encode_check(cube_codec codec, VencTab tab, double coef, int64_t n, uint64_t seed,
                               unsigned long long* __restrict__ bad) {
  unsigned long long nb = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull + seed;
    h ^= h >> 31; h *= 0xBF58476D1CE4E5B9ull; h ^= h >> 27; h *= 0x94D049BB133111EBull; h ^= h >> 31;
    const double u = (double)(h >> 11) * 0x1p-53;                        // [0,1)
    const double half = 0.5 * (double)codec.nvbin_m1_f;
    const double code = floor(u * (double)codec.nvbin_m1_f) - half;       // whole code range
    const int cls = (int)(h & 7);
    const double off = cls < 3 ? ((double)((h >> 3) & 0xFF) - 128.0) * 1e-10 + 0.5       // near x.5
                     : cls < 5 ? ((double)((h >> 3) & 0xFFFF) - 32768.0) * 1e-9 + 0.5     // across the
                                                                                          // table's bands
                               : ((double)((h >> 3) & 0xFFFF) / 65536.0 - 0.5);          // anywhere
    const double ang = 3.141592653589793 * (code + off) / (double)codec.nvbin_m1_f;
    if (fabs(ang) >= 1.5707963) continue;
    const double v = tan(ang) / coef;
    const int32_t ex = cube_vencode(&codec, v, coef);
    nb += cube_vencode_step(&codec, tab, v, coef) != ex;
  }
  if (nb) atomicAdd(bad, nb);
}
}  // namespace

namespace {
// splitmix64 stream for the division check
__device__ __forceinline__ uint64_t smix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// quotients of the PP pair term x/r^3 (x a separation component on the 2^-14 or 2^-6
// grid of int2/int1 positions within +-8 fine cells, r^3 from three such components,
// r > 0.3) and of random doubles over wide ranges: cube_div_rcp against __ddiv_rn
__global__ void k_division_check(int64_t n, uint64_t seed, unsigned long long* bad) {
  unsigned long long nb = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t st = seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(i + 1));
    const int kind = (int)(i & 3);
    double a[3], b;
    if (kind < 3) {
      const double res = kind == 2 ? 0.015625 : 6.103515625e-05;  // 2^-6 or 2^-14
      const int span = kind == 2 ? 1024 : 262144;                // +-8 fine cells
      double r2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        a[d] = res * (double)((int64_t)(smix(st) % (uint64_t)(2 * span + 1)) - span);
        r2 = __dadd_rn(r2, __dmul_rn(a[d], a[d]));
      }
      const double rm = sqrt(r2);
      if (!(rm > 0.3)) continue;
      b = __dmul_rn(__dmul_rn(rm, rm), rm);
    } else {
      const uint64_t u = smix(st);
      b = ldexp(1.0 + (double)(u >> 12) * 0x1p-52, (int)(smix(st) % 50) - 10);
      for (int d = 0; d < 3; ++d) {
        const uint64_t v = smix(st);
        a[d] = ldexp(1.0 + (double)(v >> 12) * 0x1p-52, (int)(smix(st) % 60) - 30) * ((v & 1) ? -1.0 : 1.0);
      }
    }
    const double y = __drcp_rn(b);
    for (int d = 0; d < 3; ++d) {
      const double q1 = cube_div_rcp(a[d], b, y), q2 = __ddiv_rn(a[d], b);
      if (__double_as_longlong(q1) != __double_as_longlong(q2)) ++nb;
    }
  }
  if (nb) atomicAdd(bad, nb);
}
}  // namespace

int32_t cube_debug_division_check(cube_ctx* ctx, int64_t n, uint64_t seed, int64_t* mismatches) {
  if (!ctx || !mismatches || n < 0) return CUBE_ERR_PARAM;
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(ctx->red_tmp);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, 8, ctx->stream));
  k_division_check<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(n, seed, bad);
  CUBE_LAUNCH_CHECK(ctx);
  unsigned long long h = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&h, bad, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *mismatches = (int64_t)h;
  return CUBE_OK;
}

int32_t cube_debug_encode_check(cube_ctx* ctx, int64_t n, uint64_t seed, float sigma, int64_t* mismatches) {
  if (!ctx || !mismatches || n < 0) return CUBE_ERR_PARAM;
  unsigned long long* bad = reinterpret_cast<unsigned long long*>(ctx->red_tmp);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, 8, ctx->stream));
  const double coef = cube_vcoef(&ctx->codec, sigma);
  k_encode_check<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(ctx->codec, cube_venc_tab(ctx), coef, n,
                                                            seed, bad);
  CUBE_LAUNCH_CHECK(ctx);
  unsigned long long h = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&h, bad, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *mismatches = (int64_t)h;
  return CUBE_OK;
}
