/*
 * k_noalloc.cu -- coarse CIC density without any device allocation.
 *
 * cube_coarse_density_noalloc() computes the same coarse density r3 as the
 * coarse half of the deposit in k_deposit.cu (the nc^3 CIC mass field of
 * pm.f90:192-278, accumulated as 64-bit fixed point, weight * 2^32), for
 * callers that may not call cudaMalloc: a host whose device memory is owned
 * by another allocator, or a scheduler that hands a fixed HBM budget to each
 * box at start-up and forbids allocation afterwards.  Such a caller passes
 * device pointers to its particles, its cell starts and the output mesh; the
 * accumulator the deposit needs lives in the file-scope array below, which
 * every GPU that loads the library holds until the process exits.
 *
 * Limits and sharing:
 *   - nc <= CUBE_NOALLOC_MAX_NC (64): the accumulator holds 64^3 int64 (2 MiB);
 *     larger meshes are rejected with CUBE_ERR_CAPACITY before any launch;
 *   - all calls on a device share the one accumulator; each call clears it
 *     first, so calls that overlap on the GPU (different streams, or threads)
 *     race and must be serialised by the caller;
 *   - the first call on a device looks up the accumulator's device address
 *     (cudaGetSymbolAddress, with that device current) and caches it; make that
 *     first call before any stream capture.
 */
#include "cube_internal.cuh"

#include <mutex>

#define CUBE_NOALLOC_MAX_NC 64
#define CUBE_NOALLOC_MAX_DEV 64

static __device__ __align__(256) unsigned long long g_noalloc_acc[CUBE_NOALLOC_MAX_NC * CUBE_NOALLOC_MAX_NC *
                                                                   CUBE_NOALLOC_MAX_NC];

namespace {

constexpr int NCELLS_PER_CTA = 64;

__global__ void k_noalloc_clear(unsigned long long* __restrict__ acc, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    acc[i] = 0ull;
}

// one thread per particle; weights as in k_deposit.cu (coarse part): position
// (i-1)+frac-0.5 formed in FP64 and rounded to FP32, FP32 weight products
template <int ZX>
__global__ void k_noalloc_deposit(const void* __restrict__ xp_, const int64_t* __restrict__ cell_start, int64_t cap,
                                  int64_t ncells, int nc, int nt, int nnt, float mass,
                                  unsigned long long* __restrict__ acc) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  __shared__ int64_t cs[NCELLS_PER_CTA + 1];
  const int64_t c0 = (int64_t)blockIdx.x * NCELLS_PER_CTA;
  const int ncl = (int)min((int64_t)NCELLS_PER_CTA, ncells - c0);
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = cell_start[c0 + i];
  __syncthreads();
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
    int n0[3];
    float w1[3], w2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX);
      const float tc = (float)cube_dsub(cube_dadd((double)l[d], fr), 0.5);
      const float ci = floorf(tc) + 1.f;
      w1[d] = cube_fsub(ci, tc);
      w2[d] = cube_fsub(1.f, w1[d]);
      n0[d] = t[d] * nt + (int)ci - 1;  // global coarse node of the lower corner, may be -1
    }
#pragma unroll
    for (int c8 = 0; c8 < 8; ++c8) {
      const int sx = c8 & 1, sy = (c8 >> 1) & 1, sz = c8 >> 2;
      const float w = cube_fmul(cube_fmul(cube_fmul(sx ? w2[0] : w1[0], sy ? w2[1] : w1[1]), sz ? w2[2] : w1[2]), mass);
      const unsigned long long q = (unsigned long long)__double2ll_rn((double)w * 4294967296.0);
      const int gx = (n0[0] + sx + nc) % nc, gy = (n0[1] + sy + nc) % nc, gz = (n0[2] + sz + nc) % nc;
      atomicAdd(&acc[((size_t)gz * nc + gy) * nc + gx], q);
    }
  }
}

__global__ void k_noalloc_finalize(const unsigned long long* __restrict__ acc, float* __restrict__ rho, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    rho[i] = (float)((double)acc[i] * (1.0 / 4294967296.0));
}

std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[CUBE_NOALLOC_MAX_DEV];
bool g_noalloc_ready[CUBE_NOALLOC_MAX_DEV];

// device address of the accumulator for the current device, looked up once per device
int noalloc_scratch(unsigned long long** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= CUBE_NOALLOC_MAX_DEV) return CUBE_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ready[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_acc) != cudaSuccess || !p) return CUBE_ERR_CUDA;
    g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
    g_noalloc_ready[dev] = true;
  }
  *out = g_noalloc_ptr[dev];
  return CUBE_OK;
}

}  // namespace

extern "C" int32_t cube_coarse_density_noalloc(int32_t nc, int32_t nnt, int32_t izipx, int64_t np_capacity,
                                               const void* xp, const int64_t* cell_start, float mass_p_cdm,
                                               float* rho, void* stream) {
  if (nc <= 0 || nnt <= 0 || nc % nnt || (izipx != 1 && izipx != 2) || np_capacity < 0 || !xp || !cell_start ||
      !rho)
    return CUBE_ERR_PARAM;
  if (nc > CUBE_NOALLOC_MAX_NC) return CUBE_ERR_CAPACITY;
  unsigned long long* acc = nullptr;
  int rc = noalloc_scratch(&acc);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t ncells = (int64_t)nc * nc * nc;
  const int nt = nc / nnt;
  k_noalloc_clear<<<64, 256, 0, st>>>(acc, ncells);
  const unsigned blocks = (unsigned)((ncells + NCELLS_PER_CTA - 1) / NCELLS_PER_CTA);
  if (izipx == 1)
    k_noalloc_deposit<1><<<blocks, 256, 0, st>>>(xp, cell_start, np_capacity, ncells, nc, nt, nnt, mass_p_cdm, acc);
  else
    k_noalloc_deposit<2><<<blocks, 256, 0, st>>>(xp, cell_start, np_capacity, ncells, nc, nt, nnt, mass_p_cdm, acc);
  k_noalloc_finalize<<<64, 256, 0, st>>>(acc, rho, ncells);
  return cudaGetLastError() == cudaSuccess ? CUBE_OK : CUBE_ERR_CUDA;
}
