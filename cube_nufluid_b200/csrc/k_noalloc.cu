/*
 * k_noalloc.cu -- coarse CIC density without any device allocation.
 *
 * cube_coarse_density_noalloc() computes the same particle (CDM) coarse density
 * r3 as the deposit in k_deposit.cu (the nc^3 CIC mass field of pm.f90:192-278,
 * as the exact 64-bit restriction of the fixed-point fine node sums), for
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
 *     first call before any stream capture;
 *   - with fluid neutrinos on, the context's coarse density also holds their
 *     mass; this entry point deposits the particles only;
 *   - errors are returned as status codes only (there is no context, so
 *     cube_last_error has no text for them); a CUDA error already pending when
 *     the call starts is returned as CUBE_ERR_CUDA without launching anything.
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

// one thread per particle.  The coarse density of k_deposit.cu is the restriction
// of the 64-bit fine node sums with the tent weights (4 - |d|), |d| <= 3, per
// dimension (scale 2^38); a particle's share of it is its eight quantised fine
// weights q = RN(w * 2^32) (w the FP32 product of pm.f90:87's linear factors)
// restricted the same way, which reaches at most three coarse nodes per
// dimension.  Integer sums make the result the same bits in any order.
template <int ZX>
__global__ void k_noalloc_deposit(const void* __restrict__ xp_, const int64_t* __restrict__ cell_start, int64_t cap,
                                  int64_t ncells, int nc, int nt, int nnt, unsigned long long* __restrict__ acc) {
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
    int j0[3];
    int tw[3][2][3];  // restriction weight x4 of the corner's fine node (0, 1) onto coarse node j0 + k
    float w1[3], w2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX);
      const float tf = (float)cube_dadd(4.0 * (double)l[d], cube_dmul(4.0, fr));
      const float f = floorf(tf) + 1.f;
      w1[d] = cube_fsub(f, tf);
      w2[d] = cube_fsub(1.f, w1[d]);
      const int n1 = 4 * t[d] * nt + (int)f - 1;  // global fine node of the lower corner, >= 0
      j0[d] = (n1 + 2) / 4 - 1;                    // floor((n1 - 2) / 4): the lowest coarse node reached
#pragma unroll
      for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int dd = n1 + e - 4 * (j0[d] + k) - 2;
          const int ad = dd < 0 ? -dd : dd;
          tw[d][e][k] = ad <= 3 ? 4 - ad : 0;
        }
    }
    unsigned long long part[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) part[k] = 0ull;
#pragma unroll
    for (int c8 = 0; c8 < 8; ++c8) {
      const int sx = c8 & 1, sy = (c8 >> 1) & 1, sz = c8 >> 2;
      const float w = cube_fmul(cube_fmul(sx ? w2[0] : w1[0], sy ? w2[1] : w1[1]), sz ? w2[2] : w1[2]);
      const unsigned long long q = __double2ull_rn((double)w * 4294967296.0);
#pragma unroll
      for (int kz = 0; kz < 3; ++kz)
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
          for (int kx = 0; kx < 3; ++kx)
            part[(kz * 3 + ky) * 3 + kx] +=
                (unsigned long long)(tw[0][sx][kx] * tw[1][sy][ky] * tw[2][sz][kz]) * q;
    }
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
      for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const unsigned long long v = part[(kz * 3 + ky) * 3 + kx];
          if (!v) continue;
          const int gx = (j0[0] + kx + nc) % nc, gy = (j0[1] + ky + nc) % nc, gz = (j0[2] + kz + nc) % nc;
          atomicAdd(&acc[((size_t)gz * nc + gy) * nc + gx], v);
        }
  }
}

// the coarse density mass * sum * 2^-38, as k_coarse_finalize writes it without neutrinos
__global__ void k_noalloc_finalize(const unsigned long long* __restrict__ acc, float* __restrict__ rho, int64_t n,
                                   double unit_c) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    rho[i] = (float)((double)acc[i] * unit_c);
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
  // an error left by the caller's earlier work is theirs: report it, launch nothing
  if (cudaPeekAtLastError() != cudaSuccess) return CUBE_ERR_CUDA;
  unsigned long long* acc = nullptr;
  int rc = noalloc_scratch(&acc);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t ncells = (int64_t)nc * nc * nc;
  const int nt = nc / nnt;
  const double unit_c = (double)mass_p_cdm * (1.0 / (64.0 * 4294967296.0));  // exact
  k_noalloc_clear<<<64, 256, 0, st>>>(acc, ncells);
  if (cudaGetLastError() != cudaSuccess) return CUBE_ERR_CUDA;
  const unsigned blocks = (unsigned)((ncells + NCELLS_PER_CTA - 1) / NCELLS_PER_CTA);
  if (izipx == 1)
    k_noalloc_deposit<1><<<blocks, 256, 0, st>>>(xp, cell_start, np_capacity, ncells, nc, nt, nnt, acc);
  else
    k_noalloc_deposit<2><<<blocks, 256, 0, st>>>(xp, cell_start, np_capacity, ncells, nc, nt, nnt, acc);
  if (cudaGetLastError() != cudaSuccess) return CUBE_ERR_CUDA;
  k_noalloc_finalize<<<64, 256, 0, st>>>(acc, rho, ncells, unit_c);
  return cudaGetLastError() == cudaSuccess ? CUBE_OK : CUBE_ERR_CUDA;
}
