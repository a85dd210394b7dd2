/*
 * k_deposit.cu -- fine and coarse CIC mass deposit (pm.f90:76-107, :192-278).
 *
 * One CTA owns a brick of BX x BY x BZ coarse cells and the 4B^3 fine nodes
 * inside it.  It reads the particles of its cells plus the one-cell layer on
 * the low side of each dimension (the only outside particles whose CIC cloud
 * reaches the brick's first node plane), accumulates every weight into
 * shared memory as a 64-bit fixed-point integer (weight * 2^32, rounded to
 * nearest), and writes each fine node once as FP32.  Integer accumulation
 * makes the density independent of particle order: the fine mesh is
 * bit-identical to the fixed-point mode of the CPU oracle.
 *
 * Each 64-bit accumulator is kept as two 32-bit words updated with native
 * 32-bit shared atomics: the low word's add returns the old value, and the
 * carry out of it goes into the high word with the weight's high half.  The
 * words then hold the 64-bit sum exactly (the number of low-word wraps is
 * floor(sum of low halves / 2^32) whatever the order).  A 64-bit shared
 * atomic add is a compare-and-swap loop whose colliding lanes retry: in
 * clustered states, where thousands of particles of one coarse cell add into
 * the same nodes, it took six times the atomic instructions of an unclustered
 * state of the same size.
 *
 * Weights follow the reference expressions in FP32, with the position formed
 * in FP64 and rounded to FP32 exactly where the reference assigns it to its
 * real tempx (tile-relative coordinates, as in pm.f90:87 and :255).
 *
 * The coarse deposit (ncell coarser, node at the cell centre) is accumulated
 * from the brick's own particles into a (B+2)^3 shared region and added to a
 * global 64-bit accumulator with atomics; the nc^3 accumulator stays in L2.
 *
 * A brick whose region holds more than DMAX particles (clustered states) is
 * split over several blocks, each taking DMAX of them: a block adds its fine
 * nodes into the brick's 64-bit global slot, and the block that finishes last
 * (a fence, then a counter: no block waits for another) writes the brick's
 * nodes.  Integer sums make the split invisible in the result.
 */
#include "cube_internal.cuh"

#include <algorithm>

namespace {

constexpr int BX = 8, BY = 4, BZ = 4;
constexpr int HX = BX + 1, HY = BY + 1, HZ = BZ + 1;
constexpr int NHC = HX * HY * HZ;  // cells read (with the low-side layer)
constexpr int FX = 4 * BX, FY = 4 * BY, FZ = 4 * BZ;
constexpr int CX = BX + 2, CY = BY + 2, CZ = BZ + 2;
constexpr double FIX_SCALE = 4294967296.0;  // 2^32
constexpr int DMAX = 8192;  // region particles per deposit block
static_assert(32 * NHC <= DMAX, "regions of cells of at most 32 particles need no split");

// 64-bit fixed-point add into the word pair (lo[i], hi[i]); q >= 0
__device__ __forceinline__ void fix_add(unsigned* lo, unsigned* hi, int i, unsigned long long q) {
  const unsigned ql = (unsigned)q;
  const unsigned old = atomicAdd(&lo[i], ql);
  const unsigned h = (unsigned)(q >> 32) + ((unsigned)(old + ql) < old ? 1u : 0u);
  if (h) atomicAdd(&hi[i], h);
}
__device__ __forceinline__ unsigned long long fix_get(const unsigned* lo, const unsigned* hi, int i) {
  return ((unsigned long long)hi[i] << 32) | lo[i];
}

// the coarse cell of region cell q of the brick at (x0, y0, z0)
__device__ __forceinline__ int64_t region_cell(int q, int x0, int y0, int z0, int nc, int nt, int nnt) {
  const int cx = q % HX - 1, cy = (q / HX) % HY - 1, cz = q / (HX * HY) - 1;
  return cube_cell_of(cube_wrap(x0 + cx, nc), cube_wrap(y0 + cy, nc), cube_wrap(z0 + cz, nc), nt, nnt);
}

// deposit work items [brick, first, end region particle, split slot or -1]: item b
// is brick b's first (or only) block, the further blocks of split bricks follow
// the bricks.  One warp per brick, one lane per (y, z) row of its region: a row's
// cells with consecutive indices form runs, each counted from two cell starts.
__global__ void __launch_bounds__(256) k_dep_items(const int64_t* __restrict__ cell_start, int nc, int nt, int nnt,
                                                   int64_t* __restrict__ items, int64_t items_max, DevScal* dscal) {
  const int nbx = nc / BX, nby = nc / BY;
  const int64_t nbricks = (int64_t)nbx * nby * (nc / BZ);
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (b >= nbricks) return;  // whole warps
  const int x0 = (int)(b % nbx) * BX, y0 = (int)((b / nbx) % nby) * BY, z0 = (int)(b / ((int64_t)nbx * nby)) * BZ;
  int64_t total = 0;
  if (lane < HY * HZ) {
    const int gy = cube_wrap(y0 + lane % HY - 1, nc), gz = cube_wrap(z0 + lane / HY - 1, nc);
    int64_t first = cube_cell_of(cube_wrap(x0 - 1, nc), gy, gz, nt, nnt), prev = first;
    for (int xi = 1; xi < HX; ++xi) {
      const int64_t c = cube_cell_of(cube_wrap(x0 - 1 + xi, nc), gy, gz, nt, nnt);
      if (c != prev + 1) {
        total += cell_start[prev + 1] - cell_start[first];
        first = c;
      }
      prev = c;
    }
    total += cell_start[prev + 1] - cell_start[first];
  }
  for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
  if (lane) return;
  int64_t* it = items + 4 * b;
  if (total <= DMAX) {
    it[0] = b; it[1] = 0; it[2] = total; it[3] = -1;
    return;
  }
  const int64_t slot = (int64_t)atomicAdd(&dscal->n_split, 1ull);
  it[0] = b; it[1] = 0; it[2] = DMAX; it[3] = slot;
  for (int64_t t = DMAX; t < total; t += DMAX) {
    const int64_t idx = nbricks + (int64_t)atomicAdd(&dscal->n_dep_extra, 1ull);
    if (idx >= items_max) {
      cube_dev_error(dscal, CUBE_ERR_CAPACITY, (int)(b & 0x7fffffff));
      return;
    }
    int64_t* e = items + 4 * idx;
    e[0] = b; e[1] = t; e[2] = min(t + DMAX, total); e[3] = slot;
  }
}

template <int ZX>
__global__ void __launch_bounds__(256) k_deposit(const void* __restrict__ xp_, const int64_t* __restrict__ cell_start,
                                                 int64_t cap, int nc, int nt, int nnt, float mass,
                                                 float* __restrict__ rho, int rp, size_t plane,
                                                 unsigned long long* __restrict__ rho_c_acc,
                                                 unsigned long long* __restrict__ mass_total,
                                                 const int64_t* __restrict__ items,
                                                 unsigned long long* __restrict__ split_nodes,
                                                 unsigned int* __restrict__ split_done) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  extern __shared__ unsigned smem_u32[];
  unsigned* flo = smem_u32;                  // FX*FY*FZ low words
  unsigned* fhi = flo + FX * FY * FZ;        // high words
  unsigned* clo = fhi + FX * FY * FZ;        // CX*CY*CZ
  unsigned* chi = clo + CX * CY * CZ;
  __shared__ int64_t cst[NHC];
  __shared__ int cpre[NHC + 1];
  __shared__ int lt[3][HX];  // in-tile coordinate of region cell -1..B-1 per dimension

  __shared__ int last_block;
  int64_t brick = blockIdx.x, slot = -1;  // without items: block b = brick b, all of it
  int t0 = 0, t1 = 0x7fffffff;
  if (items) {
    const int64_t* item = items + 4 * (int64_t)blockIdx.x;
    brick = item[0];
    t0 = (int)item[1];
    t1 = (int)item[2];
    slot = item[3];
  }
  const int nbx = nc / BX, nby = nc / BY;
  const int bx = (int)(brick % nbx), by = (int)((brick / nbx) % nby), bz = (int)(brick / ((int64_t)nbx * nby));
  const int x0 = bx * BX, y0 = by * BY, z0 = bz * BZ;

  for (int i = threadIdx.x; i < 2 * (FX * FY * FZ + CX * CY * CZ); i += blockDim.x) smem_u32[i] = 0u;
  if (threadIdx.x >= 32 && threadIdx.x < 32 + 3 * HX) {
    const int d = (threadIdx.x - 32) / HX, c = (threadIdx.x - 32) % HX;
    const int base = d == 0 ? x0 : d == 1 ? y0 : z0;
    lt[d][c] = cube_wrap(base + c - 1, nc) % nt;
  }
  if (threadIdx.x < 32) {
    // cell table of the (B+1)^3 region in (z,y,x) order; warp 0 builds the prefix
    int run = 0;
    for (int base = 0; base < NHC; base += 32) {
      const int q = base + threadIdx.x;
      int cnt = 0;
      if (q < NHC) {
        const int64_t c = region_cell(q, x0, y0, z0, nc, nt, nnt);
        const int64_t s0 = cell_start[c];
        cst[q] = s0;
        cnt = (int)(cell_start[c + 1] - s0);
      }
      int inc = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)threadIdx.x >= o) inc += v;
      }
      if (q < NHC) cpre[q] = run + inc - cnt;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (threadIdx.x == 0) cpre[NHC] = run;
  }
  __syncthreads();
  const int total = cpre[NHC];
  const int tend = min(t1, total);
  for (int t = t0 + threadIdx.x; t < tend; t += blockDim.x) {
    int lo = 0, hi = NHC - 1;  // last q with cpre[q] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cpre[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int q = lo;
    const int64_t ip = cst[q] + (t - cpre[q]);
    const int cx = q % HX - 1, cy = (q / HX) % HY - 1, cz = q / (HX * HY) - 1;
    const int cu[3] = {x0 + cx, y0 + cy, z0 + cz};     // unwrapped global coarse cell
    const int cr[3] = {cx + 1, cy + 1, cz + 1};        // region index
    const int own = (cx >= 0 && cy >= 0 && cz >= 0);
    int o1[3], c1[3];
    float dx1[3], dx2[3], cd1[3], cd2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int l = lt[d][cr[d]];
      const double fr = cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX);
      // fine: tempx = ncell*(i-1) + ncell*frac (tile-relative), FP64 -> FP32
      const float tf = (float)cube_dadd(4.0 * (double)l, cube_dmul(4.0, fr));
      const float f = floorf(tf) + 1.f;
      dx1[d] = cube_fsub(f, tf);
      dx2[d] = cube_fsub(1.f, dx1[d]);
      o1[d] = 4 * (cu[d] - (d == 0 ? x0 : d == 1 ? y0 : z0)) + ((int)f - 1 - 4 * l);
      // coarse: tempx = (i-1) + frac - 0.5, FP64 -> FP32
      const float tc = (float)cube_dsub(cube_dadd((double)l, fr), 0.5);
      const float ci = floorf(tc) + 1.f;
      cd1[d] = cube_fsub(ci, tc);
      cd2[d] = cube_fsub(1.f, cd1[d]);
      c1[d] = (cu[d] - (d == 0 ? x0 : d == 1 ? y0 : z0)) + ((int)ci - 1 - l) + 1;  // +1: region starts at -1
    }
#pragma unroll
    for (int c8 = 0; c8 < 8; ++c8) {
      const int sx = c8 & 1, sy = (c8 >> 1) & 1, sz = c8 >> 2;
      const int nx = o1[0] + sx, ny = o1[1] + sy, nz = o1[2] + sz;
      if (nx >= 0 && nx < FX && ny >= 0 && ny < FY && nz >= 0 && nz < FZ) {
        const float w = cube_fmul(cube_fmul(cube_fmul(sx ? dx2[0] : dx1[0], sy ? dx2[1] : dx1[1]),
                                            sz ? dx2[2] : dx1[2]), mass);
        const unsigned long long qv = (unsigned long long)__double2ll_rn((double)w * FIX_SCALE);
        fix_add(flo, fhi, (nz * FY + ny) * FX + nx, qv);
      }
      if (own) {
        const float w = cube_fmul(cube_fmul(cube_fmul(sx ? cd2[0] : cd1[0], sy ? cd2[1] : cd1[1]),
                                            sz ? cd2[2] : cd1[2]), mass);
        const unsigned long long qv = (unsigned long long)__double2ll_rn((double)w * FIX_SCALE);
        fix_add(clo, chi, ((c1[2] + sz) * CY + (c1[1] + sy)) * CX + (c1[0] + sx), qv);
      }
    }
  }
  __syncthreads();
  unsigned long long msum = 0ull;
  unsigned long long* sacc = slot >= 0 ? split_nodes + (size_t)slot * (FX * FY * FZ) : nullptr;
  for (int i = threadIdx.x; i < FX * FY * FZ; i += blockDim.x) {
    const int nx = i % FX, ny = (i / FX) % FY, nz = i / (FX * FY);
    const unsigned long long a = fix_get(flo, fhi, i);
    msum += a;
    if (!sacc)
      rho[(size_t)(4 * z0 + nz) * plane + (size_t)(4 * y0 + ny) * rp + (4 * x0 + nx)] =
          (float)((double)a * (1.0 / FIX_SCALE));
    else if (a)
      atomicAdd(&sacc[i], a);
  }
  if (sacc) {  // the last of the brick's blocks writes its nodes
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last_block = atomicAdd(&split_done[slot], 1u) == (unsigned)((total + DMAX - 1) / DMAX - 1);
    __syncthreads();
    if (last_block) {
      __threadfence();
      for (int i = threadIdx.x; i < FX * FY * FZ; i += blockDim.x) {
        const int nx = i % FX, ny = (i / FX) % FY, nz = i / (FX * FY);
        rho[(size_t)(4 * z0 + nz) * plane + (size_t)(4 * y0 + ny) * rp + (4 * x0 + nx)] =
            (float)((double)__ldcg(&sacc[i]) * (1.0 / FIX_SCALE));
      }
    }
  }
  for (int i = threadIdx.x; i < CX * CY * CZ; i += blockDim.x) {
    const unsigned long long a = fix_get(clo, chi, i);
    if (a) {
      const int nx = i % CX - 1, ny = (i / CX) % CY - 1, nz = i / (CX * CY) - 1;
      const int gx = cube_wrap(x0 + nx, nc), gy = cube_wrap(y0 + ny, nc), gz = cube_wrap(z0 + nz, nc);
      atomicAdd(&rho_c_acc[((size_t)gz * nc + gy) * nc + gx], a);
    }
  }
  for (int o = 16; o > 0; o >>= 1) msum += __shfl_xor_sync(0xffffffffu, msum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(mass_total, msum);
}

// coarse accumulator -> FP32 density (pitch rp), accumulator cleared for the next step
__global__ void k_coarse_finalize(unsigned long long* __restrict__ acc, float* __restrict__ r3, int nc, int rp,
                                  unsigned long long* __restrict__ mass_total) {
  const int64_t n = (int64_t)nc * nc * nc;
  unsigned long long msum = 0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long a = acc[i];
    acc[i] = 0ull;
    msum += a;
    const int64_t x = i % nc, yz = i / nc;
    r3[yz * rp + x] = (float)((double)a * (1.0 / FIX_SCALE));
  }
  for (int o = 16; o > 0; o >>= 1) msum += __shfl_xor_sync(0xffffffffu, msum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(mass_total, msum);
}

}  // namespace

int cube_deposit(cube_ctx* ctx, cube_scalars* io) {
  const int nc = ctx->nc;
  if (nc % BX || nc % BY || nc % BZ) {
    ctx->err = "nc must be a multiple of 8";
    return CUBE_ERR_PARAM;
  }
  unsigned long long* mtot = reinterpret_cast<unsigned long long*>(ctx->red_tmp);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(mtot, 0, 2 * sizeof(unsigned long long), ctx->stream));
  // work items: one per brick, more for bricks beyond DMAX region particles; not
  // needed when no cell holds more than 32 particles (a region of 225 cells then
  // holds at most 7200 <= DMAX)
  const int64_t nbricks = (int64_t)(nc / BX) * (nc / BY) * (nc / BZ);
  const int64_t items_max = cube_rebin_items_max(ctx->ncells, ctx->cap);
  unsigned long long hv[2] = {0ull, 0ull};  // n_dep_extra, n_split
  const int64_t* items = nullptr;
  if (!ctx->cells_le32) {
    CUBE_CUDA_TRY(ctx, cudaMemsetAsync(&ctx->dscal->n_dep_extra, 0, 2 * sizeof(unsigned long long), ctx->stream));
    k_dep_items<<<(unsigned)((nbricks + 7) / 8), 256, 0, ctx->stream>>>(ctx->cell_start, nc, ctx->nt, ctx->nnt,
                                                                        ctx->rebin_items, items_max, ctx->dscal);
    CUBE_LAUNCH_CHECK(ctx);
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(hv, &ctx->dscal->n_dep_extra, sizeof(hv), cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    items = ctx->rebin_items;
  }
  const int64_t blocks = std::min<int64_t>(nbricks + (int64_t)hv[0], items_max);
  unsigned long long* split_nodes = nullptr;
  unsigned int* split_done = nullptr;
  if (hv[1]) {
    const size_t node_bytes = sizeof(unsigned long long) * FX * FY * FZ * hv[1];
    const size_t need = node_bytes + sizeof(unsigned int) * hv[1];
    if (need > ctx->dep_scratch_bytes) {
      if (ctx->dep_scratch) cudaFree(ctx->dep_scratch);
      ctx->dep_scratch = nullptr;
      ctx->dep_scratch_bytes = 0;
      const size_t grow = need + need / 2;
      CUBE_CUDA_TRY(ctx, cudaMalloc(&ctx->dep_scratch, grow));
      ctx->dep_scratch_bytes = grow;
    }
    CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dep_scratch, 0, need, ctx->stream));
    split_nodes = reinterpret_cast<unsigned long long*>(ctx->dep_scratch);
    split_done = reinterpret_cast<unsigned int*>(reinterpret_cast<char*>(ctx->dep_scratch) + node_bytes);
  }
  const size_t smem = 2 * sizeof(unsigned) * (FX * FY * FZ + CX * CY * CZ);
  if (ctx->izipx == 1) {
    CUBE_CUDA_TRY(ctx, cube_smem_limit(k_deposit<1>, smem));
    k_deposit<1><<<(unsigned)blocks, 256, smem, ctx->stream>>>(
        ctx->xp, ctx->cell_start, ctx->cap, nc, ctx->nt, ctx->nnt, io->mass_p_cdm, ctx->fine.rho, ctx->fine.rp,
        ctx->fine.plane, ctx->rho_c_acc, mtot, items, split_nodes, split_done);
  } else {
    CUBE_CUDA_TRY(ctx, cube_smem_limit(k_deposit<2>, smem));
    k_deposit<2><<<(unsigned)blocks, 256, smem, ctx->stream>>>(
        ctx->xp, ctx->cell_start, ctx->cap, nc, ctx->nt, ctx->nnt, io->mass_p_cdm, ctx->fine.rho, ctx->fine.rp,
        ctx->fine.plane, ctx->rho_c_acc, mtot, items, split_nodes, split_done);
  }
  CUBE_LAUNCH_CHECK(ctx);
  if (ctx->nu.on) {  // neutrino density into both meshes (pm.f90:55-74, :198-242)
    const int rc = cube_nu_density(ctx, io);
    if (rc) return rc;
  }
  k_coarse_finalize<<<592, 256, 0, ctx->stream>>>(ctx->rho_c_acc, ctx->coarse.rho, nc, ctx->coarse.rp, mtot + 1);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}
