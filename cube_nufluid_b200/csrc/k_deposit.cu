/*
 * k_deposit.cu -- fine and coarse CIC mass deposit (pm.f90:76-107, :192-278).
 *
 * One CTA owns a brick of BX x BY x BZ coarse cells and the 4B^3 fine nodes
 * inside it.  It reads the particles of its cells plus the one-cell layer on
 * the low side of each dimension (the only outside particles whose CIC cloud
 * reaches the brick's first node plane) and accumulates every CIC weight as a
 * 64-bit fixed-point integer q = RN(w * 2^32) in shared memory.  The weight is
 * the reference's FP32 product of the three linear factors; the particle mass
 * is applied once per node when the node is written, so q <= 2^32 and every
 * node sum is exact and independent of particle order: the fine mesh is
 * bit-identical to the fixed-point mode of the CPU oracle.
 *
 * A node sum S is held as two 32-bit words, A = sum(q mod 2^16) and
 * B = sum(q div 2^16), S = A + 2^16 B, each updated by a 32-bit shared add whose
 * result is not needed (a no-return reduction, no round trip).  A block takes at
 * most DMAX <= 65535 particles, so neither word can wrap.  Node slots are
 * rotated within their 32-word row by two bits of (y, z), so the lanes of a warp,
 * which hold neighbouring particles of a few cells, hit different banks.
 *
 * The coarse density is not deposited particle by particle.  The coarse CIC
 * kernel of a particle at fine coordinate x, seen from the coarse node whose
 * centre is the fine node 4J+2, is the tent T(x) = 1 - |x - 4J - 2|/4; T is
 * linear between fine nodes, and CIC interpolation reproduces linear functions,
 * so sum_n W_fine(x - n) T(n) = T(x) exactly.  The coarse density is therefore
 * the fine node sums restricted with the weights (4 - |d|)/4, |d| <= 3, per
 * dimension -- the identity holds for each particle's quantised fine weights
 * too, so the coarse sums are exact integers (scale 2^38 = 2^32 * 4^3) and
 * order-independent.  Each brick restricts its own fine nodes (z, then y, then x
 * passes in shared memory) into the (B+2)^3 coarse nodes they reach and adds
 * them to a global 64-bit accumulator (nc^3, resident in L2).  This removes the
 * per-particle coarse atomics, whose lanes (the eight particles of a cell) all
 * hit the same coarse nodes.
 *
 * A brick whose region holds more than DMAX particles (clustered states) is
 * split over several blocks, each taking DMAX of them: a block adds its fine
 * node sums into the brick's 64-bit global slot, and the block that finishes
 * last (a fence, then a counter: no block waits for another) writes the
 * brick's fine nodes and restricts them.
 */
#include "cube_internal.cuh"

#include <algorithm>

namespace {

constexpr int BX = 8, BY = 4, BZ = 4;
constexpr int HX = BX + 1, HY = BY + 1, HZ = BZ + 1;
constexpr int NHC = HX * HY * HZ;  // cells read (with the low-side layer)
constexpr int FX = 4 * BX, FY = 4 * BY, FZ = 4 * BZ;
constexpr int NFN = FX * FY * FZ;  // fine nodes of a brick
constexpr int CX = BX + 2, CY = BY + 2, CZ = BZ + 2;  // coarse nodes a brick's fine nodes reach
constexpr int DEP_THREADS = 512;
constexpr double FIX_SCALE = 4294967296.0;  // 2^32
constexpr int DMAX = 8192;  // region particles per deposit block
static_assert(32 * NHC <= DMAX, "regions of cells of at most 32 particles need no split");
static_assert(DMAX <= 65535, "the split words of a node take at most 65535 adds");
static_assert(FX == 32, "a fine row of the brick is one bank cycle");
static_assert(FX * FY == DEP_THREADS, "one (x, y) column of the brick per thread in the z pass");
static_assert(CX * CY * CZ <= DEP_THREADS && CZ * FX <= DEP_THREADS, "restriction passes fit one block");

// shared-memory slot of fine node (nx, ny, nz) of the brick: the row is rotated
// by 16 (ny bit 1) + (nz bit 1) words
__device__ __forceinline__ int node_slot(int nx, int ny, int nz) {
  return ((nz * FY + ny) << 5) + ((nx + (((ny >> 1) & 1) << 4) + ((nz >> 1) & 1)) & 31);
}

// restriction weight x4 of fine node n = 4m + r onto coarse nodes: node n feeds
// local coarse index m (= J + 1 for the node J = m - 1), m + 1 and m + 2
template <int R>
__device__ __forceinline__ void tent_add(unsigned long long* acc, int m, unsigned long long s) {
  if (R == 0) { acc[m] += 2ull * s; acc[m + 1] += 2ull * s; }
  if (R == 1) { acc[m] += s; acc[m + 1] += 3ull * s; }
  if (R == 2) { acc[m + 1] += 4ull * s; }
  if (R == 3) { acc[m + 1] += 3ull * s; acc[m + 2] += s; }
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

// RT: the fine mesh's element type (float; double in the FP64 Poisson mode)
template <int ZX, typename RT>
__global__ void __launch_bounds__(DEP_THREADS, 3) k_deposit(
    const void* __restrict__ xp_, const int64_t* __restrict__ cell_start, int64_t cap, int nc, int nt, int nnt,
    double unit, RT* __restrict__ rho, int rp, size_t plane, unsigned long long* __restrict__ rho_c_acc,
    unsigned long long* __restrict__ mass_total, const int64_t* __restrict__ items,
    unsigned long long* __restrict__ split_nodes, unsigned int* __restrict__ split_done) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  extern __shared__ unsigned smem_u32[];
  unsigned* wa = smem_u32;   // NFN words: sums of q mod 2^16
  unsigned* wb = wa + NFN;   // NFN words: sums of q div 2^16
  __shared__ int64_t cst[NHC];
  __shared__ int cpre[NHC + 1];
  __shared__ float ltf[3][HX];  // 4 x in-tile coordinate of region cell -1..B-1 per dimension
  __shared__ int last_block;
  const int tid = threadIdx.x;
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

  for (int i = tid; i < 2 * NFN; i += DEP_THREADS) smem_u32[i] = 0u;
  if (tid >= 32 && tid < 32 + 3 * HX) {
    const int d = (tid - 32) / HX, c = (tid - 32) % HX;
    const int base = d == 0 ? x0 : d == 1 ? y0 : z0;
    ltf[d][c] = 4.f * (float)(cube_wrap(base + c - 1, nc) % nt);
  }
  {
    // cell table of the (B+1)^3 region in (z,y,x) order: one region cell per thread,
    // then a block-wide exclusive prefix of the counts (warp scans + warp totals)
    __shared__ int wtot[(NHC + 31) / 32];
    int cnt = 0;
    if (tid < NHC) {
      const int64_t c = region_cell(tid, x0, y0, z0, nc, nt, nnt);
      const int64_t s0 = cell_start[c];
      cst[tid] = s0;
      cnt = (int)(cell_start[c + 1] - s0);
    }
    const int lane = tid & 31, warp = tid >> 5;
    int inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    if (tid < NHC && (lane == 31 || tid == NHC - 1)) wtot[warp] = inc;
    __syncthreads();
    if (tid < NHC) {
      int before = 0;
      for (int w = 0; w < warp; ++w) before += wtot[w];
      cpre[tid] = before + inc - cnt;
      if (tid == NHC - 1) cpre[NHC] = before + inc;
    }
  }
  __syncthreads();
  const int total = cpre[NHC];
  const int tend = min(t1, total);
  const float xres = ZX == 1 ? 0.00390625f : 1.52587890625e-05f;  // 2^-8, 2^-16
  for (int t = t0 + tid; t < tend; t += DEP_THREADS) {
    int lo = 0, hi = NHC - 1;  // last q with cpre[q] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cpre[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int q = lo;
    const int64_t ip = cst[q] + (t - cpre[q]);
    const int cr[3] = {q % HX, (q / HX) % HY, q / (HX * HY)};  // region index (cell + 1)
    int o1[3];
    float dx1[3], dx2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float l4 = ltf[d][cr[d]];
      const uint32_t u = (uint32_t)(int32_t)xp[(size_t)d * cap + ip] & (ZX == 1 ? 0xFFu : 0xFFFFu);
      const float fr = __fmul_rn((float)u + 0.5f, xres);  // exact
      // tempx = ncell*(i-1) + ncell*frac (tile-relative) rounded once to real(4) (pm.f90:87):
      // both terms are exact in FP32, so the FP32 add is that single rounding
      const float tf = __fadd_rn(l4, __fmul_rn(4.f, fr));
      const float f = floorf(tf);
      dx1[d] = cube_fsub(f + 1.f, tf);
      dx2[d] = cube_fsub(1.f, dx1[d]);
      o1[d] = 4 * (cr[d] - 1) + (int)(f - l4);  // brick-local fine node of the lower corner
    }
    // a particle of the low-side layer reaches the brick only from the last fine cell
    // of its coarse cell (o1 = -1); the other three quarters touch no node here
    if (o1[0] < -1 || o1[1] < -1 || o1[2] < -1) continue;
#pragma unroll
    for (int c8 = 0; c8 < 8; ++c8) {
      const int sx = c8 & 1, sy = (c8 >> 1) & 1, sz = c8 >> 2;
      const int nx = o1[0] + sx, ny = o1[1] + sy, nz = o1[2] + sz;
      if (nx >= 0 && nx < FX && ny >= 0 && ny < FY && nz >= 0 && nz < FZ) {
        const float w = cube_fmul(cube_fmul(sx ? dx2[0] : dx1[0], sy ? dx2[1] : dx1[1]), sz ? dx2[2] : dx1[2]);
        // w * 2^32 is exact in FP32 (w <= 1); its nearest integer as in the FP64 form
        const unsigned long long qv = __float2ull_rn(__fmul_rn(w, 4294967296.f));  // <= 2^32
        const int s = node_slot(nx, ny, nz);
        atomicAdd(&wa[s], (unsigned)(qv & 0xFFFFull));
        atomicAdd(&wb[s], (unsigned)(qv >> 16));
      }
    }
  }
  __syncthreads();
  unsigned long long* sacc = slot >= 0 ? split_nodes + (size_t)slot * NFN : nullptr;
  if (sacc) {  // partial sums into the brick's slot; the last of its blocks goes on
    for (int i = tid; i < NFN; i += DEP_THREADS) {
      const unsigned long long s = (unsigned long long)wa[i] + ((unsigned long long)wb[i] << 16);
      if (s) atomicAdd(&sacc[i], s);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last_block = atomicAdd(&split_done[slot], 1u) == (unsigned)((total + DMAX - 1) / DMAX - 1);
    __syncthreads();
    if (!last_block) return;
    __threadfence();
  }
  // z pass: one (x, y) column per thread writes its fine nodes and restricts them in z
  const int cxl = tid & 31, cyl = tid >> 5;
  unsigned long long rz[CZ];
#pragma unroll
  for (int k = 0; k < CZ; ++k) rz[k] = 0ull;
  unsigned long long msum = 0ull;
  RT* rrow = rho + (size_t)(4 * z0) * plane + (size_t)(4 * y0 + cyl) * rp + (4 * x0 + cxl);
#pragma unroll
  for (int m = 0; m < BZ; ++m) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int nz = 4 * m + r;
      const int s = node_slot(cxl, cyl, nz);
      const unsigned long long S =
          sacc ? __ldcg(&sacc[s]) : (unsigned long long)wa[s] + ((unsigned long long)wb[s] << 16);
      msum += S;
      rrow[(size_t)nz * plane] = (RT)((double)S * unit);
      if (r == 0) tent_add<0>(rz, m, S);
      if (r == 1) tent_add<1>(rz, m, S);
      if (r == 2) tent_add<2>(rz, m, S);
      if (r == 3) tent_add<3>(rz, m, S);
    }
  }
  __syncthreads();  // every node read: the words are free for the restriction
  unsigned long long* R1 = reinterpret_cast<unsigned long long*>(smem_u32);  // [CZ][FY][FX]
  unsigned long long* R2 = R1 + CZ * FY * FX;                                // [CZ][CY][FX]
#pragma unroll
  for (int k = 0; k < CZ; ++k) R1[(k * FY + cyl) * FX + cxl] = rz[k];
  __syncthreads();
  // y pass: one (z node, x) column per thread
  if (tid < CZ * FX) {
    const int k = tid >> 5, x = tid & 31;
    unsigned long long ry[CY];
#pragma unroll
    for (int j = 0; j < CY; ++j) ry[j] = 0ull;
#pragma unroll
    for (int m = 0; m < BY; ++m) {
      tent_add<0>(ry, m, R1[(k * FY + 4 * m) * FX + x]);
      tent_add<1>(ry, m, R1[(k * FY + 4 * m + 1) * FX + x]);
      tent_add<2>(ry, m, R1[(k * FY + 4 * m + 2) * FX + x]);
      tent_add<3>(ry, m, R1[(k * FY + 4 * m + 3) * FX + x]);
    }
#pragma unroll
    for (int j = 0; j < CY; ++j) R2[(k * CY + j) * FX + x] = ry[j];
  }
  __syncthreads();
  // x pass: one coarse node per thread, added to the global accumulator
  if (tid < CX * CY * CZ) {
    const int i = tid % CX, j = (tid / CX) % CY, k = tid / (CX * CY);
    const unsigned long long* row = R2 + (k * CY + j) * FX;
    const int c = 4 * i - 2;  // brick-local fine node of coarse node i - 1's centre (4(i-1)+2)
    unsigned long long s = 0ull;
#pragma unroll
    for (int d = -3; d <= 3; ++d) {
      const int n = c + d;
      if (n >= 0 && n < FX) s += (unsigned long long)(4 - (d < 0 ? -d : d)) * row[n];
    }
    if (s) {
      const int gx = cube_wrap(x0 + i - 1, nc), gy = cube_wrap(y0 + j - 1, nc), gz = cube_wrap(z0 + k - 1, nc);
      atomicAdd(&rho_c_acc[((size_t)gz * nc + gy) * nc + gx], s);
    }
  }
  for (int o = 16; o > 0; o >>= 1) msum += __shfl_xor_sync(0xffffffffu, msum, o);
  if ((tid & 31) == 0) atomicAdd(mass_total, msum);
}

// coarse accumulators -> FP32 density (pitch rp), accumulators cleared for the next
// step: mass * (particle sum) * 2^-38 + (neutrino sum) * 2^-32; the mass totals are
// the particle sums / 64 (scale 2^32, without the mass) and the neutrino sums
template <typename RT>
__global__ void k_coarse_finalize(unsigned long long* __restrict__ acc, unsigned long long* __restrict__ acc_nu,
                                  RT* __restrict__ r3, int nc, int rp, double unit_c,
                                  unsigned long long* __restrict__ mass_total) {
  const int64_t rows = (int64_t)nc * nc;  // (y, z) rows of nc nodes, one row per block at a time
  unsigned long long msum = 0ull, nsum = 0ull;
  for (int64_t yz = blockIdx.x; yz < rows; yz += gridDim.x)
    for (int x = threadIdx.x; x < nc; x += blockDim.x) {
      const int64_t i = yz * nc + x;
      const unsigned long long a = acc[i];
      acc[i] = 0ull;
      msum += a >> 6;
      double v = (double)a * unit_c;
      if (acc_nu) {
        const unsigned long long b = acc_nu[i];
        acc_nu[i] = 0ull;
        nsum += b;
        v = v + (double)b * (1.0 / FIX_SCALE);
      }
      r3[yz * rp + x] = (RT)v;
    }
  for (int o = 16; o > 0; o >>= 1) {
    msum += __shfl_xor_sync(0xffffffffu, msum, o);
    nsum += __shfl_xor_sync(0xffffffffu, nsum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(mass_total, msum);
    if (nsum) atomicAdd(mass_total + 1, nsum);
  }
}

}  // namespace

int cube_deposit(cube_ctx* ctx, cube_scalars* io) {
  const int nc = ctx->nc;
  if (nc % BX || nc % BY || nc % BZ) {
    ctx->err = "nc must be a multiple of 8";
    return CUBE_ERR_PARAM;
  }
  unsigned long long* mtot = reinterpret_cast<unsigned long long*>(ctx->red_tmp);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(mtot, 0, 3 * sizeof(unsigned long long), ctx->stream));
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
    const size_t node_bytes = sizeof(unsigned long long) * NFN * hv[1];
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
  const size_t smem = 2 * sizeof(unsigned) * NFN;
  const double unit = (double)io->mass_p_cdm * (1.0 / FIX_SCALE);  // exact
  auto launch = [&](auto kern, auto* rho) -> int {
    CUBE_CUDA_TRY(ctx, cube_smem_limit(kern, smem));
    kern<<<(unsigned)blocks, DEP_THREADS, smem, ctx->stream>>>(ctx->xp, ctx->cell_start, ctx->cap, nc, ctx->nt,
                                                              ctx->nnt, unit, rho, ctx->fine.rp, ctx->fine.plane,
                                                              ctx->rho_c_acc, mtot, items, split_nodes, split_done);
    CUBE_LAUNCH_CHECK(ctx);
    return CUBE_OK;
  };
  double* rho_d = reinterpret_cast<double*>(ctx->fine.rho);
  int lrc;
  if (ctx->fine.fp64)
    lrc = ctx->izipx == 1 ? launch(k_deposit<1, double>, rho_d) : launch(k_deposit<2, double>, rho_d);
  else
    lrc = ctx->izipx == 1 ? launch(k_deposit<1, float>, ctx->fine.rho) : launch(k_deposit<2, float>, ctx->fine.rho);
  if (lrc) return lrc;
  if (ctx->nu.on) {  // neutrino density into both meshes (pm.f90:55-74, :198-242)
    const int rc = cube_nu_density(ctx, io);
    if (rc) return rc;
  }
  const double unit_c = (double)io->mass_p_cdm * (1.0 / (64.0 * FIX_SCALE));  // exact
  if (ctx->coarse.fp64)
    k_coarse_finalize<double><<<8 * ctx->num_sms, 256, 0, ctx->stream>>>(ctx->rho_c_acc, nullptr,
                                                            reinterpret_cast<double*>(ctx->coarse.rho), nc,
                                                            ctx->coarse.rp, unit_c, mtot + 1);
  else
    k_coarse_finalize<float><<<8 * ctx->num_sms, 256, 0, ctx->stream>>>(ctx->rho_c_acc, ctx->nu.on ? ctx->rho_c_nu : nullptr,
                                                           ctx->coarse.rho, nc, ctx->coarse.rp, unit_c, mtot + 1);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}
