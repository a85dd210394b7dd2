/*
 * k_pp.cu -- ext_pp_force: particle-particle correction over the fine cells
 * within +-pp_range of each particle's fine cell (ext_pp_force.f90:34-143).
 *
 * The reference builds a head-of-chain linked list per fine cell (LIFO, over
 * the coarse cells 0..nt+1 of a tile) and, for every particle of a physical
 * fine cell, sums m*(dx/r^3)*(1-7/4 rho^3+3/4 rho^5), rho=r/nf_cutoff, zero
 * for r <= rsoft, over the neighbour cells in (k,j,i) order, each chain
 * newest-first.  A fine cell lies inside exactly one coarse cell, so its chain
 * is that coarse cell's particles in reverse storage order, filtered by fine
 * cell.
 *
 * Targets in bricks of 4^3 coarse cells whose region (the brick and a one-cell
 * halo) holds no cell of more than PP_DENSE particles walk their windows over
 * per-cell fine-occupancy masks in global memory (k_pp_masks, k_pp_walk below),
 * 32 targets per warp with the pair terms evaluated pair-parallel.  Crowded
 * bricks go to k_pp_brick: one CTA stages the particles of the brick and of its
 * halo (6^3 coarse cells, 24^3 fine cells) in shared memory, and the targets add
 * the pair terms of the 27 (or (2 pp_range+1)^3) window cells in the reference's
 * (k,j,i) order, each cell's particles newest-first:
 *   - sparse bricks (up to PB_SPARSE staged) keep the reference's chains: one
 *     thread per region coarse cell threads its particles into per-fine-cell
 *     lists in storage order, and each warp evaluates its 32 targets' entries
 *     pair-parallel;
 *   - dense bricks sort the staged particles by fine cell (counting sort, each
 *     fine cell's particles newest-first, the brick's own fine cells numbered
 *     first so that the targets are the first T slots), so each window cell is
 *     a contiguous range and the targets of one fine cell, which share their
 *     window, sit in the same warp: where particles cluster the lanes walk ranges
 *     of equal length instead of chains of different lengths.
 * The pair arithmetic is FP64 as in the reference (xvec* are real(8)), so the
 * kicked codes are bit-identical to the oracle.  Bricks with more than PB_CAP
 * staged particles build the sorted arrays in global memory (one CTA per brick)
 * and spread their targets over many CTAs.
 */
#include "cube_internal.cuh"

#include <vector>

namespace {

constexpr int PB = 4;                     // brick edge in coarse cells
constexpr int PR = PB + 2;                // with the halo
constexpr int PRC = PR * PR * PR;         // 216 region cells
constexpr int PF = 4 * PR;                // region edge in fine cells (24)
constexpr int NFC = PF * PF * PF;         // 13824 region fine cells
constexpr int NOWN = 16 * 16 * 16;        // the brick's own fine cells, numbered first
constexpr int PB_CAP = 4096;              // particles staged per brick in shared memory
constexpr int PB_SPARSE = 2560;           // up to this many: the chains; above: the fine-cell sort
constexpr int PP_THREADS = 256;
constexpr int PP_PMAX = 4096;             // staged window entries of the block's warps, evaluated pair-parallel
constexpr int PPW_MAX = PP_PMAX / (PP_THREADS / 32);  // per warp (32 targets)

// fine cell (region coordinates, 0..23) -> sort index: own cells (4..19 in every
// dimension) first in (z,y,x) order, then the halo cells in raster order
__device__ __forceinline__ int pp_fidx(int fx, int fy, int fz) {
  const bool ox = (unsigned)(fx - 4) < 16u, oy = (unsigned)(fy - 4) < 16u, oz = (unsigned)(fz - 4) < 16u;
  if (ox && oy && oz) return ((fz - 4) * 16 + (fy - 4)) * 16 + (fx - 4);
  int before = min(max(fz - 4, 0), 16) * 256;  // own cells ahead of this one in raster order
  if (oz) {
    before += min(max(fy - 4, 0), 16) * 16;
    if (oy) before += min(max(fx - 4, 0), 16);
  }
  return NOWN + (fz * PF + fy) * PF + fx - before;
}

// FP64 pair term of ext_pp_force.f90:99-107 for a separation x21 (exact in FP64).
// rc = rmag/nf_cutoff is evaluated as rmag*(1/nf_cutoff) only when nf_cutoff is
// a power of two, where both are the same exact scaling.
__device__ __forceinline__ void pp_pair(const double x21[3], double mass, double rsoft, int nf_cutoff,
                                        bool pow2_cut, double inv_cut, double fp[3]) {
  double rmag = sqrt(cube_dadd(cube_dadd(cube_dmul(x21[0], x21[0]), cube_dmul(x21[1], x21[1])),
                               cube_dmul(x21[2], x21[2])));
  if (rmag == 0.0) rmag = 1.0;
  const double rc = pow2_cut ? cube_dmul(rmag, inv_cut) : cube_ddiv(rmag, (double)nf_cutoff);
  const double rc2 = cube_dmul(rc, rc);
  const double rc3 = cube_dmul(rc2, rc);
  const double rc5 = cube_dmul(cube_dmul(rc2, rc2), rc);
  const double pcut = cube_dadd(cube_dsub(1.0, cube_dmul(1.75, rc3)), cube_dmul(0.75, rc5));
  const double r3 = cube_dmul(cube_dmul(rmag, rmag), rmag);
  const bool keep = rmag > rsoft;
  const double y = __drcp_rn(r3);  // the three IEEE quotients x21/r3 through one reciprocal
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double f = cube_dmul(cube_dmul(mass, cube_div_rcp(x21[d], r3, y)), pcut);
    if (!keep) f = cube_dmul(f, 0.0);
    fp[d] = f;
  }
}

struct PPArgs {
  int pr, nf_cutoff;
  double rsoft, mass, a_mid, dt, pi_d, coef;
  double rcp6, rcp_pi;  // RN(1/6), RN(1/pi_d)
  VencTab tab;
  const double* dec;  // tan(code)/coef per code (cube_vdec_table)
  int half_nvbin;
  cube_codec codec;
  int64_t cap;
};

// the fine-cell-sorted particles of one region: end offsets per sort index (the
// start of index f is the end of f-1) and the three position codes per slot
template <typename OffT>
struct Sorted {
  const OffT* off;
  const uint16_t* c0;
  const uint16_t* c1;
  const uint16_t* c2;
  __device__ __forceinline__ int start(int f) const { return f ? (int)off[f - 1] : 0; }
  __device__ __forceinline__ int end(int f) const { return (int)off[f]; }
};

struct PPAcc {
  unsigned long long n1 = 0, npair = 0;
  float f2max = 0.f;
};

// the brick's chains (sparse bricks): head per region fine cell (raster order),
// next per staged particle, staged codes [m][3]
struct Chains {
  const uint16_t* head;
  const uint16_t* nxt;
  const uint16_t* code;
};

// kick of one target by its pair sum ft (ext_pp_force.f90:115-127): velocity codes
// vc (index code + nvbin/2) decoded, v + ((ft*a_mid)*dt)/6/pi, re-encoded; f2 max
template <int ZV>
__device__ __forceinline__ void pp_apply(const double ft[3], const int vc[3], int64_t ip, const PPArgs& A,
                                         void* __restrict__ vp_, PPAcc& acc) {
  typedef typename CodeT<ZV>::T TV;
  TV* vp = reinterpret_cast<TV*>(vp_);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // a zero sum gives k = +-0 and v + k = v: a code that re-encodes to itself stays
    if (ft[d] == 0.0 && cube_vfixed(A.dec, 2 * A.half_nvbin, vc[d])) continue;
    double k = cube_dmul(ft[d], A.a_mid);
    k = cube_dmul(k, A.dt);
    k = cube_div_rcp(k, 6.0, A.rcp6);   // the IEEE quotients /6 and /pi (Markstein, one
    k = cube_div_rcp(k, A.pi_d, A.rcp_pi);  // correctly rounded reciprocal each)
    const double v = cube_dadd(__ldg(&A.dec[vc[d]]), k);
    vp[(size_t)d * A.cap + ip] = (TV)cube_wrap_code(cube_vencode_step(&A.codec, A.tab, v, A.coef), ZV);
  }
  const double f2 = cube_dadd(cube_dadd(cube_dmul(ft[0], ft[0]), cube_dmul(ft[1], ft[1])), cube_dmul(ft[2], ft[2]));
  acc.f2max = fmaxf(acc.f2max, (float)f2);
}

// one target with codes tc, global index ip, region coarse cell cc; neighbours
// from the sorted ranges S (CHAIN = false) or the chains H (CHAIN = true)
template <int ZX, int ZV, bool CHAIN, typename OffT>
__device__ __forceinline__ void pp_target(const Sorted<OffT>& S, const Chains& H, const uint16_t tc[3], int64_t ip,
                                          const int cc[3], const PPArgs& A, void* __restrict__ vp_, PPAcc& acc) {
  typedef typename CodeT<ZV>::T TV;
  TV* vp = reinterpret_cast<TV*>(vp_);
  double x1[3], ft[3] = {0.0, 0.0, 0.0};
  int g1[3], vc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double fr = cube_xfrac((int32_t)(int16_t)tc[d], ZX);
    x1[d] = cube_dadd(4.0 * (double)cc[d], cube_dmul(4.0, fr));
    g1[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, fr));
    vc[d] = (int)vp[(size_t)d * A.cap + ip] + A.half_nvbin;
  }
  ++acc.n1;
  const bool pow2_cut = (A.nf_cutoff & (A.nf_cutoff - 1)) == 0;
  const double inv_cut = 1.0 / (double)A.nf_cutoff;
  const int pr = A.pr;
  auto pair = [&](const uint16_t nc3[3], const double cf[3]) {
    double x21[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double fr = cube_xfrac((int32_t)(int16_t)nc3[d], ZX);
      x21[d] = cube_dsub(cube_dadd(cf[d], cube_dmul(4.0, fr)), x1[d]);
    }
    // a coincident particle (the target itself included) adds exactly +0
    if (x21[0] == 0.0 && x21[1] == 0.0 && x21[2] == 0.0) return;
    double fp[3];
    pp_pair(x21, A.mass, A.rsoft, A.nf_cutoff, pow2_cut, inv_cut, fp);
#pragma unroll
    for (int d = 0; d < 3; ++d) ft[d] = cube_dadd(ft[d], fp[d]);
  };
  for (int kk = g1[2] - pr; kk <= g1[2] + pr; ++kk)
    for (int jj = g1[1] - pr; jj <= g1[1] + pr; ++jj) {
      if (CHAIN) {
        const int rbase = (kk * PF + jj) * PF;
        for (int ii = g1[0] - pr; ii <= g1[0] + pr; ++ii) {
          int m2 = H.head[rbase + ii];
          if (m2 == 0xFFFF) continue;
          const double cf[3] = {4.0 * (double)(ii >> 2), 4.0 * (double)(jj >> 2), 4.0 * (double)(kk >> 2)};
          while (m2 != 0xFFFF) {
            ++acc.npair;
            const uint16_t nc3[3] = {H.code[3 * m2], H.code[3 * m2 + 1], H.code[3 * m2 + 2]};
            pair(nc3, cf);
            m2 = H.nxt[m2];
          }
        }
      } else {
        // sort indices along the row (kk, jj): pp_fidx with the row terms hoisted
        const bool orow = (unsigned)(kk - 4) < 16u && (unsigned)(jj - 4) < 16u;
        int before = min(max(kk - 4, 0), 16) * 256;
        if ((unsigned)(kk - 4) < 16u) before += min(max(jj - 4, 0), 16) * 16;
        const int hbase = NOWN + (kk * PF + jj) * PF - before;
        const int obase = ((kk - 4) * 16 + (jj - 4)) * 16 - 4;
        for (int ii = g1[0] - pr; ii <= g1[0] + pr; ++ii) {
          const bool own = orow && (unsigned)(ii - 4) < 16u;
          const int f = own ? obase + ii : hbase + ii - ((orow && ii >= 20) ? 16 : 0);
          const int s0 = S.start(f), s1 = S.end(f);
          if (s0 == s1) continue;
          const double cf[3] = {4.0 * (double)(ii >> 2), 4.0 * (double)(jj >> 2), 4.0 * (double)(kk >> 2)};
          acc.npair += (unsigned long long)(s1 - s0);
          for (int s = s0; s < s1; ++s) {
            const uint16_t nc3[3] = {S.c0[s], S.c1[s], S.c2[s]};
            pair(nc3, cf);
          }
        }
      }
    }
  pp_apply<ZV>(ft, vc, ip, A, vp_, acc);
}

__device__ __forceinline__ void pp_flush(PPAcc& acc, DevScal* dscal) {
  for (int o = 16; o > 0; o >>= 1) {
    acc.n1 += __shfl_xor_sync(0xffffffffu, acc.n1, o);
    acc.npair += __shfl_xor_sync(0xffffffffu, acc.npair, o);
    acc.f2max = fmaxf(acc.f2max, __shfl_xor_sync(0xffffffffu, acc.f2max, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&dscal->itest1, acc.n1);
    atomicAdd(&dscal->npairs, acc.npair);
    atomicMax(&dscal->f2_pp_bits, __float_as_uint(acc.f2max));
  }
}

// exclusive prefix sum of a[0..n) in place, by the whole CTA
template <typename T>
__device__ void block_exscan(T* a, int n) {
  __shared__ unsigned int ws[PP_THREADS / 32];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b = min(n, (int)threadIdx.x * per), e = min(n, b + per);
  unsigned int sum = 0;
  for (int i = b; i < e; ++i) sum += (unsigned int)a[i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned int inc = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned int v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    unsigned int w = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int v = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += v;
    }
    if (lane < (int)(blockDim.x >> 5)) ws[lane] = w;
  }
  __syncthreads();
  unsigned int run = (warp ? ws[warp - 1] : 0u) + inc - sum;
  for (int i = b; i < e; ++i) {
    const unsigned int v = (unsigned int)a[i];
    a[i] = (T)run;
    run += v;
  }
  __syncthreads();
}

// region of brick b: per region coarse cell its first particle and the prefix of
// counts (cpre[PRC] = particles staged); run by the whole CTA
__device__ void pp_region(int brick, const int64_t* __restrict__ cell_start, int nc, int nt, int nnt,
                          int64_t* cst, int* cpre) {
  const int nb = nc / PB;
  const int bx = brick % nb, by = (brick / nb) % nb, bz = brick / (nb * nb);
  const int x0 = bx * PB - 1, y0 = by * PB - 1, z0 = bz * PB - 1;  // region origin (global coarse, unwrapped)
  if (threadIdx.x < 32) {
    int run = 0;
    for (int base = 0; base < PRC; base += 32) {
      const int q = base + threadIdx.x;
      int cnt = 0;
      if (q < PRC) {
        const int cx = q % PR, cy = (q / PR) % PR, cz = q / (PR * PR);
        const int gx = (x0 + cx + nc) % nc, gy = (y0 + cy + nc) % nc, gz = (z0 + cz + nc) % nc;
        const int64_t c = cube_cell_of(gx, gy, gz, nt, nnt);
        cst[q] = cell_start[c];
        cnt = (int)(cell_start[c + 1] - cst[q]);
      }
      int inc = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)threadIdx.x >= o) inc += v;
      }
      if (q < PRC) cpre[q] = run + inc - cnt;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (threadIdx.x == 0) cpre[PRC] = run;
  }
  __syncthreads();
}

__device__ __forceinline__ int pp_cell_of_slot(const int* cpre, int m) {
  int lo = 0, hi = PRC - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cpre[mid] <= m) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// counting sort of the region's M particles by fine cell into slots: off (NFC
// counters -> end offsets), codes per slot and, per slot, the staging index m
// (sidx) and/or the global index (sip).  fidx holds the sort index per m.
template <int ZX, typename OffT, typename IdxT>
__device__ void pp_sort(const void* __restrict__ xp_, int64_t cap, const int64_t* cst, const int* cpre, int M,
                        OffT* off, IdxT* fidx, uint16_t* c0, uint16_t* c1, uint16_t* c2, uint16_t* sidx,
                        int64_t* sip) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  for (int i = threadIdx.x; i < NFC; i += blockDim.x) off[i] = 0;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    const int q = pp_cell_of_slot(cpre, m);
    const int64_t ip = cst[q] + (m - cpre[q]);
    const int cc[3] = {q % PR, (q / PR) % PR, q / (PR * PR)};
    int f[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      f[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, cube_xfrac((int)xp[(size_t)d * cap + ip], ZX)));
    fidx[m] = (IdxT)pp_fidx(f[0], f[1], f[2]);
  }
  __syncthreads();
  // a fine cell lies in one coarse cell: its thread counts it, no atomics
  for (int q = threadIdx.x; q < PRC; q += blockDim.x)
    for (int m = cpre[q]; m < cpre[q + 1]; ++m) off[fidx[m]] = (OffT)(off[fidx[m]] + 1);
  __syncthreads();
  block_exscan(off, NFC);
  // newest first inside each fine cell: the chain order of the reference
  for (int q = threadIdx.x; q < PRC; q += blockDim.x)
    for (int m = cpre[q + 1] - 1; m >= cpre[q]; --m) {
      const int f = (int)fidx[m];
      const int s = (int)off[f];
      off[f] = (OffT)(s + 1);
      const int64_t ip = cst[q] + (m - cpre[q]);
      c0[s] = (uint16_t)xp[ip];
      c1[s] = (uint16_t)xp[(size_t)cap + ip];
      c2[s] = (uint16_t)xp[2 * (size_t)cap + ip];
      if (sidx) sidx[s] = (uint16_t)m;
      if (sip) sip[s] = ip;
    }
  __syncthreads();
}

// pp_sort for a region staged in shared memory: the slot of particle m is the
// start of its fine cell plus the number of later particles of its coarse cell in
// the same fine cell (newest first), so every particle is placed by its own
// thread, with its codes read once from global memory, in parallel.  Leaves
// end offsets in off, as pp_sort does.
template <int ZX>
__device__ void pp_sort_par(const void* __restrict__ xp_, int64_t cap, const int64_t* cst, const int* cpre, int M,
                            uint16_t* off, uint16_t* fidx, uint16_t* c0, uint16_t* c1, uint16_t* c2,
                            uint16_t* sidx) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  for (int i = threadIdx.x; i < NFC; i += blockDim.x) off[i] = 0;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    const int q = pp_cell_of_slot(cpre, m);
    const int64_t ip = cst[q] + (m - cpre[q]);
    const int cc[3] = {q % PR, (q / PR) % PR, q / (PR * PR)};
    int f[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
      f[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, cube_xfrac((int)xp[(size_t)d * cap + ip], ZX)));
    fidx[m] = (uint16_t)pp_fidx(f[0], f[1], f[2]);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < PRC; q += blockDim.x)
    for (int m = cpre[q]; m < cpre[q + 1]; ++m) off[fidx[m]] = (uint16_t)(off[fidx[m]] + 1);
  __syncthreads();
  block_exscan(off, NFC);  // start offsets
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    const int q = pp_cell_of_slot(cpre, m);
    const int fm = fidx[m];
    int rank = 0;
    for (int j = m + 1; j < cpre[q + 1]; ++j) rank += fidx[j] == fm;
    const int sl = off[fm] + rank;
    const int64_t ip = cst[q] + (m - cpre[q]);
    c0[sl] = (uint16_t)xp[ip];
    c1[sl] = (uint16_t)xp[(size_t)cap + ip];
    c2[sl] = (uint16_t)xp[2 * (size_t)cap + ip];
    sidx[sl] = (uint16_t)m;
  }
  // start offsets -> end offsets (end of f = start of f+1, the last one M)
  const int per = (NFC + blockDim.x - 1) / blockDim.x;
  const int b = min(NFC, (int)threadIdx.x * per), e = min(NFC, b + per);
  const int next = e < NFC ? off[e] : M;
  __syncthreads();
  for (int i = b; i < e; ++i) off[i] = (uint16_t)(i + 1 < e ? off[i + 1] : next);
  __syncthreads();
}

template <int ZX, int ZV>
__global__ void __launch_bounds__(PP_THREADS, 2) k_pp_brick(const void* __restrict__ xp_, void* __restrict__ vp_,
                                                         const int64_t* __restrict__ cell_start, int nc, int nt,
                                                         int nnt, PPArgs A, int32_t* __restrict__ spill,
                                                         DevScal* __restrict__ dscal,
                                                         const int32_t* __restrict__ bricks) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  extern __shared__ unsigned char pbsm[];
  __shared__ int64_t cst[PRC];
  __shared__ int cpre[PRC + 1];
  __shared__ int tpre[PB * PB * PB + 1];  // prefix of the brick's own cells (chain targets)
  const int brick = bricks ? bricks[blockIdx.x] : (int)blockIdx.x;
  pp_region(brick, cell_start, nc, nt, nnt, cst, cpre);
  const int M = cpre[PRC];
  if (M > PB_CAP) {  // crowded: sorted in global memory by k_pp_build
    if (threadIdx.x == 0) {
      const unsigned long long q = atomicAdd(&dscal->n_big, 1ull);
      spill[2 * q] = brick;
      spill[2 * q + 1] = M;
    }
    return;
  }
  PPAcc acc;
  if (M > PB_SPARSE) {
    // dense: fine-cell sorted slots, targets grouped by fine cell
    uint16_t* off = reinterpret_cast<uint16_t*>(pbsm);  // NFC
    uint16_t* fidx = off + NFC;                         // PB_CAP
    uint16_t* c0 = fidx + PB_CAP;                       // PB_CAP each
    uint16_t* c1 = c0 + PB_CAP;
    uint16_t* c2 = c1 + PB_CAP;
    uint16_t* sidx = c2 + PB_CAP;
    pp_sort_par<ZX>(xp_, A.cap, cst, cpre, M, off, fidx, c0, c1, c2, sidx);
    const Sorted<uint16_t> S = {off, c0, c1, c2};
    const Chains H = {nullptr, nullptr, nullptr};
    const int T = off[NOWN - 1];
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
      const int m = sidx[t];
      const int q = pp_cell_of_slot(cpre, m);
      const int cc[3] = {q % PR, (q / PR) % PR, q / (PR * PR)};
      const uint16_t tc[3] = {c0[t], c1[t], c2[t]};
      pp_target<ZX, ZV, false>(S, H, tc, cst[q] + (m - cpre[q]), cc, A, vp_, acc);
    }
  } else {
    // sparse: the reference's chains in shared memory, targets in storage order
    uint16_t* head = reinterpret_cast<uint16_t*>(pbsm);  // NFC, raster order
    uint16_t* nxt = head + NFC;                          // PB_CAP
    uint16_t* fr = nxt + PB_CAP;                         // PB_CAP: raster fine cell per m
    uint16_t* code = fr + PB_CAP;                        // 3 * PB_CAP
    if (threadIdx.x < 32) {  // own cells in (z,y,x) order, two per lane
      int n2[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = 2 * threadIdx.x + h;
        const int q = (((t >> 4) + 1) * PR + ((t >> 2) & 3) + 1) * PR + (t & 3) + 1;
        n2[h] = cpre[q + 1] - cpre[q];
      }
      int inc = n2[0] + n2[1];
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)threadIdx.x >= o) inc += v;
      }
      tpre[2 * threadIdx.x] = inc - n2[0] - n2[1];
      tpre[2 * threadIdx.x + 1] = inc - n2[1];
      if (threadIdx.x == 31) tpre[PB * PB * PB] = inc;
    }
    for (int i = threadIdx.x; i < NFC; i += blockDim.x) head[i] = 0xFFFFu;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
      const int q = pp_cell_of_slot(cpre, m);
      const int64_t ip = cst[q] + (m - cpre[q]);
      const int cc[3] = {q % PR, (q / PR) % PR, q / (PR * PR)};
      int f[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const int cd = (int)xp[(size_t)d * A.cap + ip];
        code[3 * m + d] = (uint16_t)cd;
        f[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, cube_xfrac(cd, ZX)));
      }
      fr[m] = (uint16_t)((f[2] * PF + f[1]) * PF + f[0]);
    }
    __syncthreads();
    // the thread of region cell q inserts q's particles in storage order: each
    // chain is newest-first, as the linked list of ext_pp_force.f90:51-73
    for (int q = threadIdx.x; q < PRC; q += blockDim.x)
      for (int m = cpre[q]; m < cpre[q + 1]; ++m) {
        const int f = fr[m];
        nxt[m] = head[f];
        head[f] = (uint16_t)m;
      }
    __syncthreads();
    const Sorted<uint16_t> S = {nullptr, nullptr, nullptr, nullptr};
    const Chains H = {head, nxt, code};
    const int T = tpre[PB * PB * PB];
    // Targets in groups of 32, one group per warp and one target per lane: each lane
    // counts the entries of its window (the chains it walks), a warp scan places them,
    // each lane writes its entries in window order (with its lane number beside each),
    // and then the warp evaluates the FP64 pair terms of its list 32 at a time while
    // every lane adds its own terms in that order.  A coincident pair gives +0, which
    // leaves the running sum unchanged (it is never -0), so the sums are those of the
    // per-target walk.  Warps only meet at __syncwarp; a group whose windows hold more
    // than PPW_MAX entries walks per target.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint16_t* plist = code + 3 * PB_CAP + warp * PPW_MAX;                            // staged indices
    double* term = reinterpret_cast<double*>(code + 3 * PB_CAP + PP_PMAX) + warp * 3 * 32;  // [3][32]
    uint8_t* ptgt = reinterpret_cast<uint8_t*>(reinterpret_cast<double*>(code + 3 * PB_CAP + PP_PMAX) +
                                               (PP_THREADS / 32) * 3 * 32) + warp * PPW_MAX;  // lane of each entry
    const bool pow2_cut = (A.nf_cutoff & (A.nf_cutoff - 1)) == 0;
    const double inv_cut = 1.0 / (double)A.nf_cutoff;
    const int pr = A.pr;
    for (int g0 = warp * 32; g0 < T; g0 += PP_THREADS) {
      const int t = g0 + lane;
      const bool valid = t < T;
      int cc[3] = {0, 0, 0}, g1[3] = {0, 0, 0}, q = 0, m = 0, nt = 0;
      int64_t ip = 0;
      double x1[3] = {0.0, 0.0, 0.0};
      if (valid) {
        int lo = 0, hi = PB * PB * PB - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (tpre[mid] <= t) lo = mid; else hi = mid - 1;
        }
        cc[0] = (lo & 3) + 1; cc[1] = ((lo >> 2) & 3) + 1; cc[2] = (lo >> 4) + 1;
        q = (cc[2] * PR + cc[1]) * PR + cc[0];
        m = cpre[q] + (t - tpre[lo]);
        ip = cst[q] + (t - tpre[lo]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double fr = cube_xfrac((int32_t)(int16_t)code[3 * m + d], ZX);
          x1[d] = cube_dadd(4.0 * (double)cc[d], cube_dmul(4.0, fr));
          g1[d] = 4 * cc[d] + (int)floor(cube_dmul(4.0, fr));
        }
        for (int kk = g1[2] - pr; kk <= g1[2] + pr; ++kk)
          for (int jj = g1[1] - pr; jj <= g1[1] + pr; ++jj) {
            const int rbase = (kk * PF + jj) * PF;
            for (int ii = g1[0] - pr; ii <= g1[0] + pr; ++ii)
              for (int m2 = head[rbase + ii]; m2 != 0xFFFF; m2 = nxt[m2]) ++nt;
          }
      }
      int inc = nt;
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += v;
      }
      const int off = inc - nt;
      const int P = __shfl_sync(0xffffffffu, inc, 31);
      if (P > PPW_MAX) {  // too many entries for the warp's list: the per-target walk
        if (valid) {
          const uint16_t tc[3] = {code[3 * m], code[3 * m + 1], code[3 * m + 2]};
          pp_target<ZX, ZV, true>(S, H, tc, ip, cc, A, vp_, acc);
        }
        continue;
      }
      if (valid) {
        int k = off;
        for (int kk = g1[2] - pr; kk <= g1[2] + pr; ++kk)
          for (int jj = g1[1] - pr; jj <= g1[1] + pr; ++jj) {
            const int rbase = (kk * PF + jj) * PF;
            for (int ii = g1[0] - pr; ii <= g1[0] + pr; ++ii)
              for (int m2 = head[rbase + ii]; m2 != 0xFFFF; m2 = nxt[m2]) {
                plist[k] = (uint16_t)m2;
                ptgt[k] = (uint8_t)lane;
                ++k;
              }
          }
      }
      __syncwarp();
      double ft[3] = {0.0, 0.0, 0.0};
      for (int cb = 0; cb < P; cb += 32) {
        const int p = cb + lane;
        const int tg = p < P ? ptgt[p] : lane;
        double tx[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) tx[d] = __shfl_sync(0xffffffffu, x1[d], tg);
        if (p < P) {
          const int m2 = plist[p];
          const int f2 = fr[m2];
          const int fi[3] = {f2 % PF, (f2 / PF) % PF, f2 / (PF * PF)};
          double x21[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double cf = 4.0 * (double)(fi[d] >> 2);
            const double frn = cube_xfrac((int32_t)(int16_t)code[3 * m2 + d], ZX);
            x21[d] = cube_dsub(cube_dadd(cf, cube_dmul(4.0, frn)), tx[d]);
          }
          double fp[3] = {0.0, 0.0, 0.0};
          if (!(x21[0] == 0.0 && x21[1] == 0.0 && x21[2] == 0.0))
            pp_pair(x21, A.mass, A.rsoft, A.nf_cutoff, pow2_cut, inv_cut, fp);
#pragma unroll
          for (int d = 0; d < 3; ++d) term[d * 32 + lane] = fp[d];
        }
        __syncwarp();
        if (valid) {
          const int e0 = max(off, cb), e1 = min(off + nt, cb + 32);
          for (int e = e0; e < e1; ++e)
#pragma unroll
            for (int d = 0; d < 3; ++d) ft[d] = cube_dadd(ft[d], term[d * 32 + (e - cb)]);
        }
        __syncwarp();
      }
      if (valid) {
        ++acc.n1;
        acc.npair += (unsigned long long)nt;
        typedef typename CodeT<ZV>::T TV;
        const TV* vpr = reinterpret_cast<const TV*>(vp_);
        int vc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) vc[d] = (int)vpr[(size_t)d * A.cap + ip] + A.half_nvbin;
        pp_apply<ZV>(ft, vc, ip, A, vp_, acc);
      }
    }
  }
  pp_flush(acc, dscal);
}

// crowded bricks: per brick, its fine-cell counters (NFC, global), staged sort
// indices and slot arrays at base .. base+M of the global slot arrays
struct PPCrowd {
  const int32_t* list;       // (brick, M) pairs
  const int64_t* base;       // slot base per crowded brick
  const int64_t* chunk0;     // first target CTA per crowded brick (n+1 entries)
  int n;
  uint32_t* off;             // [n][NFC]
  uint32_t* fidx;            // [slots]
  uint16_t *c0, *c1, *c2;    // [slots]
  int64_t* sip;              // [slots]
  uint8_t* scell;            // [slots] region coarse cell of the slot
};

template <int ZX>
__global__ void __launch_bounds__(PP_THREADS) k_pp_build(const void* __restrict__ xp_,
                                                         const int64_t* __restrict__ cell_start, int nc, int nt,
                                                         int nnt, int64_t cap, PPCrowd C) {
  __shared__ int64_t cst[PRC];
  __shared__ int cpre[PRC + 1];
  const int b = blockIdx.x;
  const int brick = C.list[2 * b];
  pp_region(brick, cell_start, nc, nt, nnt, cst, cpre);
  const int M = cpre[PRC];
  const int64_t base = C.base[b];
  uint32_t* off = C.off + (size_t)b * NFC;
  pp_sort<ZX>(xp_, cap, cst, cpre, M, off, C.fidx + base, C.c0 + base, C.c1 + base, C.c2 + base,
              (uint16_t*)nullptr, C.sip + base);
  // region coarse cell of each target slot (the own fine cells are the first NOWN indices)
  const int T = (int)off[NOWN - 1];
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    int lo = 0, hi = NOWN - 1;  // first own fine cell whose end exceeds t
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((int)off[mid] > t) hi = mid; else lo = mid + 1;
    }
    const int fz = lo >> 8, fy = (lo >> 4) & 15, fx = lo & 15;  // own fine cell, 0..15
    C.scell[base + t] = (uint8_t)(((fz / 4 + 1) * PR + fy / 4 + 1) * PR + fx / 4 + 1);
  }
}

template <int ZX, int ZV>
__global__ void __launch_bounds__(PP_THREADS) k_pp_crowd(void* __restrict__ vp_, PPArgs A, PPCrowd C,
                                                         DevScal* __restrict__ dscal) {
  int lo = 0, hi = C.n - 1;  // the crowded brick of this CTA
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (C.chunk0[mid] <= (int64_t)blockIdx.x) lo = mid; else hi = mid - 1;
  }
  const int b = lo;
  const int64_t base = C.base[b];
  const uint32_t* off = C.off + (size_t)b * NFC;
  const int T = (int)off[NOWN - 1];
  const int t = (int)(blockIdx.x - C.chunk0[b]) * PP_THREADS + threadIdx.x;
  PPAcc acc;
  if (t < T) {
    const Sorted<uint32_t> S = {off, C.c0 + base, C.c1 + base, C.c2 + base};
    const Chains H = {nullptr, nullptr, nullptr};
    const int q = C.scell[base + t];
    const int cc[3] = {q % PR, (q / PR) % PR, q / (PR * PR)};
    const uint16_t tc[3] = {S.c0[t], S.c1[t], S.c2[t]};
    pp_target<ZX, ZV, false>(S, H, tc, C.sip[base + t], cc, A, vp_, acc);
  }
  pp_flush(acc, dscal);
}

// ---- particle-parallel path (every brick whose region holds no crowded cell) ----
//   k_pp_masks  one thread per coarse cell: 64-bit masks of the fine cells holding
//               at least one and at least two particles, and each particle's fine
//               cell; a cell of more than PP_DENSE particles instead marks every
//               brick whose region (brick +- 1 cell) holds it as crowded;
//   k_pp_walk   the targets of the other bricks over the re-bin's work items, 32 per
//               warp: each lane walks its window in the reference's (k,j,i) order,
//               each fine cell's particles newest-first (reverse storage order within
//               the coarse cell), and records the partners; the warp then evaluates
//               the FP64 pair terms of all its lanes 32 at a time and every lane adds
//               its own in walk order, so the sums and the codes are those of the
//               chains of ext_pp_force.f90:51-73,76-127;
//   k_pp_crowd_list  the crowded bricks, for k_pp_brick.
// A target in a brick that is not crowded has its window inside that brick's region,
// which holds no crowded cell, so no window reads a crowded cell's masks (which are
// not built) and no scan of a coarse cell takes more than PP_DENSE particles.
constexpr int PP_DENSE = 32;

struct PPPar {
  const int64_t* cell_start;
  int64_t ncells;
  int nc, nt, nnt, nb;          // nb = nc / PB bricks per dimension
  unsigned long long* occ;      // [ncells] fine cells (bit (z*4+y)*4+x) holding a particle
  unsigned long long* multi;    // [ncells] fine cells holding two or more
  uint8_t* pfine;               // [cap] each particle's fine cell within its coarse cell
  unsigned int* crowded;        // [nb^3] 1: the brick's region holds a crowded cell
  int32_t* dense_list;          // crowded bricks for k_pp_brick, pp_dense of them
  int32_t* list_ip;             // listed targets (a neighbour in the window): particle, coarse cell
  int32_t* list_cell;
  DevScal* dscal;
};

// coarse cell ids of the neighbours -1, 0, +1 of (tile t, in-tile l) along one
// dimension whose tile stride is st and in-tile stride sl (cell ids are sums of
// the three dimensions' terms)
__device__ __forceinline__ void pp_sep3(int l, int t, int nt, int nnt, int64_t st, int64_t sl, int64_t out[3]) {
  out[1] = t * st + l * sl;
  out[0] = l > 0 ? out[1] - sl : (int64_t)((t + nnt - 1) % nnt) * st + (int64_t)(nt - 1) * sl;
  out[2] = l < nt - 1 ? out[1] + sl : (int64_t)((t + 1) % nnt) * st;
}

// the three per-dimension id terms of a cell's neighbours
__device__ __forceinline__ void pp_neighbours(int64_t c, int nt, int nnt, int64_t X[3], int64_t Y[3], int64_t Z[3],
                                              int g[3]) {
  const int64_t nt3 = (int64_t)nt * nt * nt;
  const int64_t tile = c / nt3;
  const int rem = (int)(c - tile * nt3);
  const int l[3] = {rem % nt, (rem / nt) % nt, rem / (nt * nt)};
  const int t[3] = {(int)(tile % nnt), (int)((tile / nnt) % nnt), (int)(tile / ((int64_t)nnt * nnt))};
  pp_sep3(l[0], t[0], nt, nnt, nt3, 1, X);
  pp_sep3(l[1], t[1], nt, nnt, nt3 * nnt, nt, Y);
  pp_sep3(l[2], t[2], nt, nnt, nt3 * nnt * nnt, (int64_t)nt * nt, Z);
#pragma unroll
  for (int d = 0; d < 3; ++d) g[d] = t[d] * nt + l[d];
}

// 4-bit mask of the fine cells [lo, hi] (coarse-cell relative) inside coarse offset o
__device__ __forceinline__ unsigned pp_range4(int lo, int hi, int o) {
  const int a = max(lo - 4 * o, 0), b = min(hi - 4 * o, 3);
  return a > b ? 0u : ((2u << b) - (1u << a));
}

template <int ZX>
__global__ void __launch_bounds__(256) k_pp_masks(const void* __restrict__ xp_, int64_t cap, PPPar Q) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= Q.ncells) return;
  const int64_t s0 = Q.cell_start[c], s1 = Q.cell_start[c + 1];
  if (s1 - s0 > PP_DENSE) {
    int l[3], tb[3];
    cube_cell_coords(c, Q.nt, Q.nnt, l, tb);
    int blo[3], bhi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int g = tb[d] + l[d];
      blo[d] = cube_wrap(g - 1, Q.nc) / PB;
      bhi[d] = cube_wrap(g + 1, Q.nc) / PB;
    }
    for (int kz = 0; kz < 2; ++kz)
      for (int ky = 0; ky < 2; ++ky)
        for (int kx = 0; kx < 2; ++kx) {
          if ((kz && bhi[2] == blo[2]) || (ky && bhi[1] == blo[1]) || (kx && bhi[0] == blo[0])) continue;
          Q.crowded[((kz ? bhi[2] : blo[2]) * Q.nb + (ky ? bhi[1] : blo[1])) * Q.nb + (kx ? bhi[0] : blo[0])] = 1u;
        }
    return;
  }
  unsigned long long occ = 0ull, multi = 0ull;
  for (int64_t ip = s0; ip < s1; ++ip) {
    int f = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d)
      f |= (int)floor(cube_dmul(4.0, cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX))) << (2 * d);
    Q.pfine[ip] = (uint8_t)f;
    const unsigned long long b = 1ull << f;
    multi |= occ & b;
    occ |= b;
  }
  Q.occ[c] = occ;
  Q.multi[c] = multi;
}

// nibble spread of a 4-bit mask (bit y -> bit 4y) and its 16-bit spread (bit z -> bit 16z)
__device__ __forceinline__ unsigned pp_spread4(unsigned m) {
  return (m & 1u) | ((m & 2u) << 3) | ((m & 4u) << 6) | ((m & 8u) << 9);
}
__device__ __forceinline__ unsigned long long pp_spread16(unsigned m) {
  return (unsigned long long)(m & 1u) | ((unsigned long long)(m & 2u) << 15) | ((unsigned long long)(m & 4u) << 30) |
         ((unsigned long long)(m & 8u) << 45);
}

// true if the window of +-pr fine cells around fine cell f of a coarse cell holds no
// particle but the target: nb[9] are the ids of the coarse neighbours -1..1 per
// dimension as separable terms (x, y, z; three each)
__device__ __forceinline__ bool pp_isolated(const PPPar& Q, int f, int pr, const int32_t* nb) {
  unsigned m[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int fl = (f >> (2 * d)) & 3;
#pragma unroll
    for (int o = 0; o < 3; ++o) m[d][o] = pp_range4(fl - pr, fl + pr, o - 1);
  }
  const unsigned long long own = 1ull << f;
#pragma unroll
  for (int oz = 0; oz < 3; ++oz)
#pragma unroll
    for (int oy = 0; oy < 3; ++oy)
#pragma unroll
      for (int ox = 0; ox < 3; ++ox) {
        if (!(m[2][oz] && m[1][oy] && m[0][ox])) continue;
        const int64_t C = (int64_t)nb[6 + oz] + nb[3 + oy] + nb[ox];
        const unsigned long long w = (unsigned long long)(m[0][ox] * pp_spread4(m[1][oy])) * pp_spread16(m[2][oz]);
        unsigned long long hit = __ldg(&Q.occ[C]) & w;
        if (ox == 1 && oy == 1 && oz == 1) hit = (hit & ~own) | (__ldg(&Q.multi[C]) & own);
        if (hit) return false;
      }
  return true;
}

// one thread per coarse cell of a brick that is not crowded: a target alone in its
// window (the masks decide) has a zero pair sum and is finished here (one window
// entry, the zero kick); the others are listed for k_pp_walk.  (One thread per
// target over the re-bin's work items left 7 of 32 lanes active in the branching
// window test; one CTA per brick with the 6^3 masks of brick and halo staged in
// shared memory read the halo 3.4 times over: both slower at 512^3.)
template <int ZV>
__global__ void __launch_bounds__(256, 3) k_pp_cells(PPPar Q, PPArgs A, void* __restrict__ vp_) {
  typedef typename CodeT<ZV>::T TV;
  const TV* vp = reinterpret_cast<const TV*>(vp_);
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  PPAcc acc;
  unsigned nonmask = 0u;  // targets of this cell with a neighbour (at most PP_DENSE = 32)
  int64_t s0 = 0;
  if (c < Q.ncells) {
    int64_t X[3], Y[3], Z[3];
    int g[3];
    pp_neighbours(c, Q.nt, Q.nnt, X, Y, Z, g);
    const int b = ((g[2] / PB) * Q.nb + g[1] / PB) * Q.nb + g[0] / PB;
    s0 = Q.cell_start[c];
    const int n = (int)(Q.cell_start[c + 1] - s0);
    if (!Q.crowded[b] && n > 0) {
      const int32_t nb9[9] = {(int32_t)X[0], (int32_t)X[1], (int32_t)X[2], (int32_t)Y[0], (int32_t)Y[1],
                              (int32_t)Y[2], (int32_t)Z[0], (int32_t)Z[1], (int32_t)Z[2]};
      for (int k = 0; k < n; ++k) {
        const int64_t ip = s0 + k;
        if (!pp_isolated(Q, Q.pfine[ip], A.pr, nb9)) {
          nonmask |= 1u << k;
        } else {
          ++acc.n1;
          ++acc.npair;
          const double ft[3] = {0.0, 0.0, 0.0};
          int vc[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) vc[d] = (int)vp[(size_t)d * A.cap + ip] + A.half_nvbin;
          if (!(cube_vfixed(A.dec, 2 * A.half_nvbin, vc[0]) && cube_vfixed(A.dec, 2 * A.half_nvbin, vc[1]) &&
                cube_vfixed(A.dec, 2 * A.half_nvbin, vc[2])))
            pp_apply<ZV>(ft, vc, ip, A, vp_, acc);
        }
      }
    }
  }
  const unsigned cnt = (unsigned)__popc(nonmask);
  unsigned inc = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned v = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += v;
  }
  const unsigned tot = __shfl_sync(0xffffffffu, inc, 31);
  unsigned long long base = 0;
  if (lane == 31 && tot) base = atomicAdd(&Q.dscal->pp_list, (unsigned long long)tot);
  base = __shfl_sync(0xffffffffu, base, 31);
  if (cnt) {
    unsigned long long k = base + inc - cnt;
    for (unsigned m = nonmask; m; m &= m - 1, ++k) {
      Q.list_ip[k] = (int32_t)(s0 + __ffs(m) - 1);
      Q.list_cell[k] = (int32_t)c;
    }
  }
  pp_flush(acc, Q.dscal);
}

// the crowded bricks, for k_pp_brick (one thread per brick)
__global__ void k_pp_crowd_list(PPPar Q, int nbricks) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbricks) return;
  if (Q.crowded[b]) Q.dense_list[atomicAdd(&Q.dscal->pp_dense, 1ull)] = b;
}

constexpr int PPL = 24;        // window entries per lane for the warp's pair pass

// one target's window walk in the reference's order: calls put(k, ip2, o) for each
// particle of each window fine cell, newest first; o = (oz+1)*9 + (oy+1)*3 + (ox+1) is
// the partner's coarse cell offset; returns the number of entries.  A window row
// (kk, jj) is read as the 4-bit nibble of each coarse cell it crosses (occupancy
// bits of fine cells x = 0..3), and the particles of an occupied fine cell are found
// four at a time by a byte compare of the coarse cell's fine-cell bytes, from the top
template <typename Put>
__device__ __forceinline__ int pp_walk_window(const PPPar& Q, const int32_t* nb9, int f, int pr, Put put) {
  const int fl[3] = {f & 3, (f >> 2) & 3, (f >> 4) & 3};
  unsigned m0[3];
#pragma unroll
  for (int o = 0; o < 3; ++o) m0[o] = pp_range4(fl[0] - pr, fl[0] + pr, o - 1);
  const uint32_t* pw = reinterpret_cast<const uint32_t*>(Q.pfine);
  int n = 0;
  for (int kk = fl[2] - pr; kk <= fl[2] + pr; ++kk) {
    const int oz = (kk + 4) / 4 - 1;  // floor(kk / 4), kk >= -4
    const int fz = kk - 4 * oz;
    for (int jj = fl[1] - pr; jj <= fl[1] + pr; ++jj) {
      const int oy = (jj + 4) / 4 - 1;
      const int fy = jj - 4 * oy;
      const int64_t CYZ = (int64_t)nb9[6 + oz + 1] + nb9[3 + oy + 1];
      const int rs = (fz * 4 + fy) * 4;  // bit of fine cell (0, fy, fz)
#pragma unroll
      for (int ox = -1; ox <= 1; ++ox) {
        if (!m0[ox + 1]) continue;
        const int64_t C = CYZ + nb9[ox + 1];
        unsigned nib = (unsigned)(__ldg(&Q.occ[C]) >> rs) & m0[ox + 1];
        if (!nib) continue;
        const unsigned mnib = (unsigned)(__ldg(&Q.multi[C]) >> rs);
        const int o = (oz + 1) * 9 + (oy + 1) * 3 + (ox + 1);
        const int64_t s0 = __ldg(&Q.cell_start[C]), s1 = __ldg(&Q.cell_start[C + 1]);
        for (; nib; nib &= nib - 1) {
          const int fx = __ffs(nib) - 1;
          const uint32_t key = (uint32_t)(rs + fx) * 0x01010101u;
          const bool one = !((mnib >> fx) & 1u);
          for (int64_t w = (s1 - 1) >> 2; w >= (s0 >> 2); --w) {  // newest first
            uint32_t eq = __vcmpeq4(__ldg(&pw[w]), key);
            const int64_t b0 = w << 2;
            if (b0 < s0) eq &= 0xFFFFFFFFu << (8 * (int)(s0 - b0));
            if (b0 + 4 > s1) eq &= 0xFFFFFFFFu >> (8 * (int)(b0 + 4 - s1));
            bool done = false;
            while (eq) {
              const int byte = (31 - __clz(eq)) >> 3;
              put(n, b0 + byte, o);
              ++n;
              eq &= ~(0xFFu << (8 * byte));
              if (one) { done = true; break; }
            }
            if (done) break;
          }
        }
      }
    }
  }
  return n;
}

// pair term of target position x1 (coarse-cell relative, FP64 exact) and partner ip2 in
// the coarse cell at offset o; +0 for a coincident particle (the target itself included)
template <int ZX>
__device__ __forceinline__ void pp_term(const void* __restrict__ xp_, const PPArgs& A, bool pow2_cut, double inv_cut,
                                        const double x1[3], int64_t ip2, int o, double fp[3]) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  const int od[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
  double x21[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double fr = cube_xfrac((int32_t)xp[(size_t)d * A.cap + ip2], ZX);
    x21[d] = cube_dsub(cube_dadd(4.0 * (double)od[d], cube_dmul(4.0, fr)), x1[d]);
  }
  fp[0] = fp[1] = fp[2] = 0.0;
  if (!(x21[0] == 0.0 && x21[1] == 0.0 && x21[2] == 0.0))
    pp_pair(x21, A.mass, A.rsoft, A.nf_cutoff, pow2_cut, inv_cut, fp);
}

// the listed targets (grid-stride), 32 per warp
template <int ZX, int ZV>
__global__ void __launch_bounds__(256, 2) k_pp_walk(const void* __restrict__ xp_, void* __restrict__ vp_, PPPar Q,
                                                 PPArgs A) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  const TV* vpr = reinterpret_cast<const TV*>(vp_);
  __shared__ uint32_t rip[8][32 * PPL];   // partners per lane (lane-major)
  __shared__ uint8_t ro[8][32 * PPL];     // their coarse offsets
  __shared__ uint8_t ptg[8][32 * PPL];    // lane of each entry of the warp's list
  __shared__ double term[8][3][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t nlist = (int64_t)*(volatile unsigned long long*)&Q.dscal->pp_list;
  const bool pow2_cut = (A.nf_cutoff & (A.nf_cutoff - 1)) == 0;
  const double inv_cut = 1.0 / (double)A.nf_cutoff;
  const int pr = A.pr;
  uint32_t* wrip = rip[warp];
  uint8_t* wro = ro[warp];
  uint8_t* wtg = ptg[warp];
  PPAcc acc;
  for (int64_t base = ((int64_t)blockIdx.x * 8 + warp) * 32; base < nlist; base += (int64_t)gridDim.x * 256) {
    const int64_t k = base + lane;
    const bool valid = k < nlist;
    int64_t ip = 0;
    int32_t nb9[9];
    double x1[3] = {0.0, 0.0, 0.0};
    int n = 0, f = 0;
    if (valid) {
      ip = Q.list_ip[k];
      int64_t X[3], Y[3], Z[3];
      int g[3];
      pp_neighbours(Q.list_cell[k], Q.nt, Q.nnt, X, Y, Z, g);
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        nb9[t] = (int32_t)X[t];
        nb9[3 + t] = (int32_t)Y[t];
        nb9[6 + t] = (int32_t)Z[t];
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) x1[d] = cube_dmul(4.0, cube_xfrac((int32_t)xp[(size_t)d * A.cap + ip], ZX));
      f = Q.pfine[ip];
      n = pp_walk_window(Q, nb9, f, pr, [&](int e, int64_t ip2, int o) {
        if (e < PPL) {
          wrip[lane * PPL + e] = (uint32_t)ip2;
          wro[lane * PPL + e] = (uint8_t)o;
        }
      });
    }
    const bool over = n > PPL;  // this lane evaluates its walk again on its own
    const int nl = over ? 0 : n;
    int inc = nl;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += v;
    }
    const int off = inc - nl;
    const int P = __shfl_sync(0xffffffffu, inc, 31);
    for (int e = 0; e < nl; ++e) wtg[off + e] = (uint8_t)lane;
    __syncwarp();
    double ft[3] = {0.0, 0.0, 0.0};
    for (int cb = 0; cb < P; cb += 32) {
      const int p = cb + lane;
      const int tg = p < P ? wtg[p] : lane;
      const int toff = __shfl_sync(0xffffffffu, off, tg);
      double tx[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) tx[d] = __shfl_sync(0xffffffffu, x1[d], tg);
      if (p < P) {
        const int e = p - toff;
        double fp[3];
        pp_term<ZX>(xp_, A, pow2_cut, inv_cut, tx, (int64_t)wrip[tg * PPL + e], wro[tg * PPL + e], fp);
#pragma unroll
        for (int d = 0; d < 3; ++d) term[warp][d][lane] = fp[d];
      }
      __syncwarp();
      if (nl) {
        const int e0 = max(off, cb), e1 = min(off + nl, cb + 32);
        for (int e = e0; e < e1; ++e)
#pragma unroll
          for (int d = 0; d < 3; ++d) ft[d] = cube_dadd(ft[d], term[warp][d][e - cb]);
      }
      __syncwarp();
    }
    if (over) {
      pp_walk_window(Q, nb9, f, pr, [&](int, int64_t ip2, int o) {
        double fp[3];
        pp_term<ZX>(xp_, A, pow2_cut, inv_cut, x1, ip2, o, fp);
#pragma unroll
        for (int d = 0; d < 3; ++d) ft[d] = cube_dadd(ft[d], fp[d]);
      });
    }
    if (valid) {
      ++acc.n1;
      acc.npair += (unsigned long long)n;
      int vc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) vc[d] = (int)vpr[(size_t)d * A.cap + ip] + A.half_nvbin;
      pp_apply<ZV>(ft, vc, ip, A, vp_, acc);
    }
  }
  pp_flush(acc, Q.dscal);
}

template <int ZX, int ZV>
int launch_pp(cube_ctx* ctx, const cube_scalars* io) {
  if (ctx->nc % PB) {
    ctx->err = "nc must be a multiple of 4 for the PP bricks";
    return CUBE_ERR_PARAM;
  }
  PPArgs A;
  A.pr = ctx->P.pp_range;
  A.nf_cutoff = ctx->P.nf_cutoff;
  A.rsoft = (double)ctx->P.rsoft;
  A.mass = (double)io->mass_p_cdm;
  A.a_mid = (double)io->a_mid;
  A.dt = (double)io->dt;
  A.pi_d = (double)ctx->codec.pi_f;
  A.rcp6 = 1.0 / 6.0;
  A.rcp_pi = 1.0 / A.pi_d;
  A.tab = cube_venc_tab(ctx);
  A.coef = cube_vcoef(&ctx->codec, io->sigma_vi);
  int rc;
  A.dec = cube_vdec_table(ctx, A.coef, &rc);
  if (rc) return rc;
  A.half_nvbin = ctx->nvbin / 2;
  A.codec = ctx->codec;
  A.cap = ctx->cap;
  // re-bin scratch, free outside update_x: per-cell masks in cell_stats, fine cells in
  // pkey, per-brick flags in cursor, and in big_list the (brick, M) pairs of crowded
  // bricks followed by the crowded-brick list
  const int nb = ctx->nc / PB;
  const int nbricks = nb * nb * nb;
  int32_t* spill = ctx->big_list;
  PPPar Q;
  Q.cell_start = ctx->cell_start;
  Q.ncells = ctx->ncells;
  Q.nc = ctx->nc; Q.nt = ctx->nt; Q.nnt = ctx->nnt; Q.nb = nb;
  Q.occ = reinterpret_cast<unsigned long long*>(ctx->cell_stats);
  Q.multi = Q.occ + ctx->ncells;
  Q.pfine = reinterpret_cast<uint8_t*>(ctx->pkey);
  Q.crowded = reinterpret_cast<unsigned int*>(ctx->cursor);
  Q.dense_list = ctx->big_list + 2 * (size_t)nbricks;
  Q.list_ip = ctx->perm;
  Q.list_cell = ctx->tcell;
  Q.dscal = ctx->dscal;
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(Q.crowded, 0, sizeof(unsigned int) * nbricks, ctx->stream));
  const unsigned cblocks = (unsigned)((ctx->ncells + 255) / 256);
  k_pp_masks<ZX><<<cblocks, 256, 0, ctx->stream>>>(ctx->xp, ctx->cap, Q);
  CUBE_LAUNCH_CHECK(ctx);
  k_pp_cells<ZV><<<cblocks, 256, 0, ctx->stream>>>(Q, A, ctx->vp);
  CUBE_LAUNCH_CHECK(ctx);
  k_pp_walk<ZX, ZV><<<(unsigned)(4 * ctx->num_sms), 256, 0, ctx->stream>>>(ctx->xp, ctx->vp, Q, A);
  CUBE_LAUNCH_CHECK(ctx);
  k_pp_crowd_list<<<(unsigned)((nbricks + 255) / 256), 256, 0, ctx->stream>>>(Q, nbricks);
  CUBE_LAUNCH_CHECK(ctx);
  unsigned long long ndense = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&ndense, &ctx->dscal->pp_dense, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (!ndense) return CUBE_OK;
  // bricks whose region holds a crowded cell: one CTA per brick as before
  const size_t smem =
      sizeof(uint16_t) * ((size_t)NFC + 5 * (size_t)PB_CAP + PP_PMAX) + sizeof(double) * 3 * 32 * (PP_THREADS / 32) +
      (size_t)PP_PMAX;
  auto kb = k_pp_brick<ZX, ZV>;
  CUBE_CUDA_TRY(ctx, cube_smem_limit(kb, smem));
  kb<<<(unsigned)ndense, PP_THREADS, smem, ctx->stream>>>(ctx->xp, ctx->vp, ctx->cell_start, ctx->nc, ctx->nt,
                                                          ctx->nnt, A, spill, ctx->dscal, Q.dense_list);
  CUBE_LAUNCH_CHECK(ctx);
  unsigned long long nspill = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&nspill, &ctx->dscal->n_big, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (!nspill) return CUBE_OK;
  // crowded bricks: slot bases, target CTAs and scratch from the (brick, M) list
  const int n = (int)nspill;
  std::vector<int32_t> lst(2 * (size_t)n);
  CUBE_CUDA_TRY(ctx, cudaMemcpy(lst.data(), spill, sizeof(int32_t) * 2 * n, cudaMemcpyDeviceToHost));
  std::vector<int64_t> meta(2 * (size_t)n + 1);  // base[n], chunk0[n+1]
  int64_t slots = 0, chunks = 0;
  for (int b = 0; b < n; ++b) {
    meta[b] = slots;
    meta[n + b] = chunks;
    slots += lst[2 * b + 1];
    chunks += (lst[2 * b + 1] + PP_THREADS - 1) / PP_THREADS;  // targets <= M
  }
  meta[2 * (size_t)n] = chunks;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t b_meta = al(sizeof(int64_t) * meta.size()), b_off = al(sizeof(uint32_t) * (size_t)n * NFC),
               b_fidx = al(4 * (size_t)slots), b_code = al(2 * (size_t)slots), b_sip = al(8 * (size_t)slots),
               b_cell = al((size_t)slots);
  const size_t need = b_meta + b_off + b_fidx + 3 * b_code + b_sip + b_cell;
  if (need > ctx->pp_scratch_bytes) {
    if (ctx->pp_scratch) cudaFree(ctx->pp_scratch);
    ctx->pp_scratch = nullptr;
    ctx->pp_scratch_bytes = 0;
    CUBE_CUDA_TRY(ctx, cudaMalloc(&ctx->pp_scratch, need + need / 4));
    ctx->pp_scratch_bytes = need + need / 4;
  }
  char* p = reinterpret_cast<char*>(ctx->pp_scratch);
  int64_t* dmeta = reinterpret_cast<int64_t*>(p);
  p += b_meta;
  PPCrowd C;
  C.list = spill;
  C.base = dmeta;
  C.chunk0 = dmeta + n;
  C.n = n;
  C.off = reinterpret_cast<uint32_t*>(p); p += b_off;
  C.fidx = reinterpret_cast<uint32_t*>(p); p += b_fidx;
  C.c0 = reinterpret_cast<uint16_t*>(p); p += b_code;
  C.c1 = reinterpret_cast<uint16_t*>(p); p += b_code;
  C.c2 = reinterpret_cast<uint16_t*>(p); p += b_code;
  C.sip = reinterpret_cast<int64_t*>(p); p += b_sip;
  C.scell = reinterpret_cast<uint8_t*>(p);
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dmeta, meta.data(), sizeof(int64_t) * meta.size(), cudaMemcpyHostToDevice,
                                     ctx->stream));
  k_pp_build<ZX><<<n, PP_THREADS, 0, ctx->stream>>>(ctx->xp, ctx->cell_start, ctx->nc, ctx->nt, ctx->nnt, ctx->cap,
                                                     C);
  CUBE_LAUNCH_CHECK(ctx);
  k_pp_crowd<ZX, ZV><<<(unsigned)chunks, PP_THREADS, 0, ctx->stream>>>(ctx->vp, A, C, ctx->dscal);
  CUBE_LAUNCH_CHECK(ctx);
  // the host copy of meta must outlive the asynchronous upload
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return CUBE_OK;
}

}  // namespace

int cube_pp(cube_ctx* ctx, cube_scalars* io) {
  if (ctx->P.pp_range < 0 || ctx->P.pp_range > 4) {
    ctx->err = "pp_range must be in 0..4";
    return CUBE_ERR_PARAM;
  }
  if (!ctx->P.ext_pp_force) {
    ctx->err = "the context was created with PP off";
    return CUBE_ERR_PARAM;
  }
  if (ctx->izipx == 1 && ctx->izipv == 1) return launch_pp<1, 1>(ctx, io);
  if (ctx->izipx == 1 && ctx->izipv == 2) return launch_pp<1, 2>(ctx, io);
  if (ctx->izipx == 2 && ctx->izipv == 1) return launch_pp<2, 1>(ctx, io);
  return launch_pp<2, 2>(ctx, io);
}
