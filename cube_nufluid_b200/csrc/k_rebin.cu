/*
 * k_rebin.cu -- update_x: drift, re-bin by counting sort, re-encode
 * (update_particle.f90:13-259).
 *
 * The reference drifts every particle of a tile plus its ncb-cell buffer,
 * counts the new cells, builds the spine, scatters in its loop order
 * (layer, k, j, i, l) with nlayer = 2*ceiling(dt_mid*vz_max/ncell)+1, and
 * keeps the particles that land in the tile.  Inside a new cell the particles
 * therefore sit in that loop order, and the cell's new mean velocity is an
 * FP32 running sum in the same order.  The GPU reproduces both exactly:
 *
 *   count   : per particle, target cell (computed in the coordinates of the
 *             target tile, as the reference does) and a 32-bit order key
 *             ((layer*nte + k)*nte + j)*nte + i of the source cell in those
 *             coordinates; count per target cell
 *   scan    : cell starts
 *   place   : slot = start + atomic cursor (arbitrary order inside the cell)
 *   sortsum : per target cell, sort its entries by (key, source index) --
 *             the reference order -- then run the FP32 velocity sum in that
 *             order and the division by (n + weight_v); cells with more than
 *             32 particles go to a warp sorter (one warp per cell, many cells
 *             per SM, so the serial sums of different cells overlap), those
 *             beyond 256 to a block-wide sorter in shared memory, those beyond
 *             4096 to one in a global scratch grown on demand
 *   emit    : per particle in the old order (coalesced reads; the sort pass
 *             records each particle's slot), re-encode, move and copy the PID
 *   stats   : per cell |vfield|^2; with the per-slot terms of emit, summed
 *             by the fixed tree
 * Positions move by nint(dt_mid*v/(x_resolution*ncell)) with the integer
 * wrap of the 1- or 2-byte store (update_particle.f90:117).
 */
#include "cube_internal.cuh"

#include <algorithm>
#include <cmath>

namespace {

constexpr int RCELLS = 64;  // cube_cell_item assumes 64-cell groups
constexpr int PMAX = 4096;     // particles per work item of the count and emit passes
constexpr int SMALL = 32;
constexpr int WARP_MAX = 256;  // warp sorter: keys + 3 velocity columns, 8 KB per warp
constexpr int WARP_WARPS = 8;
constexpr int BIG_MAX = 4096;

struct RebinArgs {
  const void* xp; const void* vp; const int32_t* pid;
  const int64_t* cell_start; const float* vfield;
  void* xp2; void* vp2; int32_t* pid2;
  int32_t* cnt2; int64_t* start2; float* vfield2;
  int32_t* tcell; uint32_t* tkey; int32_t* perm; uint32_t* pkey; int32_t* cursor;
  int32_t* big_list; double* stats; int32_t* slot_cell;  // new cell of each slot
  const int64_t* items; int64_t items_max;
  const double* dec; int half_nvbin;  // tan(code)/coef per code (cube_vdec_table)
  cube_codec codec; double coef; VencTab tab;
  double inv_ncell, inv_xstep;  // 1/ncell and 1/(x_resolution*ncell), exact powers of two
  int64_t cap, ncells;
  int nc, nt, nnt, ncb, nte, ncell, nlayer, use_pid;
  float dt_mid;
  DevScal* dscal;
};

__device__ __forceinline__ int floordiv(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

template <int ZX, int ZV>
__device__ __forceinline__ double decode_v(const RebinArgs& A, int64_t ip, int d) {
  typedef typename CodeT<ZV>::T TV;
  const TV* vp = reinterpret_cast<const TV*>(A.vp);
  const int code = (int)vp[(size_t)d * A.cap + ip];
  return __ldg(&A.dec[code + A.half_nvbin]);
}

// Work items of the count and emit passes (and of the kick): a run of at most
// RCELLS cells and a particle range inside it of at most PMAX particles.  Item
// g < ngroups is the 64-cell group g (all of it when it holds at most PMAX
// particles); a crowded group is cut greedily into runs of whole cells, a cell
// beyond PMAX particles into ranges of PMAX, and the items after its first are
// appended after the groups.  A group of cnt > PMAX particles makes at most
// 4 cnt/PMAX items.
__device__ __forceinline__ void put_item(int64_t* items, int64_t items_max, int64_t ngroups, DevScal* dscal, int64_t g,
                                         bool& first, int64_t c0, int64_t ncl, int64_t p0, int64_t p1) {
  int64_t idx = g;
  if (!first) {
    idx = ngroups + (int64_t)atomicAdd(&dscal->n_items, 1ull);
    if (idx >= items_max) {
      cube_dev_error(dscal, CUBE_ERR_CAPACITY, (int)(g & 0x7fffffff));
      return;
    }
  }
  first = false;
  int64_t* it = items + 4 * idx;
  it[0] = c0; it[1] = ncl; it[2] = p0; it[3] = p1;
}

__global__ void k_cell_items(const int64_t* __restrict__ cs, int64_t ncells, int64_t* __restrict__ items,
                             int64_t items_max, DevScal* dscal) {
  const int64_t ngroups = (ncells + RCELLS - 1) / RCELLS;
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const int64_t c0 = g * RCELLS;
  const int64_t ncl = min((int64_t)RCELLS, ncells - c0);
  bool first = true;
  if (cs[c0 + ncl] - cs[c0] <= PMAX) {
    put_item(items, items_max, ngroups, dscal, g, first, c0, ncl, cs[c0], cs[c0 + ncl]);
    return;
  }
  int64_t ic = c0;  // first cell of the open run
  for (int64_t c = c0; c < c0 + ncl; ++c) {
    const int64_t a = cs[c], e = cs[c + 1];
    if (e - a > PMAX) {
      if (c > ic) put_item(items, items_max, ngroups, dscal, g, first, ic, c - ic, cs[ic], a);
      for (int64_t q = a; q < e; q += PMAX)
        put_item(items, items_max, ngroups, dscal, g, first, c, 1, q, min(q + PMAX, e));
      ic = c + 1;
    } else if (e - cs[ic] > PMAX) {  // cell c does not fit the open run (c > ic here)
      put_item(items, items_max, ngroups, dscal, g, first, ic, c - ic, cs[ic], a);
      ic = c;
    }
  }
  if (c0 + ncl > ic) put_item(items, items_max, ngroups, dscal, g, first, ic, c0 + ncl - ic, cs[ic], cs[c0 + ncl]);
}

// item of this block, or false past the last
__device__ __forceinline__ bool get_item(const RebinArgs& A, int64_t& c0, int& ncl, int64_t& p0, int64_t& p1) {
  return cube_cell_item(A.items, A.ncells, A.items_max, A.dscal, c0, ncl, p0, p1);
}

template <int ZX, int ZV>
__global__ void __launch_bounds__(256) k_rebin_count(RebinArgs A) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(A.xp);
  __shared__ int64_t cs[RCELLS + 1];
  __shared__ int cl[RCELLS][3], ctt[RCELLS][3];  // per cell: local coords, tile coords
  int64_t c0, p0, p1;
  int ncl;
  if (!get_item(A, c0, ncl, p0, p1)) return;
  const int nt = A.nt, nnt = A.nnt, ncb = A.ncb, nte = A.nte;
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = A.cell_start[c0 + i];
  for (int i = threadIdx.x; i < ncl; i += blockDim.x) {
    int tb[3];
    cube_cell_coords(c0 + i, nt, nnt, cl[i], tb);
    ctt[i][0] = tb[0] / nt;
    ctt[i][1] = tb[1] / nt;
    ctt[i][2] = tb[2] / nt;
  }
  __syncthreads();
  typedef typename CodeT<ZV>::T TV;
  const TV* vp = reinterpret_cast<const TV*>(A.vp);
  // two particles per thread, their code and cell-mean reads issued together
  for (int64_t ib = p0 + threadIdx.x; ib < p1; ib += 2 * blockDim.x) {
    int lov[2];
    int xcv[2][3];
    double vv[2][3];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int64_t q = ib + u * (int64_t)blockDim.x < p1 ? ib + u * (int64_t)blockDim.x : ib;
      int lo = 0, hi = ncl - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cs[mid] <= q) lo = mid; else hi = mid - 1;
      }
      lov[u] = lo;
      const int64_t c = c0 + lo;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        xcv[u][d] = (int32_t)xp[(size_t)d * A.cap + q];
        vv[u][d] = cube_dadd(__ldg(&A.dec[(int)vp[(size_t)d * A.cap + q] + A.half_nvbin]),
                             (double)__ldg(&A.vfield[(size_t)d * A.ncells + c]));
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int64_t ip = ib + u * (int64_t)blockDim.x;
      if (ip >= p1) continue;
      const int lo = lov[u];
      const int l[3] = {cl[lo][0], cl[lo][1], cl[lo][2]};
      const int t[3] = {ctt[lo][0], ctt[lo][1], ctt[lo][2]};
      int tg[3], src[3];
      bool bad = false;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double fr = cube_xfrac(xcv[u][d], ZX);
        const double v = vv[u][d];
        // /ncell: ncell = 4 (cube_create), and a quotient by a power of two is the product by
        // its reciprocal, bit for bit
        const double dx = cube_dmul(cube_dmul((double)A.dt_mid, v), A.inv_ncell);
        // ig = ceiling(xq + deltax), xq = (i-1) + frac in the coordinates of the tile that keeps it
        int ig = (int)ceil(cube_dadd(cube_dadd((double)l[d], fr), dx));
        int ls = l[d], tt = t[d];
        if (ig < 1 || ig > nt) {
          const int sh = floordiv(ig - 1, nt);
          ls = l[d] - sh * nt;
          tt = ((t[d] + sh) % nnt + nnt) % nnt;
          const int ig2 = (int)ceil(cube_dadd(cube_dadd((double)ls, fr), dx));
          if (ig2 >= 1 && ig2 <= nt) ig = ig2;
          else { ig = ig - sh * nt; atomicAdd(&A.dscal->moved_far, 1ull); }
        }
        if (ls + 1 < 1 - ncb || ls + 1 > nt + ncb) bad = true;
        tg[d] = tt * nt + ig - 1;
        src[d] = ls + ncb;  // 0-based index in the target tile's extended range
      }
      if (bad) {
        cube_dev_error(A.dscal, CUBE_ERR_MOVE, (int)(ip & 0x7fffffff));
        src[0] = min(max(src[0], 0), nte - 1);
        src[1] = min(max(src[1], 0), nte - 1);
        src[2] = min(max(src[2], 0), nte - 1);
      }
      const int64_t tc = cube_cell_of(tg[0], tg[1], tg[2], nt, nnt);
      const uint32_t layer = (uint32_t)(src[2] % A.nlayer);
      const uint32_t key = ((layer * nte + src[2]) * nte + src[1]) * nte + src[0];
      A.tcell[ip] = (int32_t)tc;
      A.tkey[ip] = key;
      atomicAdd(&A.cnt2[tc], 1);
    }
  }
}

__global__ void k_rebin_place(RebinArgs A, int64_t np) {
  for (int64_t ip = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; ip < np; ip += (int64_t)gridDim.x * blockDim.x) {
    const int32_t tc = A.tcell[ip];
    const int64_t slot = A.start2[tc] + atomicAdd(&A.cursor[tc], 1);
    A.perm[slot] = (int32_t)ip;
    A.pkey[slot] = A.tkey[ip];
  }
}

// source cell of an entry from its key and the target cell's tile
__device__ __forceinline__ int64_t src_cell(const RebinArgs& A, uint32_t key, const int tt[3]) {
  const int nte = A.nte, nt = A.nt, nc = A.nc, ncb = A.ncb;
  const int i = key % nte, j = (key / nte) % nte, k = (key / (nte * nte)) % nte;
  const int gx = cube_wrap(tt[0] * nt + i - ncb, nc);
  const int gy = cube_wrap(tt[1] * nt + j - ncb, nc);
  const int gz = cube_wrap(tt[2] * nt + k - ncb, nc);
  return cube_cell_of(gx, gy, gz, nt, A.nnt);
}

__device__ __forceinline__ void cell_tile(const RebinArgs& A, int64_t c, int tt[3]) {
  const int nt3 = A.nt * A.nt * A.nt;
  const int64_t tile = c / nt3;
  tt[0] = (int)(tile % A.nnt);
  tt[1] = (int)((tile / A.nnt) % A.nnt);
  tt[2] = (int)(tile / ((int64_t)A.nnt * A.nnt));
}

// F1: per target cell, sort its entries into the reference order and run the
// cell's FP32 velocity sum in that order (update_particle.f90:74,83-85).
// Crowded cells are listed for the sorter of their size: up to WARP_MAX entries
// at the front of big_list (k_rebin_warp), up to BIG_MAX at its back
// (k_rebin_big), beyond that in cursor, which is free after the place pass
// (k_rebin_huge).
template <int ZX, int ZV>
__global__ void __launch_bounds__(256) k_rebin_sortsum(RebinArgs A) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= A.ncells) return;
  const int n = A.cnt2[c];
  const int64_t s = A.start2[c];
  if (n > SMALL) {
    if (n <= WARP_MAX) {
      const unsigned long long q = atomicAdd(&A.dscal->n_big, 1ull);
      A.big_list[q] = (int32_t)c;
    } else if (n <= BIG_MAX) {
      const unsigned long long q = atomicAdd(&A.dscal->n_mid, 1ull);
      A.big_list[A.ncells - 1 - (int64_t)q] = (int32_t)c;
    } else {
      const unsigned long long q = atomicAdd(&A.dscal->n_huge, 1ull);
      A.cursor[q] = (int32_t)c;
      atomicMax(&A.dscal->max_huge, (unsigned long long)n);
    }
    return;
  }
  // insertion sort of the cell's (key, source) entries, ascending
  for (int i = 1; i < n; ++i) {
    const uint32_t kk = A.pkey[s + i];
    const int32_t pp = A.perm[s + i];
    int j = i - 1;
    while (j >= 0) {
      const uint32_t kj = A.pkey[s + j];
      const int32_t pj = A.perm[s + j];
      if (kj > kk || (kj == kk && pj > pp)) {
        A.pkey[s + j + 1] = kj;
        A.perm[s + j + 1] = pj;
        --j;
      } else break;
    }
    A.pkey[s + j + 1] = kk;
    A.perm[s + j + 1] = pp;
  }
  int tt[3];
  cell_tile(A, c, tt);
  float acc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) acc[d] = (float)cube_dmul((double)A.vfield[(size_t)d * A.ncells + c], 0.1);
  // one entry ahead: the next entry's particle, key and codes are read while this
  // entry is decoded and added (the adds keep their order)
  typedef typename CodeT<ZV>::T TV;
  const TV* vpr = reinterpret_cast<const TV*>(A.vp);
  int64_t ipn = n > 0 ? A.perm[s] : 0;
  uint32_t keyn = n > 0 ? A.pkey[s] : 0u;
  int coden[3] = {0, 0, 0};
  if (n > 0)
#pragma unroll
    for (int d = 0; d < 3; ++d) coden[d] = (int)vpr[(size_t)d * A.cap + ipn];
  for (int r = 0; r < n; ++r) {
    const int64_t ip = ipn;
    const uint32_t key = keyn;
    const int code[3] = {coden[0], coden[1], coden[2]};
    if (r + 1 < n) {
      ipn = A.perm[s + r + 1];
      keyn = A.pkey[s + r + 1];
#pragma unroll
      for (int d = 0; d < 3; ++d) coden[d] = (int)vpr[(size_t)d * A.cap + ipn];
    }
    A.tkey[ip] = (uint32_t)(s + r);  // the particle's slot (tkey is free after the place pass)
    A.slot_cell[s + r] = (int32_t)c;
    const int64_t sc = src_cell(A, key, tt);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = cube_dadd(__ldg(&A.dec[code[d] + A.half_nvbin]), (double)__ldg(&A.vfield[(size_t)d * A.ncells + sc]));
      acc[d] = (float)cube_dadd((double)acc[d], v);
    }
  }
  const double den = cube_dadd((double)n, 0.1);
#pragma unroll
  for (int d = 0; d < 3; ++d) A.vfield2[(size_t)d * A.ncells + c] = (float)cube_ddiv((double)acc[d], den);
}

// acc + x[0] + x[1] + ... + x[n-1] left to right, each partial sum rounded to FP32
// through FP64 (the reference's real(4) accumulation of real(8) terms); the
// loads of eight terms are issued ahead of their adds
__device__ __forceinline__ float ordered_sum(float acc, const double* x, int n) {
  int i = 0;
  for (; i + 8 <= n; i += 8) {
    double t[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) t[u] = x[i + u];
#pragma unroll
    for (int u = 0; u < 8; ++u) acc = (float)cube_dadd((double)acc, t[u]);
  }
  for (; i < n; ++i) acc = (float)cube_dadd((double)acc, x[i]);
  return acc;
}

// ascending bitonic sort of m (a power of two) keys by the whole CTA, in place
// (shared or global memory)
__device__ __forceinline__ void bitonic_block(unsigned long long* sk, int m) {
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = sk[i], bb = sk[ixj];
          const bool up = (i & k) == 0;
          if ((a > bb) == up) { sk[i] = bb; sk[ixj] = a; }
        }
      }
      __syncthreads();
    }
}

// one pass (k, j < T) of the bitonic network on a tile of T keys that starts at
// key `base` (the direction follows the key's global index)
__device__ __forceinline__ void tile_pass(unsigned long long* t, int T, int base, int j, int k) {
  for (int i = threadIdx.x; i < T; i += blockDim.x) {
    const int ixj = i ^ j;
    if (ixj > i) {
      const unsigned long long a = t[i], bb = t[ixj];
      const bool up = ((base + i) & k) == 0;
      if ((a > bb) == up) { t[i] = bb; t[ixj] = a; }
    }
  }
}

// The same sort for m > T keys in global memory with a shared tile of T keys
// (both powers of two): the stages up to T and, in every later stage, the passes
// of stride below T run tile by tile in shared memory; only the passes of stride
// T and above go through global memory, four compare-exchanges per thread in
// flight (their pairs are disjoint, so the loads of a batch precede its stores).
__device__ __forceinline__ void bitonic_tiled(unsigned long long* g, int m, unsigned long long* t, int T) {
  const int nthr = blockDim.x;
  for (int base = 0; base < m; base += T) {
    for (int i = threadIdx.x; i < T; i += nthr) t[i] = g[base + i];
    __syncthreads();
    for (int k = 2; k <= T; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        tile_pass(t, T, base, j, k);
        __syncthreads();
      }
    for (int i = threadIdx.x; i < T; i += nthr) g[base + i] = t[i];
    __syncthreads();
  }
  const int npairs = m >> 1;
  for (int k = 2 * T; k <= m; k <<= 1) {
    for (int j = k >> 1; j >= T; j >>= 1) {
      for (int p0 = threadIdx.x; p0 < npairs; p0 += 4 * nthr) {
        unsigned long long a[4], bb[4];
        int ii[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int p = p0 + u * nthr;
          ii[u] = -1;
          if (p < npairs) {
            const int i = ((p & ~(j - 1)) << 1) | (p & (j - 1));  // bit j of i clear
            ii[u] = i;
            a[u] = g[i];
            bb[u] = g[i | j];
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (ii[u] >= 0) {
            const bool up = (ii[u] & k) == 0;
            if ((a[u] > bb[u]) == up) { g[ii[u]] = bb[u]; g[ii[u] | j] = a[u]; }
          }
      }
      __syncthreads();
    }
    for (int base = 0; base < m; base += T) {
      for (int i = threadIdx.x; i < T; i += nthr) t[i] = g[base + i];
      __syncthreads();
      for (int j = T >> 1; j > 0; j >>= 1) {
        tile_pass(t, T, base, j, k);
        __syncthreads();
      }
      for (int i = threadIdx.x; i < T; i += nthr) g[base + i] = t[i];
      __syncthreads();
    }
  }
}

// one crowded cell by the whole CTA: bitonic sort of (key<<32|source) in sk (m =
// next power of two of n entries; through the shared tile of T keys when sk is in
// global memory and m > T), the sorted order back to the slots, the per-particle
// velocities into sv[d * vstride + i] in parallel, the FP32 sum by one thread per
// component in order.  sk and sv may be shared or global memory.
template <int ZX, int ZV>
__device__ __forceinline__ void sort_sum_cell(const RebinArgs& A, int64_t c, int n, int64_t s, unsigned long long* sk,
                                              double* sv, int vstride, unsigned long long* tile = nullptr, int T = 0,
                                              double* stage = nullptr, int stage_len = 0) {
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    sk[i] = i < n ? (((unsigned long long)A.pkey[s + i] << 32) | (uint32_t)A.perm[s + i]) : ~0ull;
  __syncthreads();
  if (tile && m > T) bitonic_tiled(sk, m, tile, T);
  else bitonic_block(sk, m);
  int tt[3];
  cell_tile(A, c, tt);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const uint32_t key = (uint32_t)(sk[i] >> 32);
    const int32_t ip = (int32_t)(uint32_t)(sk[i] & 0xffffffffu);
    A.pkey[s + i] = key;  // sorted order back to the slots
    A.perm[s + i] = ip;
    A.tkey[ip] = (uint32_t)(s + i);  // the particle's slot
    A.slot_cell[s + i] = (int32_t)c;
    const int64_t sc = src_cell(A, key, tt);
    for (int d = 0; d < 3; ++d)
      sv[(size_t)d * vstride + i] =
          cube_dadd(decode_v<ZX, ZV>(A, ip, d), (double)__ldg(&A.vfield[(size_t)d * A.ncells + sc]));
  }
  __syncthreads();
  const int d = threadIdx.x;
  float acc = 0.f;
  if (d < 3) acc = (float)cube_dmul((double)A.vfield[(size_t)d * A.ncells + c], 0.1);
  if (stage) {
    // sv in global memory: the CTA copies the next chunk of the three columns into
    // shared memory (free after the sort), the three sums read it from there
    const int ch = stage_len / 3;
    for (int j0 = 0; j0 < n; j0 += ch) {
      const int len = min(ch, n - j0);
      for (int i = threadIdx.x; i < 3 * len; i += blockDim.x) {
        const int dd = i / len, k = i - dd * len;
        stage[dd * ch + k] = sv[(size_t)dd * vstride + j0 + k];
      }
      __syncthreads();
      if (d < 3) acc = ordered_sum(acc, stage + d * ch, len);
      __syncthreads();
    }
  } else if (d < 3) {
    acc = ordered_sum(acc, sv + (size_t)d * vstride, n);
  }
  if (d < 3) A.vfield2[(size_t)d * A.ncells + c] = (float)cube_ddiv((double)acc, cube_dadd((double)n, 0.1));
  __syncthreads();
}

// the same for one cell of at most WARP_MAX entries by one warp, in the warp's
// own shared-memory segment (sk: WARP_MAX keys, sv: [3][WARP_MAX] velocities)
template <int ZX, int ZV>
__device__ __forceinline__ void sort_sum_cell_warp(const RebinArgs& A, int64_t c, int n, int64_t s, unsigned long long* sk,
                                   double* sv) {
  const int lane = threadIdx.x & 31;
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = lane; i < m; i += 32)
    sk[i] = i < n ? (((unsigned long long)A.pkey[s + i] << 32) | (uint32_t)A.perm[s + i]) : ~0ull;
  __syncwarp();
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < m; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = sk[i], bb = sk[ixj];
          const bool up = (i & k) == 0;
          if ((a > bb) == up) { sk[i] = bb; sk[ixj] = a; }
        }
      }
      __syncwarp();
    }
  int tt[3];
  cell_tile(A, c, tt);
  for (int i = lane; i < n; i += 32) {
    const uint32_t key = (uint32_t)(sk[i] >> 32);
    const int32_t ip = (int32_t)(uint32_t)(sk[i] & 0xffffffffu);
    A.pkey[s + i] = key;
    A.perm[s + i] = ip;
    A.tkey[ip] = (uint32_t)(s + i);
    A.slot_cell[s + i] = (int32_t)c;
    const int64_t sc = src_cell(A, key, tt);
    for (int d = 0; d < 3; ++d)
      sv[d * WARP_MAX + i] = cube_dadd(decode_v<ZX, ZV>(A, ip, d), (double)__ldg(&A.vfield[(size_t)d * A.ncells + sc]));
  }
  __syncwarp();
  if (lane < 3) {
    const int d = lane;
    const float acc = ordered_sum((float)cube_dmul((double)A.vfield[(size_t)d * A.ncells + c], 0.1),
                                  sv + d * WARP_MAX, n);
    A.vfield2[(size_t)d * A.ncells + c] = (float)cube_ddiv((double)acc, cube_dadd((double)n, 0.1));
  }
  __syncwarp();
}

// F1 for cells of SMALL+1..WARP_MAX entries: one warp per cell
template <int ZX, int ZV>
__global__ void __launch_bounds__(32 * WARP_WARPS) k_rebin_warp(RebinArgs A) {
  extern __shared__ unsigned long long wsm[];
  const int w = threadIdx.x >> 5;
  unsigned long long* sk = wsm + (size_t)w * 4 * WARP_MAX;
  double* sv = reinterpret_cast<double*>(sk + WARP_MAX);
  const unsigned long long nw = A.dscal->n_big;
  const unsigned long long stride = (unsigned long long)gridDim.x * WARP_WARPS;
  for (unsigned long long b = (unsigned long long)blockIdx.x * WARP_WARPS + w; b < nw; b += stride) {
    const int64_t c = A.big_list[b];
    sort_sum_cell_warp<ZX, ZV>(A, c, A.cnt2[c], A.start2[c], sk, sv);
  }
}

// F1 for cells of WARP_MAX+1..BIG_MAX entries: one CTA per cell, keys sorted in
// shared memory (32 KB, so four CTAs share an SM and their serial sums overlap),
// the velocity columns in the CTA's global slot of 3 BIG_MAX doubles; cells are
// taken as CTAs become free
template <int ZX, int ZV>
__global__ void __launch_bounds__(512) k_rebin_big(RebinArgs A, double* __restrict__ scratch) {
  extern __shared__ unsigned long long sk[];
  __shared__ unsigned long long qs;
  double* sv = scratch + (size_t)blockIdx.x * 3 * BIG_MAX;
  const unsigned long long nmid = A.dscal->n_mid;
  while (true) {
    if (threadIdx.x == 0) qs = atomicAdd(&A.dscal->mid_next, 1ull);
    __syncthreads();
    const unsigned long long b = qs;
    __syncthreads();
    if (b >= nmid) break;
    const int64_t c = A.big_list[A.ncells - 1 - (int64_t)b];
    sort_sum_cell<ZX, ZV>(A, c, A.cnt2[c], A.start2[c], sk, sv, BIG_MAX, nullptr, 0, reinterpret_cast<double*>(sk),
                          BIG_MAX);
  }
}

// F1 for cells beyond BIG_MAX: the same in a global scratch slot per CTA
// (slot_u64 = keys for the largest cell padded to a power of two, then its
// velocities)
constexpr int HUGE_TILE = 8192;  // keys per shared tile of the huge-cell sort (64 KB)
template <int ZX, int ZV>
__global__ void __launch_bounds__(1024) k_rebin_huge(RebinArgs A, unsigned long long* __restrict__ scratch,
                                                     size_t slot_u64, int mmax) {
  extern __shared__ unsigned long long tile[];
  __shared__ unsigned long long qs;
  unsigned long long* sk = scratch + (size_t)blockIdx.x * slot_u64;
  double* sv = reinterpret_cast<double*>(sk + mmax);
  const unsigned long long nh = A.dscal->n_huge;
  const int vstride = (int)((slot_u64 - mmax) / 3);
  while (true) {  // cells taken in list order (largest first) as blocks become free
    if (threadIdx.x == 0) qs = atomicAdd(&A.dscal->huge_next, 1ull);
    __syncthreads();
    const unsigned long long q = qs;
    __syncthreads();
    if (q >= nh) break;
    const int64_t c = A.cursor[q];
    sort_sum_cell<ZX, ZV>(A, c, A.cnt2[c], A.start2[c], sk, sv, vstride, tile, HUGE_TILE,
                          reinterpret_cast<double*>(tile), HUGE_TILE);
  }
}

// the huge-cell list in decreasing particle count (bitonic sort of (~n, cell) in
// shared memory), so that the largest cells start first; lists longer than
// HUGE_ORDER stay in arrival order
constexpr int HUGE_ORDER = 4096;
__global__ void __launch_bounds__(1024) k_rebin_huge_order(RebinArgs A) {
  __shared__ unsigned long long h[HUGE_ORDER];
  const int nh = (int)A.dscal->n_huge;
  if (nh < 2 || nh > HUGE_ORDER) return;
  int m = 1;
  while (m < nh) m <<= 1;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    if (i < nh) {
      const int32_t c = A.cursor[i];
      h[i] = ((unsigned long long)(~(uint32_t)A.cnt2[c]) << 32) | (uint32_t)c;
    } else {
      h[i] = ~0ull;
    }
  }
  __syncthreads();
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = h[i], bb = h[ixj];
          const bool up = (i & k) == 0;
          if ((a > bb) == up) { h[i] = bb; h[ixj] = a; }
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < nh; i += blockDim.x) A.cursor[i] = (int32_t)(uint32_t)(h[i] & 0xffffffffu);
}

// F2: one thread per particle in its old storage order (coalesced reads of its
// codes and PID): re-encode, move and copy it to its slot of the new layout (the
// slots of neighbouring particles are close, so the writes gather in L2); the
// statistics terms are formed from the new codes by the tree pass (k_stats_first)
template <int ZX, int ZV>
__global__ void __launch_bounds__(256) k_rebin_emit(RebinArgs A, int64_t np) {
  typedef typename CodeT<ZX>::T TX;
  typedef typename CodeT<ZV>::T TV;
  const TX* xp = reinterpret_cast<const TX*>(A.xp);
  const TV* vp = reinterpret_cast<const TV*>(A.vp);
  TX* xp2 = reinterpret_cast<TX*>(A.xp2);
  TV* vp2 = reinterpret_cast<TV*>(A.vp2);
  __shared__ int64_t cs[RCELLS + 1];
  int64_t c0, p0, p1;
  int ncl;
  if (!get_item(A, c0, ncl, p0, p1)) return;
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = A.cell_start[c0 + i];
  __syncthreads();
  // two particles per thread, their reads issued together (each read depends on one
  // before it at most: slot and new cell, codes, then the decode table and cell means)
  for (int64_t ib = p0 + threadIdx.x; ib < p1; ib += 2 * blockDim.x) {
    int64_t ip[2], sc[2], c[2], slot[2];
    int vc[2][3], xc[2][3];
    int32_t pv[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      ip[u] = ib + u * (int64_t)blockDim.x;
      const int64_t q = ip[u] < p1 ? ip[u] : ib;
      int lo = 0, hi = ncl - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (cs[mid] <= q) lo = mid; else hi = mid - 1;
      }
      sc[u] = c0 + lo;  // the particle's cell before the drift
      c[u] = A.tcell[q];
      slot[u] = A.tkey[q];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        vc[u][d] = (int)vp[(size_t)d * A.cap + q];
        xc[u][d] = (int)xp[(size_t)d * A.cap + q];
      }
      pv[u] = A.use_pid ? A.pid[q] : 0;
    }
    double v[2][3];
    float vfn[2][3];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        v[u][d] = cube_dadd(__ldg(&A.dec[vc[u][d] + A.half_nvbin]), (double)__ldg(&A.vfield[(size_t)d * A.ncells + sc[u]]));
        vfn[u][d] = A.vfield2[(size_t)d * A.ncells + c[u]];
      }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (ip[u] >= p1 || slot[u] >= np) continue;  // past the item, or its cell overflowed the sorter (error reported)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        // /(x_resolution*ncell), a power of two: the product by its reciprocal, bit for bit
        const int64_t mv = cube_nint(cube_dmul(cube_dmul((double)A.dt_mid, v[u][d]), A.inv_xstep));
        xp2[(size_t)d * A.cap + slot[u]] = (TX)cube_wrap_code((int64_t)xc[u][d] + (int32_t)mv, ZX);
        const int code =
            cube_wrap_code(cube_vencode_step(&A.codec, A.tab, cube_dsub(v[u][d], (double)vfn[u][d]), A.coef), ZV);
        vp2[(size_t)d * A.cap + slot[u]] = (TV)code;
      }
      if (A.use_pid) A.pid2[slot[u]] = pv[u];
    }
  }
}

// F3: per cell, |vfield|^2 in FP32 (update_particle.f90:183); the per-particle
// terms are formed and summed by k_stats_first and the fixed tree
__global__ void k_rebin_stats(RebinArgs A) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= A.ncells) return;
  float vfn[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) vfn[d] = A.vfield2[(size_t)d * A.ncells + c];
  const float f2 = cube_fadd(cube_fadd(cube_fmul(vfn[0], vfn[0]), cube_fmul(vfn[1], vfn[1])), cube_fmul(vfn[2], vfn[2]));
  A.stats[c] = (double)f2;
}

template <int ZX, int ZV>
int run_rebin(cube_ctx* ctx, RebinArgs& A) {
  int64_t ni = 0;  // one block per item (blocks past the last item return at once)
  int rc = cube_cell_items(ctx, ctx->cell_start, &ni);
  if (rc) return rc;
  k_rebin_count<ZX, ZV><<<(unsigned)ni, 256, 0, ctx->stream>>>(A);
  CUBE_LAUNCH_CHECK(ctx);
  rc = cube_exclusive_scan(ctx, A.cnt2, ctx->ncells, A.start2);
  if (rc) return rc;
  k_rebin_place<<<1184, 256, 0, ctx->stream>>>(A, ctx->np);
  CUBE_LAUNCH_CHECK(ctx);
  const unsigned cb = (unsigned)((ctx->ncells + 255) / 256);
  k_rebin_sortsum<ZX, ZV><<<cb, 256, 0, ctx->stream>>>(A);
  CUBE_LAUNCH_CHECK(ctx);
  // sizes of the sorters' lists: n_huge, max_huge, n_mid, and n_big
  unsigned long long hv[4] = {0ull, 0ull, 0ull, 0ull};
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(hv, &ctx->dscal->n_huge, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                     ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(hv + 3, &ctx->dscal->n_big, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                     ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->cells_le32 = (hv[0] | hv[2] | hv[3]) == 0ull;
  const size_t wsmem = sizeof(unsigned long long) * 4 * WARP_MAX * WARP_WARPS;
  CUBE_CUDA_TRY(ctx, cube_smem_limit(k_rebin_warp<ZX, ZV>, wsmem));
  k_rebin_warp<ZX, ZV><<<3 * ctx->num_sms, 32 * WARP_WARPS, wsmem, ctx->stream>>>(A);
  CUBE_LAUNCH_CHECK(ctx);
  if (hv[2]) {
    const int nblk = 4 * ctx->num_sms;
    if (!ctx->rebin_mid_scratch)
      CUBE_CUDA_TRY(ctx, cudaMalloc(&ctx->rebin_mid_scratch, sizeof(double) * 3 * BIG_MAX * (size_t)nblk));
    const size_t smem = sizeof(unsigned long long) * BIG_MAX;
    CUBE_CUDA_TRY(ctx, cube_smem_limit(k_rebin_big<ZX, ZV>, smem));
    const int grid = (int)std::min<unsigned long long>(hv[2], (unsigned long long)nblk);
    k_rebin_big<ZX, ZV><<<grid, 512, smem, ctx->stream>>>(A, reinterpret_cast<double*>(ctx->rebin_mid_scratch));
    CUBE_LAUNCH_CHECK(ctx);
  }
  // cells beyond the block sorter: global scratch sized for the largest
  if (hv[0]) {
    // one slot per SM of keys (mmax, a power of two) and three velocity columns
    // of mmax: the scratch is reallocated only when mmax doubles
    int mmax = 1;
    while ((unsigned long long)mmax < hv[1]) mmax <<= 1;
    const size_t slot = 4 * (size_t)mmax;
    const int grid = (int)std::min<unsigned long long>(hv[0], (unsigned long long)ctx->num_sms);
    const size_t need = sizeof(unsigned long long) * slot * ctx->num_sms;
    if (need > ctx->rebin_scratch_bytes) {
      if (ctx->rebin_scratch) cudaFree(ctx->rebin_scratch);
      ctx->rebin_scratch = nullptr;
      ctx->rebin_scratch_bytes = 0;
      CUBE_CUDA_TRY(ctx, cudaMalloc(&ctx->rebin_scratch, need));
      ctx->rebin_scratch_bytes = need;
    }
    k_rebin_huge_order<<<1, 1024, 0, ctx->stream>>>(A);
    CUBE_LAUNCH_CHECK(ctx);
    const size_t tsmem = sizeof(unsigned long long) * HUGE_TILE;
    CUBE_CUDA_TRY(ctx, cube_smem_limit(k_rebin_huge<ZX, ZV>, tsmem));
    k_rebin_huge<ZX, ZV><<<grid, 1024, tsmem, ctx->stream>>>(
        A, reinterpret_cast<unsigned long long*>(ctx->rebin_scratch), slot, mmax);
    CUBE_LAUNCH_CHECK(ctx);
  }
  k_rebin_emit<ZX, ZV><<<(unsigned)ni, 256, 0, ctx->stream>>>(A, ctx->np);
  CUBE_LAUNCH_CHECK(ctx);
  k_rebin_stats<<<cb, 256, 0, ctx->stream>>>(A);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

}  // namespace

int64_t cube_rebin_items_max(int64_t ncells, int64_t cap) {
  return (ncells + RCELLS - 1) / RCELLS + 4 * (cap / PMAX + 1) + 64;
}

int cube_cell_items(cube_ctx* ctx, const int64_t* cell_start, int64_t* blocks) {
  const int64_t ngroups = (ctx->ncells + RCELLS - 1) / RCELLS;
  const int64_t items_max = cube_rebin_items_max(ctx->ncells, ctx->cap);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(&ctx->dscal->n_items, 0, sizeof(unsigned long long), ctx->stream));
  k_cell_items<<<(unsigned)((ngroups + 255) / 256), 256, 0, ctx->stream>>>(cell_start, ctx->ncells, ctx->rebin_items,
                                                                         items_max, ctx->dscal);
  CUBE_LAUNCH_CHECK(ctx);
  *blocks = std::min<int64_t>(items_max, ngroups + 4 * (ctx->np / PMAX + 1));
  return CUBE_OK;
}

int cube_rebin(cube_ctx* ctx, cube_scalars* io) {
  io->dt_mid = (io->dt_old + io->dt) / 2;
  const float q = cube_fdiv(cube_fmul(io->dt_mid, io->vz_max), (float)ctx->ncell);
  const int nlayer = 2 * (int)ceilf(q) + 1;
  io->nlayer = nlayer;
  RebinArgs A;
  A.xp = ctx->xp; A.vp = ctx->vp; A.pid = ctx->pid;
  A.cell_start = ctx->cell_start; A.vfield = ctx->vfield;
  A.xp2 = ctx->xp2; A.vp2 = ctx->vp2; A.pid2 = ctx->pid2;
  A.cnt2 = ctx->rhoc2; A.start2 = ctx->cell_start2; A.vfield2 = ctx->vfield2;
  A.tcell = ctx->tcell; A.tkey = ctx->tkey; A.perm = ctx->perm; A.pkey = ctx->pkey; A.cursor = ctx->cursor;
  A.big_list = ctx->big_list; A.stats = ctx->cell_stats;
  A.items = ctx->rebin_items; A.items_max = cube_rebin_items_max(ctx->ncells, ctx->cap);
  A.slot_cell = reinterpret_cast<int32_t*>(ctx->slot_r2);
  A.half_nvbin = ctx->nvbin / 2;
  A.codec = ctx->codec; A.coef = cube_vcoef(&ctx->codec, io->sigma_vi);
  A.tab = cube_venc_tab(ctx);
  {
    int trc;
    A.dec = cube_vdec_table(ctx, A.coef, &trc);
    if (trc) return trc;
  }
  A.cap = ctx->cap; A.ncells = ctx->ncells;
  A.nc = ctx->nc; A.nt = ctx->nt; A.nnt = ctx->nnt; A.ncb = ctx->ncb; A.nte = ctx->nte; A.ncell = ctx->ncell;
  A.nlayer = nlayer; A.use_pid = ctx->P.use_pid; A.dt_mid = io->dt_mid; A.dscal = ctx->dscal;
  A.inv_ncell = 1.0 / (double)ctx->ncell;
  A.inv_xstep = 1.0 / (ctx->codec.x_resolution * (double)ctx->ncell);
  {
    int e1, e2;  // both divisors must be powers of two for the products to equal the quotients
    if (std::frexp((double)ctx->ncell, &e1) != 0.5 || std::frexp(ctx->codec.x_resolution * ctx->ncell, &e2) != 0.5) {
      ctx->err = "re-bin: ncell and x_resolution*ncell must be powers of two";
      return CUBE_ERR_PARAM;
    }
  }
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->rhoc2, 0, sizeof(int32_t) * ctx->ncells, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->cursor, 0, sizeof(int32_t) * ctx->ncells, ctx->stream));
  int rc;
  if (ctx->izipx == 1 && ctx->izipv == 1) rc = run_rebin<1, 1>(ctx, A);
  else if (ctx->izipx == 1) rc = run_rebin<1, 2>(ctx, A);
  else if (ctx->izipv == 1) rc = run_rebin<2, 1>(ctx, A);
  else rc = run_rebin<2, 2>(ctx, A);
  return rc;
}
