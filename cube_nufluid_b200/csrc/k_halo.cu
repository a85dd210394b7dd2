/*
 * k_halo.cu -- run-time spherical-overdensity halo finder (halofind.f90:18-598)
 * on the device-resident particles, for the whole periodic box of one image.
 *
 * The reference works tile by tile on a buffered fine mesh and keeps halos whose
 * refined centre lies in the tile; here the same steps run once on the global
 * periodic fine mesh (as the PM step does), so every halo is found once:
 *
 *   density  CIC of every particle with nodes at fine-cell centres (pos - 1/2,
 *            halofind.f90:144-177), positions from the exact codes, weights
 *            dx*dy*dz exact in FP64, accumulated as 64-bit fixed point (w * 2^32),
 *            which makes the mesh independent of the summation order;
 *   peaks    nodes that no neighbour of their 3^3 block exceeds and above
 *            den_peak_cutoff = 100 (:179-183); the mesh mass m_mesh summed over the
 *            nodes in order of distance, whole shells of equal distance at a time,
 *            until the mean drops below den_odc once at least 19 nodes are in
 *            (:185-195); kept if m_mesh > min_halo_particles/2 = 50 particle masses
 *            (:197); position by parabolic interpolation (:203-208);
 *   halos    peaks in order of decreasing density (ties by node index), one after
 *            the other, since each tags the particles it takes (:231-421): the
 *            untagged particles within rsearch = min(2 r_proxy, (ncb-1) ncell),
 *            r_proxy = (3 m_mesh/(4 pi den_odc))^(1/3) (:236-238); the centre refined
 *            on a grid 3x finer over the coarse cells within r_proxy (CIC of the
 *            particles within r_proxy, first maximum in Fortran maxloc order, then
 *            parabolic interpolation whose z denominator repeats the k0-1 node as
 *            the reference's does, :341-357); the gathered particles sorted by
 *            distance from it; the radius where the enclosed density first drops
 *            below den_odc, log-interpolated (:385-401); a halo if at least
 *            min_halo_particles = 100 particles lie inside, which are tagged.
 *
 * Properties follow :408-513: mean position and its variance, mean velocity and
 * dispersion, angular momentum and second-moment tensor about the mean position
 * (raw velocities), the redshift-space mean position along the line of sight of
 * the reference's fixed viewer, and the Lagrangian mean position and tensor from
 * the PIDs (PID - 1 = fine-mesh index of the particle's lattice point), in FP64.
 *
 * Where the reference's result depends on its FP32 rounding or is undefined, the
 * choices here are: peak ties in the sort broken by node index; gathered particles
 * at equal distance ordered by storage index; a parabolic denominator of zero at a
 * mesh peak leaves that coordinate at the node centre (the reference divides by
 * zero there and stops on the NaN box); a zero denominator at the refined maximum
 * rejects the peak (the reference's NaN or infinite centre yields i_odc < 100);
 * the moment accumulators start from zero for every halo (the reference never
 * resets its inertia, dx_mean and q-space sums).
 *
 * A candidate is processed by one CTA, which parallelises its gather, refined grid,
 * sort and sums.  Candidates are independent when their search balls do not meet
 * (a candidate only gathers, and tags, untagged particles within its rsearch of its
 * peak), so the host groups them into waves: a candidate goes one wave after the
 * latest earlier candidate whose ball meets its own, and each wave runs as one
 * launch of many CTAs, each with its own scratch slot.  A candidate a slot cannot
 * hold (more particles or a larger refined grid) is left untouched and runs after
 * its wave in a single CTA with the full-size scratch.  The result is the sequential
 * one: halo numbers, records and member lists are assembled in candidate order at
 * the end.  Distances and centres use explicitly rounded FP64 operations so that
 * the CPU restatement reproduces them bit for bit.
 */
#include "cube_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

constexpr double HFIX = 4294967296.0;  // 2^32
constexpr int H_THREADS = 1024;
constexpr int NB_MAX = 300;             // refined cells per dimension (newbox_max, :26)
constexpr int64_t GCAP = 1 << 22;       // particles gathered per halo (max_halo_np = 3.6M, :29)
constexpr int CAND_CAP = 1 << 21;       // density peaks
constexpr int RMAX = 64;                // radius of the shell list in fine cells
constexpr int MIN_NP = 100;             // min_halo_particles (:37)
constexpr int W_THREADS = 256;          // threads of a wave CTA
constexpr int W_GCAP = 1 << 16;         // particles a wave slot gathers
constexpr int W_NB = 72;                // refined cells per dimension a wave slot holds

struct HaloCand {
  int64_t node;             // fine node index (x fastest)
  unsigned long long acc;   // density at the node, fixed point
  double mass;              // m_mesh
  double pos[3];            // peak position, fine units
  double rp;                // r_proxy, filled in by the host after the sort
};

__device__ __forceinline__ double pmod(double a, double p) {  // Fortran modulo for reals
  return __dsub_rn(a, __dmul_rn(floor(__ddiv_rn(a, p)), p));
}

template <int ZX>
__device__ __forceinline__ double h_pos(const void* xp_, int64_t cap, int64_t ip, int d, int gcell) {
  typedef typename CodeT<ZX>::T TX;
  const TX* xp = reinterpret_cast<const TX*>(xp_);
  return 4.0 * ((double)gcell + cube_xfrac((int32_t)xp[(size_t)d * cap + ip], ZX));
}

// fine density with nodes at cell centres, fixed point, unit mass per particle
template <int ZX>
__global__ void __launch_bounds__(256) k_halo_density(const void* __restrict__ xp, const int64_t* __restrict__ cell_start,
                                                      int64_t cap, int64_t ncells, int nt, int nnt, int nf,
                                                      unsigned long long* __restrict__ acc) {
  constexpr int HC = 64;
  __shared__ int64_t cs[HC + 1];
  __shared__ int cg[HC][3];
  const int64_t c0 = (int64_t)blockIdx.x * HC;
  const int ncl = (int)min((int64_t)HC, ncells - c0);
  for (int i = threadIdx.x; i <= ncl; i += blockDim.x) cs[i] = cell_start[c0 + i];
  if (threadIdx.x < ncl) {
    int l[3], tb[3];
    cube_cell_coords(c0 + threadIdx.x, nt, nnt, l, tb);
    for (int d = 0; d < 3; ++d) cg[threadIdx.x][d] = tb[d] + l[d];
  }
  __syncthreads();
  for (int64_t ip = cs[0] + threadIdx.x; ip < cs[ncl]; ip += blockDim.x) {
    int lo = 0, hi = ncl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cs[mid] <= ip) lo = mid; else hi = mid - 1;
    }
    int i1[3];
    double w1[3], w2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double p = h_pos<ZX>(xp, cap, ip, d, cg[lo][d]) - 0.5;
      const double f = floor(p);
      w1[d] = (f + 1.0) - p;  // exact
      w2[d] = 1.0 - w1[d];
      i1[d] = (int)f;
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
      const double w = __dmul_rn(__dmul_rn(ox ? w2[0] : w1[0], oy ? w2[1] : w1[1]), oz ? w2[2] : w1[2]);  // exact
      const int gx = cube_wrap(i1[0] + ox, nf), gy = cube_wrap(i1[1] + oy, nf), gz = cube_wrap(i1[2] + oz, nf);
      atomicAdd(&acc[((size_t)gz * nf + gy) * nf + gx], (unsigned long long)__double2ll_rn(w * HFIX));
    }
  }
}

// parabolic offset 0.5 (p - m) / den from fixed-point values (exact differences)
__device__ __forceinline__ double parab(long long m, long long p, long long den) {
  return __ddiv_rn(0.5 * (double)(p - m), (double)den);
}

// local maxima above the cutoff, their mesh mass and parabolic position
__global__ void __launch_bounds__(256) k_halo_peaks(const unsigned long long* __restrict__ acc, int nf, double mass,
                                                    double den_odc, const int4* __restrict__ shells, int nshell,
                                                    HaloCand* __restrict__ cand, unsigned int* __restrict__ ncand) {
  const int64_t n3 = (int64_t)nf * nf * nf;
  const double unit = mass / HFIX;
  for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n3; n += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long a0 = acc[n];
    if (!((double)a0 * unit > 100.0)) continue;  // den_peak_cutoff
    const int x = (int)(n % nf), y = (int)((n / nf) % nf), z = (int)(n / ((int64_t)nf * nf));
    // offsets in (-nf, nf]: the wrapped index stays in [-nf, 2nf)
    auto at = [&](int dx, int dy, int dz) -> long long {
      return (long long)acc[((size_t)cube_wrap(z + dz, nf) * nf + cube_wrap(y + dy, nf)) * nf + cube_wrap(x + dx, nf)];
    };
    bool peak = true;
    for (int dz = -1; dz <= 1 && peak; ++dz)
      for (int dy = -1; dy <= 1 && peak; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
          if ((unsigned long long)at(dx, dy, dz) > a0) { peak = false; break; }
    if (!peak) continue;
    unsigned long long m = 0;
    for (int i = 0; i < nshell; ++i) {
      const int4 o = shells[i];
      m += (unsigned long long)at(o.x % nf, o.y % nf, o.z % nf);
      if (i + 1 < nshell && shells[i + 1].w == o.w) continue;  // complete the shell
      if (i + 1 >= 19 && (double)m * unit / (double)(i + 1) < den_odc) break;
    }
    const double mm = (double)m * unit;
    if (!(mm > mass * 50.0)) continue;
    HaloCand h;
    h.node = n;
    h.acc = a0;
    h.mass = mm;
    h.rp = 0.0;
    const int c[3] = {x, y, z};
    const long long a = (long long)a0;
    for (int d = 0; d < 3; ++d) {
      const int e0 = d == 0, e1 = d == 1, e2 = d == 2;
      const long long am = at(-e0, -e1, -e2), ap = at(e0, e1, e2);
      const long long den = 2 * a - am - ap;
      h.pos[d] = ((double)c[d] + 0.5) + (den != 0 ? parab(am, ap, den) : 0.0);
    }
    const unsigned int q = atomicAdd(ncand, 1u);
    if (q < (unsigned)CAND_CAP) cand[q] = h;
  }
}

// per-candidate result, assembled into the outputs in candidate order at the end
struct HaloRec {
  int is_halo;
  int iodc;              // particles in the halo
  long long moff;        // first of its member PIDs in the unordered member buffer
  cube_halo H;
};

struct HaloArgs {
  const void* xp; const void* vp; const int32_t* pid; const int64_t* cell_start; const float* vfield;
  const double* dec;         // decoded velocity per code at sigma_vi, index code + nvbin/2
  int half_nvbin, use_pid;
  int64_t cap, ncells;
  int nc, nt, nnt, nf, ncb, ncell, cmax;
  double mass, den_odc, pi;  // particle mass; threshold; the reference's FP32 pi
  double vsim2phys, a, h0, box;
  const HaloCand* cand;
  uint8_t* tag;              // per particle (storage index)
  HaloRec* rec;              // per candidate
  int32_t* mtmp;             // member PIDs, unordered by candidate
  long long* mcount;         // next free entry of mtmp
  long long mcap;
  int* err;                  // 2: refined grid beyond 300, 3: gather beyond GCAP, 4: box wraps
  int* overflow;             // candidates a slot could not hold (wave kernel): [0] count, then indices
};

// scratch of one CTA: gathered particles (capacity gcap) and the refined grid
struct HaloSlot {
  double* gx; double* gv;    // [3][gcap]
  int64_t* gip;
  double* key;
  int32_t* ord;
  unsigned long long* grid;  // (nbmax + 3)^3
  int gcap, nbmax;
};

struct HaloShared {
  double hpos[3], rp, rs;
  int flo[3], nbx[3], mx[3], clo[3], cn[3];
  unsigned int cnt;
  unsigned long long best;
  int bidx, iodc, skip;
  long long ws[32];
  double red[33];
};

__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

// exclusive block scan of one int64 per thread; *total gets the sum
__device__ long long block_scan(long long v, long long* ws, long long* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) ws[w] = x;
  __syncthreads();
  if (w == 0) {
    long long s = lane < nw ? ws[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  const long long ex = x - v + (w ? ws[w - 1] : 0);
  *total = ws[nw - 1];
  return ex;
}

__device__ __forceinline__ double dist3(const double a[3], const double b[3]) {
  const double d0 = __dsub_rn(a[0], b[0]), d1 = __dsub_rn(a[1], b[1]), d2 = __dsub_rn(a[2], b[2]);
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(d0, d0), __dmul_rn(d1, d1)), __dmul_rn(d2, d2)));
}

__device__ __forceinline__ void search_cell(const int clo[3], const int cn[3], int q, int nc, int nt, int nnt,
                                            int cu[3], int64_t* c) {
  cu[0] = clo[0] + q % cn[0];
  cu[1] = clo[1] + (q / cn[0]) % cn[1];
  cu[2] = clo[2] + q / (cn[0] * cn[1]);
  *c = cube_cell_of(cube_wrap(cu[0] % nc, nc), cube_wrap(cu[1] % nc, nc), cube_wrap(cu[2] % nc, nc), nt, nnt);
}

// One candidate by the whole CTA (halofind.f90:231-513).  Returns 0 when done (halo or
// not), 1 when the slot cannot hold it (nothing written, no particle tagged), and a
// negative error code.  Every thread returns the same value.
template <int ZX, int ZV>
__device__ int halo_candidate(const HaloArgs& A, int ic, const HaloSlot& S, HaloShared& sh, long long* s_first,
                              long long* s_pref) {
  typedef typename CodeT<ZV>::T TV;
  const TV* vp = reinterpret_cast<const TV*>(A.vp);
  const int nf = A.nf, nc = A.nc, ncell = A.ncell;
  const double ng = 1.0 / 3.0, half_ng = 0.5 / 3.0;
  __syncthreads();  // the previous candidate's shared values are consumed
  if (threadIdx.x == 0) {
    const HaloCand& h = A.cand[ic];
    for (int d = 0; d < 3; ++d) sh.hpos[d] = h.pos[d];
    const double rp = h.rp;
    const double rs = fmin(2.0 * rp, (double)((A.ncb - 1) * ncell));
    sh.rp = rp;
    sh.rs = rs;
    int bad = 0;
    for (int d = 0; d < 3; ++d) {
      sh.clo[d] = (int)floor((sh.hpos[d] - rs) / ncell);
      sh.cn[d] = (int)floor((sh.hpos[d] + rs) / ncell) - sh.clo[d] + 1;
      const int rlo = (int)floor((sh.hpos[d] - rp) / ncell), rhi = (int)floor((sh.hpos[d] + rp) / ncell);
      sh.flo[d] = ncell * rlo;
      sh.nbx[d] = 3 * ncell * (rhi - rlo + 1);
      sh.mx[d] = min(sh.nbx[d] + 1, NB_MAX);
      if (sh.nbx[d] > NB_MAX) bad = -2;
      else if (sh.nbx[d] > S.nbmax && !bad) bad = 1;
      if (sh.cn[d] > nc) bad = -4;
    }
    if (!bad && sh.cn[0] * sh.cn[1] * sh.cn[2] > A.cmax) bad = -4;
    sh.cnt = 0;
    sh.best = 0ull;
    sh.bidx = 0x7fffffff;
    sh.iodc = 0x7fffffff;
    sh.skip = bad;
  }
  __syncthreads();
  if (sh.skip) return sh.skip;
  const int gxn = sh.nbx[0] + 3, gyn = sh.nbx[1] + 3, gzn = sh.nbx[2] + 3;
  const int64_t gtot = (int64_t)gxn * gyn * gzn;
  for (int64_t i = threadIdx.x; i < gtot; i += blockDim.x) S.grid[i] = 0ull;
  // cells of the search box: first particle and count prefix
  const int ncl = sh.cn[0] * sh.cn[1] * sh.cn[2];
  const int per = (ncl + blockDim.x - 1) / blockDim.x;
  const int q0 = min(ncl, (int)threadIdx.x * per), q1 = min(ncl, q0 + per);
  long long mine = 0;
  for (int q = q0; q < q1; ++q) {
    int cu[3];
    int64_t c;
    search_cell(sh.clo, sh.cn, q, nc, A.nt, A.nnt, cu, &c);
    s_first[q] = A.cell_start[c];
    mine += A.cell_start[c + 1] - A.cell_start[c];
  }
  long long tot;
  long long run = block_scan(mine, sh.ws, &tot);
  for (int q = q0; q < q1; ++q) {
    int cu[3];
    int64_t c;
    search_cell(sh.clo, sh.cn, q, nc, A.nt, A.nnt, cu, &c);
    s_pref[q] = run;
    run += A.cell_start[c + 1] - A.cell_start[c];
  }
  __syncthreads();
  // gather the untagged particles within rsearch; CIC of those within r_proxy
  const double rs = sh.rs, rpx = sh.rp;
  const double hp[3] = {sh.hpos[0], sh.hpos[1], sh.hpos[2]};
  const int flo[3] = {sh.flo[0], sh.flo[1], sh.flo[2]};
  const int gcap = S.gcap;
  for (long long t = threadIdx.x; t < tot; t += blockDim.x) {
    int lo = 0, hi = ncl - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (s_pref[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int64_t ip = s_first[lo] + (t - s_pref[lo]);
    if (A.tag[ip]) continue;
    int cu[3];
    int64_t c;
    search_cell(sh.clo, sh.cn, lo, nc, A.nt, A.nnt, cu, &c);
    double x[3];
    for (int d = 0; d < 3; ++d) x[d] = h_pos<ZX>(A.xp, A.cap, ip, d, cu[d]);  // unwrapped next to the peak
    const double r = dist3(x, hp);
    if (!(r < rs)) continue;
    const unsigned int s = atomicAdd(&sh.cnt, 1u);
    if (s < (unsigned)gcap) {
      for (int d = 0; d < 3; ++d) {
        S.gx[(size_t)d * gcap + s] = x[d];
        const int code = (int)vp[(size_t)d * A.cap + ip];
        S.gv[(size_t)d * gcap + s] = __dadd_rn(A.dec[code + A.half_nvbin], (double)A.vfield[(size_t)d * A.ncells + c]);
      }
      S.gip[s] = ip;
    }
    if (r < rpx) {  // nodes at refined-cell centres, 1-based refined index
      int i1[3];
      double w1[3], w2[3];
      for (int d = 0; d < 3; ++d) {
        const double p = __ddiv_rn(__dsub_rn(__dsub_rn(x[d], half_ng), (double)flo[d]), ng);
        const double f = floor(p);
        w1[d] = (f + 1.0) - p;
        w2[d] = 1.0 - w1[d];
        i1[d] = (int)f + 1;
      }
      for (int cc = 0; cc < 8; ++cc) {
        const int ox = cc & 1, oy = (cc >> 1) & 1, oz = cc >> 2;
        const int ix = i1[0] + ox, iy = i1[1] + oy, iz = i1[2] + oz;
        if (ix < 0 || iy < 0 || iz < 0 || ix >= gxn || iy >= gyn || iz >= gzn) continue;
        const double w = __dmul_rn(__dmul_rn(ox ? w2[0] : w1[0], oy ? w2[1] : w1[1]), oz ? w2[2] : w1[2]);
        atomicAdd(&S.grid[((size_t)iz * gyn + iy) * gxn + ix], (unsigned long long)__double2ll_rn(w * HFIX));
      }
    }
  }
  __syncthreads();
  const unsigned int nraw = sh.cnt;
  if (nraw > (unsigned)gcap) return gcap < GCAP ? 1 : -3;
  const int n = (int)nraw;
  // refined maximum: the first one in x-fastest order over nodes 1..min(nb+1, 300)
  unsigned long long bv = 0ull;
  int bi = 0x7fffffff;
  const int mx0 = sh.mx[0], mx1 = sh.mx[1], mx2 = sh.mx[2];
  const int64_t inner = (int64_t)mx0 * mx1 * mx2;
  for (int64_t i = threadIdx.x; i < inner; i += blockDim.x) {
    const int ix = (int)(i % mx0) + 1, iy = (int)((i / mx0) % mx1) + 1, iz = (int)(i / ((int64_t)mx0 * mx1)) + 1;
    const unsigned long long v = S.grid[((size_t)iz * gyn + iy) * gxn + ix];
    if (v > bv || (v == bv && (int)i < bi)) { bv = v; bi = (int)i; }
  }
  atomicMax(&sh.best, bv);
  __syncthreads();
  if (bv == sh.best) atomicMin(&sh.bidx, bi);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int i = sh.bidx;
    const int i0 = i % mx0 + 1, j0 = (i / mx0) % mx1 + 1, k0 = i / (mx0 * mx1) + 1;
    auto g = [&](int a, int b, int c) { return (long long)S.grid[((size_t)c * gyn + b) * gxn + a]; };
    const long long g0 = g(i0, j0, k0);
    const long long dxn = 2 * g0 - g(i0 - 1, j0, k0) - g(i0 + 1, j0, k0);
    const long long dyn = 2 * g0 - g(i0, j0 - 1, k0) - g(i0, j0 + 1, k0);
    const long long dzn = 2 * g0 - g(i0, j0, k0 - 1) - g(i0, j0, k0 - 1);  // the reference's z denominator
    if (dxn == 0 || dyn == 0 || dzn == 0) {
      sh.skip = 2;
    } else {
      const double hr[3] = {(i0 - 0.5) + parab(g(i0 - 1, j0, k0), g(i0 + 1, j0, k0), dxn),
                            (j0 - 0.5) + parab(g(i0, j0 - 1, k0), g(i0, j0 + 1, k0), dyn),
                            (k0 - 0.5) + parab(g(i0, j0, k0 - 1), g(i0, j0, k0 + 1), dzn)};
      for (int d = 0; d < 3; ++d) sh.hpos[d] = __dadd_rn((double)flo[d], __dmul_rn(ng, hr[d]));
    }
  }
  __syncthreads();
  if (sh.skip) return 0;  // a zero denominator: not a halo
  // distances from the refined centre; sort by (distance, storage index)
  const double hc[3] = {sh.hpos[0], sh.hpos[1], sh.hpos[2]};
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  for (int i = threadIdx.x; i < np2; i += blockDim.x) {
    if (i < n) {
      const double x[3] = {S.gx[i], S.gx[(size_t)gcap + i], S.gx[2 * (size_t)gcap + i]};
      S.key[i] = dist3(x, hc);
    }
    S.ord[i] = i;
  }
  __syncthreads();
  for (int k = 2; k <= np2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < np2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const int a = S.ord[i], b = S.ord[l];
          bool gt;
          if (a >= n || b >= n) {
            gt = a >= n && (b < n || a > b);  // padding sorts last
          } else {
            const double ka = S.key[a], kb = S.key[b];
            gt = ka > kb || (ka == kb && S.gip[a] > S.gip[b]);
          }
          if (gt == ((i & k) == 0)) { S.ord[i] = b; S.ord[l] = a; }
        }
      }
      __syncthreads();
    }
  // i_odc: the first ii >= 2 (1-based) whose enclosed density is below den_odc
  const double c43 = 0.75 / A.pi;
  for (int ii = threadIdx.x + 2; ii <= n; ii += blockDim.x) {
    const double r = S.key[S.ord[ii - 1]];
    if (c43 * ii * A.mass / (r * r * r) < A.den_odc) atomicMin(&sh.iodc, ii);
  }
  __syncthreads();
  const int iis = sh.iodc;
  const int iodc = iis == 0x7fffffff ? 0 : iis - 1;
  if (iodc < MIN_NP) return 0;
  // a halo: tag its particles, record its PIDs
  __shared__ long long s_moff;
  if (threadIdx.x == 0)
    s_moff = A.use_pid ? (long long)atomicAdd(reinterpret_cast<unsigned long long*>(A.mcount),
                                              (unsigned long long)iodc)
                       : 0;
  __syncthreads();
  const long long moff = s_moff;
  for (int i = threadIdx.x; i < iodc; i += blockDim.x) {
    const int64_t ip = S.gip[S.ord[i]];
    A.tag[ip] = 1;
    if (A.use_pid && moff + i < A.mcap) A.mtmp[moff + i] = A.pid[ip];
  }
  double xm[3], vm[3], xl[3] = {0, 0, 0}, vl[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < iodc; i += blockDim.x) {
    const int o = S.ord[i];
    for (int d = 0; d < 3; ++d) {
      xl[d] += S.gx[(size_t)d * gcap + o];
      vl[d] += S.gv[(size_t)d * gcap + o];
    }
  }
  for (int d = 0; d < 3; ++d) xm[d] = block_sum(xl[d], sh.red) / iodc;
  for (int d = 0; d < 3; ++d) vm[d] = block_sum(vl[d], sh.red) / iodc;
  double xw[3];
  for (int d = 0; d < 3; ++d) xw[d] = pmod(xm[d], (double)nf);
  // second moments about the means; Lagrangian offsets from the wrapped mean
  double sxx[3] = {0, 0, 0}, svv = 0, am[3] = {0, 0, 0}, in[6] = {0, 0, 0, 0, 0, 0}, dq[3] = {0, 0, 0}, nq = 0;
  const long long nfl = nf;
  const double hnf = (double)(nf / 2);
  for (int i = threadIdx.x; i < iodc; i += blockDim.x) {
    const int o = S.ord[i];
    double dx[3], v[3];
    for (int d = 0; d < 3; ++d) {
      dx[d] = S.gx[(size_t)d * gcap + o] - xm[d];
      v[d] = S.gv[(size_t)d * gcap + o];
      sxx[d] += dx[d] * dx[d];
      svv += (v[d] - vm[d]) * (v[d] - vm[d]);
    }
    am[0] += dx[1] * v[2] - dx[2] * v[1];
    am[1] += dx[2] * v[0] - dx[0] * v[2];
    am[2] += dx[0] * v[1] - dx[1] * v[0];
    in[0] += dx[0] * dx[0]; in[1] += dx[1] * dx[1]; in[2] += dx[2] * dx[2];
    in[3] += dx[0] * dx[1]; in[4] += dx[1] * dx[2]; in[5] += dx[2] * dx[0];
    if (A.use_pid) {
      const long long qt = (long long)A.pid[S.gip[o]] - 1;
      if (qt >= 0) {
        const long long qz = qt / (nfl * nfl), qy = (qt - qz * nfl * nfl) / nfl, qx = qt % nfl;
        const double qp[3] = {qx + 0.5, qy + 0.5, qz + 0.5};
        for (int d = 0; d < 3; ++d) dq[d] += pmod(__dadd_rn(__dsub_rn(qp[d], xw[d]), hnf), (double)nf) - hnf;
        nq += 1.0;
      }
    }
  }
  for (int d = 0; d < 3; ++d) sxx[d] = block_sum(sxx[d], sh.red);
  svv = block_sum(svv, sh.red);
  for (int d = 0; d < 3; ++d) am[d] = block_sum(am[d], sh.red);
  for (int q = 0; q < 6; ++q) in[q] = block_sum(in[q], sh.red);
  for (int d = 0; d < 3; ++d) dq[d] = block_sum(dq[d], sh.red);
  nq = block_sum(nq, sh.red);
  double qm[3] = {0, 0, 0}, iq[6] = {0, 0, 0, 0, 0, 0};
  if (A.use_pid && nq > 0) {
    for (int d = 0; d < 3; ++d) qm[d] = pmod(xw[d] + dq[d] / nq, (double)nf);
    for (int i = threadIdx.x; i < iodc; i += blockDim.x) {
      const long long qt = (long long)A.pid[S.gip[S.ord[i]]] - 1;
      if (qt < 0) continue;
      const long long qz = qt / (nfl * nfl), qy = (qt - qz * nfl * nfl) / nfl, qx = qt % nfl;
      const double qp[3] = {qx + 0.5, qy + 0.5, qz + 0.5};
      double e[3];
      for (int d = 0; d < 3; ++d)  // the reference adds 1/2 once more here
        e[d] = pmod(__dadd_rn(__dsub_rn(__dadd_rn(qp[d], 0.5), qm[d]), hnf), (double)nf) - hnf;
      iq[0] += e[0] * e[0]; iq[1] += e[1] * e[1]; iq[2] += e[2] * e[2];
      iq[3] += e[0] * e[1]; iq[4] += e[1] * e[2]; iq[5] += e[2] * e[0];
    }
    for (int q = 0; q < 6; ++q) iq[q] = block_sum(iq[q], sh.red);
  }
  if (threadIdx.x == 0) {
    HaloRec& R = A.rec[ic];
    cube_halo& H = R.H;
    for (int d = 0; d < 3; ++d) H.hpos[d] = (float)pmod(sh.hpos[d], (double)nf);
    H.mass_odc = (float)iodc;
    {
      const double r2 = S.key[S.ord[iis - 1]], r1 = S.key[S.ord[iis - 2]];
      const double den2 = c43 * iis * A.mass / (r2 * r2 * r2), den1 = c43 * (iis - 1) * A.mass / (r1 * r1 * r1);
      const double lr2 = log10(r2), lr1 = log10(r1), d2 = log10(den2), d1 = log10(den1), lo = log10(A.den_odc);
      H.radius_odc = (float)pow(10.0, ((lo - d2) * lr1 + (d1 - lo) * lr2) / (d1 - d2));
    }
    H.v_disp = (float)sqrt(svv / (iodc - 1));
    for (int d = 0; d < 3; ++d) {
      H.x_mean[d] = (float)xw[d];
      H.v_mean[d] = (float)vm[d];
      H.var_x[d] = (float)(sxx[d] / (iodc - 1));
      H.ang_mom[d] = (float)am[d];
      H.q_mean[d] = (float)qm[d];
    }
    const int sym[9] = {0, 3, 5, 3, 1, 4, 5, 4, 2};  // (3,3) column-major from xx,yy,zz,xy,yz,zx
    for (int k = 0; k < 9; ++k) {
      H.inertia[k] = (float)in[sym[k]];
      H.inertia_q[k] = (float)iq[sym[k]];
    }
    // redshift-space mean position along the line of sight (:425-430)
    double los[3], ln = 0.0, vlos = 0.0;
    const double cen[3] = {30.0, 370.0, 370.0};
    for (int d = 0; d < 3; ++d) {
      los[d] = xw[d] - cen[d] / 500.0 * (double)nc;
      ln += los[d] * los[d];
    }
    ln = sqrt(ln);
    for (int d = 0; d < 3; ++d) {
      los[d] /= ln;
      vlos += vm[d] * los[d];
    }
    for (int d = 0; d < 3; ++d) {
      const double sx = vlos * los[d] * A.vsim2phys / A.a / (100.0 * A.h0) / (A.h0 * A.box / nf);
      H.s_mean[d] = (float)pmod(xw[d] + sx, (double)nf);
    }
    R.iodc = iodc;
    R.moff = moff;
    R.is_halo = 1;
  }
  return 0;
}

// candidates list[0..n) one after the other in one CTA (large ones, or every one)
template <int ZX, int ZV>
__global__ void __launch_bounds__(H_THREADS) k_halo_seq(HaloArgs A, const int* __restrict__ list, int n, HaloSlot S) {
  extern __shared__ long long hsm[];
  __shared__ HaloShared sh;
  for (int i = 0; i < n; ++i) {
    const int rc = halo_candidate<ZX, ZV>(A, list[i], S, sh, hsm, hsm + A.cmax);
    if (rc < 0) {
      if (threadIdx.x == 0) atomicCAS(A.err, 0, -rc);
      return;
    }
  }
}

// one wave of mutually independent candidates: CTA b takes list[b], list[b + grid], ...
// with its own slot; candidates a slot cannot hold go to the overflow list untouched
template <int ZX, int ZV>
__global__ void __launch_bounds__(W_THREADS) k_halo_wave(HaloArgs A, const int* __restrict__ list, int n,
                                                         HaloSlot S0, size_t gstride, size_t grid_stride) {
  extern __shared__ long long hsm[];
  __shared__ HaloShared sh;
  HaloSlot S = S0;
  S.gx += (size_t)blockIdx.x * 3 * gstride;
  S.gv += (size_t)blockIdx.x * 3 * gstride;
  S.gip += (size_t)blockIdx.x * gstride;
  S.key += (size_t)blockIdx.x * gstride;
  S.ord += (size_t)blockIdx.x * gstride;
  S.grid += (size_t)blockIdx.x * grid_stride;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int rc = halo_candidate<ZX, ZV>(A, list[i], S, sh, hsm, hsm + A.cmax);
    if (rc < 0) {
      if (threadIdx.x == 0) atomicCAS(A.err, 0, -rc);
      return;
    }
    if (rc == 1 && threadIdx.x == 0) A.overflow[1 + atomicAdd(A.overflow, 1)] = list[i];
  }
}

__global__ void k_halo_flags(const HaloRec* __restrict__ rec, int n, int2* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_int2(rec[i].is_halo, rec[i].iodc);
}

// the outputs in candidate order: halo number k+1 for the k-th halo, its record,
// its member PIDs at the running offset, hid per member PID
__global__ void k_halo_emit(const HaloRec* __restrict__ rec, const int* __restrict__ hnum,
                            const long long* __restrict__ foff, const int* __restrict__ halo_ids, int nh,
                            const int32_t* __restrict__ mtmp, cube_halo* __restrict__ out, int out_cap,
                            int32_t* __restrict__ member, long long member_cap, int32_t* __restrict__ hid,
                            long long hid_len, int use_pid) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int k = warp; k < nh; k += nw) {
    const int ic = halo_ids[k];
    const HaloRec& R = rec[ic];
    if (lane == 0 && k < out_cap) out[k] = R.H;
    if (!use_pid) continue;
    for (int i = lane; i < R.iodc; i += 32) {
      const int32_t p = mtmp[R.moff + i];
      if (member && foff[k] + i < member_cap) member[foff[k] + i] = p;
      if (hid && p >= 1 && p <= hid_len) hid[p - 1] = hnum[k];
    }
  }
}

// cell offsets within RMAX, (dx, dy, dz, r^2), in the reference's generation order
// (x outermost, z innermost, :68-80), stably sorted by the exact r^2
const std::vector<int4>& shell_list() {
  static const std::vector<int4> L = [] {  // built once, thread-safe
    std::vector<int4> v;
    for (int i = -RMAX; i <= RMAX; ++i)
      for (int j = -RMAX; j <= RMAX; ++j)
        for (int k = -RMAX; k <= RMAX; ++k) {
          const int r2 = i * i + j * j + k * k;
          if (r2 <= RMAX * RMAX) v.push_back(make_int4(i, j, k, r2));
        }
    std::stable_sort(v.begin(), v.end(), [](const int4& a, const int4& b) { return a.w < b.w; });
    return v;
  }();
  return L;
}

struct HaloScratch {
  std::vector<void*> p;
  ~HaloScratch() {
    for (void* q : p) cudaFree(q);
  }
  template <typename T>
  cudaError_t get(T** out, size_t bytes) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaSuccess) p.push_back(q);
    *out = reinterpret_cast<T*>(q);
    return e;
  }
};

// Waves: candidate j depends on an earlier candidate i when their search balls meet
// (i tags only particles within its rsearch of its peak, j gathers only within its
// own), wave(j) = 1 + the largest wave of those, 0 if none.  Candidates of one wave
// share no particle, so running them at once gives the sequential result.
std::vector<int> halo_waves(const std::vector<HaloCand>& hc, const std::vector<double>& rs, int nf, int* nwaves) {
  const int n = (int)hc.size();
  std::vector<int> wave(n, 0);
  double rmax = 0.0;
  for (double r : rs) rmax = std::max(rmax, r);
  const double reach = 2.0 * rmax + 1e-6;
  const int G = std::max(1, (int)std::floor(nf / std::max(reach, 1e-9)));  // buckets per dimension
  const double bw = (double)nf / G;
  std::vector<std::vector<int>> bucket((size_t)G * G * G);
  auto bidx = [&](double x) { int b = (int)std::floor(x / bw); return ((b % G) + G) % G; };
  int w_max = -1;
  for (int j = 0; j < n; ++j) {
    const int bj[3] = {bidx(hc[j].pos[0]), bidx(hc[j].pos[1]), bidx(hc[j].pos[2])};
    int w = 0;
    const int span = G >= 3 ? 1 : 0;
    auto visit = [&](int b) {
      for (int i : bucket[b]) {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          double dd = std::fabs(hc[i].pos[d] - hc[j].pos[d]);
          dd = std::fmod(dd, (double)nf);
          dd = std::min(dd, (double)nf - dd);
          d2 += dd * dd;
        }
        const double lim = rs[i] + rs[j] + 1e-6;
        if (d2 < lim * lim) w = std::max(w, wave[i] + 1);
      }
    };
    if (G < 3) {
      for (size_t b = 0; b < bucket.size(); ++b) visit((int)b);
    } else {
      for (int dz = -span; dz <= span; ++dz)
        for (int dy = -span; dy <= span; ++dy)
          for (int dx = -span; dx <= span; ++dx)
            visit((((bj[2] + dz + G) % G) * G + (bj[1] + dy + G) % G) * G + (bj[0] + dx + G) % G);
    }
    wave[j] = w;
    w_max = std::max(w_max, w);
    bucket[((size_t)bj[2] * G + bj[1]) * G + bj[0]].push_back(j);
  }
  *nwaves = w_max + 1;
  return wave;
}

template <int ZX, int ZV>
int run_halofind(cube_ctx* ctx, const cube_scalars* io, const cube_halo_args* ha, cube_halo_result* res) {
  const int nf = ctx->nf;
  const int64_t n3 = (int64_t)nf * nf * nf;
  const double den_odc = ha->den_odc > 0.f ? (double)ha->den_odc : 200.0;
  const int cm = 2 * ctx->ncb;  // coarse cells per dimension of a search box, at most 2 ncb - 1
  const int cmax = cm * cm * cm;
  const size_t smem = sizeof(long long) * (2 * (size_t)cmax + 1);
  if (smem > 200 * 1024 || ctx->nc < cm) {
    ctx->err = "halofind: needs nc >= 2 ncb and ncb <= 11";
    return CUBE_ERR_PARAM;
  }
  // the density accumulator borrows the fine force meshes (free between steps)
  if ((size_t)n3 * 8 > 3 * (size_t)nf * ctx->fine.plane * 4) {
    ctx->err = "halofind: the fine force meshes are too small for the density accumulator";
    return CUBE_ERR_CAPACITY;
  }
  unsigned long long* acc = reinterpret_cast<unsigned long long*>(ctx->fine.force);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(acc, 0, 8 * (size_t)n3, ctx->stream));
  const int64_t dblocks = (ctx->ncells + 63) / 64;
  k_halo_density<ZX><<<(unsigned)dblocks, 256, 0, ctx->stream>>>(ctx->xp, ctx->cell_start, ctx->cap, ctx->ncells,
                                                                  ctx->nt, ctx->nnt, nf, acc);
  CUBE_LAUNCH_CHECK(ctx);
  HaloScratch S;
  const std::vector<int4>& sl = shell_list();
  int4* dshell;
  HaloCand* cand;
  unsigned int* ncand;
  CUBE_CUDA_TRY(ctx, S.get(&dshell, sizeof(int4) * sl.size()));
  CUBE_CUDA_TRY(ctx, S.get(&cand, sizeof(HaloCand) * CAND_CAP));
  CUBE_CUDA_TRY(ctx, S.get(&ncand, sizeof(unsigned int)));
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dshell, sl.data(), sizeof(int4) * sl.size(), cudaMemcpyHostToDevice, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ncand, 0, sizeof(unsigned int), ctx->stream));
  const double mass = (double)io->mass_p_cdm;
  k_halo_peaks<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(acc, nf, mass, den_odc, dshell, (int)sl.size(), cand, ncand);
  CUBE_LAUNCH_CHECK(ctx);
  unsigned int nc_h = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&nc_h, ncand, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (nc_h > (unsigned)CAND_CAP) {
    ctx->err = "halofind: more density peaks than the candidate list holds";
    return CUBE_ERR_CAPACITY;
  }
  res->npeak = (int32_t)nc_h;
  // densest first, ties by node index; r_proxy = (3 m/(4 pi den_odc))^(1/3)
  std::vector<HaloCand> hc(nc_h);
  if (nc_h) {
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(hc.data(), cand, sizeof(HaloCand) * nc_h, cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  std::sort(hc.begin(), hc.end(), [](const HaloCand& a, const HaloCand& b) {
    return a.acc != b.acc ? a.acc > b.acc : a.node < b.node;
  });
  const double pi = (double)ctx->codec.pi_f;
  std::vector<double> rsv(nc_h);
  for (size_t i = 0; i < nc_h; ++i) {
    hc[i].rp = std::cbrt(0.75 / pi / den_odc * hc[i].mass);
    rsv[i] = std::min(2.0 * hc[i].rp, (double)((ctx->ncb - 1) * ctx->ncell));
  }
  if (nc_h)
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(cand, hc.data(), sizeof(HaloCand) * nc_h, cudaMemcpyHostToDevice, ctx->stream));
  // waves of independent candidates, each wave's members in candidate order
  int nwaves = 0;
  const std::vector<int> wave = halo_waves(hc, rsv, nf, &nwaves);
  std::vector<int> wstart(nwaves + 1, 0), order(nc_h);
  for (size_t i = 0; i < nc_h; ++i) wstart[wave[i] + 1]++;
  for (int w = 0; w < nwaves; ++w) wstart[w + 1] += wstart[w];
  {
    std::vector<int> fill(wstart.begin(), wstart.end() - 1);
    for (size_t i = 0; i < nc_h; ++i) order[fill[wave[i]]++] = (int)i;
  }
  HaloArgs A;
  A.xp = ctx->xp; A.vp = ctx->vp; A.pid = ctx->pid; A.cell_start = ctx->cell_start; A.vfield = ctx->vfield;
  int rc = 0;
  A.dec = cube_vdec_table(ctx, cube_vcoef(&ctx->codec, io->sigma_vi), &rc);
  if (rc) return rc;
  A.half_nvbin = ctx->nvbin / 2;
  A.use_pid = ctx->P.use_pid;
  A.cap = ctx->cap; A.ncells = ctx->ncells;
  A.nc = ctx->nc; A.nt = ctx->nt; A.nnt = ctx->nnt; A.nf = nf; A.ncb = ctx->ncb; A.ncell = ctx->ncell;
  A.cmax = cmax;
  A.mass = mass; A.den_odc = den_odc; A.pi = pi;
  A.vsim2phys = io->vsim2phys; A.a = io->a; A.h0 = ctx->P.h0; A.box = ctx->P.box;
  A.cand = cand;
  const size_t npb = (size_t)std::max<int64_t>(ctx->np, 1);
  CUBE_CUDA_TRY(ctx, S.get(&A.tag, npb));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(A.tag, 0, npb, ctx->stream));
  CUBE_CUDA_TRY(ctx, S.get(&A.rec, sizeof(HaloRec) * std::max<size_t>(nc_h, 1)));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(A.rec, 0, sizeof(HaloRec) * std::max<size_t>(nc_h, 1), ctx->stream));
  A.mcap = (long long)npb;  // members are distinct particles
  CUBE_CUDA_TRY(ctx, S.get(&A.mtmp, 4 * npb));
  int* dlists;
  CUBE_CUDA_TRY(ctx, S.get(&dlists, sizeof(int) * (2 * std::max<size_t>(nc_h, 1) + 8)));
  int* dorder = dlists;
  A.overflow = dlists + std::max<size_t>(nc_h, 1);
  long long* dcounters;
  CUBE_CUDA_TRY(ctx, S.get(&dcounters, 4 * sizeof(long long)));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(dcounters, 0, 4 * sizeof(long long), ctx->stream));
  A.mcount = dcounters;
  A.err = reinterpret_cast<int*>(dcounters + 1);
  if (nc_h)
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dorder, order.data(), sizeof(int) * nc_h, cudaMemcpyHostToDevice, ctx->stream));
  // scratch: the wave slots and one large slot for what a wave slot cannot hold
  const int nslot = ctx->num_sms * 2;
  const size_t wg = W_GCAP, wgrid = (size_t)(W_NB + 3) * (W_NB + 3) * (W_NB + 3);
  HaloSlot W;
  CUBE_CUDA_TRY(ctx, S.get(&W.gx, sizeof(double) * 3 * wg * nslot));
  CUBE_CUDA_TRY(ctx, S.get(&W.gv, sizeof(double) * 3 * wg * nslot));
  CUBE_CUDA_TRY(ctx, S.get(&W.gip, sizeof(int64_t) * wg * nslot));
  CUBE_CUDA_TRY(ctx, S.get(&W.key, sizeof(double) * wg * nslot));
  CUBE_CUDA_TRY(ctx, S.get(&W.ord, sizeof(int32_t) * wg * nslot));
  CUBE_CUDA_TRY(ctx, S.get(&W.grid, sizeof(unsigned long long) * wgrid * nslot));
  W.gcap = (int)wg;
  W.nbmax = W_NB;
  HaloSlot B;
  CUBE_CUDA_TRY(ctx, S.get(&B.gx, sizeof(double) * 3 * GCAP));
  CUBE_CUDA_TRY(ctx, S.get(&B.gv, sizeof(double) * 3 * GCAP));
  CUBE_CUDA_TRY(ctx, S.get(&B.gip, sizeof(int64_t) * GCAP));
  CUBE_CUDA_TRY(ctx, S.get(&B.key, sizeof(double) * GCAP));
  CUBE_CUDA_TRY(ctx, S.get(&B.ord, sizeof(int32_t) * GCAP));
  CUBE_CUDA_TRY(ctx, S.get(&B.grid, sizeof(unsigned long long) * (size_t)(NB_MAX + 3) * (NB_MAX + 3) * (NB_MAX + 3)));
  B.gcap = (int)GCAP;
  B.nbmax = NB_MAX;
  auto kw = k_halo_wave<ZX, ZV>;
  auto ks = k_halo_seq<ZX, ZV>;
  CUBE_CUDA_TRY(ctx, cube_smem_limit(kw, smem));
  CUBE_CUDA_TRY(ctx, cube_smem_limit(ks, smem));
  std::vector<int> ovf;
  for (int w = 0; w < nwaves; ++w) {
    const int n = wstart[w + 1] - wstart[w];
    CUBE_CUDA_TRY(ctx, cudaMemsetAsync(A.overflow, 0, sizeof(int), ctx->stream));
    kw<<<std::min(n, nslot), W_THREADS, smem, ctx->stream>>>(A, dorder + wstart[w], n, W, wg, wgrid);
    CUBE_LAUNCH_CHECK(ctx);
    int no = 0;
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&no, A.overflow, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (no) {  // this wave's large candidates, one after the other in the large slot
      ks<<<1, H_THREADS, smem, ctx->stream>>>(A, A.overflow + 1, no, B);
      CUBE_LAUNCH_CHECK(ctx);
    }
  }
  int herr = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(&herr, A.err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr) {
    ctx->err = herr == 2 ? "halofind: a refined grid exceeds 300 cells per dimension (newbox_max)"
             : herr == 3 ? "halofind: more particles within a search radius than the gather list holds"
                         : "halofind: a search box wraps onto itself (nc too small for rsearch)";
    return herr == 4 ? CUBE_ERR_PARAM : CUBE_ERR_CAPACITY;
  }
  // numbering and offsets in candidate order
  std::vector<int2> flags(nc_h);
  if (nc_h) {
    int2* dfl;
    CUBE_CUDA_TRY(ctx, S.get(&dfl, sizeof(int2) * nc_h));
    k_halo_flags<<<(nc_h + 255) / 256, 256, 0, ctx->stream>>>(A.rec, (int)nc_h, dfl);
    CUBE_LAUNCH_CHECK(ctx);
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(flags.data(), dfl, sizeof(int2) * nc_h, cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  }
  std::vector<int> halo_ids, hnum;
  std::vector<long long> foff;
  long long run = 0;
  for (size_t i = 0; i < nc_h; ++i)
    if (flags[i].x) {
      halo_ids.push_back((int)i);
      hnum.push_back((int)halo_ids.size());
      foff.push_back(run);
      run += flags[i].y;
    }
  const int nh = (int)halo_ids.size();
  res->nhalo = nh;
  res->nmember = A.use_pid ? run : 0;
  const int cap_out = std::max(ha->capacity, 0);
  cube_halo* dout = nullptr;
  int32_t* dmem = nullptr;
  int32_t* dhid = nullptr;
  if (nh) {
    int* dids;
    long long* dfoff;
    CUBE_CUDA_TRY(ctx, S.get(&dids, sizeof(int) * 2 * nh));
    CUBE_CUDA_TRY(ctx, S.get(&dfoff, sizeof(long long) * nh));
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dids, halo_ids.data(), sizeof(int) * nh, cudaMemcpyHostToDevice, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dids + nh, hnum.data(), sizeof(int) * nh, cudaMemcpyHostToDevice, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(dfoff, foff.data(), sizeof(long long) * nh, cudaMemcpyHostToDevice, ctx->stream));
    CUBE_CUDA_TRY(ctx, S.get(&dout, sizeof(cube_halo) * (size_t)std::max(cap_out, 1)));
    if (ha->member_pid && ha->member_capacity > 0) CUBE_CUDA_TRY(ctx, S.get(&dmem, 4 * (size_t)ha->member_capacity));
    if (ha->hid && ha->hid_len > 0) {
      CUBE_CUDA_TRY(ctx, S.get(&dhid, 4 * (size_t)ha->hid_len));
      CUBE_CUDA_TRY(ctx, cudaMemsetAsync(dhid, 0, 4 * (size_t)ha->hid_len, ctx->stream));
    }
    k_halo_emit<<<ctx->num_sms * 4, 256, 0, ctx->stream>>>(A.rec, dids + nh, dfoff, dids, nh, A.mtmp, dout, cap_out,
                                                           dmem, ha->member_capacity, dhid, ha->hid_len, A.use_pid);
    CUBE_LAUNCH_CHECK(ctx);
    const int nout = std::min(nh, cap_out);
    if (nout > 0)
      CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ha->halos, dout, sizeof(cube_halo) * nout, cudaMemcpyDeviceToHost, ctx->stream));
    if (dmem && run > 0)
      CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ha->member_pid, dmem, 4 * (size_t)std::min<long long>(run, ha->member_capacity),
                                         cudaMemcpyDeviceToHost, ctx->stream));
    if (dhid)
      CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ha->hid, dhid, 4 * (size_t)ha->hid_len, cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  } else if (ha->hid && ha->hid_len > 0) {
    std::fill(ha->hid, ha->hid + ha->hid_len, 0);
  }
  if (nh > cap_out || (ha->member_pid && A.use_pid && run > ha->member_capacity)) {
    ctx->err = "halofind: the output arrays are too small (the counts are returned)";
    return CUBE_ERR_CAPACITY;
  }
  return CUBE_OK;
}

}  // namespace

int cube_halofind_dev(cube_ctx* ctx, const cube_scalars* io, const cube_halo_args* ha, cube_halo_result* res) {
  if (ctx->izipx == 1 && ctx->izipv == 1) return run_halofind<1, 1>(ctx, io, ha, res);
  if (ctx->izipx == 1) return run_halofind<1, 2>(ctx, io, ha, res);
  if (ctx->izipv == 1) return run_halofind<2, 1>(ctx, io, ha, res);
  return run_halofind<2, 2>(ctx, io, ha, res);
}
