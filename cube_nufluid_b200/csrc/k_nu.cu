/*
 * k_nu.cu -- fluid neutrinos on the GPU: the dispersive sum of three isothermal
 * fluids (hydrodf.f90), their finite-volume update (hydro3d.f90, hydro1d.f90),
 * and their coupling to the particle mesh (pm.f90:55-74, :157-171, :198-242,
 * :374-422).
 *
 * Layout: each fluid is five FP32 arrays of n^3 cells, x fastest, periodic.
 * The reference keeps halo cells of ncb >= 2 and refreshes them by a periodic
 * copy before and after the three sweeps; with the stencil's reach of two
 * cells that is the same update as periodic indexing of the interior, which is
 * what these kernels do (the CPU tests check the two forms bit for bit).
 *
 * Sweeps (h3_evolve_xyz, h_evolve, h_riemann): one kernel per direction.  A CTA
 * stages a tile of lines plus two cells either side in shared memory as
 * primitive variables (rho, v_n, v_t1, v_t2, p), computes the HLL flux of each
 * interface once, and updates its cells from the two fluxes around them, in
 * the reference's FP32 operation order (explicit _rn intrinsics, no FMA), so
 * the result equals the oracle's bit for bit.  Input and output are separate
 * arrays: all fluxes of a sweep come from the state before it.
 *
 * Gravity (hg_gravity via dfld_gravity).  The reference scatters every fine
 * cell's acceleration a_n into the 8 surrounding fluid cells, in a loop order
 * under OpenMP, with E += dV (p.a + rho|a|^2/2) and p += dV rho a, where p is
 * the momentum already updated by earlier sources.  For one fluid cell the
 * sequential chain sums to the closed form
 *     p1 = p0 + rho A,   E1 = E0 + p0.A + rho|A|^2/2 + rho B/2,
 *     A = sum dV_n a_n,  B = sum dV_n (1 - dV_n) |a_n|^2,
 * independent of the order, so the GPU gathers A and B per fluid cell
 * (deterministically, fixed summation order) and applies the closed form once.
 * The weights dV are products of per-dimension CIC weights, so A, sum dV|a|^2
 * and sum dV^2|a|^2 are separable restrictions: k_nu_src_xy forms each fine
 * cell's a_fine + a_coarse and |a_fine|^2 + |a_coarse|^2 and restricts them
 * over x and y per fine z-plane, k_nu_grav_z restricts over z and applies the
 * closed form.  The source set is the reference's: fine sources at the
 * physical fine cells, coarse sources also at the two buffer layers each side
 * (pm.f90:382-385); contributions that the reference scatters into halo cells
 * are dropped there by the next hg_buffer, and simply have no target here.
 *
 * Density (hg_density / dfld_density): at fine node n the reference samples the
 * fluids at n + 1/2 (pm.f90:63-65); the value is added to the fine mesh after
 * the particle deposit, and deposited into the coarse accumulator in the same
 * 64-bit fixed point as the particles, so the coarse density stays
 * order-independent.
 */
#include "cube_internal.cuh"

namespace {

#define FM __fmul_rn
#define FA __fadd_rn
#define FS __fsub_rn
#define FD __fdiv_rn

// std::max / std::min semantics (first argument unless the second is larger /
// smaller), which is what the oracle's restatement uses
__device__ __forceinline__ float mx(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float mn(float a, float b) { return (b < a) ? b : a; }

constexpr float kLim = 1.5f;   // h_lim (hydro1d.f90:18)
constexpr float kCfl = 0.71f;  // h_cfl (hydro1d.f90:16)

__device__ __forceinline__ float minmod(float a, float b, float c) {
  const float sa = copysignf(1.f, a), sb = copysignf(1.f, b), sc = copysignf(1.f, c);
  return FM(FM(FM(0.25f, fabsf(FA(sa, sb))), FA(sa, sc)), mn(mn(fabsf(a), fabsf(b)), fabsf(c)));
}
// left-biased value at cell i from u(i-1), u(i), u(i+1)
__device__ __forceinline__ float lbias(float um, float u, float up) {
  return FA(u, FM(0.5f, minmod(FM(kLim, FS(u, um)), FM(0.5f, FS(up, um)), FM(kLim, FS(up, u)))));
}
// right-biased value at cell i from u(i), u(i+1), u(i+2)
__device__ __forceinline__ float rbias(float u, float up, float upp) {
  return FS(up, FM(0.5f, minmod(FM(kLim, FS(up, u)), FM(0.5f, FS(upp, u)), FM(kLim, FS(upp, up)))));
}
__device__ __forceinline__ float kinetic(float r, float m2, float m3, float m4) {
  return FD(FM(0.5f, FA(FA(FM(m2, m2), FM(m3, m3)), FM(m4, m4))), r);
}

struct SweepArgs {
  const float* in[5];
  float* out[5];
  int n, ts, tx;       // cells per side, tile length along the sweep, lines per tile
  float gm1, dt, inv_dx;  // g-1, half-step dt, 1/cell size (a power of two)
};

// slot order of the momentum components seen by the 1-D solver: the normal
// component first (hydro3d.f90:78-100 swaps 2<->3 for y, 2<->4 for z)
template <int AX>
__device__ __forceinline__ int slot_comp(int s) {  // s = 1..3 -> component 1..3 (0-based momentum)
  if (AX == 0) return s;
  if (AX == 1) return s == 1 ? 2 : (s == 2 ? 1 : 3);
  return s == 1 ? 3 : (s == 3 ? 1 : 2);
}

template <int AX>
__device__ __forceinline__ size_t cell_addr(int n, int q, int line, int third) {
  // AX=0: q = x, line = y, third = z; AX=1: q = y, line = x, third = z;
  // AX=2: q = z, line = x, third = y
  if (AX == 0) return ((size_t)third * n + line) * n + q;
  if (AX == 1) return ((size_t)third * n + q) * n + line;
  return ((size_t)q * n + third) * n + line;
}

template <int AX>
__global__ void __launch_bounds__(256) k_nu_sweep(SweepArgs A) {
  extern __shared__ float sm[];
  const int n = A.n, TS = A.ts, TX = A.tx, TH = TS + 4;
  float* prim = sm;                    // [5][TX][TH]
  float* flux = sm + 5 * TX * TH;      // [5][TX][TS+1]
  const int nseg = n / TS;
  const int seg = blockIdx.x % nseg, lt = blockIdx.x / nseg;
  const int s0 = seg * TS, l0 = lt * TX, third = blockIdx.y;
  const int c1 = slot_comp<AX>(1), c2 = slot_comp<AX>(2), c3 = slot_comp<AX>(3);
  // 1. primitives of the tile and two cells either side
  for (int e = threadIdx.x; e < TX * TH; e += blockDim.x) {
    int l, s;
    if (AX == 0) { l = e / TH; s = e - l * TH; } else { s = e / TX; l = e - s * TX; }
    int q = s0 + s - 2;
    q += (q < 0) ? n : 0;
    q -= (q >= n) ? n : 0;
    const size_t g = cell_addr<AX>(n, q, l0 + l, third);
    const float r = A.in[0][g], m1 = A.in[1 + c1 - 1][g], m2 = A.in[1 + c2 - 1][g], m3 = A.in[1 + c3 - 1][g];
    const float E = A.in[4][g];
    const float k = kinetic(r, m1, m2, m3);
    const int o = l * TH + s;
    prim[o] = r;
    prim[TX * TH + o] = FD(m1, r);
    prim[2 * TX * TH + o] = FD(m2, r);
    prim[3 * TX * TH + o] = FD(m3, r);
    prim[4 * TX * TH + o] = mx(0.f, FM(FS(E, k), A.gm1));
  }
  __syncthreads();
  // 2. HLL flux at interface i+1/2 for local cells i = -1..TS-1 (h_riemann)
  const int NI = TS + 1;
  for (int e = threadIdx.x; e < TX * NI; e += blockDim.x) {
    const int l = e / NI, j = e - l * NI;  // j = i + 1
    const int b = l * TH + j;              // smem index of cell i-1 (cells i-1..i+2 at b..b+3)
    float L[5], R[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const float* u = prim + v * TX * TH + b;
      L[v] = lbias(u[0], u[1], u[2]);
      R[v] = rbias(u[1], u[2], u[3]);
    }
    // states (rho, rho v_n, rho v_t1, rho v_t2, E)
    float hl[5], hr[5];
    hl[0] = L[0]; hl[1] = FM(L[0], L[1]); hl[2] = FM(L[0], L[2]); hl[3] = FM(L[0], L[3]);
    hr[0] = R[0]; hr[1] = FM(R[0], R[1]); hr[2] = FM(R[0], R[2]); hr[3] = FM(R[0], R[3]);
    const float kl = kinetic(hl[0], hl[1], hl[2], hl[3]), kr = kinetic(hr[0], hr[1], hr[2], hr[3]);
    hl[4] = FA(FD(L[4], A.gm1), kl);
    hr[4] = FA(FD(R[4], A.gm1), kr);
    // h_flux of each state (q_EQN_OF_STATE energy flux)
    const float pl = mx(0.f, FM(FS(hl[4], kl), A.gm1));
    const float pr = mx(0.f, FM(FS(hr[4], kr), A.gm1));
    const float vl = FD(hl[1], hl[0]), vr = FD(hr[1], hr[0]);
    float fl[5], fr[5];
    fl[0] = hl[1];
    fl[1] = FA(FM(hl[1], vl), pl);
    fl[2] = FM(hl[1], FD(hl[2], hl[0]));
    fl[3] = FM(hl[1], FD(hl[3], hl[0]));
    fl[4] = FM(hl[4], vl);
    fr[0] = hr[1];
    fr[1] = FA(FM(hr[1], vr), pr);
    fr[2] = FM(hr[1], FD(hr[2], hr[0]));
    fr[3] = FM(hr[1], FD(hr[3], hr[0]));
    fr[4] = FM(hr[4], vr);
    const float sl = __fsqrt_rn(FD(pl, hl[0])), sr = __fsqrt_rn(FD(pr, hr[0]));
    const float ap = mx(mx(0.f, FA(vl, sl)), FA(vr, sr));
    const float am = mx(mx(0.f, FA(-vl, sl)), FA(-vr, sr));
    const float apm = FA(ap, am), apam = FM(ap, am);
#pragma unroll
    for (int v = 0; v < 5; ++v)
      flux[(v * TX + l) * NI + j] = FD(FS(FA(FM(ap, fl[v]), FM(am, fr[v])), FM(apam, FS(hr[v], hl[v]))), apm);
  }
  __syncthreads();
  // 3. h = h + dt*(-f(i) + f(i-1))/dx
  for (int e = threadIdx.x; e < TX * TS; e += blockDim.x) {
    int l, s;
    if (AX == 0) { l = e / TS; s = e - l * TS; } else { s = e / TX; l = e - s * TX; }
    const size_t g = cell_addr<AX>(n, s0 + s, l0 + l, third);
    const int comp[5] = {0, 1 + c1 - 1, 1 + c2 - 1, 1 + c3 - 1, 4};
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const float* f = flux + (v * TX + l) * NI + s;  // f[0] = f(i-1), f[1] = f(i)
      const float r = FA(-f[1], f[0]);
      A.out[comp[v]][g] = FA(A.in[comp[v]][g], FM(FM(A.dt, r), A.inv_dx));  // x/dx = x*(1/dx) exactly
    }
  }
}

// h3_timestep / h_timestep: per x-line max |v| and max sound speed, then
// cfl*dx/(v+s); the minimum over lines by an atomic on the float bits (all
// values are positive, and min is exact)
__global__ void __launch_bounds__(128) k_nu_dt(const float* __restrict__ r_, const float* __restrict__ px,
                                               const float* __restrict__ py, const float* __restrict__ pz,
                                               const float* __restrict__ e_, int n, float gm1, float dx,
                                               unsigned int* __restrict__ dt_bits) {
  __shared__ float red[4][4];
  const size_t base = (size_t)blockIdx.x * n;
  float vx = 0.f, vy = 0.f, vz = 0.f, s = 0.f;  // |v| and sound speeds are >= 0
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float r = r_[base + i], a = px[base + i], b = py[base + i], c = pz[base + i], E = e_[base + i];
    const float ax = fabsf(FD(a, r)), ay = fabsf(FD(b, r)), az = fabsf(FD(c, r));
    const float p = mx(0.f, FM(FS(E, kinetic(r, a, b, c)), gm1));
    const float ss = __fsqrt_rn(FD(p, r));
    vx = mx(vx, ax); vy = mx(vy, ay); vz = mx(vz, az); s = mx(s, ss);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vx = mx(vx, __shfl_xor_sync(0xffffffffu, vx, o));
    vy = mx(vy, __shfl_xor_sync(0xffffffffu, vy, o));
    vz = mx(vz, __shfl_xor_sync(0xffffffffu, vz, o));
    s = mx(s, __shfl_xor_sync(0xffffffffu, s, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { red[0][w] = vx; red[1][w] = vy; red[2][w] = vz; red[3][w] = s; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < 4; ++k) {
      vx = mx(vx, red[0][k]); vy = mx(vy, red[1][k]); vz = mx(vz, red[2][k]); s = mx(s, red[3][k]);
    }
    const float v = mx(mx(mx(0.f, vx), vy), vz);
    const float dtl = FD(FM(kCfl, dx), FA(v, s));
    atomicMin(dt_bits, __float_as_uint(dtl));
  }
}

__global__ void k_nu_aos_to_soa(const float* __restrict__ aos, float* __restrict__ soa, int64_t n3) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 5 * n3; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cell = i / 5, c = i - cell * 5;
    soa[c * n3 + cell] = aos[i];
  }
}
__global__ void k_nu_soa_to_aos(const float* __restrict__ soa, float* __restrict__ aos, int64_t n3) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 5 * n3; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cell = i / 5, c = i - cell * 5;
    aos[i] = soa[c * n3 + cell];
  }
}

// ---- density -------------------------------------------------------------------
struct Rho3 {
  const float* r[3];
  int n[3];
  float dx[3], w[3];
};

// hg_density (gc=1) of one fluid at x (fine-cell units), periodic
__device__ __forceinline__ float fluid_density(const float* __restrict__ r, int n, float dx, const float x[3]) {
  int i0[3], i1[3];
  float d1[3], d2[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const float xx = FS(FM(x[e], 1.f / dx), 0.5f);  // dx is a power of two: exact
    const int lo = (int)floorf(xx);  // 0-based index of idx1
    d1[e] = FS((float)(lo + 1), xx);
    d2[e] = FS(1.f, d1[e]);
    i0[e] = cube_wrap(lo, n);
    i1[e] = cube_wrap(lo + 1, n);
  }
  // term order 111,211,121,221,112,212,122,222
  float d = 0.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int ox = c & 1, oy = (c >> 1) & 1, oz = c >> 2;
    const float f = __ldg(&r[((size_t)(oz ? i1[2] : i0[2]) * n + (oy ? i1[1] : i0[1])) * n + (ox ? i1[0] : i0[0])]);
    const float t = FM(FM(FM(f, ox ? d2[0] : d1[0]), oy ? d2[1] : d1[1]), oz ? d2[2] : d1[2]);
    d = (c == 0) ? t : FA(d, t);
  }
  return d;
}

// neutrino density at every fine node (pm.f90:55-74): nu = 0 + f_neu*sum_k w_k rho_k(n+1/2)
// (or 0 + f_neu before z_i_nu); added to the fine mesh, kept in `scratch` for the
// coarse deposit, and summed in FP64 per CTA for testrhof.  One CTA per brick of
// 32x8x8 fine nodes: each fluid's cells under the brick (plus one on each side)
// are staged in shared memory, and each node runs hg_density's CIC in its order.
constexpr int DBX = 32, DBY = 8, DBZ = 8;
constexpr int DPATCH = 3 * (DBX / 2 + 2) * (DBY / 2 + 2) * (DBZ / 2 + 2);  // three fluids, dx >= 2

__global__ void __launch_bounds__(256) k_nu_fine_density(Rho3 F, int homogeneous, float f_neu, int nf, float* __restrict__ rho,
                                                        int rp, size_t plane, float* __restrict__ scratch,
                                                        double* __restrict__ partial) {
  __shared__ float patch[DPATCH];
  __shared__ double red[256];
  const int nbx = nf / DBX, nby = nf / DBY;
  const int x0 = (blockIdx.x % nbx) * DBX, y0 = ((blockIdx.x / nbx) % nby) * DBY, z0 = (blockIdx.x / (nbx * nby)) * DBZ;
  int off[3], px[3], py[3], pz[3], lo0[3][3];
  {
    int o = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int dx = (int)F.dx[k];  // 2, 4 or 8
      px[k] = DBX / dx + 2; py[k] = DBY / dx + 2; pz[k] = DBZ / dx + 2;
      lo0[k][0] = x0 / dx - 1; lo0[k][1] = y0 / dx - 1; lo0[k][2] = z0 / dx - 1;
      off[k] = o;
      o += px[k] * py[k] * pz[k];
    }
  }
  if (!homogeneous) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int n = F.n[k];
      for (int e = threadIdx.x; e < px[k] * py[k] * pz[k]; e += blockDim.x) {
        const int ix = e % px[k], iy = (e / px[k]) % py[k], iz = e / (px[k] * py[k]);
        const int gx = cube_wrap(lo0[k][0] + ix, n), gy = cube_wrap(lo0[k][1] + iy, n), gz = cube_wrap(lo0[k][2] + iz, n);
        patch[off[k] + e] = __ldg(&F.r[k][((size_t)gz * n + gy) * n + gx]);
      }
    }
  }
  __syncthreads();
  const int lx = threadIdx.x & 31;
  const int x = x0 + lx;
  // x weights of this thread's column, per fluid (hg_density, hydrogr.f90:328-333)
  float wx1[3], wx2[3];
  int ix0[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float xx = FS(FM(FA((float)x, 0.5f), 1.f / F.dx[k]), 0.5f);
    const int lo = (int)floorf(xx);
    wx1[k] = FS((float)(lo + 1), xx);
    wx2[k] = FS(1.f, wx1[k]);
    ix0[k] = lo - lo0[k][0];
  }
  double acc = 0.0;
  for (int yz = threadIdx.x >> 5; yz < DBY * DBZ; yz += 8) {
    const int y = y0 + (yz & (DBY - 1)), z = z0 + yz / DBY;
    float val;
    if (homogeneous) {
      val = FA(0.f, f_neu);
    } else {
      float den = 0.f;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float inv = 1.f / F.dx[k];
        const float yy = FS(FM(FA((float)y, 0.5f), inv), 0.5f), zz = FS(FM(FA((float)z, 0.5f), inv), 0.5f);
        const int ylo = (int)floorf(yy), zlo = (int)floorf(zz);
        const float wy1 = FS((float)(ylo + 1), yy), wz1 = FS((float)(zlo + 1), zz);
        const float wy2 = FS(1.f, wy1), wz2 = FS(1.f, wz1);
        const float* P = patch + off[k] + ((zlo - lo0[k][2]) * py[k] + (ylo - lo0[k][1])) * px[k] + ix0[k];
        const int sy = px[k], sz = px[k] * py[k];
        // term order 111,211,121,221,112,212,122,222 (hydrogr.f90:335-342)
        float d = FM(FM(FM(P[0], wx1[k]), wy1), wz1);
        d = FA(d, FM(FM(FM(P[1], wx2[k]), wy1), wz1));
        d = FA(d, FM(FM(FM(P[sy], wx1[k]), wy2), wz1));
        d = FA(d, FM(FM(FM(P[sy + 1], wx2[k]), wy2), wz1));
        d = FA(d, FM(FM(FM(P[sz], wx1[k]), wy1), wz2));
        d = FA(d, FM(FM(FM(P[sz + 1], wx2[k]), wy1), wz2));
        d = FA(d, FM(FM(FM(P[sz + sy], wx1[k]), wy2), wz2));
        d = FA(d, FM(FM(FM(P[sz + sy + 1], wx2[k]), wy2), wz2));
        den = FA(den, FM(F.w[k], d));
      }
      val = FA(0.f, FM(den, f_neu));
    }
    const size_t g = (size_t)z * plane + (size_t)y * rp + x;
    rho[g] = FA(rho[g], val);
    scratch[g] = val;
    acc += (double)val;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// coarse deposit of the fine-node neutrino density (pm.f90:198-242) into the
// 64-bit coarse accumulator: node N gathers fine nodes 4N-2..4N+5 per dimension
// with the CIC weights of those fine-cell centres (exact dyadic values)
__global__ void __launch_bounds__(256) k_nu_coarse_deposit(const float* __restrict__ nu, int nf, int rp, size_t plane,
                                                          int nc, int homogeneous, float hom_value,
                                                          unsigned long long* __restrict__ acc) {
  const float w8[8] = {0.125f, 0.375f, 0.625f, 0.875f, 0.875f, 0.625f, 0.375f, 0.125f};
  const int64_t total = (int64_t)nc * nc * nc;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int X = (int)(i % nc);
    const int64_t yz = i / nc;
    const int Y = (int)(yz % nc), Z = (int)(yz / nc);
    long long sum = 0;
    if (homogeneous) {
      sum = __double2ll_rn((double)hom_value * 4294967296.0);
    } else {
      for (int oz = 0; oz < 8; ++oz) {
        const int qz = cube_wrap(4 * Z - 2 + oz, nf);
        for (int oy = 0; oy < 8; ++oy) {
          const int qy = cube_wrap(4 * Y - 2 + oy, nf);
          const float* row = nu + (size_t)qz * plane + (size_t)qy * rp;
#pragma unroll
          for (int ox = 0; ox < 8; ++ox) {
            const int qx = cube_wrap(4 * X - 2 + ox, nf);
            const float t = FM(FM(FM(__ldg(&row[qx]), w8[ox]), w8[oy]), w8[oz]);
            sum += __double2ll_rn((double)t * 4294967296.0);
          }
        }
      }
    }
    acc[i] += (unsigned long long)sum;
  }
}

// ---- gravity ---------------------------------------------------------------------
constexpr int GT = 32;          // fine cells per side of a k_nu_src_xy tile
constexpr int GW = GT + 8;      // source window per side (dx <= 8: dx/2 either side)
constexpr int GCN = 12;         // coarse nodes per side the window's CIC reads

// the force meshes hold kick increments (((f*a_mid)*dt)/6)/pi per node (the
// chain of pm.f90:163, :393, applied by the c2r pass)
struct GravArgs {
  const float* ff;   // fine kick increments [3][nf planes], pitch frp, plane fplane
  size_t fcomp, fplane;
  int frp;
  const float* fc;   // coarse force
  size_t ccomp, cplane;
  int crp;
  int nf, nc;
  float a_mid, dt, pi_f;
  int nfl;           // fluids
  int fn[3], fdx[3]; // fluid cells per side and cell size (2,4,8)
  float* xy[3];      // [5][nf+4][n][n] per fluid
};

// per fine z-plane qz in [-2, nf+2) and 32x32 tile of fine cells: source terms of
// the window, then their x/y restriction onto each fluid's cells of the tile.
// A and B are FP32 sums in a fixed order (deterministic); the coarse
// acceleration at the fine-cell centres is the trilinear CIC of the coarse kick
// increments evaluated separably (z per plane, then y and x), which agrees with
// the reference's FP64 sum of its eight FP32 terms to FP32 rounding.
__global__ void __launch_bounds__(256) k_nu_src_xy(GravArgs G) {
  __shared__ float src[4][GW][GW + 1];   // A.x, A.y, A.z, |a_f|^2 + |a_c|^2 (rows padded)
  __shared__ float gz[3][GCN][GCN + 1];  // coarse increments interpolated to this plane
  __shared__ float rx[5][GW][GT / 2 + 1];  // x-restricted rows, [v][window row][target x]
  __shared__ float wt[2][GT / 2][16];     // per axis: weight of source i of target t
  const int nf = G.nf, nc = G.nc, ntx = nf / GT;
  const int x0 = (blockIdx.x % ntx) * GT, y0 = (blockIdx.x / ntx) * GT;
  const int qz = (int)blockIdx.y - 2;
  // coarse CIC along z for this plane (x = qz + 1/2): xc = x/4 - 0.5
  const float zc = FS(FM(FA((float)qz, 0.5f), 0.25f), 0.5f);
  const int zlo = (int)floorf(zc);
  const float cz1 = FS((float)(zlo + 1), zc), cz2 = FS(1.f, cz1);
  const int nbx = (x0 >> 2) - 2, nby = (y0 >> 2) - 2;  // first coarse node of the window
  const int gz0 = cube_wrap(zlo, nc), gz1 = cube_wrap(zlo + 1, nc);
  for (int e = threadIdx.x; e < 3 * GCN * GCN; e += blockDim.x) {
    const int ix = e % GCN, iy = (e / GCN) % GCN, d = e / (GCN * GCN);
    const int gx = cube_wrap(nbx + ix, nc), gy = cube_wrap(nby + iy, nc);
    const float* c = G.fc + d * G.ccomp + (size_t)gy * G.crp + gx;
    gz[d][iy][ix] = cz1 * __ldg(c + (size_t)gz0 * G.cplane) + cz2 * __ldg(c + (size_t)gz1 * G.cplane);
  }
  __syncthreads();
  const bool zf = (qz >= 0 && qz < nf);  // fine sources exist on this plane
  const bool zc_in = (qz >= -2 && qz <= nf + 1);
  for (int e = threadIdx.x; e < GW * GW; e += blockDim.x) {
    const int wx = e % GW, wy = e / GW;
    const int qx = x0 - 4 + wx, qy = y0 - 4 + wy;
    float af[3] = {0.f, 0.f, 0.f}, ac[3] = {0.f, 0.f, 0.f};
    if (zf && qx >= 0 && qx < nf && qy >= 0 && qy < nf) {
      // fine increment at node q+1 (pm.f90:160-163: idx1 = floor(tempx)+1+nfb)
      const int fx = cube_wrap(qx + 1, nf), fy = cube_wrap(qy + 1, nf), fz = cube_wrap(qz + 1, nf);
      const size_t o = (size_t)fz * G.fplane + (size_t)fy * G.frp + fx;
#pragma unroll
      for (int d = 0; d < 3; ++d) af[d] = __ldg(&G.ff[d * G.fcomp + o]);
    }
    if (zc_in && qx >= -2 && qx <= nf + 1 && qy >= -2 && qy <= nf + 1) {
      // coarse sources also on the two buffer layers beyond each face (pm.f90:382-385)
      const float xc = FS(FM(FA((float)qx, 0.5f), 0.25f), 0.5f), yc = FS(FM(FA((float)qy, 0.5f), 0.25f), 0.5f);
      const int xl = (int)floorf(xc), yl = (int)floorf(yc);
      const float cx1 = FS((float)(xl + 1), xc), cx2 = FS(1.f, cx1);
      const float cy1 = FS((float)(yl + 1), yc), cy2 = FS(1.f, cy1);
      const int ix = xl - nbx, iy = yl - nby;
#pragma unroll
      for (int d = 0; d < 3; ++d)
        ac[d] = cy1 * (cx1 * gz[d][iy][ix] + cx2 * gz[d][iy][ix + 1]) +
                cy2 * (cx1 * gz[d][iy + 1][ix] + cx2 * gz[d][iy + 1][ix + 1]);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) src[d][wy][wx] = af[d] + ac[d];
    src[3][wy][wx] = (af[0] * af[0] + af[1] * af[1] + af[2] * af[2]) + (ac[0] * ac[0] + ac[1] * ac[1] + ac[2] * ac[2]);
  }
  // Restriction onto each fluid's cells: target t gets the 2dx sources from window
  // index b0 + dx t (lower target floor((q+1/2)/dx - 1/2) with weight w1 = that + 1
  // - ((q+1/2)/dx - 1/2), the upper one 1 - w1).  A (3 components), C1 = sum w|a|^2
  // and C2 = sum w^2 |a|^2; x first (one thread per window row and target), then y.
  for (int k = 0; k < G.nfl; ++k) {
    const int dx = G.fdx[k], n = G.fn[k], tb = GT / dx, nw = 2 * dx;
    const float inv_dx = 1.f / (float)dx;  // exact: dx is a power of two
    const int b0 = 4 - dx / 2;             // window index of target 0's first source
    for (int e = threadIdx.x; e < 2 * tb * nw; e += blockDim.x) {
      const int ax = e / (tb * nw), r = e - ax * tb * nw, t = r / nw, i = r - t * nw;
      const int q = (ax == 0 ? x0 : y0) - 4 + b0 + dx * t + i;
      const float xx = FS(FM(FA((float)q, 0.5f), inv_dx), 0.5f);
      const int lo = (int)floorf(xx);
      const float w1 = FS((float)(lo + 1), xx);
      wt[ax][t][i] = (lo - (ax == 0 ? x0 : y0) / dx == t) ? w1 : FS(1.f, w1);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < tb * GW; e += blockDim.x) {
      const int tx = e / GW, wy = e - tx * GW;
      float a0 = 0.f, a1 = 0.f, a2 = 0.f, c1 = 0.f, c2 = 0.f;
      for (int i = 0; i < nw; ++i) {
        const int wx = b0 + dx * tx + i;
        const float w = wt[0][tx][i];
        a0 += w * src[0][wy][wx];
        a1 += w * src[1][wy][wx];
        a2 += w * src[2][wy][wx];
        const float q2 = src[3][wy][wx];
        c1 += w * q2;
        c2 += (w * w) * q2;
      }
      rx[0][wy][tx] = a0; rx[1][wy][tx] = a1; rx[2][wy][tx] = a2; rx[3][wy][tx] = c1; rx[4][wy][tx] = c2;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < tb * tb; e += blockDim.x) {
      const int ty = e / tb, tx = e - ty * tb;
      float a0 = 0.f, a1 = 0.f, a2 = 0.f, c1 = 0.f, c2 = 0.f;
      for (int j = 0; j < nw; ++j) {
        const int wy = b0 + dx * ty + j;
        const float w = wt[1][ty][j];
        a0 += w * rx[0][wy][tx];
        a1 += w * rx[1][wy][tx];
        a2 += w * rx[2][wy][tx];
        c1 += w * rx[3][wy][tx];
        c2 += (w * w) * rx[4][wy][tx];
      }
      const int gtx = x0 / dx + tx, gty = y0 / dx + ty;
      const size_t vs = (size_t)(nf + 4) * n * n;
      const size_t o = ((size_t)(qz + 2) * n + gty) * n + gtx;
      G.xy[k][o] = a0;
      G.xy[k][vs + o] = a1;
      G.xy[k][2 * vs + o] = a2;
      G.xy[k][3 * vs + o] = c1;
      G.xy[k][4 * vs + o] = c2;
    }
    __syncthreads();
  }
}

// z restriction and the closed-form update of one fluid (hg_gravity chain)
__global__ void __launch_bounds__(256) k_nu_grav_z(const float* __restrict__ xy, int nf, int n, int dx,
                                                  float* __restrict__ r_, float* __restrict__ px,
                                                  float* __restrict__ py, float* __restrict__ pz,
                                                  float* __restrict__ e_) {
  const int64_t total = (int64_t)n * n * n;
  const float dxf = (float)dx;
  const float inv3 = 1.f / (dxf * dxf * dxf);  // exact: dx is a power of two
  const float inv6 = inv3 * inv3;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int tx = (int)(i % n);
    const int64_t yz = i / n;
    const int ty = (int)(yz % n), tz = (int)(yz / n);
    float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    const int q0 = dx * tz - dx / 2;
    for (int j = 0; j < 2 * dx; ++j) {
      const int qz = q0 + j;
      if (qz < -2 || qz > nf + 1) continue;
      const float zz = FS(FM(FA((float)qz, 0.5f), 1.f / dxf), 0.5f);
      const int zl = (int)floorf(zz);
      const float wz1 = FS((float)(zl + 1), zz);
      const float wz = (zl == tz) ? wz1 : FS(1.f, wz1);
      const size_t o = ((size_t)(qz + 2) * n + ty) * n + tx;
      const size_t vs = (size_t)(nf + 4) * n * n;
#pragma unroll
      for (int v = 0; v < 5; ++v) s[v] = FA(s[v], FM(v == 4 ? FM(wz, wz) : wz, xy[v * vs + o]));
    }
    // A = sum dV a / dx^3, B = (sum dV |a|^2 - sum dV^2 |a|^2) / dx^6
    const float Ax = FM(s[0], inv3), Ay = FM(s[1], inv3), Az = FM(s[2], inv3);
    const float B = FM(FS(s[3], s[4]), inv6);
    const float r = r_[i], mx0 = px[i], my0 = py[i], mz0 = pz[i];
    const float pa = FA(FA(FM(mx0, Ax), FM(my0, Ay)), FM(mz0, Az));
    const float a2 = FA(FA(FM(Ax, Ax), FM(Ay, Ay)), FM(Az, Az));
    e_[i] = FA(e_[i], FA(FA(pa, FM(FM(0.5f, r), a2)), FM(FM(0.5f, r), B)));
    px[i] = FA(mx0, FM(r, Ax));
    py[i] = FA(my0, FM(r, Ay));
    pz[i] = FA(mz0, FM(r, Az));
  }
}

// largest divisor of n not above m
int pick_tile(int n, int m) {
  for (int t = std::min(n, m); t > 1; --t)
    if (n % t == 0) return t;
  return 1;
}

int grid_for(const cube_ctx* ctx, int64_t work, int threads) {
  const int64_t b = (work + threads - 1) / threads;
  const int64_t cap = (int64_t)ctx->num_sms * 16;
  return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace

__global__ void k_nu_fill(float* __restrict__ p, int64_t n, float v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

// ---- launchers -----------------------------------------------------------------
// hg_setup's initial state (hydrogr.f90:79-85, q_EQN_OF_STATE): rho = 1, m = 0,
// E = cs2*rho/(g-1)
int cube_nu_init(cube_ctx* ctx, NuFluid& F) {
  const int64_t n3 = (int64_t)F.n * F.n * F.n;
  const int g = grid_for(ctx, n3, 256);
  k_nu_fill<<<g, 256, 0, ctx->stream>>>(F.a[0], n3, 1.f);
  CUBE_LAUNCH_CHECK(ctx);
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(F.a[1], 0, sizeof(float) * 3 * n3, ctx->stream));
  k_nu_fill<<<g, 256, 0, ctx->stream>>>(F.a[4], n3, cube_fdiv(cube_fmul(F.cs2, 1.f), cube_fsub(ctx->nu.g, 1.f)));
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

int cube_nu_sweeps(cube_ctx* ctx, NuFluid& F, float dt, int dir) {
  const int n = F.n;
  for (int step = 0; step < 3; ++step) {
    const int ax = dir > 0 ? step : 2 - step;
    SweepArgs A;
    for (int c = 0; c < 5; ++c) { A.in[c] = F.a[c]; A.out[c] = F.b[c]; }
    A.n = n;
    A.gm1 = cube_fsub(ctx->nu.g, 1.f);
    A.dt = dt;
    A.inv_dx = 1.f / F.dx;
    if (ax == 0) { A.ts = pick_tile(n, 64); A.tx = pick_tile(n, 16); }
    else { A.ts = pick_tile(n, 32); A.tx = pick_tile(n, 32); }
    const size_t smem = sizeof(float) * (size_t)5 * A.tx * ((A.ts + 4) + (A.ts + 1));
    dim3 grid((unsigned)((n / A.ts) * (n / A.tx)), (unsigned)n);
    if (ax == 0) {
      CUBE_CUDA_TRY(ctx, cube_smem_limit(k_nu_sweep<0>, smem));
      k_nu_sweep<0><<<grid, 256, smem, ctx->stream>>>(A);
    } else if (ax == 1) {
      CUBE_CUDA_TRY(ctx, cube_smem_limit(k_nu_sweep<1>, smem));
      k_nu_sweep<1><<<grid, 256, smem, ctx->stream>>>(A);
    } else {
      CUBE_CUDA_TRY(ctx, cube_smem_limit(k_nu_sweep<2>, smem));
      k_nu_sweep<2><<<grid, 256, smem, ctx->stream>>>(A);
    }
    CUBE_LAUNCH_CHECK(ctx);
    for (int c = 0; c < 5; ++c) std::swap(F.a[c], F.b[c]);
  }
  return CUBE_OK;
}

int cube_nu_timestep(cube_ctx* ctx, NuFluid& F, unsigned int* dt_bits) {
  k_nu_dt<<<(unsigned)((int64_t)F.n * F.n), 128, 0, ctx->stream>>>(F.a[0], F.a[1], F.a[2], F.a[3], F.a[4], F.n,
                                                                   cube_fsub(ctx->nu.g, 1.f), F.dx, dt_bits);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

int cube_nu_transpose(cube_ctx* ctx, NuFluid& F, int to_soa) {
  const int64_t n3 = (int64_t)F.n * F.n * F.n;
  const int g = grid_for(ctx, 5 * n3, 256);
  // the AoS staging copy lives in the b arrays, which are one contiguous block
  if (to_soa) k_nu_aos_to_soa<<<g, 256, 0, ctx->stream>>>(F.b[0], F.a[0], n3);
  else k_nu_soa_to_aos<<<g, 256, 0, ctx->stream>>>(F.a[0], F.b[0], n3);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

int cube_nu_density(cube_ctx* ctx, cube_scalars* io) {
  NuState& N = ctx->nu;
  MeshLevel& L = ctx->fine;
  const int homogeneous = cube_fsub(cube_fdiv(1.f, io->a_mid), 1.f) > ctx->P.z_i_nu;
  Rho3 R;
  for (int k = 0; k < 3; ++k) {
    R.r[k] = N.fl[k].a[0];
    R.n[k] = N.fl[k].n;
    R.dx[k] = N.fl[k].dx;
    R.w[k] = N.dwgts[k];
  }
  float* scratch = L.force;  // free until the force is computed
  const int nbricks = (L.n / DBX) * (L.n / DBY) * (L.n / DBZ);
  k_nu_fine_density<<<nbricks, 256, 0, ctx->stream>>>(R, homogeneous, ctx->P.f_neu, L.n, L.rho, L.rp, L.plane,
                                                      scratch, N.partial);
  CUBE_LAUNCH_CHECK(ctx);
  const float hom = cube_fmul(ctx->P.f_neu, (float)(ctx->ncell * ctx->ncell * ctx->ncell));
  k_nu_coarse_deposit<<<grid_for(ctx, ctx->ncells, 256), 256, 0, ctx->stream>>>(
      scratch, L.n, L.rp, L.plane, ctx->nc, homogeneous, hom, ctx->rho_c_nu);
  CUBE_LAUNCH_CHECK(ctx);
  return CUBE_OK;
}

int cube_nu_gravity(cube_ctx* ctx, cube_scalars* io) {
  NuState& N = ctx->nu;
  if (!(io->a_mid >= N.ai)) return CUBE_OK;  // dfld_gravity: a < ai leaves the fluids alone
  GravArgs G;
  MeshLevel& F = ctx->fine;
  MeshLevel& C = ctx->coarse;
  G.ff = F.force; G.fcomp = (size_t)F.n * F.plane; G.fplane = F.plane; G.frp = F.rp;
  G.fc = C.force; G.ccomp = (size_t)C.n * C.plane; G.cplane = C.plane; G.crp = C.rp;
  G.nf = F.n; G.nc = ctx->nc;
  G.a_mid = io->a_mid; G.dt = io->dt; G.pi_f = ctx->codec.pi_f;
  G.nfl = 3;
  for (int k = 0; k < 3; ++k) { G.fn[k] = N.fl[k].n; G.fdx[k] = (int)N.fl[k].dx; G.xy[k] = N.fl[k].xy; }
  dim3 grid((unsigned)((F.n / GT) * (F.n / GT)), (unsigned)(F.n + 4));
  k_nu_src_xy<<<grid, 256, 0, ctx->stream>>>(G);
  CUBE_LAUNCH_CHECK(ctx);
  for (int k = 0; k < 3; ++k) {
    NuFluid& Fl = N.fl[k];
    const int64_t n3 = (int64_t)Fl.n * Fl.n * Fl.n;
    k_nu_grav_z<<<grid_for(ctx, n3, 256), 256, 0, ctx->stream>>>(Fl.xy, F.n, Fl.n, (int)Fl.dx, Fl.a[0], Fl.a[1],
                                                                  Fl.a[2], Fl.a[3], Fl.a[4]);
    CUBE_LAUNCH_CHECK(ctx);
  }
  return CUBE_OK;
}
