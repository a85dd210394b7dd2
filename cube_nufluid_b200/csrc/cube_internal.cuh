/*
 * cube_internal.cuh -- device state and launch helpers of the B200 PM step.
 *
 * Device layout (one image on one GPU; tiles are only an ordering):
 *   cell id   c = ((tz*nnt+ty)*nnt+tx)*nt^3 + (lz*nt+ly)*nt + lx
 *             (Fortran rhoc(lx,ly,lz,tx,ty,tz) order, variables.f90:65)
 *   particles cell-sorted, each particle stored once (no buffer copies);
 *             SoA: xp[d][cap], vp[d][cap] (1 or 2 bytes), pid[cap]
 *   cell_start[c] (int64, exclusive prefix of rhoc), vfield[d][ncells]
 *   fine mesh nf^3 with row pitch rp = nf+32 floats (128-byte rows), used
 *             in place as the half spectrum (complex pitch cp = rp/2)
 *   coarse mesh nc^3, same convention
 */
#ifndef CUBE_INTERNAL_CUH
#define CUBE_INTERNAL_CUH

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/cube_gpu.h"
#include "cube_codec.h"

#define CUBE_MAX_RADIX_STAGES 12

struct FftPlan {
  int n;                          // transform length
  int nst;                        // number of stages
  int radix[CUBE_MAX_RADIX_STAGES];
  float2* tw;                     // device twiddles exp(-2 pi i j/n), j < n
  float2* tw2;                    // register-FFT twiddles tw[(t*k1) mod n] at [k1*T + t] (n = R*T)
  double2* twd;                   // tw in FP64 (FP64 Poisson mode)
};

// R x T split of the register-resident transforms (T threads of one warp, R
// points each); false for lengths they do not cover
inline bool cube_fast_rt(int n, int* R, int* T) {
  switch (n) {
    case 1024: *R = 32; *T = 32; return true;
    case 512: *R = 32; *T = 16; return true;
    case 256: *R = 16; *T = 16; return true;
    case 128: *R = 16; *T = 8; return true;
    case 64: *R = 8; *T = 8; return true;
    case 32: *R = 8; *T = 4; return true;
    case 768: *R = 48; *T = 16; return true;
    case 384: *R = 48; *T = 8; return true;
    case 192: *R = 24; *T = 8; return true;
    case 96: *R = 24; *T = 4; return true;
    default: return false;
  }
}

struct MeshLevel {
  int n;          // mesh points per dimension
  int rp;         // real row pitch (floats)
  int cp;         // complex row pitch (float2) = rp/2
  size_t plane;   // floats per z-plane = n*rp
  float* rho;     // density, in place as the forward half spectrum
  float* force;   // [3] force meshes, each n*plane floats, in place as spectra
  float* ext;     // scratch mesh (n*plane floats) for the transposed passes
  float* kern;    // Green multiplier (imaginary parts, /n^3)
  double* kernd = nullptr;  // the same in FP64 (FP64 Poisson mode, else null)
  int fp64 = 0;             // 1: rho, force and ext hold doubles (same element pitches)
  int kern_octant;  // 1: kern is [3][(n/2+1)^3] octant; 0: [3][n][n][cp_k]
  int kern_pitch;   // inner pitch of kern (n/2+1)
  FftPlan plan;
};

struct DevScal {
  unsigned int f2_fine_bits;   // max f^2 as float bits (non-negative floats order as ints)
  unsigned int f2_coarse_bits;
  unsigned int vmax_bits[3];
  unsigned int f2_pp_bits;
  int err;                     // first error code seen on the device
  int err_info;
  unsigned long long n_big;    // re-bin cells for the warp sorter (PP: spilled bricks)
  unsigned long long itest1, npairs;
  unsigned long long moved_far;
  unsigned int nu_dt_bits[3];  // per-fluid CFL step as float bits
  unsigned long long n_huge;   // re-bin cells beyond the shared-memory sorter
  unsigned long long max_huge; // the most particles in one of them
  unsigned long long n_mid;    // re-bin cells for the block sorter (beyond the warp sorter)
  unsigned long long huge_next;  // next cell for a k_rebin_huge block
  unsigned long long n_items;    // re-bin work items beyond the one per 64-cell group
  unsigned long long mid_next;   // next cell for a k_rebin_big block
  unsigned long long n_dep_extra;  // deposit work items beyond one per brick
  unsigned long long n_split;      // bricks whose particles are split over several deposit blocks
  unsigned long long pp_list;      // PP targets with a neighbour, listed for the pair pass
  unsigned long long pp_dense;     // PP bricks whose region holds a crowded cell
};

// one isothermal fluid of the dispersive sum (hydrogr.f90 type hydro): five FP32
// arrays of n^3 cells, x fastest, periodic; a = current state, b = the other
// half of the ping-pong (each is one contiguous block of 5 n^3)
struct NuFluid {
  int n = 0, ncb = 0;              // cells per side; halo width of the reference layout
  float dx = 0.f, cs2 = 0.f, dv = 0.f;
  float* a[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float* b[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  float* block[2] = {nullptr, nullptr};
  float* xy = nullptr;             // gravity scratch [5][nf+4][n][n]
};

// fluid neutrinos of one species (hydrodf.f90 type dfld)
struct NuState {
  bool on = false;
  float beta = 0.f, g = 0.f, ai = 0.f;
  float dwgts[3] = {0.f, 0.f, 0.f};
  NuFluid fl[3];
  double* partial = nullptr;       // per-CTA sums of the fine neutrino density
  int nparts = 0;
};

struct cube_ctx {
  cube_params P;
  int nc, nnt, nt, ncell, ncb, nte, nf, nvbin;
  int64_t ncells;
  int izipx, izipv;
  cube_codec codec;
  cudaStream_t stream;
  int own_stream;
  int64_t np, cap;
  int state_loaded;
  int cells_le32;  // the last re-bin left no cell beyond 32 particles (no deposit brick needs splitting)
  int num_sms;
  // particles (double-buffered for the re-bin)
  void* xp;  void* vp;  int32_t* pid;
  void* xp2; void* vp2; int32_t* pid2;
  int32_t* rhoc;  int32_t* rhoc2;
  int64_t* cell_start; int64_t* cell_start2;
  float* vfield; float* vfield2;
  // re-bin scratch
  int32_t* tcell; uint32_t* tkey; int32_t* perm; uint32_t* pkey; int32_t* cursor;
  int32_t* big_list;
  int64_t* rebin_items;  // [4] per item: first cell, cells, first and end particle
  double* cell_stats;   // [3][ncells]
  double* slot_r2; double* slot_s2;  // re-bin scratch: each slot's new cell (int32), tree block sums
  double* red_tmp;      // scratch for tree sums
  int64_t* scan_tmp;
  NuState nu;
  double* pk_bins;  // power-spectrum bin sums, 7 * (bins of the fine mesh + 1)
  double* vdec[2] = {nullptr, nullptr};  // decoded velocity per code, tan(code)/coef, for two coefs
  double vdec_coef[2] = {0.0, 0.0};
  int vdec_next = 0;
  void* pp_scratch = nullptr;     // sorted particles of crowded PP bricks, grown on demand
  size_t pp_scratch_bytes = 0;
  void* rebin_scratch = nullptr;  // sort slots of re-bin cells beyond 4096 particles, grown on demand
  size_t rebin_scratch_bytes = 0;
  void* rebin_mid_scratch = nullptr;  // velocity columns of the block sorter, allocated on first use
  void* dep_scratch = nullptr;   // fine nodes and block counters of split deposit bricks, grown on demand
  size_t dep_scratch_bytes = 0;
  // meshes
  MeshLevel fine, coarse;
  unsigned long long* rho_c_acc;  // coarse particle sums, 64-bit fixed point without the mass (scale 2^38)
  unsigned long long* rho_c_nu;   // coarse neutrino sums, 64-bit fixed point in mass units (scale 2^32)
  double* dep_partial;            // per-CTA fine mass partial sums
  int64_t dep_blocks;
  float* tan_table;               // tanf of each velocity code, index code+nvbin/2
  struct VencBrk* venc_brk;       // angle breakpoints of cube_vencode_brk (64 entries)
  DevScal* dscal;                 // device scalars
  DevScal* hscal;                 // pinned host mirror
  float2* sbuf;                   // spare spectrum buffer for the forward z pass
  // timing
  cudaEvent_t ev[16];
  float phase_ms[8];
  long long launches;
  std::string err;
};

// ---- error helpers ---------------------------------------------------------
#define CUBE_CUDA_TRY(ctx, call)                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);             \
      return CUBE_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

#define CUBE_LAUNCH_CHECK(ctx)                                                     \
  do {                                                                             \
    (ctx)->launches++;                                                             \
    cudaError_t e_ = cudaGetLastError();                                           \
    if (e_ != cudaSuccess) {                                                       \
      (ctx)->err = std::string("launch: ") + cudaGetErrorString(e_);               \
      return CUBE_ERR_CUDA;                                                        \
    }                                                                              \
  } while (0)

__device__ __forceinline__ void cube_dev_error(DevScal* s, int code, int info) {
  if (atomicCAS(&s->err, 0, code) == 0) s->err_info = info;
}

// Raises a kernel's dynamic shared-memory limit to the most the device allows beside
// the kernel's static shared memory.  The limit is a per-kernel global, so contexts on
// other host threads launching the same kernel with other sizes must never see it
// lowered under them: it is only ever set to that one value.  Fails if the launch
// would need more.
template <typename F>
inline cudaError_t cube_smem_limit(F* func, size_t bytes) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, func);
  if (e != cudaSuccess) return e;
  const size_t lim = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
  if (bytes > lim) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim);
}

// device-side view of the particle codes
template <int Z>
struct CodeT;
template <>
struct CodeT<1> { typedef int8_t T; };
template <>
struct CodeT<2> { typedef int16_t T; };

__device__ __forceinline__ int64_t cube_cell_of(int gx, int gy, int gz, int nt, int nnt) {
  const int tx = gx / nt, ty = gy / nt, tz = gz / nt;
  const int lx = gx - tx * nt, ly = gy - ty * nt, lz = gz - tz * nt;
  return ((((int64_t)tz * nnt + ty) * nnt + tx) * nt + lz) * (int64_t)nt * nt + (int64_t)ly * nt + lx;
}

// periodic wrap of an index that lies in [-n, 2n)
__device__ __forceinline__ int cube_wrap(int x, int n) {
  x += (x < 0) ? n : 0;
  return x - ((x >= n) ? n : 0);
}

// tile-major cell id -> coordinates inside its tile (l) and the tile's first
// global coarse cell per dimension (tb = tile index * nt)
__device__ __forceinline__ void cube_cell_coords(int64_t c, int nt, int nnt, int l[3], int tb[3]) {
  const int nt3 = nt * nt * nt;
  const int64_t tile = c / nt3;
  const int rem = (int)(c - tile * nt3);
  const int t2 = (int)tile;  // < nnt^3 < 2^31
  l[0] = rem % nt;
  l[1] = (rem / nt) % nt;
  l[2] = rem / (nt * nt);
  tb[0] = (t2 % nnt) * nt;
  tb[1] = ((t2 / nnt) % nnt) * nt;
  tb[2] = (t2 / (nnt * nnt)) * nt;
}

// The kick chain of the reference, (((f*a_mid)*dt)/6)/pi (pm.f90:146,163,358,393),
// is the same for every particle that reads a force node.  cube_particle_mesh folds
// the scalar ((a_mid*dt)/6)/pi into the Green multiply, so the force meshes come
// out of the inverse FFT as kick increments (to FP32 rounding, like the force
// itself); forces given from outside (cube_debug_kick_with_force) get the exact
// per-node chain below.
struct KickScale {
  float a_mid, dt, pi_f;
  int on;
  float inv6, inv_pi;  // RN(1/6), RN(1/pi_f)
};

// RN(x/y) for a constant y with z = RN(1/y): q0 = RN(x z), r = fma(-q0, y, x),
// q = fma(r, z, q0) (Brisebarre, Muller and Raina, IEEE Trans. Computers 53(8),
// 2004).  For y = 6 and y = pi_f the result equals IEEE division for every finite
// FP32 x with |x| >= 2^-100 (checked over all 2^32 inputs by the CPU tests); smaller
// and non-finite x take the IEEE division.
__device__ __forceinline__ float cube_div_const(float x, float y, float z) {
  const float ax = fabsf(x);
  if (!(ax >= 7.88860905e-31f && ax <= 3.40282347e38f)) return __fdiv_rn(x, y);
  const float q0 = __fmul_rn(x, z);
  const float r = __fmaf_rn(-q0, y, x);
  return __fmaf_rn(r, z, q0);
}

// RN(a/b) from y = RN(1/b) for b > 0 (normal) and finite a, by two FMA corrections
// of q0 = RN(a y): the first gives a quotient within one ulp of a/b, and then, y being
// within half an ulp of 1/b, RN(q + (a - b q) y) with the exact FMA residual is the
// correctly rounded quotient (Markstein's theorem; Markstein, IBM J. Res. Dev. 34(1),
// 1990; Muller et al., Handbook of Floating-Point Arithmetic, sec. 4.7).  It replaces
// IEEE divisions by one b shared by several a; cube_debug_division_check compares it
// with the IEEE division on the GPU.
__device__ __forceinline__ double cube_div_rcp(double a, double b, double y) {
  double q = __dmul_rn(a, y);
  double r = __fma_rn(-b, q, a);
  q = __fma_rn(r, y, q);
  r = __fma_rn(-b, q, a);
  return __fma_rn(r, y, q);
}

inline float cube_kick_scalar(const KickScale& k) {
  return k.on ? cube_fdiv(cube_fdiv(cube_fmul(k.a_mid, k.dt), 6.f), k.pi_f) : 1.f;
}

__device__ __forceinline__ float cube_kick_scale(float f, const KickScale& k) {
  const float t = __fmul_rn(__fmul_rn(f, k.a_mid), k.dt);
  return cube_div_const(cube_div_const(t, 6.f, k.inv6), k.pi_f, k.inv_pi);
}

// FP64 reciprocal from an FP32 seed and two Newton steps (relative error below 2^-49)
__device__ __forceinline__ double cube_rcp_fast(double b) {
  double y = (double)__fdividef(1.0f, (float)b);
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  return fma(y, e, y);
}

struct VencBrk;
struct VencTab {
  const VencBrk* brk;   // 64 angle breakpoints (cube_vencode_brk)
  double qscale_d;      // nvbin_m1 * (1/pi_f)
};
inline VencTab cube_venc_tab(const cube_ctx* ctx) {
  return VencTab{ctx->venc_brk, (double)ctx->codec.nvbin_m1_f * (1.0 / (double)ctx->codec.pi_f)};
}

// Velocity encode by angle breakpoints, with no reciprocal reduction and no table
// read on the dependent chain beyond 32 bytes that stay in L1.  With theta_j =
// (j + 1/2)*pi/128, c_j = tan(theta_j), j = 0..63 (extended-precision values, theta_j
// split hi + lo), atan(x) = theta_j + atan(u), u = (x - c_j)/(1 + x c_j).  j comes
// from an FP32 arctangent guess (least-squares polynomial in t^2 on [0,1], |error|
// < 1.8e-6 over every float t, reciprocal above 1; with its roundings < 2e-6), so |u| <=
// tan(pi/256 + 2e-6) < 0.0123 for every x >= 0 (c_63 = 81.6 bounds u by 1/c_63 as
// x grows), and atan(u) = u - u^3/3 + u^5/5 - u^7/7 leaves out less than 1e-18.  The
// quotient takes the FP32-seeded Newton reciprocal (relative error < 2^-49, which
// moves atan by < 3e-17 at this |u|); with the roundings of the sum and of
// q = nvbin_m1*atan*(1/pi_f), q is within 3e-11 of the exact evaluation's, so as in
// the exact evaluation's own error (< 3e-11) the integer is accepted unless q lies
// within 1e-9 of k + 1/2; there the exact FP64 evaluation decides.
struct VencBrk {
  double c, hi, lo, pad;  // tan(theta_j), theta_j = hi + lo
};

__device__ __forceinline__ int32_t cube_vencode_brk(const cube_codec* c, const VencBrk* __restrict__ brk, double v,
                                                    double coef, double qscale) {
  const double x = cube_dmul(coef, v);
  const double ax = fabs(x);
  if (!(ax < 1e30)) return cube_vencode(c, v, coef);  // beyond the FP32 guess's range, or NaN
  const float af = __double2float_rn(ax);
  const bool big = af > 1.f;
  const float t = big ? __fdividef(1.f, af) : af;
  const float s = __fmul_rn(t, t);
  float p = -0.011719122529029846f;
  p = __fmaf_rn(p, s, 0.052647314965724945f);
  p = __fmaf_rn(p, s, -0.11642644554376602f);
  p = __fmaf_rn(p, s, 0.19354036450386047f);
  p = __fmaf_rn(p, s, -0.33262282609939575f);
  p = __fmaf_rn(p, s, 0.9999772310256958f);
  const float a = __fmul_rn(t, p);
  const float th = big ? __fsub_rn(1.5707963267948966f, a) : a;
  const int j = min(max(__float2int_rd(__fmul_rn(th, 40.743665431525205f)), 0), 63);  // 128/pi
  const double2 ch = __ldg(reinterpret_cast<const double2*>(brk + j));
  const double lo = __ldg(&brk[j].lo);
  const double num = cube_dsub(ax, ch.x);
  const double den = cube_dfma(ax, ch.x, 1.0);
  const double u = cube_dmul(num, cube_rcp_fast(den));
  const double u2 = cube_dmul(u, u);
  double q7 = cube_dfma(-1.0 / 7.0, u2, 1.0 / 5.0);
  q7 = cube_dfma(q7, u2, -1.0 / 3.0);
  const double at = cube_dadd(ch.y, cube_dadd(cube_dfma(cube_dmul(u, u2), q7, u), lo));
  const double q = cube_dmul(at, qscale);  // |q|, atan >= 0 here
  const double fl = floor(q);
  const double fr = q - fl;  // exact
  if (fabs(fr - 0.5) < 1e-9) return cube_vencode(c, v, coef);
  const int32_t n = (int32_t)fl + (fr > 0.5 ? 1 : 0);
  return x < 0.0 ? -n : n;
}

// the encode of the step's kernels (kick, PP, re-bin, decode-table fixed points)
__device__ __forceinline__ int32_t cube_vencode_step(const cube_codec* c, const VencTab& T, double v, double coef) {
  return cube_vencode_brk(c, T.brk, v, coef, T.qscale_d);
}

// ---- launchers (implemented in the k_*.cu files) -----------------------------
int cube_rebin(cube_ctx* ctx, cube_scalars* io);
int64_t cube_rebin_items_max(int64_t ncells, int64_t cap);
// work items over the cells of cell_start into ctx->rebin_items (a run of at most
// 64 cells and at most 4096 of its particles each); *blocks = launch size, one
// block per item, blocks past the last return (cube_cell_item)
int cube_cell_items(cube_ctx* ctx, const int64_t* cell_start, int64_t* blocks);
__device__ __forceinline__ bool cube_cell_item(const int64_t* items, int64_t ncells, int64_t items_max,
                                               const DevScal* dscal, int64_t& c0, int& ncl, int64_t& p0, int64_t& p1) {
  const int64_t ngroups = (ncells + 63) / 64;
  const int64_t b = blockIdx.x;
  if (b >= ngroups + (int64_t)dscal->n_items || b >= items_max) return false;
  const int64_t* it = items + 4 * b;
  c0 = it[0]; ncl = (int)it[1]; p0 = it[2]; p1 = it[3];
  return true;
}
int cube_deposit(cube_ctx* ctx, cube_scalars* io);
// mass sums of a deposit (pm.f90:108,280) from the three totals it leaves at the
// start of red_tmp: fine and coarse particle sums without the mass (scale 2^32) and
// the coarse neutrino sum (mass units, scale 2^32); the caller adds the fine
// neutrino sum
inline void cube_mass_sums(const unsigned long long mt[3], float mass, double* testrhof, double* testrhoc) {
  const double m = (double)mass, s = 1.0 / 4294967296.0;
  *testrhof = (double)mt[0] * s * m;
  *testrhoc = (double)mt[1] * s * m + (double)mt[2] * s;
}
int cube_fft_poisson(cube_ctx* ctx, MeshLevel& L, unsigned int* f2_bits, KickScale ks);
int cube_force_scale(cube_ctx* ctx, MeshLevel& L, KickScale ks);
int cube_fft_forward3(cube_ctx* ctx, MeshLevel& L, float* data, int* kx_major);
int cube_pk_nbin(int ng, int logbins);
int cube_power_spectrum_dev(cube_ctx* ctx, int logbins, std::vector<double>& bins, int* nbin_out);
int cube_fft_forward3_fast(cube_ctx* ctx, MeshLevel& L, float* data, int* rc, int* kx_major);
int cube_fft_poisson_fast(cube_ctx* ctx, MeshLevel& L, unsigned int* f2_bits, KickScale ks, int* rc);
int cube_kick(cube_ctx* ctx, cube_scalars* io);
int cube_pp(cube_ctx* ctx, cube_scalars* io);
int cube_build_green(cube_ctx* ctx, const float* fk_table, const float* ck_table);
int cube_tree_sum_dev(cube_ctx* ctx, const double* in, int64_t n, double* out_host);
// the per-particle velocity statistics of update_x, sum |v_res|^2 and sum |v|^2, in the
// new layout from its codes, its cell means and each slot's cell (slot_cell)
int cube_stats_sums(cube_ctx* ctx, const int32_t* slot_cell, const double* dec, double* sum_r, double* sum_s);
int cube_exclusive_scan(cube_ctx* ctx, const int32_t* in, int64_t n, int64_t* out);
int cube_fft_plan(cube_ctx* ctx, FftPlan& p, int n);
int cube_nu_init(cube_ctx* ctx, NuFluid& F);
int cube_nu_sweeps(cube_ctx* ctx, NuFluid& F, float dt, int dir);
int cube_nu_timestep(cube_ctx* ctx, NuFluid& F, unsigned int* dt_bits);
int cube_nu_transpose(cube_ctx* ctx, NuFluid& F, int to_soa);
int cube_nu_density(cube_ctx* ctx, cube_scalars* io);
int cube_nu_gravity(cube_ctx* ctx, cube_scalars* io);
int cube_fft_r2c_x(cube_ctx* ctx, MeshLevel& L, float* data, int inverse, int ncomp, unsigned int* f2_bits);
int cube_make_ic_dev(cube_ctx* ctx, const cube_ic_params* icp, cube_scalars* io);
int cube_halofind_dev(cube_ctx* ctx, const cube_scalars* io, const cube_halo_args* ha, cube_halo_result* res);
// device table of cube_vdecode(tan_table[c], coef) for every code c (index code + nvbin/2),
// built on first use of a coefficient; the last two coefficients stay cached.  After
// the nvbin doubles follow nvbin/32 words of cube_vfixed bits.
const double* cube_vdec_table(cube_ctx* ctx, double coef, int* rc);

// true if re-encoding the decoded velocity of code index c (code + nvbin/2) at the
// table's coefficient, cube_wrap_code(cube_vencode_step(v)), gives the code back: a
// velocity kicked by exactly zero then keeps its code
__device__ __forceinline__ bool cube_vfixed(const double* dec, int nvbin, int c) {
  return (reinterpret_cast<const uint32_t*>(dec + nvbin)[c >> 5] >> (c & 31)) & 1u;
}

#endif
