/*
 * cube_api.cu -- the C-ABI of include/cube_gpu.h: context, state transfer and
 * the step entry points that replace particle_mesh, update_x, ext_pp_force
 * and timestep of the reference.
 */
#include "cube_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

static std::string g_create_error;

namespace {

template <typename T>
__global__ void k_aos_to_soa(const T* __restrict__ aos, T* __restrict__ soa, int64_t n, int64_t cap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    soa[i] = aos[3 * i];
    soa[cap + i] = aos[3 * i + 1];
    soa[2 * cap + i] = aos[3 * i + 2];
  }
}

template <typename T>
__global__ void k_soa_to_aos(const T* __restrict__ soa, T* __restrict__ aos, int64_t n, int64_t cap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    aos[3 * i] = soa[i];
    aos[3 * i + 1] = soa[cap + i];
    aos[3 * i + 2] = soa[2 * cap + i];
  }
}

// fine (octant) multiplier for debug fetch: straight copy; mesh copy with pitch
template <typename T>
__global__ void k_unpitch(const T* __restrict__ src, T* __restrict__ dst, int n, int rp, int ncomp) {
  const int64_t n3 = (int64_t)n * n * n;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n3 * ncomp; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = q / n3, r = q - c * n3;
    const int64_t x = r % n, yz = r / n;
    dst[q] = src[c * (int64_t)n * n * rp + yz * rp + x];
  }
}

__global__ void k_pitch(const float* __restrict__ src, float* __restrict__ dst, int n, int rp, int ncomp) {
  const int64_t n3 = (int64_t)n * n * n;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n3 * ncomp; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = q / n3, r = q - c * n3;
    const int64_t x = r % n, yz = r / n;
    dst[c * (int64_t)n * n * rp + yz * rp + x] = src[q];
  }
}

int alloc_level(cube_ctx* ctx, MeshLevel& L, int n, int fp64) {
  L.n = n;
  L.rp = n + 32;
  L.cp = L.rp / 2;
  L.plane = (size_t)n * L.rp;
  L.fp64 = fp64;
  const size_t vol = (size_t)n * L.plane;
  const size_t es = fp64 ? sizeof(double) : sizeof(float);  // the pitches count elements
  CUBE_CUDA_TRY(ctx, cudaMalloc(&L.rho, es * vol));
  CUBE_CUDA_TRY(ctx, cudaMalloc(&L.force, es * 3 * vol));
  CUBE_CUDA_TRY(ctx, cudaMalloc(&L.ext, es * vol));
  const int kp = n / 2 + 1;
  L.kern_octant = 1;
  L.kern_pitch = kp;
  CUBE_CUDA_TRY(ctx, cudaMalloc(&L.kern, sizeof(float) * 3 * (size_t)kp * kp * kp));
  L.kernd = nullptr;
  if (fp64) CUBE_CUDA_TRY(ctx, cudaMalloc(&L.kernd, sizeof(double) * 3 * (size_t)kp * kp * kp));
  CUBE_CUDA_TRY(ctx, cudaMemset(L.rho, 0, es * vol));
  CUBE_CUDA_TRY(ctx, cudaMemset(L.force, 0, es * 3 * vol));
  return cube_fft_plan(ctx, L.plan, n);
}

int check_device_error(cube_ctx* ctx) {
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->hscal, ctx->dscal, sizeof(DevScal), cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->hscal->err) {
    const int e = ctx->hscal->err;
    ctx->err = "device error " + std::to_string(e) + " (info " + std::to_string(ctx->hscal->err_info) + ")";
    return e;
  }
  return CUBE_OK;
}

float uint_as_float(unsigned int u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}

unsigned int float_as_uint(float f) {
  unsigned int u;
  memcpy(&u, &f, 4);
  return u;
}

/* sim%vsim2phys of particle_mesh (pm.f90:427), FP32 as the reference */
float vsim2phys(const cube_ctx* ctx, float a) {
  float v = cube_fdiv(1.5f, a);
  v = cube_fmul(v, ctx->P.box);
  v = cube_fmul(v, ctx->P.h0);
  v = cube_fmul(v, 100.f);
  v = cube_fmul(v, sqrtf(ctx->P.omega_m));
  return cube_fdiv(v, (float)ctx->nf);
}

/* dt constraints of particle_mesh (pm.f90:427-443), FP32 as the reference */
void dt_constraints(const cube_ctx* ctx, cube_scalars* s) {
  const float pi_f = ctx->codec.pi_f;
  const float GG = cube_fdiv(cube_fdiv(1.0f, 6.0f), pi_f);  // variables.f90:22
  s->vsim2phys = vsim2phys(ctx, s->a);
  s->dt_fine = sqrtf(cube_fdiv(1.0f, cube_fmul(cube_fmul(sqrtf(s->f2_max_fine), s->a_mid), GG)));
  s->dt_coarse = sqrtf(cube_fdiv((float)ctx->ncell, cube_fmul(cube_fmul(sqrtf(s->f2_max_coarse), s->a_mid), GG)));
  const float vm = std::max(s->vmax[0], std::max(s->vmax[1], s->vmax[2]));
  s->dt_vmax = cube_fdiv(cube_fmul(ctx->P.vbuf, 20.f), vm);
  s->vz_max = s->vmax[2];
  // vmax_nu is zeroed at pm.f90:40 and nothing raises it in the fluid model
  if (ctx->nu.on) s->dt_vmax_nu = cube_fdiv(cube_fmul(ctx->P.vbuf, 20.f), 0.f);
}

// dfld_setup / hg_setup (hydrodf.f90:53-84, hydrogr.f90:39-90) for one species of
// mass m_nu_ev with gamma = 5/3 (main.f90:38), on the host in FP32 with the C
// library's expf, then the device arrays in their initial state
int setup_neutrinos(cube_ctx* ctx) {
  const cube_params& P = ctx->P;
  NuState& N = ctx->nu;
  const int nf = ctx->nf;
  const float GLv[3] = {0.41577456f, 2.29428036f, 6.28994508f};
  const float GLw[3] = {0.71109301f, 0.27851773f, 0.01038926f};
  N.g = 5.f / 3.f;
  N.beta = cube_fmul(5966.34f, P.m_nu_ev);
  N.ai = cube_fdiv(1.f, cube_fadd(1.f, P.z_i_nu));  // NEUTRINO_IC: ai = ai_max (hydrodf.f90:13-15,96-97)
  const float hg_dv = cube_fdiv((float)(2 * nf), cube_fmul(cube_fmul(300.f, sqrtf(P.omega_m)), P.box));
  const int hg_nfb = P.ncb * P.ncell;
  float wsum = 0.f;
  for (int k = 0; k < 3; ++k) {
    NuFluid& F = N.fl[k];
    F.n = P.nu_nc[k] > 0 ? P.nu_nc[k] : nf >> (k + 1);
    if (F.n < 4 || nf % F.n || (nf / F.n != 2 && nf / F.n != 4 && nf / F.n != 8) || nf % 32) {
      ctx->err = "fluid meshes must be nf/2, nf/4 or nf/8 cells per side (>= 4), with nf a multiple of 32";
      return CUBE_ERR_PARAM;
    }
    F.dx = cube_fdiv(cube_fmul(1.f, (float)nf), (float)F.n);
    F.dv = hg_dv;
    F.ncb = std::max(2, 1 + (int)floorf(cube_fdiv((float)hg_nfb, F.dx)));
    const float v = cube_fmul(cube_fdiv(GLv[k], N.beta), 2.998e5f);
    const float t = cube_fmul(v, F.dv);
    F.cs2 = std::max(1e-6f, cube_fmul(t, t));
    const float f0 = cube_fdiv(cube_fmul(GLv[k], GLv[k]), cube_fadd(expf(GLv[k]), 1.f));
    N.dwgts[k] = cube_fmul(cube_fmul(GLw[k], f0), expf(GLv[k]));
    wsum = (k == 0) ? N.dwgts[0] : cube_fadd(wsum, N.dwgts[k]);
  }
  for (int k = 0; k < 3; ++k) N.dwgts[k] = cube_fdiv(N.dwgts[k], wsum);
  for (int k = 0; k < 3; ++k) {
    NuFluid& F = N.fl[k];
    const size_t n3 = (size_t)F.n * F.n * F.n;
    if (cudaMalloc((void**)&F.block[0], 4 * 5 * n3) != cudaSuccess ||
        cudaMalloc((void**)&F.block[1], 4 * 5 * n3) != cudaSuccess ||
        cudaMalloc((void**)&F.xy, 4 * (size_t)5 * (nf + 4) * F.n * F.n) != cudaSuccess) {
      ctx->err = "cudaMalloc of the fluid arrays failed";
      return CUBE_ERR_CUDA;
    }
    for (int c = 0; c < 5; ++c) {
      F.a[c] = F.block[0] + c * n3;
      F.b[c] = F.block[1] + c * n3;
    }
    int rc = cube_nu_init(ctx, F);
    if (rc) return rc;
  }
  N.nparts = (nf / 32) * (nf / 8) * (nf / 8);  // one partial sum per k_nu_fine_density brick
  if (cudaMalloc((void**)&N.partial, 8 * (size_t)N.nparts) != cudaSuccess) {
    ctx->err = "cudaMalloc failed";
    return CUBE_ERR_CUDA;
  }
  N.on = true;
  return CUBE_OK;
}

}  // namespace

extern "C" {

int32_t cube_abi_version(void) { return 1; }

const char* cube_last_error(cube_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int64_t cube_launch_count(cube_ctx* ctx) { return ctx ? ctx->launches : -1; }

int32_t cube_set_stream(cube_ctx* ctx, void* stream) {
  if (!ctx) return CUBE_ERR_PARAM;
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  ctx->own_stream = 0;
  ctx->stream = (cudaStream_t)stream;
  return CUBE_OK;
}

int32_t cube_set_params(cube_ctx* ctx, const cube_params* p) {
  if (!ctx || !p) return CUBE_ERR_PARAM;
  cube_params q = *p;  // everything but the changeable fields must match
  q.box = ctx->P.box; q.h0 = ctx->P.h0; q.omega_m = ctx->P.omega_m; q.omega_l = ctx->P.omega_l;
  q.wde = ctx->P.wde; q.ra_max = ctx->P.ra_max; q.dt_max = ctx->P.dt_max;
  if (memcmp(&q, &ctx->P, sizeof(cube_params)) != 0) {
    ctx->err = "cube_set_params: only box, h0, omega_m, omega_l, wde, ra_max and dt_max may change";
    return CUBE_ERR_PARAM;
  }
  if (!(p->box > 0.f) || !(p->h0 > 0.f) || !(p->omega_m > 0.f)) {
    ctx->err = "cube_set_params: box, h0 and omega_m must be positive";
    return CUBE_ERR_PARAM;
  }
  ctx->P.box = p->box; ctx->P.h0 = p->h0; ctx->P.omega_m = p->omega_m; ctx->P.omega_l = p->omega_l;
  ctx->P.wde = p->wde; ctx->P.ra_max = p->ra_max; ctx->P.dt_max = p->dt_max;
  return CUBE_OK;
}

void cube_destroy(cube_ctx* ctx) {
  if (!ctx) return;
  cudaStreamSynchronize(ctx->stream);
  void* ptrs[] = {ctx->xp, ctx->vp, ctx->pid, ctx->xp2, ctx->vp2, ctx->pid2, ctx->rhoc, ctx->rhoc2,
                  ctx->cell_start, ctx->cell_start2, ctx->vfield, ctx->vfield2, ctx->tcell, ctx->tkey,
                  ctx->perm, ctx->pkey, ctx->cursor, ctx->big_list, ctx->rebin_items, ctx->cell_stats, ctx->slot_r2, ctx->slot_s2,
                  ctx->red_tmp,
                  ctx->scan_tmp, ctx->fine.rho, ctx->fine.force, ctx->fine.ext, ctx->fine.kern, ctx->fine.plan.tw, ctx->fine.plan.tw2,
                  ctx->coarse.rho, ctx->coarse.force, ctx->coarse.ext, ctx->coarse.kern, ctx->coarse.plan.tw, ctx->coarse.plan.tw2,
                  ctx->fine.kernd, ctx->coarse.kernd, ctx->fine.plan.twd, ctx->coarse.plan.twd,
                  ctx->rho_c_acc,
                  ctx->tan_table, ctx->venc_brk, ctx->dscal, ctx->pk_bins};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int k = 0; k < 3; ++k) {
    NuFluid& F = ctx->nu.fl[k];
    for (float* q : {F.block[0], F.block[1], F.xy})
      if (q) cudaFree(q);
  }
  if (ctx->nu.partial) cudaFree(ctx->nu.partial);
  if (ctx->pp_scratch) cudaFree(ctx->pp_scratch);
  if (ctx->rebin_scratch) cudaFree(ctx->rebin_scratch);
  if (ctx->rebin_mid_scratch) cudaFree(ctx->rebin_mid_scratch);
  if (ctx->dep_scratch) cudaFree(ctx->dep_scratch);
  for (double* t : ctx->vdec)
    if (t) cudaFree(t);
  if (ctx->hscal) cudaFreeHost(ctx->hscal);
  for (int i = 0; i < 16; ++i)
    if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int32_t cube_create(const cube_params* params, int64_t np_capacity, const float* fk_table, const float* ck_table,
                    cube_ctx** out) {
  if (!params || !out || !fk_table || !ck_table) {
    g_create_error = "null argument";
    return CUBE_ERR_PARAM;
  }
  const cube_params& P = *params;
  if (P.nc <= 0 || P.nnt <= 0 || P.nc % P.nnt || P.ncell != 4 || (P.izipx != 1 && P.izipx != 2) ||
      (P.izipv != 1 && P.izipv != 2) || P.nf_cutoff <= 0 || P.ncb <= 0 || np_capacity <= 0 ||
      np_capacity >= ((int64_t)1 << 31)) {
    g_create_error = "invalid parameters (nc % nnt == 0, ncell == 4, izip in {1,2}, capacity < 2^31)";
    return CUBE_ERR_PARAM;
  }
  if (P.poisson_fp64 && P.neutrino) {
    g_create_error = "invalid parameters: the FP64 Poisson mode runs without neutrinos";
    return CUBE_ERR_PARAM;
  }
  cube_ctx* ctx = new cube_ctx();
  memset(ctx->ev, 0, sizeof(ctx->ev));
  ctx->P = P;
  ctx->nc = P.nc; ctx->nnt = P.nnt; ctx->nt = P.nc / P.nnt; ctx->ncell = P.ncell; ctx->ncb = P.ncb;
  ctx->nte = ctx->nt + 2 * ctx->ncb; ctx->nf = P.nc * P.ncell;
  ctx->ncells = (int64_t)P.nc * P.nc * P.nc;
  ctx->izipx = P.izipx; ctx->izipv = P.izipv;
  ctx->nvbin = 1 << (8 * P.izipv);
  ctx->codec.pi_f = 4.0f * atanf(1.0f);
  ctx->codec.sqrt_pio2_f = sqrtf(ctx->codec.pi_f / 2.0f);
  ctx->codec.nvbin_m1_f = (float)(ctx->nvbin - 1);
  ctx->codec.izipx = P.izipx; ctx->codec.izipv = P.izipv;
  ctx->codec.vrel_boost = P.vrel_boost;
  ctx->codec.x_resolution = P.izipx == 1 ? 1.0 / 256.0 : 1.0 / 65536.0;
  ctx->cap = np_capacity;
  ctx->np = 0;
  auto fail = [&](int rc) {
    g_create_error = ctx->err;
    cube_destroy(ctx);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    ctx->err = "cudaStreamCreate failed";
    ctx->stream = 0;
    return fail(CUBE_ERR_CUDA);
  }
  ctx->own_stream = 1;
  {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || ctx->num_sms <= 0)
      ctx->num_sms = 148;
  }
  for (int i = 0; i < 16; ++i)
    if (cudaEventCreate(&ctx->ev[i]) != cudaSuccess) { ctx->err = "cudaEventCreate failed"; return fail(CUBE_ERR_CUDA); }
  const int64_t cap = ctx->cap, nce = ctx->ncells;
  auto A = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) {
      ctx->err = "cudaMalloc of " + std::to_string(bytes) + " bytes failed";
      return false;
    }
    return true;
  };
  bool ok = A(&ctx->xp, 3 * cap * P.izipx) && A(&ctx->vp, 3 * cap * P.izipv) && A(&ctx->xp2, 3 * cap * P.izipx) &&
            A(&ctx->vp2, 3 * cap * P.izipv) && A((void**)&ctx->pid, 4 * cap) && A((void**)&ctx->pid2, 4 * cap) &&
            A((void**)&ctx->rhoc, 4 * nce) && A((void**)&ctx->rhoc2, 4 * nce) &&
            A((void**)&ctx->cell_start, 8 * (nce + 1)) && A((void**)&ctx->cell_start2, 8 * (nce + 1)) &&
            A((void**)&ctx->vfield, 12 * nce) && A((void**)&ctx->vfield2, 12 * nce) &&
            A((void**)&ctx->tcell, 4 * cap) && A((void**)&ctx->tkey, 4 * cap) && A((void**)&ctx->perm, 4 * cap) &&
            A((void**)&ctx->pkey, 4 * cap) && A((void**)&ctx->cursor, 4 * nce) &&
            A((void**)&ctx->big_list, 4 * nce) && A((void**)&ctx->cell_stats, 24 * nce) &&
            A((void**)&ctx->rebin_items, 32 * cube_rebin_items_max(nce, cap)) &&
            A((void**)&ctx->slot_r2, 8 * cap) && A((void**)&ctx->slot_s2, 8 * cap) &&
            A((void**)&ctx->red_tmp, 8 * (2 * (std::max<int64_t>(nce, cap) / 1024 + 64) + 64)) &&
            A((void**)&ctx->scan_tmp, 8 * (nce / 2048 + 64)) &&
            A((void**)&ctx->rho_c_acc, (P.neutrino ? 16 : 8) * nce) && A((void**)&ctx->tan_table, 4 * ctx->nvbin) &&
            A((void**)&ctx->venc_brk, sizeof(VencBrk) * 64) &&
            A((void**)&ctx->dscal, sizeof(DevScal)) &&
            A((void**)&ctx->pk_bins, 8 * 7 * (size_t)(cube_pk_nbin(ctx->nf, 0) + 1));
  if (!ok) return fail(CUBE_ERR_CUDA);
  if (cudaMallocHost((void**)&ctx->hscal, sizeof(DevScal)) != cudaSuccess) { ctx->err = "cudaMallocHost failed"; return fail(CUBE_ERR_CUDA); }
  cudaMemset(ctx->rho_c_acc, 0, (P.neutrino ? 16 : 8) * nce);
  ctx->rho_c_nu = P.neutrino ? ctx->rho_c_acc + nce : nullptr;
  cudaMemset(ctx->dscal, 0, sizeof(DevScal));
  cudaMemset(ctx->pid, 0, 4 * cap);
  int rc;
  if ((rc = alloc_level(ctx, ctx->fine, ctx->nf, P.poisson_fp64))) return fail(rc);
  if ((rc = alloc_level(ctx, ctx->coarse, ctx->nc, P.poisson_fp64))) return fail(rc);
  // FP32 tangent of every velocity code with the C library's tanf (decode table)
  std::vector<float> tt(ctx->nvbin);
  for (int c = -ctx->nvbin / 2; c < ctx->nvbin / 2; ++c) tt[c + ctx->nvbin / 2] = tanf(cube_varg(&ctx->codec, c));
  if (cudaMemcpyAsync(ctx->tan_table, tt.data(), 4 * ctx->nvbin, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
    ctx->err = "tan table upload failed";
    return fail(CUBE_ERR_CUDA);
  }
  // angle breakpoints theta_j = (j + 1/2) pi/128 and their tangents (cube_vencode_brk)
  VencBrk br[64];
  const long double pil = acosl(-1.0L);
  for (int j = 0; j < 64; ++j) {
    const long double th = ((long double)j + 0.5L) * pil / 128.0L;
    br[j].c = (double)tanl(th);
    br[j].hi = (double)th;
    br[j].lo = (double)(th - (long double)br[j].hi);
    br[j].pad = 0.0;
  }
  if (cudaMemcpy(ctx->venc_brk, br, sizeof(br), cudaMemcpyHostToDevice) != cudaSuccess) {
    ctx->err = "encode breakpoint table upload failed";
    return fail(CUBE_ERR_CUDA);
  }
  if ((rc = cube_build_green(ctx, fk_table, ck_table))) return fail(rc);
  if (P.neutrino && (rc = setup_neutrinos(ctx))) return fail(rc);
  if (cudaDeviceSynchronize() != cudaSuccess) { ctx->err = "setup failed"; return fail(CUBE_ERR_CUDA); }
  *out = ctx;
  return CUBE_OK;
}

int32_t cube_load_state(cube_ctx* ctx, int64_t nplocal, const void* xp, const void* vp, const int32_t* pid,
                        const int32_t* rhoc, const float* vfield) {
  if (!ctx || !xp || !vp || !rhoc || !vfield) return CUBE_ERR_PARAM;
  if (nplocal < 0 || nplocal > ctx->cap) {
    ctx->err = "nplocal exceeds the context capacity";
    return CUBE_ERR_CAPACITY;
  }
  const int64_t nce = ctx->ncells;
  std::vector<int64_t> dummy;
  int64_t tot = 0;
  for (int64_t c = 0; c < nce; ++c) tot += rhoc[c];
  if (tot != nplocal) {
    ctx->err = "sum(rhoc) != nplocal";
    return CUBE_ERR_PARAM;
  }
  ctx->np = nplocal;
  void* stage = ctx->tcell;  // 8 bytes per particle of scratch (tcell+tkey are adjacent in need, use two)
  // positions
  {
    const size_t bytes = 3 * (size_t)nplocal * ctx->izipx;
    void* st = bytes <= 4 * (size_t)ctx->cap ? stage : (void*)ctx->perm;
    if (bytes > 4 * (size_t)ctx->cap) st = ctx->xp2;
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->xp2, xp, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->izipx == 1) k_aos_to_soa<int8_t><<<1184, 256, 0, ctx->stream>>>((int8_t*)ctx->xp2, (int8_t*)ctx->xp, nplocal, ctx->cap);
    else k_aos_to_soa<int16_t><<<1184, 256, 0, ctx->stream>>>((int16_t*)ctx->xp2, (int16_t*)ctx->xp, nplocal, ctx->cap);
    CUBE_LAUNCH_CHECK(ctx);
    (void)st;
  }
  {
    const size_t bytes = 3 * (size_t)nplocal * ctx->izipv;
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->vp2, vp, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->izipv == 1) k_aos_to_soa<int8_t><<<1184, 256, 0, ctx->stream>>>((int8_t*)ctx->vp2, (int8_t*)ctx->vp, nplocal, ctx->cap);
    else k_aos_to_soa<int16_t><<<1184, 256, 0, ctx->stream>>>((int16_t*)ctx->vp2, (int16_t*)ctx->vp, nplocal, ctx->cap);
    CUBE_LAUNCH_CHECK(ctx);
  }
  if (pid) CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pid, pid, 4 * (size_t)nplocal, cudaMemcpyHostToDevice, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->rhoc, rhoc, 4 * (size_t)nce, cudaMemcpyHostToDevice, ctx->stream));
  {
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->vfield2, vfield, 12 * (size_t)nce, cudaMemcpyHostToDevice, ctx->stream));
    k_aos_to_soa<float><<<1184, 256, 0, ctx->stream>>>(ctx->vfield2, ctx->vfield, nce, nce);
    CUBE_LAUNCH_CHECK(ctx);
  }
  int rc = cube_exclusive_scan(ctx, ctx->rhoc, nce, ctx->cell_start);
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->state_loaded = 1;
  ctx->cells_le32 = 0;
  (void)dummy;
  return CUBE_OK;
}

int32_t cube_store_state(cube_ctx* ctx, int64_t* nplocal, void* xp, void* vp, int32_t* pid, int32_t* rhoc,
                         float* vfield) {
  if (!ctx) return CUBE_ERR_PARAM;
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  const int64_t n = ctx->np, nce = ctx->ncells;
  if (nplocal) *nplocal = n;
  if (xp) {
    if (ctx->izipx == 1) k_soa_to_aos<int8_t><<<1184, 256, 0, ctx->stream>>>((int8_t*)ctx->xp, (int8_t*)ctx->xp2, n, ctx->cap);
    else k_soa_to_aos<int16_t><<<1184, 256, 0, ctx->stream>>>((int16_t*)ctx->xp, (int16_t*)ctx->xp2, n, ctx->cap);
    CUBE_LAUNCH_CHECK(ctx);
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(xp, ctx->xp2, 3 * (size_t)n * ctx->izipx, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (vp) {
    if (ctx->izipv == 1) k_soa_to_aos<int8_t><<<1184, 256, 0, ctx->stream>>>((int8_t*)ctx->vp, (int8_t*)ctx->vp2, n, ctx->cap);
    else k_soa_to_aos<int16_t><<<1184, 256, 0, ctx->stream>>>((int16_t*)ctx->vp, (int16_t*)ctx->vp2, n, ctx->cap);
    CUBE_LAUNCH_CHECK(ctx);
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(vp, ctx->vp2, 3 * (size_t)n * ctx->izipv, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (pid) CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(pid, ctx->pid, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  if (rhoc) CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(rhoc, ctx->rhoc, 4 * (size_t)nce, cudaMemcpyDeviceToHost, ctx->stream));
  if (vfield) {
    k_soa_to_aos<float><<<1184, 256, 0, ctx->stream>>>(ctx->vfield, ctx->vfield2, nce, nce);
    CUBE_LAUNCH_CHECK(ctx);
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(vfield, ctx->vfield2, 12 * (size_t)nce, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return CUBE_OK;
}

int32_t cube_update_x(cube_ctx* ctx, cube_scalars* io) {
  if (!ctx || !io) return CUBE_ERR_PARAM;
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  int rc = cube_rebin(ctx, io);
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
  if ((rc = check_device_error(ctx))) return rc;
  // particle count of the new layout: start2[ncells]
  int64_t npn = 0;
  CUBE_CUDA_TRY(ctx, cudaMemcpy(&npn, ctx->cell_start2 + ctx->ncells, 8, cudaMemcpyDeviceToHost));
  if (npn != ctx->np) {
    ctx->err = "particle number not conserved by the re-bin (" + std::to_string(npn) + " != " + std::to_string(ctx->np) + ")";
    return CUBE_ERR_STATE;
  }
  std::swap(ctx->xp, ctx->xp2);
  std::swap(ctx->vp, ctx->vp2);
  std::swap(ctx->pid, ctx->pid2);
  std::swap(ctx->rhoc, ctx->rhoc2);
  std::swap(ctx->cell_start, ctx->cell_start2);
  std::swap(ctx->vfield, ctx->vfield2);
  // |vfield|^2 per cell, |v_res|^2 and |v|^2 per particle in the new storage order
  double sums[3];
  if ((rc = cube_tree_sum_dev(ctx, ctx->cell_stats, ctx->ncells, &sums[0]))) return rc;
  {
    int trc;
    const double* dec = cube_vdec_table(ctx, cube_vcoef(&ctx->codec, io->sigma_vi), &trc);
    if (trc) return trc;
    if ((rc = cube_stats_sums(ctx, reinterpret_cast<const int32_t*>(ctx->slot_r2), dec, &sums[1], &sums[2])))
      return rc;
  }
  const double npg = (double)(io->npglobal > 0 ? io->npglobal : ctx->np);
  io->std_vsim_c = sqrt(sums[0] / (double)ctx->ncells);
  io->std_vsim_res = sqrt(sums[1] / npg);
  io->std_vsim = sqrt(sums[2] / npg);
  io->sigma_vi_new = (float)(io->std_vsim_res / (double)sqrtf(3.f));
  io->nplocal = ctx->np;
  CUBE_CUDA_TRY(ctx, cudaEventElapsedTime(&ctx->phase_ms[0], ctx->ev[0], ctx->ev[1]));
  return CUBE_OK;
}

int32_t cube_particle_mesh(cube_ctx* ctx, cube_scalars* io) {
  if (!ctx || !io) return CUBE_ERR_PARAM;
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[2], ctx->stream));
  int rc = cube_deposit(ctx, io);
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
  const KickScale ks = {io->a_mid, io->dt, ctx->codec.pi_f, 1, 1.0f / 6.0f, 1.0f / ctx->codec.pi_f};
  if ((rc = cube_fft_poisson(ctx, ctx->fine, &ctx->dscal->f2_fine_bits, ks))) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
  if ((rc = cube_fft_poisson(ctx, ctx->coarse, &ctx->dscal->f2_coarse_bits, ks))) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
  if ((rc = cube_kick(ctx, io))) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
  if (ctx->nu.on) {
    if ((rc = cube_nu_gravity(ctx, io))) return rc;
    CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[9], ctx->stream));
  }
  unsigned long long mt[3];
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(mt, ctx->red_tmp, sizeof(mt), cudaMemcpyDeviceToHost, ctx->stream));
  if ((rc = check_device_error(ctx))) return rc;
  cube_mass_sums(mt, io->mass_p_cdm, &io->testrhof, &io->testrhoc);
  if (ctx->nu.on) {
    double nus = 0.0;
    if ((rc = cube_tree_sum_dev(ctx, ctx->nu.partial, ctx->nu.nparts, &nus))) return rc;
    io->testrhof += nus;
    cudaEventElapsedTime(&ctx->phase_ms[6], ctx->ev[6], ctx->ev[9]);
  }
  // the meshes hold force*s; max f^2 in force units
  const double s2 = (double)cube_kick_scalar(ks) * (double)cube_kick_scalar(ks);
  io->f2_max_fine = (float)((double)uint_as_float(ctx->hscal->f2_fine_bits) / s2);
  io->f2_max_coarse = (float)((double)uint_as_float(ctx->hscal->f2_coarse_bits) / s2);
  for (int d = 0; d < 3; ++d) io->vmax[d] = uint_as_float(ctx->hscal->vmax_bits[d]);
  io->sigma_vi = io->sigma_vi_new;  // pm.f90:180
  dt_constraints(ctx, io);
  cudaEventElapsedTime(&ctx->phase_ms[2], ctx->ev[2], ctx->ev[3]);
  cudaEventElapsedTime(&ctx->phase_ms[3], ctx->ev[3], ctx->ev[4]);
  cudaEventElapsedTime(&ctx->phase_ms[4], ctx->ev[4], ctx->ev[5]);
  cudaEventElapsedTime(&ctx->phase_ms[5], ctx->ev[5], ctx->ev[6]);
  return CUBE_OK;
}

int32_t cube_ext_pp_force(cube_ctx* ctx, cube_scalars* io) {
  if (!ctx || !io) return CUBE_ERR_PARAM;
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[7], ctx->stream));
  int rc = cube_pp(ctx, io);
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[8], ctx->stream));
  if ((rc = check_device_error(ctx))) return rc;
  const float f2 = uint_as_float(ctx->hscal->f2_pp_bits);
  io->f2_max_pp = std::max(io->f2_max_pp, f2);  // a saved local in the reference, never reset
  io->itest1 = (int64_t)ctx->hscal->itest1;
  io->npairs = (int64_t)ctx->hscal->npairs;
  const float pi_f = ctx->codec.pi_f;
  const float GG = cube_fdiv(cube_fdiv(1.0f, 6.0f), pi_f);
  io->dt_pp = cube_fdiv(cube_fmul(1.0f, sqrtf(1.0f)), cube_fmul(cube_fmul(sqrtf(io->f2_max_pp), io->a_mid), GG));
  cudaEventElapsedTime(&ctx->phase_ms[1], ctx->ev[7], ctx->ev[8]);
  if (io->itest1 != ctx->np) {
    ctx->err = "PP did not update every particle once";
    return CUBE_ERR_STATE;
  }
  return CUBE_OK;
}

void cube_expansion(const cube_params* p, float a0, float dt0, float* da1, float* da2) {
  // timestep.f90:136-180: third-order Taylor expansion of the Friedmann
  // equation over two half steps; real(4) interface, real(8) internals, with
  // the reference's default-real literals and parameters (4.0/9.0, 1.5*(1.0-wde),
  // dt_x**2 ...) evaluated in FP32 before promotion.
  const float om = p->omega_m, ol = p->omega_l, wde = p->wde;
  const float dt_x = dt0 / 2.0f;
  const double omHsq = (double)(4.0f / 9.0f);
  const float dt2 = dt_x * dt_x, dt3 = dt2 * dt_x;
  double a_x = (double)a0;
  float out[2];
  for (int half = 0; half < 2; ++half) {
    const double a3rlm = pow(a_x, (double)(-3.0f * wde)) * (double)ol / (double)om;
    const double arkm = a_x * (double)(1.0f - om - ol) / (double)om;
    const double a3 = a_x * a_x * a_x;
    const double adot = sqrt(omHsq * a3 * (1.0 + arkm + a3rlm));
    const double addot = (a_x * a_x) * omHsq * (1.5 + 2.0 * arkm + (double)(1.5f * (1.0f - wde)) * a3rlm);
    const double atdot =
        a_x * adot * omHsq * (3.0 + 6.0 * arkm + (double)(1.5f * (2.0f - 3.0f * wde) * (1.0f - wde)) * a3rlm);
    out[half] = (float)(adot * (double)dt_x + (addot * (double)dt2) / 2.0 + (atdot * (double)dt3) / 6.0);
    a_x = (double)(a0 + out[0]);
  }
  *da1 = out[0];
  *da2 = out[1];
}

int32_t cube_timestep(const cube_params* p, cube_scalars* s, float a_next, int32_t* hit) {
  // timestep.f90:1-95 (head image)
  s->dt_old = s->dt;
  s->timestep += 1;
  float dt_e = p->dt_max;
  float da1, da2, da, ra;
  int ntry = 0;
  for (;;) {
    ++ntry;
    cube_expansion(p, s->a, dt_e, &da1, &da2);
    da = da1 + da2;
    ra = da / (s->a + da);
    if (ra > p->ra_max) dt_e = dt_e * (p->ra_max / ra);
    else break;
    if (ntry > 10) break;
  }
  s->dt_e = dt_e;
  const float nu_lim = p->neutrino ? s->dt_vmax_nu : 1000.f;
  float dt = std::min(std::min(std::min(dt_e, s->dt_fine), std::min(s->dt_coarse, s->dt_pp)),
                      std::min(std::min(s->dt_vmax, nu_lim), s->dt_neu));
  cube_expansion(p, s->a, dt, &da1, &da2);
  da = da1 + da2;
  int h = 0;
  if (a_next > 0 && da >= a_next - s->a) {
    h = 1;
    int guard = 0;
    while (fabsf((s->a + da) / a_next - 1) >= 1e-6f && guard++ < 100) {
      dt = dt * (a_next - s->a) / da;
      cube_expansion(p, s->a, dt, &da1, &da2);
      da = da1 + da2;
    }
  }
  s->dt = dt;
  s->da = da;
  s->a_mid = s->a + (da / 2);
  s->tau += dt;
  s->t += dt;
  s->a = s->a + da;
  s->dt_neu = 1000.f;
  if (hit) *hit = h;
  return CUBE_OK;
}

int32_t cube_nu_evolve(cube_ctx* ctx, float dt, float* dtg, int32_t dir, float a) {
  if (!ctx || !dtg || (dir != 1 && dir != -1)) return CUBE_ERR_PARAM;
  if (!ctx->nu.on) {
    ctx->err = "fluid neutrinos are not enabled in this context";
    return CUBE_ERR_STATE;
  }
  NuState& N = ctx->nu;
  if (!(a >= N.ai)) return CUBE_OK;  // dfld_evolve: before the turn-on nothing moves
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[10], ctx->stream));
  const unsigned int big = float_as_uint(1e9f);
  const unsigned int init[3] = {big, big, big};
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->dscal->nu_dt_bits, init, sizeof(init), cudaMemcpyHostToDevice, ctx->stream));
  for (int k = 0; k < 3; ++k) {
    int rc = cube_nu_sweeps(ctx, N.fl[k], dt, dir);
    if (rc) return rc;
    if ((rc = cube_nu_timestep(ctx, N.fl[k], &ctx->dscal->nu_dt_bits[k]))) return rc;
  }
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[11], ctx->stream));
  unsigned int bits[3];
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(bits, ctx->dscal->nu_dt_bits, sizeof(bits), cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < 3; ++k) {  // hg_timestep: dt = min(dtg, h3_timestep) per fluid
    float d = uint_as_float(bits[k]);
    if (d == 1e9f) d = 1.f;
    *dtg = std::min(*dtg, d);
  }
  cudaEventElapsedTime(&ctx->phase_ms[6], ctx->ev[10], ctx->ev[11]);
  return CUBE_OK;
}

int32_t cube_nu_load(cube_ctx* ctx, int32_t fluid, const float* fld) {
  if (!ctx || !fld || fluid < 0 || fluid > 2) return CUBE_ERR_PARAM;
  if (!ctx->nu.on) { ctx->err = "fluid neutrinos are not enabled in this context"; return CUBE_ERR_STATE; }
  NuFluid& F = ctx->nu.fl[fluid];
  const size_t n3 = (size_t)F.n * F.n * F.n;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(F.b[0], fld, 4 * 5 * n3, cudaMemcpyHostToDevice, ctx->stream));
  int rc = cube_nu_transpose(ctx, F, 1);
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return CUBE_OK;
}

int32_t cube_nu_store(cube_ctx* ctx, int32_t fluid, float* fld) {
  if (!ctx || !fld || fluid < 0 || fluid > 2) return CUBE_ERR_PARAM;
  if (!ctx->nu.on) { ctx->err = "fluid neutrinos are not enabled in this context"; return CUBE_ERR_STATE; }
  NuFluid& F = ctx->nu.fl[fluid];
  const size_t n3 = (size_t)F.n * F.n * F.n;
  int rc = cube_nu_transpose(ctx, F, 0);
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(fld, F.b[0], 4 * 5 * n3, cudaMemcpyDeviceToHost, ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return CUBE_OK;
}

int32_t cube_debug_time_poisson(cube_ctx* ctx, int32_t reps, float* ms) {
  if (!ctx || !ms || reps <= 0) return CUBE_ERR_PARAM;
  const KickScale ks = {0.5f, 0.01f, ctx->codec.pi_f, 1, 1.0f / 6.0f, 1.0f / ctx->codec.pi_f};
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  int rc = cube_fft_poisson(ctx, ctx->fine, &ctx->dscal->f2_fine_bits, ks);  // warm-up
  if (rc) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[12], ctx->stream));
  for (int r = 0; r < reps; ++r)
    if ((rc = cube_fft_poisson(ctx, ctx->fine, &ctx->dscal->f2_fine_bits, ks))) return rc;
  CUBE_CUDA_TRY(ctx, cudaEventRecord(ctx->ev[13], ctx->stream));
  CUBE_CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev[13]));
  float t = 0.f;
  cudaEventElapsedTime(&t, ctx->ev[12], ctx->ev[13]);
  *ms = t / (float)reps;
  return CUBE_OK;
}

int32_t cube_make_ic(cube_ctx* ctx, const cube_ic_params* ic, cube_scalars* io) {
  if (!ctx || !ic || !io) return CUBE_ERR_PARAM;
  if (ctx->fine.fp64) {  // these use the FP32 meshes as scratch
    ctx->err = "not available in the FP64 Poisson mode";
    return CUBE_ERR_PARAM;
  }
  const int rc = cube_make_ic_dev(ctx, ic, io);
  if (rc == CUBE_OK) io->vsim2phys = vsim2phys(ctx, io->a);
  return rc;
}

int32_t cube_halofind(cube_ctx* ctx, const cube_scalars* io, const cube_halo_args* args, cube_halo_result* result) {
  if (!ctx || !io || !args || !result || (args->capacity > 0 && !args->halos)) return CUBE_ERR_PARAM;
  if (ctx->fine.fp64) {  // these use the FP32 meshes as scratch
    ctx->err = "not available in the FP64 Poisson mode";
    return CUBE_ERR_PARAM;
  }
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  *result = cube_halo_result{0, 0, 0};
  return cube_halofind_dev(ctx, io, args, result);
}

int32_t cube_power_spectrum(cube_ctx* ctx, int32_t log_bins, float* xip, int32_t capacity, int32_t* nbin) {
  if (!ctx || !xip || !nbin) return CUBE_ERR_PARAM;
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  if (ctx->fine.fp64) {  // it uses the FP32 meshes as scratch
    ctx->err = "not available in the FP64 Poisson mode";
    return CUBE_ERR_PARAM;
  }
  const int need = cube_pk_nbin(ctx->nf, log_bins ? 1 : 0);
  *nbin = need;
  if (capacity < need) {
    ctx->err = "xip holds fewer bins than the mesh has";
    return CUBE_ERR_CAPACITY;
  }
  std::vector<double> b;
  int nb = 0;
  int rc = cube_power_spectrum_dev(ctx, log_bins ? 1 : 0, b, &nb);
  if (rc) return rc;
  // powerspectrum.f90:113-135 for bins 1..nbin (bin 0 holds only modes with |k| < 1/2)
  const int W = nb + 1;
  const double two_pi_box = 2.0 * 3.14159265358979323846 / (double)ctx->P.box;
  for (int i = 1; i <= nb; ++i) {
    const double n = b[0 * W + i];
    float* o = xip + (size_t)(i - 1) * 10;
    o[0] = (float)n;
    o[1] = (float)(b[1 * W + i] / n * two_pi_box);
    for (int q = 2; q < 7; ++q) o[q] = (float)(b[q * W + i] / n);
    o[7] = o[4] / sqrtf(o[2] * o[3]);
    o[8] = sqrtf(o[3] / o[2]);
    o[9] = powf(o[7], 4.f) / powf(o[8], 2.f) * o[3];
  }
  return CUBE_OK;
}

int32_t cube_nu_info(cube_ctx* ctx, float* out) {
  if (!ctx || !out) return CUBE_ERR_PARAM;
  if (!ctx->nu.on) { ctx->err = "fluid neutrinos are not enabled in this context"; return CUBE_ERR_STATE; }
  const NuState& N = ctx->nu;
  out[0] = N.beta;
  for (int k = 0; k < 3; ++k) out[1 + k] = N.dwgts[k];
  for (int k = 0; k < 3; ++k) {
    const NuFluid& F = N.fl[k];
    float* q = out + 4 + 5 * k;
    q[0] = (float)F.n; q[1] = (float)F.ncb; q[2] = F.dx; q[3] = F.cs2; q[4] = F.dv;
  }
  return CUBE_OK;
}

int32_t cube_phase_times(cube_ctx* ctx, float* ms8) {
  if (!ctx || !ms8) return CUBE_ERR_PARAM;
  float tot = 0;
  for (int i = 0; i < 7; ++i) { ms8[i] = ctx->phase_ms[i]; tot += ctx->phase_ms[i]; }
  ms8[7] = tot;
  return CUBE_OK;
}

int64_t cube_debug_fetch(cube_ctx* ctx, int32_t which, void* host, int64_t capacity) {
  if (!ctx || !host) return -1;
  MeshLevel* L = nullptr;
  int ncomp = 1;
  const float* src = nullptr;
  switch (which) {
    case 0: L = &ctx->fine; src = L->rho; break;
    case 1: L = &ctx->coarse; src = L->rho; break;
    case 2: L = &ctx->fine; src = L->force; ncomp = 3; break;
    case 3: L = &ctx->coarse; src = L->force; ncomp = 3; break;
    case 4: case 5: {
      L = which == 4 ? &ctx->fine : &ctx->coarse;
      const int64_t kp = L->n / 2 + 1, n = 3 * kp * kp * kp;
      if (n > capacity) return -1;
      if (cudaMemcpyAsync(host, L->kern, 4 * n, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) return -1;
      if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return -1;
      return n;
    }
    default: return -1;
  }
  const int64_t n3 = (int64_t)L->n * L->n * L->n, n = n3 * ncomp;
  if (n > capacity) return -1;
  const size_t es = L->fp64 ? 8 : 4;  // the FP64 Poisson mode's meshes come back as doubles
  void* tmp = nullptr;
  if (cudaMalloc(&tmp, es * n) != cudaSuccess) return -1;
  if (L->fp64)
    k_unpitch<double><<<1184, 256, 0, ctx->stream>>>(reinterpret_cast<const double*>(src),
                                                     static_cast<double*>(tmp), L->n, L->rp, ncomp);
  else
    k_unpitch<float><<<1184, 256, 0, ctx->stream>>>(src, static_cast<float*>(tmp), L->n, L->rp, ncomp);
  ctx->launches++;
  cudaStreamSynchronize(ctx->stream);
  const cudaError_t e = cudaMemcpy(host, tmp, es * n, cudaMemcpyDeviceToHost);
  cudaFree(tmp);
  return e == cudaSuccess ? n : -1;
}

int32_t cube_debug_deposit(cube_ctx* ctx, cube_scalars* io) {
  if (!ctx || !io) return CUBE_ERR_PARAM;
  if (!ctx->state_loaded) return CUBE_ERR_STATE;
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  int rc = cube_deposit(ctx, io);
  if (rc) return rc;
  unsigned long long mt[3];
  CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(mt, ctx->red_tmp, sizeof(mt), cudaMemcpyDeviceToHost, ctx->stream));
  if ((rc = check_device_error(ctx))) return rc;
  cube_mass_sums(mt, io->mass_p_cdm, &io->testrhof, &io->testrhoc);
  if (ctx->nu.on) {
    double nus = 0.0;
    if ((rc = cube_tree_sum_dev(ctx, ctx->nu.partial, ctx->nu.nparts, &nus))) return rc;
    io->testrhof += nus;
  }
  return CUBE_OK;
}

int32_t cube_debug_kick_with_force(cube_ctx* ctx, cube_scalars* io, const float* fine_force,
                                   const float* coarse_force) {
  if (!ctx || !io || !fine_force || !coarse_force) return CUBE_ERR_PARAM;
  if (ctx->fine.fp64) {
    ctx->err = "not available in the FP64 Poisson mode";
    return CUBE_ERR_PARAM;
  }
  MeshLevel* Ls[2] = {&ctx->fine, &ctx->coarse};
  const float* hs[2] = {fine_force, coarse_force};
  for (int l = 0; l < 2; ++l) {
    MeshLevel& L = *Ls[l];
    const int64_t n = 3 * (int64_t)L.n * L.n * L.n;
    float* tmp = nullptr;
    CUBE_CUDA_TRY(ctx, cudaMalloc(&tmp, 4 * n));
    CUBE_CUDA_TRY(ctx, cudaMemcpyAsync(tmp, hs[l], 4 * n, cudaMemcpyHostToDevice, ctx->stream));
    k_pitch<<<1184, 256, 0, ctx->stream>>>(tmp, L.force, L.n, L.rp, 3);
    CUBE_LAUNCH_CHECK(ctx);
    CUBE_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    cudaFree(tmp);
  }
  CUBE_CUDA_TRY(ctx, cudaMemsetAsync(ctx->dscal, 0, sizeof(DevScal), ctx->stream));
  // the meshes hold kick increments once particle_mesh has run: scale the raw forces
  const KickScale ks = {io->a_mid, io->dt, ctx->codec.pi_f, 1, 1.0f / 6.0f, 1.0f / ctx->codec.pi_f};
  int rc = cube_force_scale(ctx, ctx->fine, ks);
  if (rc || (rc = cube_force_scale(ctx, ctx->coarse, ks))) return rc;
  if ((rc = cube_kick(ctx, io))) return rc;
  if (ctx->nu.on && (rc = cube_nu_gravity(ctx, io))) return rc;
  if ((rc = check_device_error(ctx))) return rc;
  for (int d = 0; d < 3; ++d) io->vmax[d] = uint_as_float(ctx->hscal->vmax_bits[d]);
  io->sigma_vi = io->sigma_vi_new;
  return CUBE_OK;
}

// One box-step of main.f90:49-64 on one context (the order of Cube.step): timestep,
// neutrino half step, drift, PP, particle mesh, neutrino half step.
static int32_t run_one_step(cube_ctx* ctx, cube_scalars* io) {
  int32_t hit = 0;
  int32_t rc = cube_timestep(&ctx->P, io, 0.0f, &hit);
  if (!rc && ctx->nu.on) rc = cube_nu_evolve(ctx, io->dt / 2.0f, &io->dt_neu, 1, io->a_mid);
  if (!rc) rc = cube_update_x(ctx, io);
  if (!rc && ctx->P.ext_pp_force) rc = cube_ext_pp_force(ctx, io);
  if (!rc) rc = cube_particle_mesh(ctx, io);
  if (!rc && ctx->nu.on) rc = cube_nu_evolve(ctx, io->dt / 2.0f, &io->dt_neu, -1, io->a_mid);
  return rc;
}

int32_t cube_run_steps(cube_ctx* const* ctxs, cube_scalars* ios, int32_t n, int32_t steps, int32_t threads,
                       int32_t* failed) {
  if (failed) *failed = -1;
  if (!ctxs || !ios || n < 0 || steps < 0 || threads < 1) return CUBE_ERR_PARAM;
  for (int32_t i = 0; i < n; ++i)
    if (!ctxs[i] || !ctxs[i]->state_loaded) {
      if (failed) *failed = i;
      return ctxs[i] ? CUBE_ERR_STATE : CUBE_ERR_PARAM;
    }
  const int32_t nt = std::min(threads, std::max(n, 1));
  std::vector<int32_t> st(nt, CUBE_OK), at(nt, -1);
  auto work = [&](int32_t t) {
    for (int32_t k = 0; k < steps; ++k)
      for (int32_t i = t; i < n; i += nt) {
        const int32_t rc = run_one_step(ctxs[i], &ios[i]);
        if (rc) {
          st[t] = rc;
          at[t] = i;
          return;
        }
      }
  };
  std::vector<std::thread> pool;
  for (int32_t t = 1; t < nt; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  int32_t rc = CUBE_OK, first = -1;
  for (int32_t t = 0; t < nt; ++t)
    if (st[t] && (first < 0 || at[t] < first)) {
      first = at[t];
      rc = st[t];
    }
  if (failed) *failed = first;
  return rc;
}

}  // extern "C"
