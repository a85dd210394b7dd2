/*
 * cube_gpu.h -- C-ABI of the B200 particle-mesh step of CUBE.
 *
 * The reference step routines take no arguments and act on Fortran module
 * globals (CUBE_v2.0/work/main/variables.f90:28-81):
 *   particle_mesh  (pm.f90:2)            -> cube_particle_mesh
 *   update_x       (update_particle.f90:5) -> cube_update_x
 *   ext_pp_force   (ext_pp_force.f90:9)  -> cube_ext_pp_force
 *   buffer_grid / buffer_x / buffer_v (buffer_grid.f90:5, buffer_particle.f90:5,13)
 *                                       -> no device work: one image on one GPU
 *                                          keeps every particle once and reads
 *                                          neighbour cells by periodic index
 *   neu(nu)%evolve (hydrodf.f90:86)     -> cube_nu_evolve
 *   neu(nu)%gravity / %density (hydrodf.f90:111,209) -> inside cube_particle_mesh
 *   neu(nu)%restart / %checkpoint (hydrodf.f90:158,134) -> cube_nu_load / cube_nu_store
 *   timestep       (timestep.f90:1)     -> cube_timestep (host arithmetic)
 *   kernel_f / kernel_c (kernel_f.f90:2, kernel_c.f90:2) -> inside cube_create
 *
 * A Fortran host keeps its no-argument wrappers (see include/cube_gpu.f90) and
 * passes the module arrays through these entry points.  The library owns the
 * device-resident particle and mesh state between calls; the host keeps the
 * scalar globals in a cube_scalars block that each call reads and updates.
 *
 * Array layouts are the reference's checkpoint layouts (checkpoint.f90:24-75):
 *   xp, vp   int8|int16 [nplocal][3]   (Fortran xp(3,nplocal)), izipx/izipv bytes
 *   pid      int32 [nplocal]
 *   rhoc     int32 [nnt][nnt][nnt][nt][nt][nt]  (Fortran rhoc(1:nt,1:nt,1:nt,nnt,nnt,nnt))
 *   vfield   float [nnt^3*nt^3][3]            (Fortran vfield(3,1:nt,1:nt,1:nt,...))
 * Particles are sorted by tile (x fastest), then by coarse cell (x fastest)
 * inside the tile, exactly as update_xp leaves them (update_particle.f90:134-149).
 *
 * Every entry point returns a cube_status; non-zero codes replace the
 * reference's print + stop (update_particle.f90:90-96, buffer_grid.f90:131-137,
 * ext_pp_force.f90:154-158).  Calls on one context come from one host thread;
 * a context is bound to one CUDA stream.
 */
#ifndef CUBE_GPU_H
#define CUBE_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum cube_status {
  CUBE_OK = 0,
  CUBE_ERR_PARAM = 1,      /* inconsistent sizes or parameters */
  CUBE_ERR_CAPACITY = 2,   /* particle count beyond the allocated capacity */
  CUBE_ERR_CUDA = 3,       /* a CUDA runtime call failed (see cube_last_error) */
  CUBE_ERR_MOVE = 4,       /* a particle moved farther than ncb coarse cells in one drift */
  CUBE_ERR_TIMEOUT = 5,    /* a bounded device wait gave up */
  CUBE_ERR_STATE = 6,      /* call made before the state it needs was loaded */
  CUBE_ERR_CELL = 7        /* one coarse cell holds more particles than a re-bin block can sort */
} cube_status;

/* Compile-time parameters of parameters.f90:8-116, as runtime fields. */
typedef struct cube_params {
  int32_t nc;            /* coarse cells per dimension of the (single) image, nc */
  int32_t nnt;           /* tiles per dimension, nnt; nt = nc/nnt */
  int32_t ncell;         /* fine cells per coarse cell per dimension (4) */
  int32_t ncb;           /* coarse buffer depth (6) */
  int32_t np_nc;         /* particles per coarse cell per dimension in the IC lattice */
  int32_t izipx;         /* bytes per position component (1 or 2) */
  int32_t izipv;         /* bytes per velocity component (1 or 2) */
  int32_t nf_cutoff;     /* fine-force cutoff in fine cells (16) */
  int32_t pp_range;      /* PP neighbour range in fine cells (1) */
  int32_t ext_pp_force;  /* 1: PP on (Extended_pp_force), zeroes the fine-kernel core */
  int32_t use_pid;       /* 1: particle IDs are carried (-DPID) */
  int32_t neutrino;      /* 1: fluid neutrinos are coupled (neutrino_flag) */
  float rsoft;           /* PP softening (0.3) */
  float tile_buffer;     /* 1.5 */
  float image_buffer;    /* 1.2 */
  float vbuf;            /* 0.9 */
  double vrel_boost;     /* 2.5 */
  /* cosmology (parameters.f90:69-100) */
  float box;             /* Mpc/h */
  float h0;
  float omega_m;
  float omega_l;
  float wde;
  float ra_max;          /* 0.2 */
  float dt_max;          /* 1 (variables.f90:20) */
  /* neutrino fluid (hydrodf.f90:22-49, parameters.f90:73-93) */
  float z_i_nu;          /* neutrino turn-on redshift */
  float f_neu;           /* sum(f_neu) = omega_neu/omega_m */
  float m_nu_ev;         /* neutrino mass per species, eV */
  float deg_nu;          /* degeneracy */
  int32_t nu_nc[3];      /* fluid mesh sizes per Gauss-Laguerre fluid (0 = nf/2,nf/4,nf/8) */
  int32_t stockham_only; /* 1: every mesh FFT takes the shared-memory Stockham passes (testing) */
  int32_t poisson_fp64;  /* 1: FP64 Poisson path (meshes, FFT, Green, interpolation in FP64);
                            no counterpart in the reference, whose meshes are FP32: the FP64
                            run of the same step that the FP32 results are measured against.
                            Needs neutrino = 0; power spectrum, halo finder and device ICs
                            need the FP32 meshes and return CUBE_ERR_PARAM. */
  int32_t reserved[6];
} cube_params;

/* Scalar globals the step reads and writes (variables.f90:28-48 and sim_header,
 * parameters.f90:129-153). */
typedef struct cube_scalars {
  float a, a_mid, da;
  float dt, dt_old, dt_mid;
  float t, tau;
  float sigma_vi, sigma_vi_new;
  float mass_p_cdm;
  float vz_max;            /* sim%vz_max */
  float dt_fine, dt_coarse, dt_pp, dt_vmax, dt_vmax_nu, dt_e, dt_neu;
  float vmax[3];
  float f2_max_fine, f2_max_coarse, f2_max_pp;
  float vsim2phys;
  int32_t nlayer;          /* update_xp ordering layers, 2*ceiling(dt_mid*vz_max/ncell)+1 */
  int32_t timestep;
  double std_vsim, std_vsim_c, std_vsim_res;
  double testrhof, testrhoc;   /* mass sums (pm.f90:108,280) */
  int64_t nplocal, npglobal;
  int64_t npairs, itest1;      /* PP diagnostics (ext_pp_force.f90:98,87) */
  int32_t reserved[16];
} cube_scalars;

typedef struct cube_ctx cube_ctx;

/* Version of this ABI; bump on layout changes of the structs above. */
int32_t cube_abi_version(void);

/* Creates a context on the current CUDA device: allocates the device state
 * for up to `np_capacity` particles and builds the fine and coarse Green's
 * functions (kernel_f.f90:14-37, kernel_c.f90:1-134) in FP64.
 *   fk_table: fine force table fk_table(16,16,16,3), Fortran order (kernel_f.f90:10-22)
 *   ck_table: coarse matching table ck_table(3,4,4,4), Fortran order (kernel_c.f90:31-39) */
int32_t cube_create(const cube_params* params, int64_t np_capacity,
                    const float* fk_table, const float* ck_table, cube_ctx** out);

/* Copies a checkpoint-layout state to the device (particle_initialization.f90:34-82).
 * Load (and store) between steps, after cube_particle_mesh, where the reference
 * reads and writes checkpoints: a state loaded between cube_update_x and
 * cube_particle_mesh was measured to change the run that follows. */
int32_t cube_load_state(cube_ctx* ctx, int64_t nplocal, const void* xp, const void* vp,
                        const int32_t* pid, const int32_t* rhoc, const float* vfield);

/* Copies the device state back in checkpoint layout (checkpoint.f90:24-75).
 * Any pointer may be NULL to skip that array. */
int32_t cube_store_state(cube_ctx* ctx, int64_t* nplocal, void* xp, void* vp, int32_t* pid,
                         int32_t* rhoc, float* vfield);

/* update_x: drift by dt_mid, re-bin by counting sort, re-encode velocities
 * against the new coarse velocity field, velocity statistics -> sigma_vi_new
 * (update_particle.f90:13-259).  Reads dt, dt_old, sigma_vi, vz_max;
 * writes dt_mid, nlayer, sigma_vi_new, std_vsim*, nplocal. */
int32_t cube_update_x(cube_ctx* ctx, cube_scalars* io);

/* ext_pp_force: particle-particle correction over +-pp_range fine cells
 * (ext_pp_force.f90:34-143).  Reads a_mid, dt, sigma_vi, mass_p_cdm; writes
 * dt_pp, f2_max_pp, npairs, itest1. */
int32_t cube_ext_pp_force(cube_ctx* ctx, cube_scalars* io);

/* particle_mesh: fine and coarse CIC deposit, Poisson solve by FFT, interpolate
 * and kick (pm.f90:2-451).  Reads a, a_mid, dt, sigma_vi, sigma_vi_new,
 * mass_p_cdm; writes sigma_vi (= sigma_vi_new), vmax, vz_max, dt_fine,
 * dt_coarse, dt_vmax, f2_max_*, testrhof, testrhoc, vsim2phys. */
int32_t cube_particle_mesh(cube_ctx* ctx, cube_scalars* io);

/* timestep (timestep.f90:1-95) in its adaptive form, host arithmetic with the
 * FP64 Friedmann expansion of timestep.f90:136-180.  If a_next > 0 the step is
 * snapped to reach a_next exactly (the checkpoint logic of timestep.f90:46-61),
 * which is also the prescribed-step mode.  Returns 1 in *hit if a_next was hit. */
int32_t cube_timestep(const cube_params* params, cube_scalars* io, float a_next, int32_t* hit);

/* Steps n independent contexts (an ensemble of boxes) `steps` times each on a pool
 * of `threads` host threads, boxes dealt round-robin: every box-step is the order
 * of main.f90:49-64 (cube_timestep in its adaptive form, the neutrino half steps if
 * the context has fluid neutrinos, cube_update_x, cube_ext_pp_force if enabled,
 * cube_particle_mesh) on that context's stream and ios[i].  No counterpart in the
 * reference, which runs one box per job; it lets a host step many small boxes
 * without a thread of its own per box.  A thread stops at its box's first error;
 * the call returns the error of the lowest-numbered failing box and its index in
 * *failed (-1 if none).  Each context must have a state loaded. */
int32_t cube_run_steps(cube_ctx* const* ctxs, cube_scalars* ios, int32_t n, int32_t steps, int32_t threads,
                       int32_t* failed);

/* Friedmann expansion of timestep.f90:136-180 (real(4) interface, FP64 inside). */
void cube_expansion(const cube_params* params, float a0, float dt0, float* da1, float* da2);

/* ---- fluid neutrinos (params.neutrino = 1) ------------------------------------
 * One species of mass m_nu_ev (Nneu = 1, parameters.f90:80) as the dispersive sum
 * of three isothermal fluids (hydrodf.f90:22-49) on meshes of nu_nc[k] cells per
 * side (0 = nf/2, nf/4, nf/8), gamma = 5/3.  cube_create sets them to hg_setup's
 * rest state; cube_particle_mesh adds their density to both meshes and applies
 * the mesh forces to them (pm.f90:55-74, :157-171, :198-242, :374-422).
 *
 * Half step neu(nu)%evolve(dt,dtg,dir,a) (hydrodf.f90:86-109): dir = +1 sweeps
 * x,y,z, -1 sweeps z,y,x; no-op while a < 1/(1+z_i_nu); *dtg is lowered to each
 * fluid's CFL step (hydrogr.f90:92-108). */
int32_t cube_nu_evolve(cube_ctx* ctx, float dt, float* dtg, int32_t dir, float a);

/* Fluid k (0..2) to / from the host as fld(1:5,1:n,1:n,1:n): float [n][n][n][5],
 * component fastest (rho, rho*vx, rho*vy, rho*vz, E), the physical cells of the
 * reference's fld array (hydrogr.f90:21; its checkpoint adds the halo cells,
 * hydrodf.f90:134-156). */
int32_t cube_nu_load(cube_ctx* ctx, int32_t fluid, const float* fld);
int32_t cube_nu_store(cube_ctx* ctx, int32_t fluid, float* fld);

/* Power spectrum of the resident particles on the fine mesh (ng = nf), the
 * checkpoint analysis of cicpower.f90:84-255 + powerspectrum.f90:27-137: CIC
 * with unit mass at pos*ng/nc - 1/2, delta = rho/mean - 1, forward FFT, modes
 * binned by nint(|k|) (log_bins = 0, the reference's linear_kbin) or 4 per
 * octave from 0.95 (log_bins = 1).  With fluid neutrinos the second field is
 * their density contrast (cross power), else zero.  Writes xip(10,nbin) as
 * float [nbin][10]: count, k (h/Mpc), Delta^2_cc, Delta^2_nn, Delta^2_cn,
 * <1/sinc^2>, <1/sinc^4>, r, b, reconstruction; *nbin = bins of the mesh
 * (CUBE_ERR_CAPACITY if capacity < *nbin).  Uses the fine meshes as scratch:
 * call it between steps, not inside one. */
int32_t cube_power_spectrum(cube_ctx* ctx, int32_t log_bins, float* xip, int32_t capacity, int32_t* nbin);

/* ---- initial conditions on the device -----------------------------------------
 * Replaces running the ic.x program (initial_conditions.f90:268-900) and loading
 * its files with cube_load_state: a Zel'dovich state on the np_nc*nc particle
 * lattice, made in place.  The linear power is Delta^2(k) = norm_d2 * T(k)^2 *
 * k^(3+n_s) with the Eisenstein-Hu (1998) no-wiggle transfer T (k in h/Mpc; the
 * host precomputes the sigma8 normalisation times D(a)^2 and the EH constants);
 * the noise is Philox4x32-10 under `seed` through the reference's Box-Muller
 * pairing along x (initial_conditions.f90:320-336).  Particles are packed as the
 * reference packs them (:797-838): sorted by coarse cell, lattice order within a
 * cell, PID = 1 + the fine-mesh index of the lattice point (iq = (ncell/np_nc)*
 * lattice index per dimension, PID = iq_x + nf iq_y + nf^2 iq_z + 1, :834-836; needs
 * nf^3 < 2^31), vfield = cell-mean velocity, velocity codes
 * relative to it with sigma_vi from the residuals. */
typedef struct cube_ic_params {
  int64_t seed;
  int32_t np_nc;        /* particles per coarse cell per dimension; np_nc*nc even */
  int32_t pad0;
  double a;             /* initial scale factor 1/(1+z_i) */
  double norm_d2;       /* sigma8^2/v8 * D(a)^2 */
  double n_s, h;
  double eh_s;          /* sound horizon, Mpc */
  double eh_alpha;      /* alpha_Gamma */
  double eh_omh;        /* Omega_m h */
  double eh_theta2;     /* (T_cmb/2.7)^2 */
  double vf;            /* a^2 H(a) f(a), simulation units (initial_conditions.f90:1068-1079) */
  double amplitude;     /* extra scale of the displacement (1) */
  double f_cdm;         /* CDM share of the matter: mass_p_cdm = f_cdm*nf^3/np */
} cube_ic_params;

/* Generates the state above for the context's box (params.box, nc, nnt, ncell,
 * izipx, izipv) and sets the scalar block as particle_initialization.f90:37-39
 * does after reading it (a, sigma_vi, mass_p_cdm, vmax, vz_max, dt_vmax, np).
 * Uses the fine meshes as scratch (np_nc <= ncell); needs np <= np_capacity. */
int32_t cube_make_ic(cube_ctx* ctx, const cube_ic_params* ic, cube_scalars* io);

/* ---- run-time halo finder ------------------------------------------------------
 * halofind (halofind.f90:18-598) on the resident particles: spherical-overdensity
 * halos grown from the peaks of the fine CIC density, densest first, each taking
 * the untagged particles inside the radius where the enclosed density falls below
 * den_odc, kept with at least 100 particles.  One record per halo, the reference's
 * type_halo_info (halofind.f90:10-15), 42 floats: */
typedef struct cube_halo {
  float hpos[3];          /* refined density peak, fine units, in [0, nf) */
  float mass_odc;         /* particles inside radius_odc */
  float radius_odc;       /* fine units */
  float v_disp;           /* 3-D velocity dispersion, simulation units */
  float x_mean[3], v_mean[3], ang_mom[3], var_x[3];
  float inertia[9];       /* (3,3), column-major, about x_mean */
  float q_mean[3];        /* Lagrangian mean position from the PIDs */
  float inertia_q[9];
  float s_mean[3];        /* redshift-space mean position (viewer at cen/500*nc) */
} cube_halo;

typedef struct cube_halo_args {
  float den_odc;          /* overdensity threshold; <= 0 selects 200 (halofind.f90:96-104) */
  int32_t capacity;       /* records `halos` holds */
  cube_halo* halos;       /* host, in order of discovery (decreasing peak density) */
  int32_t* member_pid;    /* host or NULL: each halo's PIDs by increasing radius, halos
                             concatenated (the halo_pid file without its counts) */
  int64_t member_capacity;
  int32_t* hid;           /* host or NULL: hid[pid-1] = 1-based halo number, 0 if none */
  int64_t hid_len;        /* entries of hid (nf^3 for the IC's PIDs) */
} cube_halo_args;

typedef struct cube_halo_result {
  int32_t nhalo;          /* halos found (may exceed capacity: CUBE_ERR_CAPACITY) */
  int32_t npeak;          /* density peaks examined */
  int64_t nmember;        /* PIDs written to member_pid (with params.use_pid) */
} cube_halo_result;

/* Finds the halos of the resident state.  Reads a, sigma_vi, mass_p_cdm and
 * vsim2phys (set by cube_particle_mesh or cube_make_ic) from io.  Without
 * params.use_pid the q-space fields are zero and no PIDs are written.  Uses the
 * fine force meshes as scratch: call it between steps.  CUBE_ERR_CAPACITY when
 * a halo's refined grid would exceed 300 cells per dimension (the reference's
 * newbox_max stop) or an output array is too small (the counts are still set). */
int32_t cube_halofind(cube_ctx* ctx, const cube_scalars* io, const cube_halo_args* args,
                      cube_halo_result* result);

/* Set-up constants, 19 floats: beta = m/T, the three normalised weights, then
 * per fluid (n, ncb of the reference layout, dx, cs2, hg_dv). */
int32_t cube_nu_info(cube_ctx* ctx, float* out);

/* Device time of the phases of the last step call, milliseconds:
 * [0] update_x, [1] ext_pp_force, [2] deposit, [3] fine FFT+Green, [4] coarse
 * FFT+Green, [5] kick, [6] neutrino fluid, [7] total. */
int32_t cube_phase_times(cube_ctx* ctx, float* ms8);

/* Number of kernels the library launched on this context so far. */
int64_t cube_launch_count(cube_ctx* ctx);

/* Sets the CUDA stream (cudaStream_t passed as void*) the context launches on. */
int32_t cube_set_stream(cube_ctx* ctx, void* stream);

/* Gives an existing context another box size and cosmology (box, h0, omega_m,
 * omega_l, wde, ra_max, dt_max) without reallocating, so that a host serving many
 * boxes of one mesh size can reuse a context (and not stall the device in cudaFree)
 * by following this with cube_make_ic or cube_load_state.  No counterpart in the
 * reference, whose parameters are compile-time.  Every other field must equal the
 * context's (they size its arrays or its Green's functions): CUBE_ERR_PARAM if not. */
int32_t cube_set_params(cube_ctx* ctx, const cube_params* params);

/* Text of the last error on this context (or the last create error if ctx is NULL). */
const char* cube_last_error(cube_ctx* ctx);

void cube_destroy(cube_ctx* ctx);

/* ---- inspection entry points used by the parity tests -----------------------
 * Copies device meshes to host buffers:
 *   which=0 fine density rho_f   [nf^3]   (x fastest, global periodic fine mesh)
 *   which=1 coarse density r3    [nc^3]
 *   which=2 fine force           [3][nf^3]
 *   which=3 coarse force         [3][nc^3]
 *   which=4 fine Green multiplier octant [3][(nf/2+1)^3]
 *   which=5 coarse Green multiplier      [3][nc][nc][nc/2+1]
 * In the FP64 Poisson mode (params.poisson_fp64) which=0..3 write doubles.
 * Returns the element count written, or -1. */
int64_t cube_debug_fetch(cube_ctx* ctx, int32_t which, void* host, int64_t capacity);

/* Runs only the fine and coarse CIC deposit of particle_mesh (pm.f90:76-107,
 * :192-278), so that cube_debug_fetch(0/1) returns the densities before the
 * FFT reuses their storage.  Writes testrhof and testrhoc. */
int32_t cube_debug_deposit(cube_ctx* ctx, cube_scalars* io);

/* Uploads a fine (which=2) or coarse (which=3) force mesh and runs only the
 * interpolate+kick of particle_mesh on it (parity of the kick against the oracle
 * on identical forces). */
int32_t cube_debug_kick_with_force(cube_ctx* ctx, cube_scalars* io, const float* fine_force,
                                   const float* coarse_force);

/* Compares, for n velocities spread over every code and concentrated at the
 * rounding boundaries, the step's velocity encode (angle breakpoints from an FP32
 * first guess, falling back to the exact encode near ties) with the exact FP64
 * encode under sigma; *mismatches counts the disagreements (0 expected). */
int32_t cube_debug_encode_check(cube_ctx* ctx, int64_t n, uint64_t seed, float sigma, int64_t* mismatches);

/* Compares, for n quotients shaped like the PP pair term (separation components on
 * the int1/int2 position grids over +-8 fine cells divided by r^3, r > 0.3) and
 * random doubles over wide ranges, the library's division through one shared
 * reciprocal (two FMA corrections) with the IEEE division; *mismatches counts the
 * quotients that differ in any bit (0 expected). */
int32_t cube_debug_division_check(cube_ctx* ctx, int64_t n, uint64_t seed, int64_t* mismatches);

/* Device time of the fine-mesh Poisson solve (FFT passes + Green multiply) on
 * whatever the fine density array holds, averaged over reps runs, in *ms. */
int32_t cube_debug_time_poisson(cube_ctx* ctx, int32_t reps, float* ms);

/* ---- allocation-free coarse density ------------------------------------------
 * No counterpart in the reference.  For hosts that may not allocate device memory
 * during a run (their HBM is owned by another allocator, or a fixed budget per box
 * was handed out at start-up): computes the particle (CDM) coarse CIC density of
 * pm.f90:192-278 from caller-owned device buffers and allocates nothing.  It is
 * bit-identical to the coarse density of cube_particle_mesh when neutrinos are
 * off (with params.neutrino = 1 the context's coarse density also holds the
 * neutrino mass, which this call does not add).
 *   xp         device, int8|int16 [3][np_capacity] position codes (structure of arrays)
 *   cell_start device, int64 [nc^3+1] first particle of each cell, tile-major order
 *   rho        device, float [nc^3] output (x fastest), overwritten
 *   stream     cudaStream_t (may be NULL) the kernels are launched on
 * Its 64-bit accumulator is a static device array sized for nc <= 64 (2 MiB, held
 * by every GPU that loads the library until exit); larger nc returns
 * CUBE_ERR_CAPACITY.  Every call shares that array and clears it first, so calls
 * that overlap on the GPU race.  The first call on a device looks up the array's
 * address and should come before any stream capture.  Errors come back as the
 * status only (no context, so cube_last_error has no text for them); a CUDA
 * error already pending when the call starts is returned as CUBE_ERR_CUDA and
 * nothing is launched. */
int32_t cube_coarse_density_noalloc(int32_t nc, int32_t nnt, int32_t izipx, int64_t np_capacity, const void* xp,
                                    const int64_t* cell_start, float mass_p_cdm, float* rho, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUBE_GPU_H */
