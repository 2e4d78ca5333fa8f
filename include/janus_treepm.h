/*
 * janus_treepm.h -- C ABI of the B200 bimetric TreePM force-and-step engine.
 *
 * Two species of opposite gravitational mass (m+ and m-) in a periodic cube
 * [-L/2, L/2)^3.  Same signs attract, opposite signs repel (janus-sim
 * src/lib.rs:94-121).  Per-species particle arrays in, per-species
 * accelerations out.  Arrays are AoS float3 (x,y,z per particle), the layout
 * of the reference's Vec<f32> position/velocity buffers
 * (src/nbody_gpu_twopass.rs:2159-2176).
 *
 * Conventions (the reference's FFI returns 0 or -1 after printing to stderr,
 * cuda/cufft_wrapper.cu:13-27; here every entry point returns 0 or one of the
 * negative JT_E* codes below and prints nothing):
 *   - the caller owns every array it passes; `mem` says whether the pointers
 *     are host (JT_MEM_HOST) or device (JT_MEM_DEVICE, current device) memory;
 *   - a handle owns all its device state, cuFFT plans and a private stream;
 *     handles are independent (no process-global state), one host thread per
 *     handle at a time;
 *   - every call returns after its GPU work has finished.
 */
#ifndef JANUS_TREEPM_H
#define JANUS_TREEPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---- */
#define JT_OK          0
#define JT_EINVAL     -1   /* bad argument (the reference's only error value) */
#define JT_ENOMEM     -2   /* device or host allocation failed */
#define JT_ECUDA      -3   /* a CUDA or cuFFT call failed */
#define JT_ETIMEDOUT  -4   /* a bounded device-side wait gave up */
#define JT_ENOTIMPL   -5   /* feature not available in this build */
#define JT_ESTATE     -6   /* call out of order (e.g. no particles set) */
#define JT_EOVERFLOW  -7   /* a fixed-capacity device list overflowed */
#define JT_EBUSY      -8   /* admission refused (batch / serve) */

/* ---- memory kinds ---- */
#define JT_MEM_HOST    0
#define JT_MEM_DEVICE  1

/* ---- force modes ---- */
/* ACCURATE: signed-source PM (PCS assignment with interlacing by default,
 * deconvolved, Gaussian long-range filter, spectral gradient), short-range
 * factor erfc(x) + 2x/sqrt(pi) exp(-x^2), x = r / (2 r_s), Plummer softening,
 * monopole + quadrupole nodes, hard cut at r_cut. */
#define JT_ACCURATE    0
/* RCOMPAT: the reference GPU formulas (src/nbody_gpu_twopass.rs:98-257,
 * 1670-1811; cuda/cufft_wrapper.cu:148-208): finite-difference gradient of the
 * undeconvolved potential, erfc-only short-range factor with r_s = r_cut/3,
 * 16-bit quantised theta/softening and integer r_cut/box_half, warp-uniform
 * opening decisions over groups of 32 particles of the concatenated
 * [m+ ; m-] arrays, monopole nodes with the reference's cube geometry. */
#define JT_RCOMPAT     1

/* ---- integrators ---- */
#define JT_KDK         0   /* kick(dt/2) drift(dt) force kick(dt/2) */
#define JT_DKD_REF     1   /* drift(dt/2) force kick(dt) drift(dt/2), the
                              reference's step_treepm_gpu order (:4518-4637) */

/* Configuration.  Mirrors the reference's TreePM fields
 * (TreePMForce{r_cut, r_s, softening, g_constant}, src/treepm/treepm_force.rs:
 * 17-25; GpuNBodyTwoPass{theta, softening, box_size, pm_grid_size, pm_k_min,
 * mass_factor}, src/nbody_gpu_twopass.rs:1874-1893). */
typedef struct jt_config {
    double box_L;        /* box side (Mpc); positions in [-L/2, L/2) */
    int    pm_grid;      /* PM cells per side M, power of two, 8..1024 */
    double theta;        /* Barnes-Hut opening angle */
    double softening;    /* Plummer softening eps */
    double r_s;          /* long/short split scale (ACCURATE; RCOMPAT uses r_cut/3) */
    double r_cut;        /* short-range cutoff */
    double mu;           /* total-mass ratio M- / M+ */
    double G_mass_plus;  /* G * (mass of one m+ particle); m- = mu*m+*N+/N- */
    int    k_min;        /* zero modes with max(|kx|,|ky|,|kz|) < k_min; 0 = off */
    int    mode;         /* JT_ACCURATE | JT_RCOMPAT */
    int    integrator;   /* JT_KDK | JT_DKD_REF */
    /* ACCURATE mass assignment: 0 = default (PCS), 2 = CIC, 3 = TSC, 4 = PCS
     * (the cubic B-spline, 64 cells per particle and grid).  At r_s = 1.25
     * cells with interlacing, on a Zel'dovich lattice (FP64 oracle, PM part
     * relative to the total force): TSC p50 2.4e-4 / p99 2.5e-3, PCS
     * p50 1.6e-5 / p99 2.6e-4; CIC leaves ~1e-2. */
    int    pm_order;
    /* ACCURATE interlacing (second grid shifted by half a cell, odd aliases
     * cancel): 0 = default (on), 1 = on, 2 = off. */
    int    pm_interlace;
    /* ACCURATE short-range tail: 0 = the walk cuts at r_cut as given; k > 0 =
     * the walk's cut is widened (r_cut stays the floor) to the radius where
     * the short-range factor S(r / 2 r_s) falls to k * 1e-6, so that the pairs
     * the cut drops carry at most that fraction of their Newtonian force.
     * With r_cut = 4.5 r_s, S(2.25) = 1.8 % sets the error floor against the
     * full periodic sum (p99 ~7e-3 on uniform boxes); k = 440 (S = 4.4e-4,
     * cut 6 r_s) brings that part of the error to the softening convention's
     * floor (p99 ~3e-4) at (6 / 4.5)^3 = 2.4x the pairs. */
    int    cut_tail_ppm;
    int    reserved[2];  /* zero */
} jt_config;

typedef struct jt_handle jt_handle;

/* The short-range cut an accurate-mode handle or batch box uses for this
 * config: r_cut, widened by cut_tail_ppm when that is set.  No counterpart
 * in the reference (its cut is r_cut). */
int  jt_config_short_cut(const jt_config* cfg, double* cut);

/* Stage timings of the last jt_accel / jt_step call, milliseconds of device
 * time (CUDA events on the handle's stream), summed over the call. */
typedef struct jt_timings {
    double sort_ms;      /* Morton keys + radix sort + reorder */
    double tree_ms;      /* Karras nodes + bottom-up moments */
    double deposit_ms;   /* CIC deposit of the signed source */
    double fft_ms;       /* R2C + k-space kernel + C2R */
    double kspace_ms;    /* the fused k-space kernel alone (part of fft_ms) */
    double walk_ms;      /* PM interpolation + short-range walk (+ kick) */
    double kick_drift_ms;/* kick/drift kernels outside the walk */
    double total_ms;     /* whole call */
    int64_t interactions;/* pair + node interactions evaluated by the walk */
    int64_t launches;    /* kernels launched by the library (cuFFT's not counted) */
    int64_t pair_interactions;  /* particle pairs inside r_cut (the cell walk's
                                   with the pair counters on: jt_set_counters) */
    int64_t node_interactions;  /* multipole node interactions */
    int64_t candidates;         /* particle candidates distance-tested */
    double cellwalk_ms;  /* the near-field cell walk kernel alone (part of walk_ms) */
    double interp_ms;    /* the tiled PM interpolation kernel alone (part of walk_ms) */
} jt_timings;

/* Pair counters, a diagnostic: with on != 0 the near-field cell walk counts
 * its pairs inside r_cut into pair_interactions and interactions (one
 * instruction per candidate pair, about 5 % of the walk's time).  Off by
 * default (JT_COUNTERS=1 in the environment when a handle, batch or server
 * is made turns them on), when those fields hold the tree walk's pairs and
 * nodes only.  jt_batch_set_counters and jt_server_set_counters (declared
 * with the batches and the server) do the same for their boxes. */
int  jt_set_counters(jt_handle* h, int on);

/* Create a handle on the current CUDA device.  Replaces the constructor and
 * setters of GpuNBodyTwoPass (src/nbody_gpu_twopass.rs:2159-2336) and
 * TreePMForce::new (src/treepm/treepm_force.rs:35-49). */
int  jt_create(const jt_config* cfg, jt_handle** out);

/* Load both species.  Replaces GpuNBodyTwoPass::with_custom_ics (:2159-2303)
 * with per-species arrays (the reference takes one array plus i8 signs; the
 * m+ array here is its sign>0 subset in order, the m- array its sign<0 subset).
 * vel_* may be NULL (zero velocities).  n_p or n_m may be 0. */
int  jt_set_state(jt_handle* h,
                  const float* pos_p, const float* vel_p, size_t n_p,
                  const float* pos_m, const float* vel_m, size_t n_m,
                  int mem);

/* The reference's layout: one array and i8 signs (+1 / -1), exactly the
 * arguments of with_custom_ics.  RCOMPAT groups warps in this array order. */
int  jt_set_state_signed(jt_handle* h, const float* pos, const float* vel,
                         const int8_t* signs, size_t n, int mem);

/* Accelerations at the current positions (force only; the parity entry
 * point).  Replaces compute_short_range_forces + the PM half of
 * step_treepm_gpu (:3961-4138, :4530-4600) and TreePMForce::
 * compute_all_forces (src/treepm/treepm_force.rs:124-131).  Outputs in the
 * caller's order; either pointer may be NULL. */
int  jt_accel(jt_handle* h, float* acc_p, float* acc_m, int mem);
/* Same, for a state loaded with jt_set_state_signed: acc in that order. */
int  jt_accel_signed(jt_handle* h, float* acc, int mem);
/* One part of the acceleration: JT_PART_PM (long range only, the reference's
 * pm_only mode, TreePMForce::new_pm_only src/treepm/treepm_force.rs:52-63),
 * JT_PART_SHORT (tree only), JT_PART_ALL (= jt_accel).  Per-species output. */
#define JT_PART_ALL    3
#define JT_PART_PM     1
#define JT_PART_SHORT  2
int  jt_accel_part(jt_handle* h, int part, float* acc_p, float* acc_m, int mem);

/* Advance nsteps steps of length dt.  Kick: v += (a - H v dtau_per_dt) dt,
 * the reference's kick_f32 (:50-64) with hubble = H; drift x += v dt with
 * one periodic wrap (:33-48).  Replaces step_treepm_gpu(dt, r_cut, hubble,
 * dtau_per_dt) (:4486-4649); r_cut comes from the config. */
int  jt_step(jt_handle* h, double dt, double hubble, double dtau_per_dt, int nsteps);

/* The accelerations a KDK step starts from, as part of the state: jt_get_accel
 * reads the stored ones (at the current positions, as the last step or
 * force call left them; JT_ESTATE when there are none) without computing
 * anything, and jt_set_accel loads them after jt_set_state, so that a state
 * taken out with jt_get_state + jt_get_accel and put back steps on without an
 * extra force pass (the reference's DKD step needs none: it keeps no forces
 * between steps).  Per-species layout only. */
int  jt_set_accel(jt_handle* h, const float* acc_p, const float* acc_m, int mem);
int  jt_get_accel(jt_handle* h, float* acc_p, float* acc_m, int mem);

/* One step of a state the host holds between steps, in one call: the host
 * arrays (per species AoS float3, the handle's current counts; pinned for
 * full PCIe speed) are uploaded, stepped once, and overwritten in place with
 * the new positions, velocities and (KDK) the accelerations at the new
 * positions.  It equals jt_set_state + jt_set_accel + jt_step(1) +
 * jt_get_state + jt_get_accel.  In accurate KDK mode the positions, final
 * after the drift, are copied back on a side stream while the force pass
 * runs.  With JT_DKD_REF the acc arrays are not used (may be NULL).  The
 * reference's drivers upload ICs once and call get_particles() after
 * step_treepm_gpu (src/nbody_gpu_twopass.rs:4486-4649); this is that round
 * trip for a host-resident state. */
int  jt_step_host(jt_handle* h, float* pos_p, float* vel_p, float* acc_p,
                  float* pos_m, float* vel_m, float* acc_m,
                  double dt, double hubble, double dtau_per_dt);

/* Yukawa screening of opposite-sign pairs: the reference's set_lambda_0 /
 * set_current_z (src/nbody_gpu_twopass.rs:2305-2312) as its TreePM step uses
 * them (compute_short_range_forces, :3997-4068).  With lambda_0 > 0.01 the
 * short-range walk becomes the reference's screened full-range walk
 * (forces_twopass_warpcoherent_screening, :911-1035): no r_cut prune and no
 * erfc; a same-sign pair contributes m / r_p^3, an opposite-sign pair
 * -exp(-x)(1 + x) m / r_p^3 with x = r_p / lambda(z), lambda(z) = lambda_0
 * sqrt(1 + z) quantised down to 0.1; theta and softening are rounded to
 * 1e-3.  The PM part is unchanged.  On a JT_ACCURATE handle the screening
 * is the split model's instead (jt_batch_set_screening, applied to the
 * handle's box and kept across jt_set_state).  lambda_0 <= 0.01 turns it
 * off.  Takes effect at the next force evaluation. */
int  jt_set_screening(jt_handle* h, double lambda_0, double z);

/* Read the state back in the caller's order (get_particles, :5470).  Any
 * pointer may be NULL. */
int  jt_get_state(jt_handle* h, float* pos_p, float* vel_p, float* pos_m,
                  float* vel_m, int mem);
int  jt_get_state_signed(jt_handle* h, float* pos, float* vel, int mem);

/* Topology of one species' tree built at the current positions with the
 * reference's keys ((morton30 << 32) | index in the species array), in the
 * reference's numbering (internal 0..n-2, leaves n-1..2n-2;
 * build_bvh_tp :407-447): morton[n] (sorted 30-bit codes), perm[n] (species
 * index of each sorted position), left/right/parent[2n-1] (leaf entries of
 * left/right are 0; parent[0] = -1).  species: 0 = m+, 1 = m-.  Host memory. */
int  jt_debug_tree(jt_handle* h, int species, uint32_t* morton, int32_t* perm,
                   int32_t* left, int32_t* right, int32_t* parent);

int  jt_get_timings(jt_handle* h, jt_timings* t);
/* Walk phase counters accumulated since jt_create (traversal iterations,
 * ranges streamed, candidate chunks, pair-loop trips); non-zero only in a
 * diagnostic build compiled with -DJT_WALK_COUNT.  No counterpart in the
 * reference. */
int  jt_walk_counters(jt_handle* h, int64_t* out4);
int  jt_counts(jt_handle* h, size_t* n_p, size_t* n_m);
void jt_destroy(jt_handle* h);
const char* jt_strerror(int code);
/* FP32 FMA throughput of the current device (TFLOP/s), measured by a
 * register-only FMA kernel: the roofline denominator for the walk.  No
 * counterpart in the reference. */
int  jt_fp32_peak(int iters, double* tflops);
/* The walk's launch shapes picked by its autotuner so far (one entry per
 * device and size class: register budget as blocks per SM, leaf-bucket
 * size), and the near-field cells per axis timed fastest on the first
 * force-only pass of each box of 2^22 particles or more (the default
 * L / r_cut and the one kept), as text.  No counterpart in the reference. */
int  jt_walk_tuning(char* buf, size_t len);
/* ---- in-step diagnostics (device, FP64 accumulation) ----
 * segregation: |COM+ - COM-| / L, the reference's segregation()
 * (src/nbody_gpu_twopass.rs:5364-5393); diff_over_poisson, corr and
 * exc_var_minus: compute_segregation_metrics on an n_cells^3 NGP count grid
 * (src/bin/janus_mu19_production.rs:219-276); per species the kinetic energy
 * (1/2) sum m v^2, momentum sum m v and mean position, with m the particle
 * mass of the config (G folded in).  Computed over the resident state with
 * no copy of the particles. */
typedef struct jt_diag {
    double segregation;
    double diff_over_poisson;   /* Var(n+ - n-) / (mean+ + mean-) */
    double corr;                /* Corr(delta+, delta-) */
    double exc_var_minus;       /* (Var(n-) - mean-) / mean- */
    double kinetic[2];
    double momentum[2][3];
    double com[2][3];
} jt_diag;
int  jt_diagnostics(jt_handle* h, int n_cells, jt_diag* out);

/* ---- snapshots (the reference's snapshot_v3 format) ----
 * src/snapshot_v3.rs:12-47, 260-376: a 408-byte little-endian header and
 * 36-byte particles (f32 pos[3], vel[3], mass, softening; u8 sign 1 / 255,
 * split level, star flag, flags).  The metadata the engine does not know
 * (expansion state, Hubble constant, seeds, label) comes from the caller. */
typedef struct jt_snapshot_meta {
    double   a;            /* scale factor */
    double   t_gyr;        /* cosmic time (Gyr) */
    double   h0;           /* Hubble constant (km/s/Mpc) */
    double   omega_b;
    double   z_init;       /* initial redshift of the ICs */
    double   z_start_run;  /* start redshift of this run */
    uint32_t seed_ic;
    char     run_label[256];
} jt_snapshot_meta;
/* Write n particles (host arrays; vel may be NULL) to a snapshot file. */
int  jt_snapshot_write(const char* path, const jt_snapshot_meta* meta, double box_L, double mu,
                       const float* pos, const float* vel, const int8_t* signs,
                       const float* mass, const float* eps, size_t n);
/* Read a snapshot: *n = its particle count; pos == NULL asks for the header
 * only; otherwise arrays of cap >= n particles (vel, mass, eps may be NULL). */
int  jt_snapshot_read(const char* path, jt_snapshot_meta* meta, double* box_L, double* mu,
                      float* pos, float* vel, int8_t* signs, float* mass, float* eps,
                      size_t cap, size_t* n);
/* Checkpoint a handle's state (caller order, signs, config masses and
 * softening); resume with jt_snapshot_read + jt_set_state_signed. */
int  jt_checkpoint(jt_handle* h, const char* path, const jt_snapshot_meta* meta);

/* The production driver's raw snapshot (save_snapshot,
 * src/bin/janus_mu19_production.rs:198-216): u32 n, f32 box, u32 step, f32 z,
 * then n records of f32 pos[3], f32 vel[3], i8 sign (25 bytes, little-endian,
 * no padding).  read: pos == NULL only reads the header into n/box/step/z;
 * otherwise cap >= n rows are filled (vel may be NULL). */
int  jt_snapshot_write_raw(const char* path, const float* pos, const float* vel,
                           const int8_t* signs, size_t n, double box_L, uint32_t step,
                           double z);
int  jt_snapshot_read_raw(const char* path, float* pos, float* vel, int8_t* signs,
                          size_t cap, size_t* n, double* box_L, uint32_t* step, double* z);

/* Energies in FP64 on the device, the reference's GpuNBodyTwoPass
 * diagnostics (src/nbody_gpu_twopass.rs) without the host copy of the state:
 *   kinetic    = sum |v|^2 / 2 over all particles, unit masses
 *                (kinetic_energy, :5070-5077);
 *   pe_plus / pe_minus = per species, a stride sample of at most n_sample
 *                particles (rows i * (n_s / n_sample) of the species array),
 *                -sum_{i<j} 1 / sqrt(r^2 + eps^2) with plain (non-periodic)
 *                differences, times n_s (n_s - 1) / (ns (ns - 1))
 *                (potential_energy_binding_sampled, :5081-5181);
 *   pe_binding = pe_plus + pe_minus (same-species pairs only). */
typedef struct jt_energy {
    double  kinetic;
    double  pe_binding;
    double  pe_plus, pe_minus;
    int64_t n_sampled[2];
} jt_energy;
int  jt_energy_sampled(jt_handle* h, size_t n_sample, jt_energy* out);
/* virialize_sampled (:5186-5225): multiply every velocity by alpha =
 * sqrt(|pe_binding| / (2 kinetic)) when pe_binding < 0 and kinetic >= 1e-20
 * (else alpha = 1 and nothing changes); *alpha (may be NULL) receives it. */
int  jt_virialize_sampled(jt_handle* h, size_t n_sample, double* alpha);
/* energy_drift_pct (src/janus_expansion.rs:529-534): (e_now - e_initial) /
 * |e_initial| * 100, 0 when |e_initial| < 1e-30. */
double jt_energy_drift_pct(double e_now, double e_initial);

/* Zel'dovich lattice initial conditions generated on the device (the host
 * generator it replaces is the reference's generate_zeldovich_ics,
 * src/ic_gen.rs:52-176, which builds the field with rustfft on the CPU).
 * Per species an n_side^3 lattice of spacing a = box_L / n_side, the m-
 * lattice offset by a/2 on every axis; displacements psi = i k / k^2 delta(k)
 * of a Gaussian field with P(k) = A k^-2.5 exp(-(k/k_c)^2), k_c = pi / (2 a)
 * (half the lattice Nyquist wavenumber), A such that rms |psi+| = rms_frac a;
 * psi- = -psi evaluated on the offset lattice (delta- = -delta+); velocities
 * v = vel_factor psi.  The white noise is Philox4x32-10 (counter = the cell
 * index, key = seed) through Box-Muller in FP64; the Nyquist planes and k = 0
 * are zero.  Rows are in lattice order iz n^2 + iy n + ix, AoS float3. */
typedef struct jt_ics_params {
    int      n_side;     /* lattice points per side per species, 4..1024 */
    double   box_L;
    uint64_t seed;
    double   rms_frac;   /* rms displacement / lattice spacing (0.3) */
    double   vel_factor; /* v = vel_factor * psi */
} jt_ics_params;
/* Into caller arrays of n_side^3 rows (host or device per mem; velocity
 * pointers may be NULL); generated on the current device. */
int  jt_ics_zeldovich(const jt_ics_params* p, float* pos_p, float* vel_p,
                      float* pos_m, float* vel_m, int mem);
/* Generate and load as the handle's state (as jt_set_state; no host copy). */
int  jt_set_state_zeldovich(jt_handle* h, const jt_ics_params* p);
/* The generator's counter-based stream on the host (Philox4x32-10 with 10
 * rounds), for checks against its published known-answer vectors. */
void jt_philox4x32_10(const unsigned ctr[4], const unsigned key[2], unsigned out[4]);

/* Failure-path self test: runs the sort's bounded look-back wait on a
 * status word that nothing publishes, with `limit` polls (1..2^24).  Returns
 * JT_ETIMEDOUT with *timed_out = 1 when the wait gave up and reported it (the
 * expected outcome); the device context stays usable.  No counterpart in the
 * reference. */
int  jt_wait_probe(int limit, int* timed_out);
/* Library version string, e.g. "janus-treepm-b200 0.1 sm_100a". */
const char* jt_version(void);

/* ---- batched ensembles ----
 * A batch advances many independent boxes with one kernel launch per stage
 * over the work of all chosen boxes, and one batched cuFFT R2C/C2R per
 * distinct grid size.  It replaces the reference's one-process-per-box
 * parameter scans (optim/run_tour.py:40-48, scripts/run_scan_mu.sh driving
 * step_treepm_gpu once per box).  Boxes may differ in particle counts, box
 * size, grid, theta, softening, r_s, r_cut, mu and step; all boxes of one
 * batch share pm_order, pm_interlace and k_min, and must be JT_ACCURATE with
 * JT_KDK.  Every call synchronises the batch's own stream before it returns. */
typedef struct jt_batch jt_batch;

/* Per-box step arguments of jt_batch_step (one entry per listed box). */
typedef struct jt_step_args {
    double dt;           /* step length */
    double hubble;       /* H of the kick drag term v += (a - H v dtau) dt */
    double dtau_per_dt;  /* the reference's dtau factor (step_treepm_gpu) */
} jt_step_args;

int  jt_batch_create(jt_batch** out);
void jt_batch_destroy(jt_batch* b);
/* Add one box (per-species arrays as jt_set_state); *box_id receives its id.
 * JT_EINVAL if the config is not batchable or disagrees with the batch's
 * shared fields; JT_ENOMEM if its state does not fit on the device. */
int  jt_batch_add(jt_batch* b, const jt_config* cfg,
                  const float* pos_p, const float* vel_p, size_t n_p,
                  const float* pos_m, const float* vel_m, size_t n_m,
                  int mem, int* box_id);
/* Add a box whose state is generated on the device (jt_ics_params). */
int  jt_batch_add_zeldovich(jt_batch* b, const jt_config* cfg, const jt_ics_params* p, int* box_id);
/* Checkpoint one box to a snapshot_v3 file (rows [m+ ; m-] in the caller's
 * order) without waiting for it: the state is gathered on the batch's stream,
 * copied to pinned host memory on a side stream and written by a host
 * thread, so a jt_batch_step issued right after overlaps the copy and the
 * write.  One checkpoint per batch in flight (JT_EBUSY until collected);
 * jt_batch_checkpoint_wait collects it and returns the write's status (JT_OK
 * when none is pending).  The reference's snapshots block on a full
 * device-to-host copy (src/snapshot_v3.rs:260-376). */
int  jt_batch_checkpoint_async(jt_batch* b, int box_id, const char* path,
                               const jt_snapshot_meta* meta);
int  jt_batch_checkpoint_wait(jt_batch* b);
/* Create the cuFFT plans that passes over boxes of this grid size can use
 * (one per power-of-two batch up to an execution's limit of 2^27 elements,
 * both directions), so that no later step creates one: a plan costs more to
 * make than its transforms take.  Steps create what they lack anyway; this
 * moves the cost ahead (the serving loop calls it when a job with a new
 * grid size is registered).  jt_batch_trim releases them. */
int  jt_batch_prepare(jt_batch* b, int pm_grid);
/* Yukawa screening of one box's opposite-species pairs in the split model:
 * kappa = 1 / lambda, lambda = lambda_0 sqrt(1 + z) (no quantisation; the
 * reference's set_lambda_0 / set_current_z, src/nbody_gpu_twopass.rs
 * :2305-2312, screening factor :1000-1017).  Same-species pairs stay
 * Newtonian; an opposite-species pair has the potential -e^{-kappa r} / r.
 * The Gaussian split applies to both kernels: the box deposits the signed
 * source D and the unsigned source S, the k-space kernel gives D
 * (G_N + G_Y) / 2 and S (G_N - G_Y) / 2 with G_Y = 4 pi e^{-(k^2 + kappa^2)
 * r_s^2} / (k^2 + kappa^2), and the short-range walk evaluates opposite-
 * species pairs with the Yukawa short kernel (1 / 2r) [e^{-kappa r}
 * erfc(r / 2r_s - kappa r_s) + e^{kappa r} erfc(r / 2r_s + kappa r_s)],
 * directly (no multipoles).  Costs a second deposit and twice the FFT work
 * of the box.  lambda_0 <= 0.01 turns it off. */
int  jt_batch_set_screening(jt_batch* b, int box_id, double lambda_0, double z);
/* Free one box's device state; its id may be reused by a later add. */
int  jt_batch_remove(jt_batch* b, int box_id);
/* Accelerations of the listed boxes at their current positions (JT_PART_*). */
int  jt_batch_forces(jt_batch* b, const int* box_ids, int n_ids, int part);
/* nsteps KDK steps of the listed boxes, args[k] for box_ids[k]. */
int  jt_batch_step(jt_batch* b, const int* box_ids, int n_ids,
                   const jt_step_args* args, int nsteps);
/* Per-box read-back in the caller's species order (NULL pointers skipped). */
int  jt_batch_get_accel(jt_batch* b, int box_id, float* acc_p, float* acc_m, int mem);
int  jt_batch_get_state(jt_batch* b, int box_id, float* pos_p, float* vel_p,
                        float* pos_m, float* vel_m, int mem);
int  jt_batch_box_info(jt_batch* b, int box_id, size_t* n_p, size_t* n_m, size_t* bytes);
/* Device bytes held: persistent box state, and the grow-only per-pass scratch. */
int  jt_batch_memory(jt_batch* b, size_t* persistent, size_t* scratch);
/* Device bytes one box would need (no device work): its persistent state and
 * its share of the per-pass scratch.  The serving loop's admission control. */
int  jt_batch_estimate(const jt_config* cfg, size_t n_p, size_t n_m,
                       size_t* persistent, size_t* scratch);
int  jt_batch_get_timings(jt_batch* b, jt_timings* t);
/* jt_diagnostics of one box of a batch (jt_diag is declared above). */
int  jt_batch_diagnostics(jt_batch* b, int box_id, int n_cells, jt_diag* out);

/* on != 0: jt_batch_step replays each step as a CUDA graph, captured once
 * per set of boxes (two graphs: the reorder's ping-pong buffers alternate)
 * and recaptured when a box joins or leaves or a scratch pool grows.  The
 * graphs keep the two half kicks of consecutive steps separate (kick dt/2,
 * drift, forces + kick dt/2).  Stage timings are not collected inside
 * graphs (total_ms is). */
int  jt_batch_set_graphs(jt_batch* b, int on);
/* The pair counters of the batch's passes (as jt_set_counters). */
int  jt_batch_set_counters(jt_batch* b, int on);
/* Release the batch's per-pass scratch pools and cuFFT plans (they grow
 * back on the next pass); persistent box state is kept. */
int  jt_batch_trim(jt_batch* b);

/* ---- serving loop ----
 * Simulation jobs (one box each) admitted onto the device by an HBM budget,
 * their step requests served by continuous batching: every batched step
 * advances each resident job with a pending request by one KDK step in one
 * launch per stage; requests arriving meanwhile join the next step.  A job
 * that has taken all its steps is evicted to pinned host memory; idle
 * resident jobs are swapped out to make room for waiting ones.  No
 * counterpart in the reference (it runs one process per box). */
typedef struct jt_server jt_server;
typedef struct jt_serve_stats {
    int64_t requests_served;
    int64_t batched_steps;
    int64_t particle_steps;
    int64_t admitted;          /* admissions (a swapped-out job counts again) */
    int64_t evicted;           /* jobs finished and evicted to host memory */
    int64_t admission_waits;   /* admission attempts that did not fit */
    double  p50_latency_s;     /* per step request: completion - arrival */
    double  p99_latency_s;
    double  max_latency_s;
    double  busy_s;            /* wall time inside batched steps */
    int64_t peak_device_bytes; /* batch memory after a step, maximum */
    int64_t max_jobs_per_step;
    int64_t swapped_out;       /* idle jobs moved to host to admit others */
    int64_t trims;             /* scratch pools released to make room */
    double  admit_s;           /* wall time admitting jobs (state to the device) */
    double  evict_s;           /* wall time evicting and swapping out jobs (to host) */
    double  step_device_s;     /* device time of the batched steps (CUDA events) */
    double  reserved_gb;       /* memory the server's pool holds from creation (GB) */
} jt_serve_stats;

#define JT_JOB_QUEUED    0
#define JT_JOB_RESIDENT  1
#define JT_JOB_DONE      2

/* The server reserves its budget (at most 90 % of the device's free memory)
 * in its memory pool at creation, so that admissions and the batched steps'
 * scratch are carved from memory already mapped, not grown by the driver
 * while requests wait. */
int  jt_server_create(size_t hbm_budget_bytes, jt_server** out);
void jt_server_destroy(jt_server* s);
/* Register a job (host arrays copied to pinned memory; nothing on the device
 * until a request admits it).  JT_EBUSY if it can never fit the budget. */
int  jt_server_add_job(jt_server* s, const jt_config* cfg,
                       const float* pos_p, const float* vel_p, size_t n_p,
                       const float* pos_m, const float* vel_m, size_t n_m,
                       int steps_total, const jt_step_args* args, int* job_id);
/* Budget bytes a job needs when it is the only one resident: persistent
 * state, per-pass scratch with the pools' growth headroom and the cuFFT work
 * area (no device work). */
int  jt_server_job_need(const jt_config* cfg, size_t n_p, size_t n_m, size_t* bytes);
/* One step request for a job at t_arrival seconds on the server clock
 * (negative = now). */
int  jt_server_request(jt_server* s, int job, double t_arrival);
double jt_server_clock(jt_server* s);
/* Admit what fits, run one batched step; *served = requests it served. */
int  jt_server_poll(jt_server* s, int* served);
/* Replay an arrival schedule (t ascending, seconds from the call) in real
 * time until every request is served; JT_EBUSY if some can never be. */
int  jt_server_serve(jt_server* s, const double* t, const int* job, int n);
int  jt_server_job_state(jt_server* s, int job, int* state, int* steps_done);
int  jt_server_get_state(jt_server* s, int job, float* pos_p, float* vel_p,
                         float* pos_m, float* vel_m);
/* The accelerations a job holds at its current positions (those of its last
 * step; a swapped-out or finished job keeps them in pinned host memory);
 * JT_ESTATE before its first force pass. */
int  jt_server_get_accel(jt_server* s, int job, float* acc_p, float* acc_m);
int  jt_server_stats(jt_server* s, jt_serve_stats* out);
/* Stage times and counts of every batched step the server ran, summed
 * (opening force passes included); the fields as jt_get_timings'. */
int  jt_server_get_timings(jt_server* s, jt_timings* out);
/* The pair counters of the server's batched steps (as jt_set_counters). */
int  jt_server_set_counters(jt_server* s, int on);

/* ---- Janus expansion history (FP64) ----
 * The reference's JanusExpansion (src/janus_expansion.rs:62-266): the exact
 * parametric solution of the positive sector, a+(mu) = alpha^2 cosh^2 mu,
 * t+(mu) = alpha^2 (mu + sinh^2(mu) / 2) / H0, H+(mu) = H0 sinh(2 mu) /
 * (alpha^2 cosh^2 mu (1 + sinh(2 mu) / 2)), H0 = 0.0715 / Gyr, mu0 = 1.5,
 * alpha from H+(mu0) = H0, a+ = 1 and z = 0 at mu0.  A table of n_points
 * states uniform in mu from z_init (clamped to 0.99 z_max, z_max = the
 * redshift of mu = 0) to z = 0, interpolated linearly in time or redshift
 * as the reference's at_time / at_redshift: the drivers' step schedule
 * (t = t_start + k dt) and the kick's drag factor H (hubble of jt_step).
 * The reference's production run builds it with z_init = 4 and 5000 rows
 * (src/bin/janus_mu19_production.rs:46). */
typedef struct jt_expansion_state {
    double mu;       /* parameter mu */
    double a_plus;   /* scale factor, 1 at z = 0 */
    double t_gyr;    /* cosmic time (Gyr) */
    double h_plus;   /* Hubble rate (1/Gyr) */
    double z;        /* redshift */
} jt_expansion_state;
typedef struct jt_expansion_info_t {
    double  alpha, mu_0, a_0;   /* calibration (calibrate_alpha_mu0, :247-266) */
    double  z_max, z_init;      /* parametric limit; z_init after the clamp */
    double  t_start, t_end;     /* table range in time (Gyr) */
    int64_t n_points;
} jt_expansion_info_t;
typedef struct jt_expansion jt_expansion;
/* JanusExpansion::new(z_init, n_points) (:62-123); n_points >= 2. */
int  jt_expansion_create(double z_init, int n_points, jt_expansion** out);
void jt_expansion_destroy(jt_expansion* e);
int  jt_expansion_info(const jt_expansion* e, jt_expansion_info_t* out);
/* at_time (:126-154): t clamped to the table, linear interpolation of the
 * bracketing rows (t_gyr = the clamped t). */
int  jt_expansion_at_time(const jt_expansion* e, double t_gyr, jt_expansion_state* out);
/* at_redshift (:157-180): linear interpolation in z (z = the argument;
 * outside the table the end row). */
int  jt_expansion_at_redshift(const jt_expansion* e, double z, jt_expansion_state* out);
/* compute_state (:196-230) and calibrate_alpha_mu0 (:247-266). */
int  jt_expansion_state_at_mu(double mu, double alpha, double a_0, jt_expansion_state* out);
int  jt_expansion_calibrate(double* alpha, double* mu_0);
/* Cross-species factors of an eta scan: a- = a+ (1 + z)^{-(eta - 1) / eta}
 * (src/vsl_dynamic.rs:138-142), phi = (a- / a+)^3, phi_inv = (a+ / a-)^3
 * (src/janus_expansion.rs:449-462).  Outputs may be NULL. */
int  jt_expansion_phi_factors(double a_plus, double eta, double* a_minus, double* phi, double* phi_inv);

/* ---- allocation-free Morton sort ----
 * The reference's Morton keys of n positions already on the device (float3
 * array, box [-L/2, L/2)), sorted by the key (morton30 << 32) | i, i = the
 * row of the position in `pos` (equal codes keep their row order): writes
 * morton_out[n] (sorted 30-bit codes) and perm_out[n] (row of each sorted
 * position) to device memory.  For the species array a handle was loaded
 * with (jt_set_state) these are the morton/perm outputs of jt_debug_tree,
 * whose key carries each particle's index in that array in the low word.
 * Every byte of scratch of its onesweep radix sort lives in one fixed
 * file-scope static device array of JT_STATIC_SORT_BYTES (6.5 MiB); the call
 * allocates nothing (no cudaMalloc, cudaFree or allocating library call).
 * n must be 1..JT_STATIC_SORT_MAX, else JT_EINVAL.  stream: a cudaStream_t,
 * or NULL for the legacy default stream; the call synchronises that stream
 * before it returns (it reads the sort's error word: JT_ETIMEDOUT if a
 * bounded device wait gave up).
 * For callers that cannot allocate: code running inside a fixed HBM budget
 * (a served job's admission control counts every device byte it holds) and
 * code that must not synchronise the whole device (cudaMalloc and cudaFree
 * do, stalling every other stream on it).
 * The static array keeps the last call's contents; calls that overlap in
 * time (several threads or streams) race on it and must be serialised by the
 * caller.  The first call on each device looks up the array's address
 * (cudaGetSymbolAddress, once per device): make that first call before any
 * stream capture.  Every call copies the sort's error word to a host
 * variable and synchronises `stream` before it returns.  No counterpart in
 * the reference. */
#define JT_STATIC_SORT_MAX    262144
#define JT_STATIC_SORT_BYTES  6824448
int  jt_morton_sort_static(const float* pos, size_t n, double box_L,
                           uint32_t* morton_out, int32_t* perm_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
