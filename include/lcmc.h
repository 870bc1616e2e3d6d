/*
 * lcmc.h - C ABI of the B200 Gay-Berne Monte Carlo library (liblcmc.so).
 *
 * Drop-in for the Monte Carlo sweep of MCnptColloid.c.  The reference has no
 * plugin or FFI layer; its seam is the C call
 *
 *   void attempt_monte_carlo_move(double *position_x, ..., double *orient_z,
 *        float max_displacement, double *system_energy, int *neighbor_count_array,
 *        int *neighbor_list_array, long *accepted_moves, double *desp_max,
 *        size_t *histograma)                              (MCnptColloid.c:2445-2454)
 *
 * driven once per cycle by the serial loop at MCnptColloid.c:887-1032, with the
 * intended per-cell loop of the MPI path at MCnptColloid.c:683-700.  This ABI
 * replaces that loop: the caller's SoA double arrays are copied in, whole
 * sweeps run on the GPU (8-colour checkerboard, one trial move per particle per
 * sweep with the per-move semantics of attempt_monte_carlo_move), and the arrays
 * are copied back.  Every function returns an int status: 0 = LCMC_OK, negative
 * = LCMC_E* (the reference calls exit(1) instead).  There is no CPU fallback:
 * without a CUDA device every device call returns LCMC_ENODEV.
 *
 * Threading: one host thread per context; a context owns one CUDA stream and
 * is not reentrant.  A batch of 8 or more replicas also owns one helper
 * stream per further replica group: inside every sweep the colour phases of
 * each group run on its stream, forked from the context's stream after the
 * rebin and joined back into it before the statistics.
 */
#ifndef LCMC_H
#define LCMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LCMC_ABI_VERSION 2

enum {
    LCMC_OK = 0,
    LCMC_EINVAL = -1,    /* bad argument */
    LCMC_ENOFILE = -2,   /* parameter / configuration file cannot be opened */
    LCMC_EPARAM = -3,    /* missing or unparsable parameter (load_initial_conditions exits here) */
    LCMC_ECUDA = -4,     /* CUDA runtime error */
    LCMC_ENOMEM = -5,    /* device or host allocation failed */
    LCMC_ECELLCAP = -6,  /* a cell or its stencil holds more particles than the kernel's capacity */
    LCMC_ENUMERIC = -7,  /* NaN or Inf energy */
    LCMC_EBOX = -8,      /* box too small for the cutoff (L < 2 rc) or inconsistent sizes */
    LCMC_ENODEV = -9,    /* no CUDA device */
    LCMC_EOVERLAP = -10, /* a particle centre inside the colloid (check_no_colloid_overlaps, MCnptColloid.c:1324-1340) */
    LCMC_ETIMEOUT = -11, /* a bounded wait inside a tensor-core kernel gave up (the kernel returned cleanly) */
    LCMC_EDRIFT = -12    /* a periodic FP64 energy check found the running energy out of tolerance
                            (EnergyCheck, MCnptColloid.c:1343-1362, only prints); the running energy
                            was reset to the recomputed value and the chain is unchanged */
};

enum { LCMC_PREC_FP64 = 0, LCMC_PREC_FP32 = 1 };
enum { LCMC_NVT = 1, LCMC_NPT = 2 };

/* The 23 keys of parametersFile.txt (read by load_initial_conditions,
 * MCnptColloid.c:3933-4133) and the keys this library adds.  Added keys are
 * ignored with a warning by the reference parser (MCnptColloid.c:4093), so one
 * file serves both. */
typedef struct {
    int mc_ensemble_type;            /* 1 = NVT, 2 = NPT */
    int num_particles;
    double system_density;
    double system_temperature;
    double system_pressure;
    double gb_sigma_sidetoside;      /* sigma_0 */
    double gb_epsilon0;
    double gb_kappa;
    double gb_kappa_prime;
    double gb_mu_exponent;
    double gb_nu_exponent;
    float max_displacement;          /* full width of the trial translation */
    float max_rotation;
    int initial_configuration_type;  /* 0 file, 1 random, 2 lattice */
    double cutoff_radius;
    double verlet_radius;            /* parsed; the cell grid replaces the Verlet list */
    int total_mc_cycles;
    int configuration_save_interval;
    int statistics_print_interval;
    int colloid_wall_option;         /* 1 = colloid term on */
    double colloid_interaction_epsilon;   /* parsed, unused (as in the reference) */
    double colloid_interaction_amplitude; /* parsed, unused (as in the reference) */
    double colloid_radius;
    /* added keys */
    uint64_t rng_seed;
    int total_mc_sweeps;             /* sweeps of a run_simulation driver run; 0 = ceil(total_mc_cycles / num_particles) */
    int cell_capacity;               /* active-cell capacity of the FP32 kernel (<= 48: small class, six
                                        blocks per SM; <= 64: large class); 0 = automatic: NVT from the
                                        creation density, NPT the large class.  A cell holding more
                                        particles is attempted in FP64 (counted in overcap_cells) */
    double npt_max_dlnV;
    int volume_moves_per_sweep;      /* 0 or 1 */
    int precision_mode;              /* LCMC_PREC_FP64 / LCMC_PREC_FP32 */
    double init_orientation_cone_deg;/* 180 = uniform on the sphere */
    int n_read;                      /* out: number of reference keys found */
    int missing_mask;                /* out: bit i = reference key i missing */
    /* added keys (continued) */
    int energy_check_interval;       /* sweeps between periodic FP64 energy checks, 0 = off (the reference's
                                        check_energy / EnergyCheck, MCnptColloid.c:946-955, 1343-1362) */
    double energy_check_tolerance;   /* relative tolerance of the check against max(|E|, N 4 eps0) plus the
                                        sum of |dE| accepted since the last check; 0 = automatic: 1e-4 for
                                        the FP32 kernel, 1e-9 for the FP64 kernel */
    int init_lattice;                /* lattice of initial_configuration_type 2: 0 = simple cubic (the
                                        reference's), 1 = body-centred tetragonal with the long axis along z,
                                        spacing 1.05 sigma_ee along z (a start for orientations near z
                                        with no pair in the overlap clamp) */
    int cell_grid;                   /* 0 = even cell count per axis, 8-colour checkerboard (the CPU oracle's
                                        schedule); 1 = fine: the largest count of cells at least
                                        cutoff + max_displacement wide, odd counts taking 3 colours on that
                                        axis (up to 27 colour phases), so small boxes keep cells about one
                                        cutoff wide (and on the FP32 kernel) instead of up to 1.5 cutoffs */
} lcmc_params;

typedef struct {
    int64_t sweeps;              /* sweeps done on this replica */
    int64_t attempted;           /* trial moves (one per particle per sweep) */
    int64_t accepted;
    int64_t hardcore_rejected;   /* trial centre inside the colloid */
    int64_t volume_attempted;
    int64_t volume_accepted;
    double energy;               /* running total energy: last recompute + accepted dE (FP64) */
    double box[3];
    double last_recompute;       /* last FP64 total-energy recompute */
    double drift;                /* running minus recomputed energy at the last recompute */
    int64_t pairs_in_cutoff;     /* sum over attempts of in-cutoff pairs, old + new states */
    int64_t stencil_candidates;  /* sum over attempts of 27-cell stencil candidates, excluding self */
    int error_flags;             /* LCMC_F* bits seen by the kernels */
    int kernel;                  /* 0 = FP64 kernel, 1 = FP32 kernel */
    int64_t volume_stage1_rejected; /* volume moves the surrogate rejected (no exact energy computed) */
    int64_t fp64_cells;          /* FP32-kernel cell attempts run in FP64: a pair term above 100 eps0 (an
                                    overlap), or the cell above the kernel's capacity */
    int64_t overcap_cells;       /* of which: above the cell, staged-candidate or list capacity */
    int64_t energy_checks;       /* periodic FP64 energy checks run */
    int64_t drift_breaches;      /* checks out of tolerance */
    double drift_bound;          /* tolerance of the last check (absolute energy) */
    double abs_dE_since_check;   /* sum of |dE| of accepted moves since the last check */
} lcmc_stats;

/* error_flags bits */
enum {
    LCMC_F_CELLCAP = 1,     /* not set by this version: a cell above the FP32 kernel's capacity (active,    */
    LCMC_F_STENCILCAP = 2,  /* staged-candidate or list) is attempted in FP64 and counted in overcap_cells; */
    LCMC_F_LISTCAP = 4,     /* the bits stay reserved                                                       */
    LCMC_F_NONFINITE = 8,   /* NaN/Inf energy change */
    LCMC_F_GRIDCAP = 16,    /* box grew past the allocated cell grid (cells kept wider) */
    LCMC_F_DRIFT = 32       /* a periodic FP64 energy check was out of tolerance */
};

/* ---- parameters (host only) ---- */
int lcmc_params_defaults(lcmc_params *p);
/* load_initial_conditions (MCnptColloid.c:3933-4133): 23 required keys,
 * unknown keys ignored, missing keys -> LCMC_EPARAM with p->missing_mask set. */
int lcmc_params_load(const char *path, lcmc_params *p);

/* ---- context ---- */
typedef struct lcmc_ctx lcmc_ctx;
/* One system (replica 0). */
int lcmc_create(const lcmc_params *p, lcmc_ctx **out);
/* n independent systems sweeping together in shared launches (replica r has params[r]). */
int lcmc_create_batch(const lcmc_params *params, int n_replicas, lcmc_ctx **out);
int lcmc_destroy(lcmc_ctx *ctx);
int lcmc_num_replicas(const lcmc_ctx *ctx);

/* get_initial_config (MCnptColloid.c:4215-4235) for initial_configuration_type 2:
 * seeded simple-cubic lattice, box V = N/rho + V_colloid; uploads it. */
int lcmc_init_config(lcmc_ctx *ctx, int replica);
/* Host lattice only (no device): fills the caller's arrays and box. */
int lcmc_lattice(const lcmc_params *p, int replica, double *px, double *py, double *pz, double *ox, double *oy,
                 double *oz, double box[3]);

/* Copy the caller's SoA arrays (positions in [0, L], orientations) to the
 * device and recompute the total energy in FP64.  The arrays are checked on
 * the device (box bounds, no rod centre inside the colloid as in
 * check_no_colloid_overlaps, MCnptColloid.c:1324-1340, finite non-zero
 * orientations); a rejected upload leaves the replica's state unchanged. */
int lcmc_upload(lcmc_ctx *ctx, int replica, const double *px, const double *py, const double *pz, const double *ox,
                const double *oy, const double *oz, int n, const double box[3]);
/* As lcmc_upload, with the caller's running energy in place of the FP64
 * recompute: the energy in/out argument of attempt_monte_carlo_move
 * (MCnptColloid.c:2445-2454, `double *system_energy`), whose caller carries
 * the energy from call to call.  The replica's energy becomes `energy`. */
int lcmc_upload_with_energy(lcmc_ctx *ctx, int replica, const double *px, const double *py, const double *pz,
                            const double *ox, const double *oy, const double *oz, int n, const double box[3],
                            double energy);
int lcmc_download(lcmc_ctx *ctx, int replica, double *px, double *py, double *pz, double *ox, double *oy, double *oz,
                  int n, double box[3]);

/* n_sweeps checkerboard sweeps on every replica (each: N trial moves; NPT
 * replicas add one ln V volume move per sweep). */
int lcmc_sweep(lcmc_ctx *ctx, int n_sweeps);
int lcmc_get_stats(lcmc_ctx *ctx, int replica, lcmc_stats *out);

/* tot_ene (MCnptColloid.c:1598-1622): fresh total energy of one replica,
 * pair terms in `precision`, sums in FP64.  Also resets the running energy. */
int lcmc_total_energy(lcmc_ctx *ctx, int replica, int precision, double *energy);

/* compute_liquid_crystal_order_parameters (MCnptColloid.c:2117-2218): Q tensor
 * (xx, xy, xz, yy, yz, zz), P2 = 1.5 lambda_max and director. */
int lcmc_order_parameter(lcmc_ctx *ctx, int replica, double Q[6], double *P2, double director[3]);

/* Per-particle outcome of the last sweep, indexed by particle id:
 * 0 rejected, 1 accepted, 2 colloid hard-core reject (for parity tests). */
int lcmc_last_outcomes(lcmc_ctx *ctx, int replica, unsigned char *out, int n);

/* Override the kernel choice (for tests): -1 auto, LCMC_PREC_FP64, LCMC_PREC_FP32. */
int lcmc_set_kernel(lcmc_ctx *ctx, int kernel);

/* Error flags are sticky: lcmc_sweep keeps returning the error of a set flag
 * until the caller clears them. */
int lcmc_clear_error_flags(lcmc_ctx *ctx);

/* FP64 energy check now (the reference's EnergyCheck, MCnptColloid.c:1343-1362,
 * which prints the running and the recomputed energy): recomputes every
 * replica's total energy in FP64, records drift = running - recomputed,
 * resets the running energy to the recomputed value and returns LCMC_EDRIFT
 * (setting LCMC_F_DRIFT) when |drift| exceeds the replica's tolerance (see
 * energy_check_tolerance).  lcmc_sweep runs the same check after every
 * energy_check_interval sweeps of a replica.  The chain is unchanged. */
int lcmc_energy_check(lcmc_ctx *ctx);

/* Per-particle record of the moves of each sweep (for tests that compare
 * kernels decision by decision): on = 1 starts recording, 0 stops and frees.
 * lcmc_get_move_records returns, by particle id, the energy change dE of the
 * last sweep's attempt (0 for a colloid hard-core reject) and the log of its
 * Metropolis draw ln u (accepted iff dE <= 0 or ln u <= -beta dE). */
int lcmc_record_moves(lcmc_ctx *ctx, int on);
int lcmc_get_move_records(lcmc_ctx *ctx, int replica, double *dE, double *log_u, int n);

/* ---- measurement (no counterpart in the reference, which only times with clock()) ---- */
/* The CUDA stream (cudaStream_t) of this context: every sweep starts and ends
 * on it (work enqueued on it after lcmc_sweep returns follows the sweep). */
int lcmc_get_stream(lcmc_ctx *ctx, void **stream);
/* Kernel launches in one sweep of this context (all replicas). */
int lcmc_kernels_per_sweep(lcmc_ctx *ctx);
/* Device time of the last sweep run by lcmc_sweep, part by part, from CUDA
 * event nodes inside the sweep graph: ms[0] rebin, ms[1] the colour-phase
 * kernels (all 8 phases), ms[2] the phases' statistics and the volume move,
 * ms[3] the sweep counter (and history). */
int lcmc_last_sweep_timing(lcmc_ctx *ctx, double ms[4]);

/* Gay-Berne pair term of n given configurations on the GPU, in the FP32
 * kernel's arithmetic (out32) and in the FP64 kernel's arithmetic (out64):
 * pij_GB (MCnptColloid.c:2618-2681) for separation d = r_j - r_i (3n values),
 * orientations ei, ej (3n each), with the cutoff and the constants of p.
 * Pairs beyond the cutoff give 0.  For tests and error statistics. */
int lcmc_pair_terms(const lcmc_params *p, int n, const double *d, const double *ei, const double *ej, double *out32,
                    double *out64);

/* ---- learned volume-move surrogate (no counterpart in the reference, which has
 *      no NPT move: system_pressure is parsed at MCnptColloid.c:3978 and unused) ----
 * An MLP n_in -> 128 -> 128 -> 1 (SiLU), BF16 weights and activations, FP32
 * accumulation; its matrix products run on the tensor cores (tcgen05). */
typedef struct lcmc_mlp lcmc_mlp;
int lcmc_mlp_create(int n_in, int hidden, int max_batch, uint64_t seed, lcmc_mlp **out);
int lcmc_mlp_destroy(lcmc_mlp *m);
/* Adam on mean squared error; x: n rows of n_in floats, t: n targets (host). */
int lcmc_mlp_train(lcmc_mlp *m, const float *x, const float *t, int n, int epochs, int batch, float lr, uint64_t seed,
                   float *final_loss);
int lcmc_mlp_predict(lcmc_mlp *m, const float *x, int n, float *y);
/* Gradient of the batch MSE w.r.t. all parameters without updating them, and
 * parameter get/set (layout: W1 [128 x k1] | b1 | W2 [128 x 128] | b2 | w3 | b3,
 * k1 = n_in rounded up to 128); for gradient checks. */
int lcmc_mlp_num_params(const lcmc_mlp *m);
int lcmc_mlp_gradients(lcmc_mlp *m, const float *x, const float *t, int n, float *grad, float *loss);
int lcmc_mlp_get_params(lcmc_mlp *m, float *params);
int lcmc_mlp_set_params(lcmc_mlp *m, const float *params);
/* C[M x N] = A[M x K] B[N x K]^T with A, B rounded to BF16, FP32 accumulate, on
 * the tensor cores (host arrays; K a multiple of 64).  For tests. */
int lcmc_gemm_bf16(const float *A, const float *B, float *C, int M, int N, int K);
/* Limit, in tries, of the tensor-core kernels' bounded mbarrier waits for
 * launches made from now on (0 restores the default, 2^24).  A wait that runs
 * out sets the kernel's error flag, waits (with the full bound) for the MMAs
 * it issued, frees its TMEM and returns; the call then reports LCMC_ETIMEOUT.
 * For tests of that path (a limit of 1 makes the first wait give up).  Sweep
 * graphs captured earlier keep the limit they were captured with.  No
 * counterpart in the reference. */
int lcmc_set_wait_limit(unsigned int tries);

/* Delayed-acceptance volume moves (Christen & Fox 2005) for the NPT replicas of
 * a context: stage 1 tests the surrogate's energy change
 *   dU~ = N s delta [g(phi(x), |delta|) + g(phi(y), |delta|)] / 2
 * (features phi: density, Q tensor and radial alignment on an 8^3 grid, 4097
 * inputs with |delta ln V|; g predicts the slope dU / (N delta)), which is odd
 * under x <-> y, and only moves that pass it get the exact FP64 recompute and
 * stage 2, exp(-beta (dU - dU~)).  s = target_scale converts the network
 * output to dU / (N delta).  m = NULL switches it off.  The network must stay
 * alive while set. */
int lcmc_set_surrogate(lcmc_ctx *ctx, lcmc_mlp *m, double target_scale);
/* Delayed-acceptance volume moves whose stage 1 tests the energy change
 * evaluated with FP32 pair terms (FP64 sums; the same in-cutoff pairs as the
 * FP64 recompute, each pair term a function of the two particles' FP64
 * coordinates, so the screen is odd under x <-> y), with the plain move's
 * random draw; stage 2 tests exp(-beta (dU - dU~)) with the exact FP64 dU.
 * |dU - dU~| is about 1e-3 kT, so the two stages decide as the plain move
 * does, but the FP64 recompute runs only for moves that pass stage 1.  NPT
 * replicas on the FP32 kernel only; on = 0 switches it off.  Setting it
 * clears the learned surrogate, and lcmc_set_surrogate clears it.  No
 * counterpart in the reference (it has no volume move). */
int lcmc_set_fp32_screen(lcmc_ctx *ctx, int on);
#define LCMC_FEATURES 4097
/* Record (features of x, exact dU / (N delta)) of every exactly evaluated
 * volume move (capacity samples; 0 stops and frees); fetch them (x: n x 4097). */
int lcmc_record_volume_samples(lcmc_ctx *ctx, int capacity);
int lcmc_get_volume_samples(lcmc_ctx *ctx, float *x, float *y, int max_n);
/* Per-sweep history (last `capacity` sweeps): rows of 9 doubles = sweep,
 * sums of ux ux, ux uy, ux uz, uy uy, uy uz, uz uz, energy, volume.
 * lcmc_get_history returns the number of rows written, in sweep order. */
int lcmc_record_history(lcmc_ctx *ctx, int capacity);
int lcmc_get_history(lcmc_ctx *ctx, int replica, double *rows, int max_rows);

/* Adaptive step (MCnptColloid.c:987-1031), for equilibration only (off by
 * default, off in parity and production runs): after every block of at least
 * 10,000 attempts (whole sweeps) a replica's max displacement shrinks by 5 %
 * below 30 % acceptance and grows by 5 % above 55 %, with the reference's
 * resets at 1e-4 and 1.5 min(sigma_ee, sigma_ss) (which also scale the
 * rotation), and never grows beyond its value at creation, which the
 * checkerboard's cell width was sized for.  Changes the trial moves, so a run
 * with it on is not a Markov chain with fixed moves: equilibrate with it, then
 * switch it off. */
int lcmc_set_adaptive_step(lcmc_ctx *ctx, int on);
/* Current max displacement and rotation of a replica. */
int lcmc_get_step(lcmc_ctx *ctx, int replica, double *max_displacement, double *max_rotation);
/* The parameters a replica was created with. */
int lcmc_get_params(lcmc_ctx *ctx, int replica, lcmc_params *out);
/* Position of a replica's counter-based random streams: sweep s of a replica
 * draws from counters (seed, particle, s); set it to resume a run. */
int lcmc_set_sweep_counter(lcmc_ctx *ctx, int replica, int64_t sweep);

/* Active-cell capacity the FP32 kernel takes for a system created with *p (no
 * counterpart in the reference, whose cells are unbounded host arrays): the
 * caller's cell_capacity when given; else, from the creation density, the
 * mean occupancy of a cell m plus four standard deviations of its count
 * (variance m for a gas, rho* <= 0.15, and 0.3 m for a dense liquid,
 * rho* >= 0.25) plus 4, and at least 56 for NPT.  A cell holding more (a
 * lattice start's fullest cells, a rare fluctuation) is attempted in FP64.
 * class_capacity: the kernel class used (48, 56 or 64).  Host only. */
int lcmc_cell_capacity(const lcmc_params *p, int *capacity, int *class_capacity);

/* Autotuner (no counterpart in the reference): times `sweeps` sweeps (after
 * one warm-up sweep) of every candidate configuration -- each FP32 phase-kernel
 * capacity class the capacity rule allows (the per-block tile of the active
 * cell: threads, cell capacity, staged candidates per warp, list capacity) and,
 * for NPT systems with >= 4 cells per axis, the per-cell or the per-particle
 * kernel for the volume move's exact energies -- and keeps the fastest.  The
 * state, statistics, sweep counters and last outcomes are restored after every
 * trial, so the chain continues as if autotune had not run.  With a
 * cache_path, a choice stored for the same device and workload signature is
 * applied without timing, and a new choice is appended to the file (one line:
 * signature, class, volume kernel, ms per sweep).  Call it with history and
 * volume-sample recording off (LCMC_EINVAL otherwise). */
typedef struct {
    int capacity;        /* active-cell capacity of the chosen phase-kernel class */
    int volume_by_cell;  /* 1: per-cell volume-energy kernel, 0: per-particle */
    double ms_per_sweep; /* measured time of the chosen configuration */
    int from_cache;      /* 1: taken from cache_path without timing */
    int trials;          /* configurations timed */
} lcmc_tuning;
int lcmc_autotune(lcmc_ctx *ctx, int sweeps, const char *cache_path, lcmc_tuning *out);

/* The reference's configuration files, byte for byte (host only, no device):
 * fortSphere.1 as esc_fort1 writes it (MCnptColloid.c:3193-3212) and as
 * read_initial_configuration reads it (2786-2831: the first n_max particles of
 * a file holding n_read >= n_max); Configuraciones.dat as print_Trayectoria
 * (3081-3107) and qmga_mcnvtGB.cnf as print_Qmga (3110-3158) write them,
 * append = the reference's option 1. */
int lcmc_write_fort1(const char *path, int n, const double *px, const double *py, const double *pz, const double *ox,
                     const double *oy, const double *oz, const double box[3], double colloid_radius);
int lcmc_read_fort1(const char *path, int n_max, double *px, double *py, double *pz, double *ox, double *oy,
                    double *oz, double box[3], double *colloid_radius, int *n_read);
int lcmc_write_trajectory(const char *path, int append, int n, const double *px, const double *py, const double *pz,
                          const double *ox, const double *oy, const double *oz, const double box[3]);
int lcmc_write_qmga(const char *path, int append, int n, const double *px, const double *py, const double *pz,
                    const double *ox, const double *oy, const double *oz, const double box[3]);
/* Restart of one replica: fortSphere.1 at `path` plus a binary sidecar
 * `path`.lcmc with the exact FP64 state, box, running energy and sweep
 * counter.  Loading uses the sidecar when present (the resumed run makes
 * exactly the decisions of the uninterrupted one; its seed must match) and
 * otherwise the text file, with an FP64 energy recompute, as the reference's
 * initial_configuration_type 1 restart does. */
int lcmc_save_restart(lcmc_ctx *ctx, int replica, const char *path);
int lcmc_load_restart(lcmc_ctx *ctx, int replica, const char *path);

/* ---- allocation-free total energy (no counterpart in the reference) ----
 * Some callers cannot let this library allocate device memory: a host program
 * that has already reserved the GPU's memory for its own pool, or a time-step
 * loop that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
 * imply.  For them this call computes the FP64 total energy (what tot_ene
 * computes) of a configuration the caller already holds in device memory, using
 * only a fixed scratch area compiled into liblcmc.so (1.7 MB on every GPU that
 * loads the library, held until the process exits).
 *   d_px..d_oz  device arrays of n doubles (positions in [0, L], orientations)
 *   box         host array, box edges; cells of width >= cutoff_radius
 *   d_energy    device pointer receiving the energy
 *   stream      cudaStream_t to enqueue on (NULL = legacy default stream)
 * Limits: n <= LCMC_NOALLOC_MAX_PARTICLES and (L/rc) cells per axis with at most
 * LCMC_NOALLOC_MAX_CELLS cells in total; larger inputs return LCMC_EINVAL with a
 * message (lcmc_last_error(NULL, ...)).  Asynchronous: synchronise the stream
 * before reading d_energy.  The first call on a device looks up the scratch
 * area's device address; make that first call before any stream capture.  All
 * calls share the one scratch area: calls that overlap on the GPU (other
 * streams, other host threads) race and give wrong results. */
#define LCMC_NOALLOC_MAX_PARTICLES 65536
#define LCMC_NOALLOC_MAX_CELLS 32768
int lcmc_total_energy_noalloc(const lcmc_params *p, int n, const double *d_px, const double *d_py, const double *d_pz,
                              const double *d_ox, const double *d_oy, const double *d_oz, const double box[3],
                              double *d_energy, void *stream);

const char *lcmc_strerror(int code);
/* Last error message of this context (or of the last failed create when ctx is NULL). */
int lcmc_last_error(const lcmc_ctx *ctx, char *buf, size_t len);
int lcmc_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
