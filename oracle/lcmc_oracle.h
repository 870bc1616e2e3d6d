/*
 * lcmc_oracle.h - CPU oracle for the Gay-Berne Monte Carlo sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, FP64 restatement of the
 * reference's Monte Carlo path (MCnptColloid.c) used by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker.
 * The product (the CUDA library under parellel_mc_mpi_for_liquidcrystalsystems_b200/)
 * never includes, links or calls it.
 *
 * Two arithmetic modes for the pair and colloid terms:
 *   LCO_ARITH_REFERENCE  libm pow() for the mu/nu exponents and libm log() in
 *                        Metropolis, exactly as the reference; pinned bit-exact
 *                        against the reference's own functions built into
 *                        oracle/_ref/ (tests/golden/).
 *   LCO_ARITH_CANONICAL  integer exponents specialised to products (mu = 2 ->
 *                        x*x, nu = 1 -> x) and a project-written log, so that
 *                        the GPU FP64 kernel can reproduce every bit.  Differs
 *                        from the reference by at most one ulp per pair term
 *                        (glibc pow(x, 2.0) != x*x in ~0.1% of arguments).
 */
#ifndef LCMC_ORACLE_H
#define LCMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LCO_ARITH_REFERENCE = 0, LCO_ARITH_CANONICAL = 1 };

/* The 23 keys of the reference's parameter file (MCnptColloid.c:3954-4091)
 * plus the keys this project adds (unknown keys only warn in the reference,
 * MCnptColloid.c:4093, so the added keys stay compatible with it). */
typedef struct {
    int mc_ensemble_type;
    int num_particles;
    double system_density;
    double system_temperature;
    double system_pressure;
    double gb_sigma_sidetoside;
    double gb_epsilon0;
    double gb_kappa;
    double gb_kappa_prime;
    double gb_mu_exponent;
    double gb_nu_exponent;
    float max_displacement; /* parsed with %f as in the reference */
    float max_rotation;     /* parsed with %f as in the reference */
    int initial_configuration_type;
    double cutoff_radius;
    double verlet_radius;
    int total_mc_cycles;
    int configuration_save_interval;
    int statistics_print_interval;
    int colloid_wall_option;
    double colloid_interaction_epsilon;
    double colloid_interaction_amplitude;
    double colloid_radius;
    /* added keys */
    uint64_t rng_seed;
    int total_mc_sweeps;
    int cell_capacity;
    double npt_max_dlnV;
    int volume_moves_per_sweep;
    int precision_mode; /* 0 = fp64, 1 = fp32 */
    double init_orientation_cone_deg;
    int n_read;         /* how many of the 23 reference keys were found */
    int missing_mask;   /* bit i set = reference key i missing */
} lco_params;

/* Derived constants (get_system_const, MCnptColloid.c:2752-2783), with chi
 * computed after kappa^2 (the reference computes it before, 2772-2773). */
typedef struct {
    double beta, four_eps0, rc, rc2, sigma0, sigma_ee, kappa_sq;
    double chi, chi_sq, chi_prime, k_imu, mu, nu, kappa_prime;
    double coll_R, coll_cutoff;
    int coll_on;       /* colloid_wall_option == 1 */
    double max_disp, max_rot;
    double wmin;       /* minimum checkerboard cell width: (rc + max_disp), times
                          (1 + npt_max_dlnV) for NPT so scaled boxes keep rc */
    int arith;         /* LCO_ARITH_* */
} lco_consts;

int lco_params_defaults(lco_params *p);
int lco_params_load(const char *path, lco_params *p);
void lco_consts_from_params(const lco_params *p, int arith, lco_consts *c);

/* ---- geometry (MCnptColloid.c:2420-2430, 2690-2721) ---- */
double lco_distance_sq(double x1, double y1, double z1, double x2, double y2, double z2, const double box[3],
                       double *dx, double *dy, double *dz);
void lco_apply_pbc(double *x, double *y, double *z, const double box[3]);

/* ---- energies ---- */
double lco_pij_gb(const lco_consts *c, const double ei[3], const double ej[3], double rij, double irij, double iei,
                  double iej, double eiej, const double dr[3]);
/* pair term as GBij_PosMod builds it from coordinates (MCnptColloid.c:1573-1591);
 * *in_cut = 1 when r^2 < rc^2 (otherwise the return is 0). */
double lco_pair(const lco_consts *c, const double ri[3], const double ei[3], const double rj[3], const double ej[3],
                const double box[3], int *in_cut);
double lco_colloid_rod(const lco_consts *c, const double ri[3], const double ei[3], const double box[3]);
double lco_tot_ene(const lco_consts *c, int n, const double *px, const double *py, const double *pz,
                   const double *ox, const double *oy, const double *oz, const double box[3]);

/* ---- reference-semantics single move with injected libc rand() values ---- */
int lco_move_refsem(const lco_consts *c, int n, double *px, double *py, double *pz, double *ox, double *oy,
                    double *oz, const double box[3], const int *nb_count, const int *nb_list, const float *rvx,
                    const float *rvy, const float *rvz, const int *rands, int n_rands, int *rand_pos,
                    double *energy, long *accepted, double *tracker, int gate_colloid);
int lco_ref_particle_index(int r, int n);
int lco_ref_table_index(int r);

/* ---- Philox4x32-10 (Salmon et al., SC'11) and the draws built on it ---- */
void lco_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double lco_u01(uint32_t x);
double lco_log(double u);     /* project-written log for u in (0, 1) */
double lco_expm1(double x);   /* project-written e^x - 1 for |x| <= 1.5 */
void lco_key(uint64_t seed, int replica, uint32_t key[2]);
void lco_sphere_point(const uint32_t key[2], uint32_t id, uint64_t sweep, double v[3]);

/* ---- initial configurations (MCnptColloid.c:2920-3033, seeded) ---- */
int lco_init_lattice(const lco_params *p, int replica, double *px, double *py, double *pz, double *ox, double *oy,
                     double *oz, double box[3]);

/* ---- checkerboard cell grid and sweep ---- */
typedef struct {
    int nc[3];
    double w[3];
    double shift[3];
    int ncell;
    int *cell_start; /* ncell + 1 */
    int *order;      /* particle ids, cell-major, ascending id inside a cell */
} lco_grid;

int lco_grid_dims(double L, double wmin, int *nc);
void lco_sweep_shift(const uint32_t key[2], uint64_t sweep, const int nc[3], const double box[3], double shift[3]);
void lco_colour_order(const uint32_t key[2], uint64_t sweep, int perm[8]);
int lco_cell_of(double x, double shift, double w, int nc, double L);
int lco_grid_build(lco_grid *g, int n, const double *px, const double *py, const double *pz, const double box[3],
                   double wmin, const double shift[3]);
void lco_grid_free(lco_grid *g);

typedef struct {
    long attempted, accepted, hardcore_rejected;
    double dE_sum;
} lco_sweep_stats;

/* One checkerboard sweep in the canonical FP64 order that the GPU FP64 kernel
 * reproduces bit for bit.  accept_bits (may be NULL) receives one byte per
 * attempt in processing order: 0 reject, 1 accept, 2 hard-core reject. */
int lco_sweep(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int n, double *px, double *py, double *pz,
              double *ox, double *oy, double *oz, const double box[3], lco_sweep_stats *st, unsigned char *accept_bits,
              int *order_out);
/* The same sweep on the even grid (fine = 0, what lco_sweep runs) or on the
 * fine grid (fine = 1, cell_grid 1: odd cell counts take 3 colours on their
 * axis, up to 27 colours, drawn and ordered as the GPU's k_sweep_setup does). */
int lco_sweep_grid(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int fine, int n, double *px,
                   double *py, double *pz, double *ox, double *oy, double *oz, const double box[3], lco_sweep_stats *st,
                   unsigned char *accept_bits, int *order_out);
int lco_grid_dims_fine(double L, double wmin, int fine, int *nc);

/* lco_sweep with each colour's active cells shared among OpenMP threads (in
 * the -fopenmp build, oracle/_build/liblcmc_oracle_omp.so): the same final
 * state; the checkerboard port timed as a CPU baseline. */
int lco_sweep_parallel(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int n, double *px, double *py,
                       double *pz, double *ox, double *oy, double *oz, const double box[3], lco_sweep_stats *st);

/* Total energy over the cell stencil (cutoff rc, minimum image), FP64. */
double lco_total_energy_cells(const lco_consts *c, int n, const double *px, const double *py, const double *pz,
                              const double *ox, const double *oy, const double *oz, const double box[3]);

/* NPT ln V move: returns 1 accepted, 0 rejected, 2 hard-core reject. */
typedef struct {
    double delta, lambda, U_old, U_new, dV, lnA;
    int accepted;
} lco_volume_info;
int lco_volume_move(const lco_consts *c, const uint32_t key[2], uint64_t sweep, double pressure, double dlnV_max,
                    int n, double *px, double *py, double *pz, const double *ox, const double *oy, const double *oz,
                    double box[3], lco_volume_info *info);

/* Q tensor, P2 and director with a cyclic Jacobi eigen-solver (double). */
void lco_order_parameter(int n, const double *ox, const double *oy, const double *oz, double Q[6], double *P2,
                         double director[3]);

#ifdef __cplusplus
}
#endif
#endif
