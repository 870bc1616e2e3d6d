/*
 * ref_driver.c - drives the reference's OWN serial Monte Carlo functions.
 *
 * Test infrastructure only.  oracle/build_ref.sh compiles the reference file
 * MCnptColloid.c (from where it lies, with six one-line compile fixes applied
 * on the fly) together with this driver and a no-op MPI stub into
 * oracle/_ref/libmcref*.so.  Tests and the CPU baseline call the reference's
 * functions (pij_GB, GBCollRod, tot_ene, attempt_monte_carlo_move, ...) through
 * ctypes; this file only adds set-up helpers and a timing loop that mirrors the
 * reference's serial cycle loop (MCnptColloid.c:887-927).
 *
 * Nothing in the product links against this file.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define REF_POINTS_ON_SPHERE 1000000

/* ---- the reference's globals (MCnptColloid.c:96-145) ---- */
extern int num_particles;
extern int colloid_wall_option;
extern int mc_ensemble_type;
extern float max_displacement;
extern float max_rotation;
extern float rot_vec_x[], rot_vec_y[], rot_vec_z[];
extern double box_volume, system_density, system_temperature, system_pressure;
extern double gb_epsilon0, gb_kappa, gb_kappa_prime, gb_mu_exponent, gb_nu_exponent;
extern double gb_sigma_endtoend, gb_sigma_sidetoside, cutoff_radius, verlet_radius;
extern double gb_beta, gb_4eps0, cutoff_radius_sq, r_verlet_sq, gb_kappa_sq, gb_chi_sq;
extern double gb_chi, gb_chi_prime, gb_k_imu, colloid_radius, colloid_radius_sq, colloid_volume;
extern double box_size[3], colloid_coords[3], colloid_rod_cutoff;

/* ---- the reference's functions ---- */
void load_initial_conditions(const char *filename);
void get_system_const(void);
void Marsaglia4MC(float *arr_x, float *arr_y, float *arr_z, float radio);
void build_neighbor_lists(int nvest, double *px, double *py, double *pz, double *rxo, double *ryo, double *rzo,
                          int *count, int *list);
void attempt_monte_carlo_move(double *px, double *py, double *pz, double *ox, double *oy, double *oz,
                              float max_disp, double *energy, int *count, int *list, long *accepted,
                              double *desp_max, size_t *histogram);
double tot_ene(double *px, double *py, double *pz, double *ox, double *oy, double *oz);
double tot_ene_lstnb(double *px, double *py, double *pz, double *ox, double *oy, double *oz, int *count, int *list);

/* Index expression of the reference's table look-ups (MCnptColloid.c:2486-2487). */
int refdrv_table_index(int r)
{
    return (int)(r * (1.0f / RAND_MAX) * REF_POINTS_ON_SPHERE);
}

/* Particle-selection expression of MCnptColloid.c:2475. */
int refdrv_particle_index(int r)
{
    return (int)(r * (1.0f / RAND_MAX) * num_particles);
}

/*
 * Put a configuration into the reference's globals: box, colloid centre at the
 * box centre (MCnptColloid.c:2847-2849), and the derived constants.
 * get_system_const() is called twice because its first call computes gb_chi
 * from gb_kappa_sq before gb_kappa_sq is assigned (MCnptColloid.c:2772-2773).
 */
void refdrv_set_box(int n, const double box[3])
{
    num_particles = n;
    for (int k = 0; k < 3; k++) {
        box_size[k] = box[k];
        colloid_coords[k] = 0.5 * box[k];
    }
    box_volume = box[0] * box[1] * box[2];
    get_system_const();
    get_system_const();
}

/* Fill the reference's 10^6-entry rotation table from libc rand() (seeded by the caller). */
void refdrv_fill_rotation_table(void)
{
    Marsaglia4MC(rot_vec_x, rot_vec_y, rot_vec_z, 1.0f);
}

/*
 * Build the reference's CSR Verlet list (count[i] = cumulative end offset,
 * list = neighbour ids in ascending j) with a cell grid instead of the
 * reference's O(N^2) double loop (MCnptColloid.c:1395-1468).  The content and
 * order are the same as build_neighbor_lists produces; this only makes large N
 * set-up feasible for timing.  Returns the number of list entries, or -1 if
 * `cap` is too small.
 */
long refdrv_build_verlet_cells(const double *px, const double *py, const double *pz, int *count, int *list, long cap)
{
    int n = num_particles;
    double rv = verlet_radius, rv2 = rv * rv;
    int nc[3];
    for (int k = 0; k < 3; k++) {
        nc[k] = (int)floor(box_size[k] / rv);
        if (nc[k] < 3) nc[k] = 1;
    }
    long ncell = (long)nc[0] * nc[1] * nc[2];
    int *head = malloc(sizeof(int) * (size_t)ncell);
    int *next = malloc(sizeof(int) * (size_t)n);
    int *cid = malloc(sizeof(int) * (size_t)n);
    int *tmp = malloc(sizeof(int) * 4096);
    for (long c = 0; c < ncell; c++) head[c] = -1;
    for (int i = n - 1; i >= 0; i--) {
        int c3[3];
        double p[3] = {px[i], py[i], pz[i]};
        for (int k = 0; k < 3; k++) {
            int c = (int)floor(p[k] / box_size[k] * nc[k]);
            c = ((c % nc[k]) + nc[k]) % nc[k];
            c3[k] = c;
        }
        int c = (c3[2] * nc[1] + c3[1]) * nc[0] + c3[0];
        cid[i] = c;
        next[i] = head[c];
        head[c] = i;
    }
    long pos = 0;
    for (int i = 0; i < n; i++) {
        int c = cid[i];
        int cx = c % nc[0], cy = (c / nc[0]) % nc[1], cz = c / (nc[0] * nc[1]);
        int m = 0;
        int seen[27];
        int nseen = 0;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    int x = ((cx + dx) % nc[0] + nc[0]) % nc[0];
                    int y = ((cy + dy) % nc[1] + nc[1]) % nc[1];
                    int z = ((cz + dz) % nc[2] + nc[2]) % nc[2];
                    int cc = (z * nc[1] + y) * nc[0] + x;
                    int dup = 0;
                    for (int s = 0; s < nseen; s++) dup |= (seen[s] == cc);
                    if (dup) continue;
                    seen[nseen++] = cc;
                    for (int j = head[cc]; j >= 0; j = next[j]) {
                        if (j == i) continue;
                        double d[3] = {px[j] - px[i], py[j] - py[i], pz[j] - pz[i]};
                        for (int k = 0; k < 3; k++) {
                            if (d[k] > 0.5 * box_size[k]) d[k] -= box_size[k];
                            else if (d[k] < -0.5 * box_size[k]) d[k] += box_size[k];
                        }
                        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                        if (r2 < rv2 && m < 4096) tmp[m++] = j;
                    }
                }
        /* ascending j, as the reference's j = 0..N-1 loop produces */
        for (int a = 1; a < m; a++) {
            int v = tmp[a], b = a - 1;
            while (b >= 0 && tmp[b] > v) { tmp[b + 1] = tmp[b]; b--; }
            tmp[b + 1] = v;
        }
        if (pos + m > cap) { pos = -1; break; }
        memcpy(list + pos, tmp, sizeof(int) * (size_t)m);
        pos += m;
        count[i] = (int)pos;
    }
    free(head); free(next); free(cid); free(tmp);
    return pos;
}

/*
 * Timed loop over the reference's attempt_monte_carlo_move, following its
 * serial cycle loop (MCnptColloid.c:887-927): one attempt per cycle and a
 * Verlet rebuild plus tot_ene_lstnb when the displacement tracker passes
 * factor*(r_v - r_c)^2 (estima_vecinos, MCnptColloid.c:2725-2749).
 * rebuild = 0: the tracker is ignored and only the move is timed;
 * rebuild = 1: the reference's own O(N^2) build_neighbor_lists, as coded;
 * rebuild = 2: the same list built through refdrv_build_verlet_cells.
 * Returns wall seconds (CLOCK_MONOTONIC).
 */
double refdrv_run_attempts(long n_attempts, int rebuild, double *px, double *py, double *pz, double *ox, double *oy,
                           double *oz, int *count, int *list, long list_cap, double *energy, long *accepted,
                           long *rebuilds)
{
    size_t *hist = calloc((size_t)num_particles, sizeof(size_t));
    double *rxi = malloc(sizeof(double) * (size_t)num_particles);
    double *ryi = malloc(sizeof(double) * (size_t)num_particles);
    double *rzi = malloc(sizeof(double) * (size_t)num_particles);
    double tracker = 0.0;
    double skin2 = (verlet_radius - cutoff_radius) * (verlet_radius - cutoff_radius);
    float factor = 1.0f;
    if (num_particles > 100) factor = num_particles * 0.01;
    long acc = 0, nreb = 0;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (long c = 0; c < n_attempts; c++) {
        attempt_monte_carlo_move(px, py, pz, ox, oy, oz, max_displacement, energy, count, list, &acc, &tracker, hist);
        if (rebuild && tracker > factor * skin2) {
            tracker = 0.0;
            if (rebuild == 1)
                build_neighbor_lists((int)list_cap, px, py, pz, rxi, ryi, rzi, count, list);
            else if (refdrv_build_verlet_cells(px, py, pz, count, list, list_cap) < 0)
                break;
            *energy = tot_ene_lstnb(px, py, pz, ox, oy, oz, count, list);
            nreb++;
        }
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    free(hist); free(rxi); free(ryi); free(rzi);
    *accepted = acc;
    *rebuilds = nreb;
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/*
 * As refdrv_run_attempts, for ensemble averages: the Verlet list (cell-built,
 * same content as build_neighbor_lists) is rebuilt every `period` attempts
 * instead of by the reference's tracker (which sums the rotation-table
 * magnitude, not the real displacement, MCnptColloid.c:2584-2595), so the
 * old energies of GBij_lstnb stay exact when period * max_displacement is
 * small against the skin verlet_radius - cutoff_radius.  The energy is
 * recomputed (tot_ene_lstnb) after every rebuild.
 */
double refdrv_run_attempts_periodic(long n_attempts, long period, double *px, double *py, double *pz, double *ox,
                                    double *oy, double *oz, int *count, int *list, long list_cap, double *energy,
                                    long *accepted)
{
    size_t *hist = calloc((size_t)num_particles, sizeof(size_t));
    double tracker = 0.0;
    long acc = 0;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (long c = 0; c < n_attempts; c++) {
        if (c % period == 0) {
            if (refdrv_build_verlet_cells(px, py, pz, count, list, list_cap) < 0) break;
            *energy = tot_ene_lstnb(px, py, pz, ox, oy, oz, count, list);
        }
        attempt_monte_carlo_move(px, py, pz, ox, oy, oz, max_displacement, energy, count, list, &acc, &tracker, hist);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    free(hist);
    *accepted += acc;
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}
