/*
 * lcmc_oracle.c - CPU oracle (FP64 restatement) of the reference's Gay-Berne
 * Monte Carlo path.  TEST INFRASTRUCTURE ONLY: used by tests/, smoke() and the
 * CPU-baseline leg of bench.py as the checker; the product never links it.
 *
 * Every function cites the lines of MCnptColloid.c it restates.  Compiled with
 * -ffp-contract=off so that no multiply-add is fused (the reference's plain
 * build on x86-64 has no FMA either).
 */
#include "lcmc_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* parameter file (load_initial_conditions / read_next_parameter,            */
/* MCnptColloid.c:3894-4133)                                                 */
/* ------------------------------------------------------------------------ */

static const char *k_ref_keys[23] = {
    "mc_ensemble_type", "num_particles", "system_density", "system_temperature", "system_pressure",
    "gb_sigma_sidetoside", "gb_epsilon0", "gb_kappa", "gb_kappa_prime", "gb_mu_exponent", "gb_nu_exponent",
    "max_displacement", "max_rotation", "initial_configuration_type", "cutoff_radius", "verlet_radius",
    "total_mc_cycles", "configuration_save_interval", "statistics_print_interval", "colloid_wall_option",
    "colloid_interaction_epsilon", "colloid_interaction_amplitude", "colloid_radius"};

int lco_params_defaults(lco_params *p)
{
    memset(p, 0, sizeof(*p));
    p->rng_seed = 12345u;
    p->total_mc_sweeps = 0;
    p->cell_capacity = 0;
    p->npt_max_dlnV = 0.01;
    p->volume_moves_per_sweep = 1;
    p->precision_mode = 0;
    p->init_orientation_cone_deg = 180.0;
    return 0;
}

/* Same line grammar as read_next_parameter (MCnptColloid.c:3894-3910): lines
 * starting with '\n', '#' or NUL are skipped; "<name> <rest of line>". */
static int next_param(FILE *f, char *name, char *value)
{
    char line[256];
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '\n' || line[0] == '#' || line[0] == '\0') continue;
        value[0] = '\0';
        if (sscanf(line, "%255s %255[^\n]", name, value) >= 1) return 1;
    }
    return 0;
}

int lco_params_load(const char *path, lco_params *p)
{
    char name[256], value[256];
    int seen[23] = {0};
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    while (next_param(f, name, value)) {
        int k = -1;
        for (int i = 0; i < 23; i++)
            if (strcmp(name, k_ref_keys[i]) == 0) k = i;
        int ok = 1;
        switch (k) {
        case 0: ok = sscanf(value, "%d", &p->mc_ensemble_type); break;
        case 1: ok = sscanf(value, "%d", &p->num_particles); break;
        case 2: ok = sscanf(value, "%lf", &p->system_density); break;
        case 3: ok = sscanf(value, "%lf", &p->system_temperature); break;
        case 4: ok = sscanf(value, "%lf", &p->system_pressure); break;
        case 5: ok = sscanf(value, "%lf", &p->gb_sigma_sidetoside); break;
        case 6: ok = sscanf(value, "%lf", &p->gb_epsilon0); break;
        case 7: ok = sscanf(value, "%lf", &p->gb_kappa); break;
        case 8: ok = sscanf(value, "%lf", &p->gb_kappa_prime); break;
        case 9: ok = sscanf(value, "%lf", &p->gb_mu_exponent); break;
        case 10: ok = sscanf(value, "%lf", &p->gb_nu_exponent); break;
        case 11: ok = sscanf(value, "%f", &p->max_displacement); break;
        case 12: ok = sscanf(value, "%f", &p->max_rotation); break;
        case 13: ok = sscanf(value, "%d", &p->initial_configuration_type); break;
        case 14: ok = sscanf(value, "%lf", &p->cutoff_radius); break;
        case 15: ok = sscanf(value, "%lf", &p->verlet_radius); break;
        case 16: ok = sscanf(value, "%d", &p->total_mc_cycles); break;
        case 17: ok = sscanf(value, "%d", &p->configuration_save_interval); break;
        case 18: ok = sscanf(value, "%d", &p->statistics_print_interval); break;
        case 19: ok = sscanf(value, "%d", &p->colloid_wall_option); break;
        case 20: ok = sscanf(value, "%lf", &p->colloid_interaction_epsilon); break;
        case 21: ok = sscanf(value, "%lf", &p->colloid_interaction_amplitude); break;
        case 22: ok = sscanf(value, "%lf", &p->colloid_radius); break;
        default:
            if (strcmp(name, "rng_seed") == 0) {
                unsigned long long s;
                ok = sscanf(value, "%llu", &s);
                p->rng_seed = s;
            } else if (strcmp(name, "total_mc_sweeps") == 0) ok = sscanf(value, "%d", &p->total_mc_sweeps);
            else if (strcmp(name, "cell_capacity") == 0) ok = sscanf(value, "%d", &p->cell_capacity);
            else if (strcmp(name, "npt_max_dlnV") == 0) ok = sscanf(value, "%lf", &p->npt_max_dlnV);
            else if (strcmp(name, "volume_moves_per_sweep") == 0) ok = sscanf(value, "%d", &p->volume_moves_per_sweep);
            else if (strcmp(name, "precision_mode") == 0) {
                ok = 1;
                if (strncmp(value, "fp32", 4) == 0) p->precision_mode = 1;
                else if (strncmp(value, "fp64", 4) == 0) p->precision_mode = 0;
                else ok = sscanf(value, "%d", &p->precision_mode);
            } else if (strcmp(name, "init_orientation_cone_deg") == 0)
                ok = sscanf(value, "%lf", &p->init_orientation_cone_deg);
            /* other unknown keys only warn in the reference (MCnptColloid.c:4093) */
            break;
        }
        if (ok != 1) {
            fclose(f);
            return -3; /* error_checker exits here (MCnptColloid.c:3862-3868) */
        }
        if (k >= 0) seen[k] = 1;
    }
    fclose(f);
    p->n_read = 0;
    p->missing_mask = 0;
    for (int i = 0; i < 23; i++) {
        if (seen[i]) p->n_read++;
        else p->missing_mask |= 1 << i;
    }
    return p->n_read == 23 ? 0 : -2; /* MCnptColloid.c:4100-4127 */
}

/* get_system_const (MCnptColloid.c:2752-2783) with chi computed after kappa^2. */
void lco_consts_from_params(const lco_params *p, int arith, lco_consts *c)
{
    memset(c, 0, sizeof(*c));
    c->beta = 1.0 / p->system_temperature;
    c->four_eps0 = 4.0 * p->gb_epsilon0;
    c->rc = p->cutoff_radius;
    c->rc2 = p->cutoff_radius * p->cutoff_radius;
    c->sigma0 = p->gb_sigma_sidetoside;
    c->sigma_ee = p->gb_sigma_sidetoside * p->gb_kappa; /* MCnptColloid.c:4130 */
    c->k_imu = pow(p->gb_kappa_prime, 1.0 / p->gb_mu_exponent);
    c->kappa_sq = p->gb_kappa * p->gb_kappa;
    c->chi = (c->kappa_sq - 1.0) / (c->kappa_sq + 1.0);
    c->chi_sq = c->chi * c->chi;
    c->chi_prime = (c->k_imu - 1.0) / (c->k_imu + 1.0);
    c->mu = p->gb_mu_exponent;
    c->nu = p->gb_nu_exponent;
    c->kappa_prime = p->gb_kappa_prime;
    c->coll_cutoff = 4.0 * c->sigma_ee;
    c->coll_R = p->colloid_radius;
    c->coll_on = p->colloid_wall_option == 1;
    c->max_disp = (double)p->max_displacement;
    c->max_rot = (double)p->max_rotation;
    c->wmin = p->cutoff_radius + (double)p->max_displacement;
    if (p->mc_ensemble_type == 2) c->wmin *= 1.0 + p->npt_max_dlnV;
    c->arith = arith;
}

/* ------------------------------------------------------------------------ */
/* geometry                                                                  */
/* ------------------------------------------------------------------------ */

/* compute_distance_sq (MCnptColloid.c:2690-2721): d = r2 - r1, one fold per axis. */
double lco_distance_sq(double x1, double y1, double z1, double x2, double y2, double z2, const double box[3],
                       double *dx, double *dy, double *dz)
{
    *dx = x2 - x1;
    *dy = y2 - y1;
    *dz = z2 - z1;
    if (box[0] > 0.0) {
        if (*dx > 0.5 * box[0]) *dx -= box[0];
        else if (*dx < -0.5 * box[0]) *dx += box[0];
    }
    if (box[1] > 0.0) {
        if (*dy > 0.5 * box[1]) *dy -= box[1];
        else if (*dy < -0.5 * box[1]) *dy += box[1];
    }
    if (box[2] > 0.0) {
        if (*dz > 0.5 * box[2]) *dz -= box[2];
        else if (*dz < -0.5 * box[2]) *dz += box[2];
    }
    double x_sq = (*dx) * (*dx), y_sq = (*dy) * (*dy), z_sq = (*dz) * (*dz);
    return x_sq + y_sq + z_sq;
}

/* apply_pbc (MCnptColloid.c:2420-2430): a single +-L fold per axis. */
void lco_apply_pbc(double *x, double *y, double *z, const double box[3])
{
    if (*x > box[0]) *x -= box[0];
    else if (*x < 0.0) *x += box[0];
    if (*y > box[1]) *y -= box[1];
    else if (*y < 0.0) *y += box[1];
    if (*z > box[2]) *z -= box[2];
    else if (*z < 0.0) *z += box[2];
}

static inline double dot3(double x1, double y1, double z1, double x2, double y2, double z2)
{
    return x1 * x2 + y1 * y2 + z1 * z2; /* compute_dot_product, MCnptColloid.c:2685-2687 */
}

/* ------------------------------------------------------------------------ */
/* Gay-Berne pair term (g_omega + pij_GB, MCnptColloid.c:2607-2681)          */
/* ------------------------------------------------------------------------ */

static inline double g_omega(double eiej, double amasb2, double amenb2, double omega)
{
    double ome = omega * eiej;
    double gmas = amasb2 / (1.0 + ome);
    double gmen = amenb2 / (1.0 - ome);
    return 1.0 - 0.50 * omega * (gmas + gmen);
}

/* x^e: libm pow in reference arithmetic; exact products for e in {1, 2} in
 * canonical arithmetic. */
static inline double powe(const lco_consts *c, double x, double e)
{
    if (c->arith == LCO_ARITH_CANONICAL) {
        if (e == 1.0) return x;
        if (e == 2.0) return x * x;
    }
    return pow(x, e);
}

double lco_pij_gb(const lco_consts *c, const double ei[3], const double ej[3], double rij, double irij, double iei,
                  double iej, double eiej, const double dr[3])
{
    double eirij = irij * iei * dot3(dr[0], dr[1], dr[2], ei[0], ei[1], ei[2]);
    double ejrij = irij * iej * dot3(dr[0], dr[1], dr[2], ej[0], ej[1], ej[2]);
    double amasb = eirij + ejrij;
    double amenb = eirij - ejrij;
    double amab2 = amasb * amasb;
    double ameb2 = amenb * amenb;
    double eps1 = 1.0 / sqrt(1.0 - c->chi_sq * eiej * eiej);
    double ctep1 = powe(c, eps1, c->nu);
    double eps2 = g_omega(eiej, amab2, ameb2, c->chi_prime);
    double ctep2 = powe(c, eps2, c->mu);
    double s_chi = g_omega(eiej, amab2, ameb2, c->chi);
    double sigma = c->sigma0 / sqrt(s_chi);
    double distreal = (rij - sigma + c->sigma0);
    if (distreal < 0.001) return 1000000000; /* MCnptColloid.c:2670 */
    double erre = c->sigma0 / distreal;
    double erre2 = erre * erre;
    double erre6 = erre2 * erre2 * erre2;
    double epsil = ctep1 * ctep2;
    return c->four_eps0 * epsil * erre6 * (erre6 - 1.0);
}

/* Per-pair preamble of GBij_PosMod (MCnptColloid.c:1573-1591): j relative to i,
 * cutoff r^2 < rc^2, orientation norms recomputed for every pair. */
double lco_pair(const lco_consts *c, const double ri[3], const double ei[3], const double rj[3], const double ej[3],
                const double box[3], int *in_cut)
{
    double dr[3];
    double r2 = lco_distance_sq(ri[0], ri[1], ri[2], rj[0], rj[1], rj[2], box, &dr[0], &dr[1], &dr[2]);
    if (!(r2 < c->rc2)) {
        *in_cut = 0;
        return 0.0;
    }
    *in_cut = 1;
    double rij = sqrt(r2);
    double irij = 1.0 / rij;
    double ei2 = dot3(ei[0], ei[1], ei[2], ei[0], ei[1], ei[2]);
    double ej2 = dot3(ej[0], ej[1], ej[2], ej[0], ej[1], ej[2]);
    double nei = sqrt(ei2), nej = sqrt(ej2);
    double iei = 1.0 / nei, iej = 1.0 / nej;
    double eiej = iei * iej * dot3(ei[0], ei[1], ei[2], ej[0], ej[1], ej[2]);
    return lco_pij_gb(c, ei, ej, rij, irij, iei, iej, eiej, dr);
}

/* GBCollRod (MCnptColloid.c:1758-1854): colloid of radius R at the box centre. */
double lco_colloid_rod(const lco_consts *c, const double ri[3], const double ei[3], const double box[3])
{
    double C[3] = {0.5 * box[0], 0.5 * box[1], 0.5 * box[2]};
    double px, py, pz;
    double d_nc = sqrt(lco_distance_sq(ri[0], ri[1], ri[2], C[0], C[1], C[2], box, &px, &py, &pz));
    double dij = d_nc - c->coll_R;
    if (d_nc <= 1e-12) return 1.0e8;
    if (dij > c->coll_cutoff) return 0.0;
    px = ri[0] - C[0];
    py = ri[1] - C[1];
    pz = ri[2] - C[2];
    double rhx = px / d_nc, rhy = py / d_nc, rhz = pz / d_nc;
    double ct = rhx * ei[0] + rhy * ei[1] + rhz * ei[2];
    if (ct > 1.0) ct = 1.0;
    if (ct < -1.0) ct = -1.0;
    double sin2 = 1.0 - ct * ct;
    double sigma0 = c->sigma0;
    double sigma_CR, eps_CR;
    {
        double denom = 1.0 - c->chi;
        double numer = 1.0 - c->chi * sin2;
        if (denom <= 0.0) denom = 1e-12;
        if (numer <= 1e-12) numer = 1e-12;
        sigma_CR = sigma0 * sqrt(numer / denom);
    }
    {
        double denom_eps = 1.0 - c->chi_prime * sin2;
        double numer_eps = 1.0 - c->chi_prime;
        if (denom_eps <= 1e-12) denom_eps = 1e-12;
        eps_CR = c->kappa_prime * powe(c, numer_eps / denom_eps, c->mu); /* eps_CR0 = kappa' (MCnptColloid.c:1821) */
    }
    double x = dij - sigma_CR + sigma0;
    if (x <= 1e-10) return 1.0e8;
    double s3 = sigma0 * sigma0 * sigma0;
    double s9 = s3 * s3 * s3;
    double x2 = x * x, x3 = x2 * x, x8 = x3 * x3 * x2, x9 = x8 * x;
    double term1 = s9 / (45.0 * x9);
    double term2 = s3 / (6.0 * x3);
    double term3 = s9 / (40.0 * d_nc * x8);
    double term4 = s3 / (4.0 * d_nc * x2);
    return eps_CR * (term1 - term2 - term3 + term4);
}

/* tot_ene (MCnptColloid.c:1598-1622) with GBij's sequential j loop (1501-1559). */
double lco_tot_ene(const lco_consts *c, int n, const double *px, const double *py, const double *pz,
                   const double *ox, const double *oy, const double *oz, const double box[3])
{
    double dumv = 0.0, wall = 0.0;
    for (int i = 0; i < n; i++) {
        double ri[3] = {px[i], py[i], pz[i]}, ei[3] = {ox[i], oy[i], oz[i]};
        double e = 0.0;
        for (int j = 0; j < n; j++) {
            if (i == j) continue;
            double rj[3] = {px[j], py[j], pz[j]}, ej[3] = {ox[j], oy[j], oz[j]};
            int in;
            double v = lco_pair(c, ri, ei, rj, ej, box, &in);
            if (in) e += v;
        }
        dumv += e;
    }
    if (c->coll_on)
        for (int i = 0; i < n; i++) {
            double ri[3] = {px[i], py[i], pz[i]}, ei[3] = {ox[i], oy[i], oz[i]};
            wall += lco_colloid_rod(c, ri, ei, box);
        }
    return 0.5 * dumv + wall;
}

/* ------------------------------------------------------------------------ */
/* reference-semantics move (attempt_monte_carlo_move, MCnptColloid.c:2445-2604) */
/* ------------------------------------------------------------------------ */

#define REF_POINTS 1000000
#define REF_IMAX (1.0f / 2147483647) /* I_MAX_RAND with glibc RAND_MAX (MCnptColloid.c:14) */

int lco_ref_particle_index(int r, int n) { return (int)(r * REF_IMAX * n); }
int lco_ref_table_index(int r) { return (int)(r * REF_IMAX * REF_POINTS); }

static int take(const int *rands, int n_rands, int *pos)
{
    if (*pos >= n_rands) return -1;
    return rands[(*pos)++];
}

/* One attempt with the reference's exact arithmetic, consuming libc rand()
 * values from `rands` in the reference's order: particle (2475), two table
 * indices (2486-2487), three displacements (2502-2509), and one acceptance
 * draw only when dE > 0 (2567-2572).  Old energy over the CSR Verlet list
 * (GBij_lstnb, 1647-1699), new energy over all j (GBij_PosMod, 1562-1595).
 * gate_colloid = 0 adds GBCollRod in both energies regardless of
 * colloid_wall_option, as the reference does (2495, 2560).
 * Returns 1 accepted, 0 rejected, 2 colloid hard-core reject, -1 out of rands. */
int lco_move_refsem(const lco_consts *c, int n, double *px, double *py, double *pz, double *ox, double *oy,
                    double *oz, const double box[3], const int *nb_count, const int *nb_list, const float *rvx,
                    const float *rvy, const float *rvz, const int *rands, int n_rands, int *rand_pos,
                    double *energy, long *accepted, double *tracker, int gate_colloid)
{
    int r;
    if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
    int sel = lco_ref_particle_index(r, n);
    if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
    int didx = lco_ref_table_index(r);
    if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
    int ridx = lco_ref_table_index(r);
    int coll = gate_colloid ? c->coll_on : 1;

    double ri[3] = {px[sel], py[sel], pz[sel]}, ei[3] = {ox[sel], oy[sel], oz[sel]};
    double old_e = 0.0;
    {
        int start = sel > 0 ? nb_count[sel - 1] : 0, end = nb_count[sel];
        for (int k = start; k < end; k++) {
            int j = nb_list[k];
            double rj[3] = {px[j], py[j], pz[j]}, ej[3] = {ox[j], oy[j], oz[j]};
            int in;
            double v = lco_pair(c, ri, ei, rj, ej, box, &in);
            if (in) old_e += v;
        }
    }
    if (coll) old_e += lco_colloid_rod(c, ri, ei, box);

    double nw[3];
    if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
    nw[0] = ri[0] + (double)(float)c->max_disp * ((double)r * REF_IMAX - 0.5);
    if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
    nw[1] = ri[1] + (double)(float)c->max_disp * ((double)r * REF_IMAX - 0.5);
    if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
    nw[2] = ri[2] + (double)(float)c->max_disp * ((double)r * REF_IMAX - 0.5);
    lco_apply_pbc(&nw[0], &nw[1], &nw[2], box);

    double dx, dy, dz;
    double r2 = lco_distance_sq(nw[0], nw[1], nw[2], 0.5 * box[0], 0.5 * box[1], 0.5 * box[2], box, &dx, &dy, &dz);
    if (!(r2 > c->coll_R * c->coll_R)) return 2;

    float mr = (float)c->max_rot;
    double ne[3];
    ne[0] = rvx[ridx] * mr + ei[0];
    ne[1] = rvy[ridx] * mr + ei[1];
    ne[2] = rvz[ridx] * mr + ei[2];
    double norm2 = ne[0] * ne[0] + ne[1] * ne[1] + ne[2] * ne[2];
    if (norm2 <= 1e-12) {
        ne[0] = ei[0]; ne[1] = ei[1]; ne[2] = ei[2];
    } else {
        ne[0] /= sqrt(norm2); ne[1] /= sqrt(norm2); ne[2] /= sqrt(norm2);
    }

    double new_e = 0.0;
    for (int j = 0; j < n; j++) {
        if (j == sel) continue;
        double rj[3] = {px[j], py[j], pz[j]}, ej[3] = {ox[j], oy[j], oz[j]};
        int in;
        double v = lco_pair(c, nw, ne, rj, ej, box, &in);
        if (in) new_e += v;
    }
    if (coll) new_e += lco_colloid_rod(c, nw, ne, box);

    double de = new_e - old_e;
    int acc;
    if (de <= 0.0) acc = 1;
    else {
        if ((r = take(rands, n_rands, rand_pos)) < 0) return -1;
        double u = (double)r * REF_IMAX;
        double lu = (c->arith == LCO_ARITH_REFERENCE) ? log(u) : (u > 0.0 ? lco_log(u) : -INFINITY);
        acc = lu <= (-c->beta * de);
    }
    if (!acc) return 0;
    px[sel] = nw[0]; py[sel] = nw[1]; pz[sel] = nw[2];
    ox[sel] = ne[0]; oy[sel] = ne[1]; oz[sel] = ne[2];
    {
        double a = fabs(rvx[didx]), b = fabs(rvy[didx]), cc = fabs(rvz[didx]);
        double m = a > b ? a : b;
        m = m > cc ? m : cc;
        *tracker += 3.0 * m * m;
    }
    *energy += de;
    *accepted += 1;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 and draws                                                   */
/* ------------------------------------------------------------------------ */

/* Philox4x32 with 10 rounds (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11): multipliers and Weyl key increments
 * as published there. */
void lco_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* uniform in (0, 1): (x + 1/2) / 2^32, exact in double */
double lco_u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

/* Natural log for u in (0, 1], written for this project: u = m 2^e with m in
 * [sqrt(1/2), sqrt(2)), log m = 2 atanh(t), t = (m-1)/(m+1), |t| < 0.1716,
 * atanh by its odd Taylor series to t^21 (truncation < 1e-18), ln 2 split in a
 * 32-bit head and a tail so that e*ln2_hi is exact. */
double lco_log(double u)
{
    int e;
    double m = frexp(u, &e);
    if (m < 0.70710678118654752440) {
        m = m * 2.0;
        e = e - 1;
    }
    double t = (m - 1.0) / (m + 1.0);
    double t2 = t * t;
    double p = 1.0 / 21.0;
    p = p * t2 + 1.0 / 19.0;
    p = p * t2 + 1.0 / 17.0;
    p = p * t2 + 1.0 / 15.0;
    p = p * t2 + 1.0 / 13.0;
    p = p * t2 + 1.0 / 11.0;
    p = p * t2 + 1.0 / 9.0;
    p = p * t2 + 1.0 / 7.0;
    p = p * t2 + 1.0 / 5.0;
    p = p * t2 + 1.0 / 3.0;
    p = p * t2 + 1.0;
    double de = (double)e;
    const double ln2_hi = 0x1.62e42feep-1;
    const double ln2_lo = 0x1.a39ef35793c76p-33;
    return de * ln2_hi + (de * ln2_lo + 2.0 * t * p);
}

/* e^x - 1 for |x| <= 1.5 by its Taylor series to x^30 in nested form
 * (truncation below 1e-20), written for this project. */
double lco_expm1(double x)
{
    double s = 1.0;
    for (int k = 30; k >= 2; k--) s = 1.0 + s * x / (double)k;
    return x * s;
}

void lco_key(uint64_t seed, int replica, uint32_t key[2])
{
    key[0] = (uint32_t)seed ^ ((uint32_t)replica * 0x9E3779B9u);
    key[1] = (uint32_t)(seed >> 32);
}

static void philox_at(const uint32_t key[2], uint32_t id, uint64_t sweep, uint32_t tag, uint32_t out[4])
{
    uint32_t ctr[4] = {id, (uint32_t)sweep, (uint32_t)(sweep >> 32), tag};
    lco_philox(ctr, key, out);
}

#define TAG_MOVE 0u
#define TAG_SPHERE 1u        /* 1..16 */
#define TAG_SHIFT 0x100u
#define TAG_COLOUR 0x101u    /* and 0x102 */
#define TAG_VOLUME 0x103u
#define TAG_COLOUR_EXT 0x110u /* 0x110..0x114: colour order beyond 8 colours (fine grid) */
#define TAG_INIT 0x200u      /* and 0x201 */
#define SWEEP_ID 0xFFFFFFFFu /* counter word 0 for per-sweep draws */

/* Marsaglia (1972) point on the unit sphere, the method of pto_ransphr
 * (MCnptColloid.c:3050-3078) in double: x1, x2 = 1 - 2u until s < 1. */
void lco_sphere_point(const uint32_t key[2], uint32_t id, uint64_t sweep, double v[3])
{
    for (int t = 0; t < 32; t++) {
        uint32_t o[4];
        philox_at(key, id, sweep, TAG_SPHERE + (uint32_t)(t >> 1), o);
        double x1 = 1.0 - 2.0 * lco_u01(o[2 * (t & 1)]);
        double x2 = 1.0 - 2.0 * lco_u01(o[2 * (t & 1) + 1]);
        double s = x1 * x1 + x2 * x2;
        if (s < 1.0) {
            double q = sqrt(1.0 - s);
            v[0] = 2.0 * x1 * q;
            v[1] = 2.0 * x2 * q;
            v[2] = 1.0 - 2.0 * s;
            return;
        }
    }
    v[0] = 0.0; v[1] = 0.0; v[2] = 1.0;
}

/* ------------------------------------------------------------------------ */
/* initial configuration: simple-cubic lattice (MCnptColloid.c:2920-3033)    */
/* ------------------------------------------------------------------------ */

/* Box V = N/rho + V_colloid (2935), n_s = smallest with n_s^3 >= N (2955)
 * counting only sites outside the colloid (the reference runs past the last
 * site when the colloid removes sites),
 * spacing L/n_s without the reference's clamp to sigma_ee (2957-2963, which
 * pushes sites outside the box when dense), sites with |r - C|^2 <= R^2 skipped
 * when R > 0 (2967-2992).  Orientations: uniform on the sphere (Marsaglia), or
 * uniform on the cap within init_orientation_cone_deg of +z. */
int lco_init_lattice(const lco_params *p, int replica, double *px, double *py, double *pz, double *ox, double *oy,
                     double *oz, double box[3])
{
    const double pi = 3.1415926535898; /* MCnptColloid.c:10 */
    int n = p->num_particles;
    double R = p->colloid_radius;
    double vcol = (4. / 3.) * pi * pow(R, 3);
    double V = (n / p->system_density) + vcol;
    double L = pow(V, 1.0 / 3.0);
    box[0] = box[1] = box[2] = L;
    double C = 0.5 * L;
    int ns = 2;
    for (;; ns++) { /* smallest n_s whose sites outside the colloid hold N */
        long free_sites = 0;
        double d = L / (double)ns;
        for (long s = 0; s < (long)ns * ns * ns; s++) {
            double x = (double)(s % ns) * d, y = (double)((s / ns) % ns) * d, z = (double)(s / ((long)ns * ns)) * d;
            double dx, dy, dz;
            double r2 = lco_distance_sq(x, y, z, C, C, C, box, &dx, &dy, &dz);
            if (!(R > 0.0 && r2 <= R * R)) free_sites++;
        }
        if (free_sites >= n) break;
    }
    double delta = L / (double)ns;
    uint32_t key[2];
    lco_key(p->rng_seed, replica, key);
    double cone = p->init_orientation_cone_deg;
    double cmin = cos(cone * (pi / 180.0));
    long site = 0, total = (long)ns * ns * ns;
    for (int i = 0; i < n; i++) {
        double x, y, z;
        for (;;) {
            if (site >= total) return -1; /* colloid leaves too few sites */
            int ix = (int)(site % ns), iy = (int)((site / ns) % ns), iz = (int)(site / ((long)ns * ns));
            site++;
            x = (double)ix * delta;
            y = (double)iy * delta;
            z = (double)iz * delta;
            double dx, dy, dz;
            double r2 = lco_distance_sq(x, y, z, C, C, C, box, &dx, &dy, &dz);
            if (R > 0.0 && r2 <= R * R) continue;
            break;
        }
        px[i] = x; py[i] = y; pz[i] = z;
        if (cone >= 180.0) {
            double v[3];
            lco_sphere_point(key, (uint32_t)i, 0xFFFFFFFFFFFFFFFFull, v);
            ox[i] = v[0]; oy[i] = v[1]; oz[i] = v[2];
        } else {
            uint32_t o[4];
            philox_at(key, (uint32_t)i, 0xFFFFFFFFFFFFFFFFull, TAG_INIT, o);
            double ct = 1.0 - lco_u01(o[0]) * (1.0 - cmin);
            double st = sqrt(1.0 - ct * ct);
            double ph = 2.0 * pi * lco_u01(o[1]);
            ox[i] = st * cos(ph); oy[i] = st * sin(ph); oz[i] = ct;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* checkerboard cell grid                                                    */
/* ------------------------------------------------------------------------ */

/* Cells per axis: the largest even count whose width is >= wmin = rc + dmax
 * (so that same-colour cells never interact even after each particle has moved
 * once by up to dmax/2 per axis), or 1 when even 2 cells do not fit. */
int lco_grid_dims(double L, double wmin, int *nc)
{
    int m = (int)floor(L / wmin);
    *nc = m >= 2 ? m - (m & 1) : 1;
    return 0;
}

void lco_sweep_shift(const uint32_t key[2], uint64_t sweep, const int nc[3], const double box[3], double shift[3])
{
    uint32_t o[4];
    philox_at(key, SWEEP_ID, sweep, TAG_SHIFT, o);
    for (int k = 0; k < 3; k++) shift[k] = lco_u01(o[k]) * (box[k] / (double)nc[k]);
}

/* Shuffled colour order for the sweep (the reference shuffles its 8 subcells,
 * MCnptColloid.c:646-648): Fisher-Yates over 0..7. */
void lco_colour_order(const uint32_t key[2], uint64_t sweep, int perm[8])
{
    uint32_t a[4], b[4];
    philox_at(key, SWEEP_ID, sweep, TAG_COLOUR, a);
    philox_at(key, SWEEP_ID, sweep, TAG_COLOUR + 1, b);
    uint32_t r[8] = {a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3]};
    for (int i = 0; i < 8; i++) perm[i] = i;
    for (int i = 7; i >= 1; i--) {
        int j = (int)(r[7 - i] % (uint32_t)(i + 1));
        int t = perm[i];
        perm[i] = perm[j];
        perm[j] = t;
    }
}

int lco_cell_of(double x, double shift, double w, int nc, double L)
{
    double t = x - shift;
    if (t < 0.0) t += L;
    int c = (int)(t / w);
    if (c >= nc) c = nc - 1;
    if (c < 0) c = 0;
    return c;
}

/* Fine cell grid (cell_grid 1): the largest count of cells at least wmin wide,
 * odd or even (an odd count >= 3 takes 3 colours on that axis). */
int lco_grid_dims_fine(double L, double wmin, int fine, int *nc)
{
    int m = (int)floor(L / wmin);
    *nc = m >= 2 ? ((fine && m >= 3) ? m : m - (m & 1)) : 1;
    return 0;
}

static int grid_build_nc(lco_grid *g, int n, const double *px, const double *py, const double *pz,
                         const double box[3], const int nc[3], const double shift[3]);

int lco_grid_build(lco_grid *g, int n, const double *px, const double *py, const double *pz, const double box[3],
                   double wmin, const double shift[3])
{
    int nc[3];
    for (int k = 0; k < 3; k++) lco_grid_dims(box[k], wmin, &nc[k]);
    return grid_build_nc(g, n, px, py, pz, box, nc, shift);
}

static int grid_build_nc(lco_grid *g, int n, const double *px, const double *py, const double *pz,
                         const double box[3], const int nc[3], const double shift[3])
{
    for (int k = 0; k < 3; k++) {
        g->nc[k] = nc[k];
        g->w[k] = box[k] / (double)g->nc[k];
        g->shift[k] = shift[k];
    }
    g->ncell = g->nc[0] * g->nc[1] * g->nc[2];
    g->cell_start = calloc((size_t)g->ncell + 1, sizeof(int));
    g->order = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *cid = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *fill = calloc((size_t)g->ncell, sizeof(int));
    for (int i = 0; i < n; i++) {
        int cx = lco_cell_of(px[i], shift[0], g->w[0], g->nc[0], box[0]);
        int cy = lco_cell_of(py[i], shift[1], g->w[1], g->nc[1], box[1]);
        int cz = lco_cell_of(pz[i], shift[2], g->w[2], g->nc[2], box[2]);
        cid[i] = (cz * g->nc[1] + cy) * g->nc[0] + cx;
        g->cell_start[cid[i] + 1]++;
    }
    for (int c = 0; c < g->ncell; c++) g->cell_start[c + 1] += g->cell_start[c];
    for (int i = 0; i < n; i++) { /* ascending i keeps ascending id inside every cell */
        int c = cid[i];
        g->order[g->cell_start[c] + fill[c]++] = i;
    }
    free(cid);
    free(fill);
    return 0;
}

void lco_grid_free(lco_grid *g)
{
    free(g->cell_start);
    free(g->order);
    g->cell_start = g->order = NULL;
}

/* Stencil cells of cell (cx,cy,cz): offsets dz, dy, dx = -1..1 in that nesting,
 * periodic, duplicates (boxes with < 3 cells per axis) dropped at their first
 * occurrence.  Returns the count. */
static int stencil_cells(const lco_grid *g, int cx, int cy, int cz, int out[27])
{
    int m = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                int x = (cx + dx + g->nc[0]) % g->nc[0];
                int y = (cy + dy + g->nc[1]) % g->nc[1];
                int z = (cz + dz + g->nc[2]) % g->nc[2];
                int c = (z * g->nc[1] + y) * g->nc[0] + x;
                int dup = 0;
                for (int s = 0; s < m; s++) dup |= out[s] == c;
                if (!dup) out[m++] = c;
            }
    return m;
}

/* Canonical 32-way sum: term q goes to partial q mod 32, partials summed in
 * order, then combined by the xor butterfly (16, 8, 4, 2, 1) that a warp
 * reduction performs. */
static double butterfly32(double part[32])
{
    for (int off = 16; off >= 1; off >>= 1) {
        double nxt[32];
        for (int l = 0; l < 32; l++) nxt[l] = part[l] + part[l ^ off];
        memcpy(part, nxt, sizeof(nxt));
    }
    return part[0];
}

/* One checkerboard sweep: per sweep a random grid shift and shuffled colour
 * order; per colour every active cell; per active cell its particles in
 * ascending id, each attempted once with the per-move semantics of
 * attempt_monte_carlo_move (MCnptColloid.c:2474-2598), a move out of the
 * particle's cell rejected (leaves_cell):
 *   E_old = sum_j phi(old, j) + U_coll(old)          (2491-2498)
 *   trial r' = r + d (u - 1/2) per axis, wrapped       (2502-2512)
 *   colloid hard-core reject if |r' - C|^2 <= R^2     (2516-2520)
 *   trial u' = normalise(u + rot * v), v on S^2       (2526-2551)
 *   E_new = sum_j phi(new, j) + U_coll(new)           (2554-2563)
 *   accept if dE <= 0 or log(x) <= -beta dE           (2566-2574)
 * with the colloid term added only when colloid_wall_option == 1 and Philox
 * draws in place of rand().  The sums over the stencil use the canonical
 * 32-way order of butterfly32. */
/* Checkerboard rule for detailed balance: a trial translation that carries the
 * particle out of the cell (cx, cy, cz) it was binned into at the sweep's start
 * is rejected without an energy evaluation, so that the cells' contents and the
 * order of the attempts stay fixed during the sweep (the rule of parallel
 * hard-particle MC on GPUs, Anderson et al., J. Comput. Phys. 254 (2013) 27;
 * the reference's random-sequential pick needs none).  Same operations, in the
 * same order, as the GPU kernels' leaves_cell. */
static int leaves_cell(const lco_grid *g, const int cell[3], const double ro[3], const double dsp[3],
                       const double box[3])
{
    for (int a = 0; a < 3; a++) {
        double o = g->shift[a] + (double)cell[a] * g->w[a];
        double r = ro[a] - o;
        double k = rint((r - 0.5 * g->w[a]) * (1.0 / box[a]));
        double rel = r - box[a] * k;
        double nr = rel + dsp[a];
        if (!(nr >= 0.0 && nr < g->w[a])) return 1;
    }
    return 0;
}

/* One trial move of particle k of cell `cell` against the staged stencil
 * particles slots[0..S) (attempt_monte_carlo_move, MCnptColloid.c:2474-2598,
 * with the checkerboard's pick and Philox draws): 0 rejected (also a move out
 * of the cell), 1 accepted (state written, *de set), 2 hard-core reject. */
static int attempt_move(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int k, const int *slots, int S,
                        double *px, double *py, double *pz, double *ox, double *oy, double *oz, const double box[3],
                        const lco_grid *g, const int cell[3], double *de_out)
{
    uint32_t rnd[4];
    philox_at(key, (uint32_t)k, sweep, TAG_MOVE, rnd);
    double ro[3] = {px[k], py[k], pz[k]}, eo[3] = {ox[k], oy[k], oz[k]};
    double rn[3], dsp[3];
    dsp[0] = c->max_disp * (lco_u01(rnd[0]) - 0.5);
    dsp[1] = c->max_disp * (lco_u01(rnd[1]) - 0.5);
    dsp[2] = c->max_disp * (lco_u01(rnd[2]) - 0.5);
    rn[0] = ro[0] + dsp[0];
    rn[1] = ro[1] + dsp[1];
    rn[2] = ro[2] + dsp[2];
    lco_apply_pbc(&rn[0], &rn[1], &rn[2], box);
    double ddx, ddy, ddz;
    double rc2c = lco_distance_sq(rn[0], rn[1], rn[2], 0.5 * box[0], 0.5 * box[1], 0.5 * box[2], box, &ddx, &ddy,
                                  &ddz);
    if (!(rc2c > c->coll_R * c->coll_R)) return 2;
    if (leaves_cell(g, cell, ro, dsp, box)) return 0;
    double v[3];
    lco_sphere_point(key, (uint32_t)k, sweep, v);
    double en[3];
    en[0] = c->max_rot * v[0] + eo[0];
    en[1] = c->max_rot * v[1] + eo[1];
    en[2] = c->max_rot * v[2] + eo[2];
    double norm2 = en[0] * en[0] + en[1] * en[1] + en[2] * en[2];
    if (norm2 <= 1e-12) {
        en[0] = eo[0]; en[1] = eo[1]; en[2] = eo[2];
    } else {
        double nr = sqrt(norm2);
        en[0] /= nr; en[1] /= nr; en[2] /= nr;
    }
    double po[32], pn[32];
    memset(po, 0, sizeof(po));
    memset(pn, 0, sizeof(pn));
    for (int q = 0; q < S; q++) {
        int j = slots[q];
        if (j == k) continue;
        double rj[3] = {px[j], py[j], pz[j]}, ej[3] = {ox[j], oy[j], oz[j]};
        int in;
        double vo = lco_pair(c, ro, eo, rj, ej, box, &in);
        if (in) po[q & 31] += vo;
        double vn = lco_pair(c, rn, en, rj, ej, box, &in);
        if (in) pn[q & 31] += vn;
    }
    double Eo = butterfly32(po), En = butterfly32(pn);
    if (c->coll_on) {
        Eo = Eo + lco_colloid_rod(c, ro, eo, box);
        En = En + lco_colloid_rod(c, rn, en, box);
    }
    double de = En - Eo;
    int acc = (de <= 0.0) || (lco_log(lco_u01(rnd[3])) <= -c->beta * de);
    if (acc) {
        px[k] = rn[0]; py[k] = rn[1]; pz[k] = rn[2];
        ox[k] = en[0]; oy[k] = en[1]; oz[k] = en[2];
        *de_out = de;
    }
    return acc;
}

/* the staged particles of the 27-cell stencil of cell (cx, cy, cz) */
static int stage_stencil(const lco_grid *g, int cx, int cy, int cz, int *slots)
{
    int sc[27];
    int ns = stencil_cells(g, cx, cy, cz, sc);
    int S = 0;
    for (int s = 0; s < ns; s++)
        for (int q = g->cell_start[sc[s]]; q < g->cell_start[sc[s] + 1]; q++) slots[S++] = g->order[q];
    return S;
}

/* Cells of colour b along an axis of nc cells with k colours, and the index of
 * the j-th of them.  k = 2 (even nc, or a single cell): cells b, b + 2, ...
 * k = 3 (odd nc >= 3, fine grid), nc = 3q + r: colour i mod 3 for i < 3q, then
 * r = 1: cell 3q takes colour 1; r = 2: cells 3q, 3q + 1 take colours 0, 1
 * (neighbours never share a colour, and every colour holds q or q + 1 cells). */
static int axis_colour_count(int nc, int k, int b)
{
    if (k != 3) return (nc - b + 1) / 2;
    int q = nc / 3, r = nc - 3 * q;
    return q + ((r >= 1 && b == 1) ? 1 : 0) + ((r == 2 && b == 0) ? 1 : 0);
}
static int axis_colour_cell(int nc, int k, int b, int j)
{
    if (k != 3) return 2 * j + b;
    int q = nc / 3, r = nc - 3 * q;
    return j < q ? b + 3 * j : 3 * q + (r == 2 ? b : 0);
}

/* Shuffled order of K colours (K = 8: lco_colour_order's draws and result;
 * more colours draw 4 more words per TAG_COLOUR_EXT call). */
static void colour_order_k(const uint32_t key[2], uint64_t sweep, int K, int *perm)
{
    uint32_t rr[32];
    uint32_t a[4], b[4];
    philox_at(key, SWEEP_ID, sweep, TAG_COLOUR, a);
    philox_at(key, SWEEP_ID, sweep, TAG_COLOUR + 1, b);
    for (int i = 0; i < 4; i++) {
        rr[i] = a[i];
        rr[4 + i] = b[i];
    }
    for (int m = 0; 8 + 4 * m < K - 1; m++) {
        uint32_t e[4];
        philox_at(key, SWEEP_ID, sweep, TAG_COLOUR_EXT + (uint32_t)m, e);
        for (int i = 0; i < 4; i++) rr[8 + 4 * m + i] = e[i];
    }
    for (int i = 0; i < K; i++) perm[i] = i;
    for (int i = K - 1; i >= 1; i--) {
        int j = (int)(rr[K - 1 - i] % (uint32_t)(i + 1));
        int t = perm[i];
        perm[i] = perm[j];
        perm[j] = t;
    }
}

/* One checkerboard sweep on the even grid (fine = 0: 8 colours) or on the
 * fine grid (fine = 1: odd cell counts take 3 colours on their axis, up to 27
 * colours); see lco_sweep for the move. */
int lco_sweep_grid(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int fine, int n, double *px,
                   double *py, double *pz, double *ox, double *oy, double *oz, const double box[3], lco_sweep_stats *st,
                   unsigned char *accept_bits, int *order_out)
{
    int nc[3], kc[3];
    for (int k = 0; k < 3; k++) {
        lco_grid_dims_fine(box[k], c->wmin, fine, &nc[k]);
        kc[k] = ((nc[k] & 1) && nc[k] >= 3) ? 3 : 2;
    }
    double shift[3];
    lco_sweep_shift(key, sweep, nc, box, shift);
    lco_grid g;
    grid_build_nc(&g, n, px, py, pz, box, nc, shift);
    const int K = kc[0] * kc[1] * kc[2];
    int perm[27];
    colour_order_k(key, sweep, K, perm);
    memset(st, 0, sizeof(*st));
    long nb = 0;
    int *slots = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int ci = 0; ci < K; ci++) {
        int col = perm[ci];
        int b[3] = {col % kc[0], (col / kc[0]) % kc[1], col / (kc[0] * kc[1])};
        int cnt[3];
        for (int a = 0; a < 3; a++) cnt[a] = axis_colour_count(nc[a], kc[a], b[a]);
        for (int jz = 0; jz < cnt[2]; jz++)
            for (int jy = 0; jy < cnt[1]; jy++)
                for (int jx = 0; jx < cnt[0]; jx++) {
                    const int cx = axis_colour_cell(nc[0], kc[0], b[0], jx);
                    const int cy = axis_colour_cell(nc[1], kc[1], b[1], jy);
                    const int cz = axis_colour_cell(nc[2], kc[2], b[2], jz);
                    int cell = (cz * g.nc[1] + cy) * g.nc[0] + cx;
                    const int cc[3] = {cx, cy, cz};
                    int S = stage_stencil(&g, cx, cy, cz, slots);
                    for (int a = g.cell_start[cell]; a < g.cell_start[cell + 1]; a++) {
                        int k = g.order[a];
                        if (order_out) order_out[st->attempted] = k;
                        st->attempted++;
                        double de = 0.0;
                        int r = attempt_move(c, key, sweep, k, slots, S, px, py, pz, ox, oy, oz, box, &g, cc, &de);
                        if (accept_bits) accept_bits[nb] = (unsigned char)r;
                        nb++;
                        if (r == 2) st->hardcore_rejected++;
                        if (r == 1) {
                            st->accepted++;
                            st->dE_sum += de;
                        }
                    }
                }
    }
    free(slots);
    lco_grid_free(&g);
    return 0;
}

int lco_sweep(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int n, double *px, double *py, double *pz,
              double *ox, double *oy, double *oz, const double box[3], lco_sweep_stats *st, unsigned char *accept_bits,
              int *order_out)
{
    return lco_sweep_grid(c, key, sweep, 0, n, px, py, pz, ox, oy, oz, box, st, accept_bits, order_out);
}

/* lco_sweep with the active cells of each colour shared among threads
 * (OpenMP, when this file is built with it): same-colour cells never interact,
 * so the final state equals lco_sweep's bit for bit; dE_sum is summed in
 * another order.  The CPU baseline's port of the checkerboard. */
int lco_sweep_parallel(const lco_consts *c, const uint32_t key[2], uint64_t sweep, int n, double *px, double *py,
                       double *pz, double *ox, double *oy, double *oz, const double box[3], lco_sweep_stats *st)
{
    int nc[3];
    for (int k = 0; k < 3; k++) lco_grid_dims(box[k], c->wmin, &nc[k]);
    double shift[3];
    lco_sweep_shift(key, sweep, nc, box, shift);
    lco_grid g;
    lco_grid_build(&g, n, px, py, pz, box, c->wmin, shift);
    int perm[8];
    lco_colour_order(key, sweep, perm);
    long att = 0, acc = 0, hard = 0;
    double dsum = 0.0;
    for (int ci = 0; ci < 8; ci++) {
        int col = perm[ci];
        int bx = col & 1, by = (col >> 1) & 1, bz = (col >> 2) & 1;
        int hx = (g.nc[0] - bx + 1) / 2, hy = (g.nc[1] - by + 1) / 2, hz = (g.nc[2] - bz + 1) / 2;
        long ncell = (long)hx * hy * hz;
#pragma omp parallel reduction(+ : att, acc, hard, dsum)
        {
            int *slots = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 4)
            for (long e = 0; e < ncell; e++) {
                int cx = bx + 2 * (int)(e % hx), cy = by + 2 * (int)((e / hx) % hy), cz = bz + 2 * (int)(e / ((long)hx * hy));
                int cell = (cz * g.nc[1] + cy) * g.nc[0] + cx;
                const int cc[3] = {cx, cy, cz};
                int S = stage_stencil(&g, cx, cy, cz, slots);
                for (int a = g.cell_start[cell]; a < g.cell_start[cell + 1]; a++) {
                    double de = 0.0;
                    int r = attempt_move(c, key, sweep, g.order[a], slots, S, px, py, pz, ox, oy, oz, box, &g, cc,
                                         &de);
                    att++;
                    if (r == 2) hard++;
                    if (r == 1) {
                        acc++;
                        dsum += de;
                    }
                }
            }
            free(slots);
        }
    }
    st->attempted = att;
    st->accepted = acc;
    st->hardcore_rejected = hard;
    st->dE_sum = dsum;
    lco_grid_free(&g);
    return 0;
}

/* Total energy over the cell stencil: 1/2 sum_i sum_{j != i, r < rc} phi +
 * sum_i U_coll (tot_ene, MCnptColloid.c:1598-1622, with cells in place of the
 * all-pairs loop).  Cells of width >= rc, unshifted. */
double lco_total_energy_cells(const lco_consts *c, int n, const double *px, const double *py, const double *pz,
                              const double *ox, const double *oy, const double *oz, const double box[3])
{
    lco_grid g;
    double zero[3] = {0, 0, 0};
    lco_grid_build(&g, n, px, py, pz, box, c->rc, zero);
    double dumv = 0.0, wall = 0.0;
    for (int cz = 0; cz < g.nc[2]; cz++)
        for (int cy = 0; cy < g.nc[1]; cy++)
            for (int cx = 0; cx < g.nc[0]; cx++) {
                int cell = (cz * g.nc[1] + cy) * g.nc[0] + cx;
                int sc[27];
                int ns = stencil_cells(&g, cx, cy, cz, sc);
                for (int a = g.cell_start[cell]; a < g.cell_start[cell + 1]; a++) {
                    int i = g.order[a];
                    double ri[3] = {px[i], py[i], pz[i]}, ei[3] = {ox[i], oy[i], oz[i]};
                    double e = 0.0;
                    for (int s = 0; s < ns; s++)
                        for (int q = g.cell_start[sc[s]]; q < g.cell_start[sc[s] + 1]; q++) {
                            int j = g.order[q];
                            if (j == i) continue;
                            double rj[3] = {px[j], py[j], pz[j]}, ej[3] = {ox[j], oy[j], oz[j]};
                            int in;
                            double v = lco_pair(c, ri, ei, rj, ej, box, &in);
                            if (in) e += v;
                        }
                    dumv += e;
                    if (c->coll_on) wall += lco_colloid_rod(c, ri, ei, box);
                }
            }
    lco_grid_free(&g);
    return 0.5 * dumv + wall;
}

/* NPT volume move (no reference code: system_pressure is parsed at
 * MCnptColloid.c:3978 and never used).  ln V random walk: delta uniform in
 * [-dlnV_max, dlnV_max], V' = V e^delta, L' = L e^(delta/3), positions scaled
 * about the origin so that the colloid stays at the box centre; hard-core
 * reject if a rod centre lands inside the colloid; otherwise accept with
 * probability min(1, exp(-beta (dU + P dV) + (N + 1) delta)). */
int lco_volume_move(const lco_consts *c, const uint32_t key[2], uint64_t sweep, double pressure, double dlnV_max,
                    int n, double *px, double *py, double *pz, const double *ox, const double *oy, const double *oz,
                    double box[3], lco_volume_info *info)
{
    uint32_t o[4];
    philox_at(key, SWEEP_ID, sweep, TAG_VOLUME, o);
    double delta = dlnV_max * (2.0 * lco_u01(o[0]) - 1.0);
    double lam = 1.0 + lco_expm1(delta / 3.0);
    double V = box[0] * box[1] * box[2];
    double dV = V * lco_expm1(delta);
    double nb[3] = {box[0] * lam, box[1] * lam, box[2] * lam};
    double *qx = malloc(sizeof(double) * (size_t)n), *qy = malloc(sizeof(double) * (size_t)n),
           *qz = malloc(sizeof(double) * (size_t)n);
    int hard = 0;
    for (int i = 0; i < n; i++) {
        qx[i] = px[i] * lam;
        qy[i] = py[i] * lam;
        qz[i] = pz[i] * lam;
        double dx, dy, dz;
        double r2 = lco_distance_sq(qx[i], qy[i], qz[i], 0.5 * nb[0], 0.5 * nb[1], 0.5 * nb[2], nb, &dx, &dy, &dz);
        if (!(r2 > c->coll_R * c->coll_R)) hard = 1;
    }
    info->delta = delta;
    info->lambda = lam;
    info->dV = dV;
    info->U_old = lco_total_energy_cells(c, n, px, py, pz, ox, oy, oz, box);
    int ret;
    if (hard) {
        info->U_new = 0.0;
        info->lnA = -INFINITY;
        ret = 2;
    } else {
        info->U_new = lco_total_energy_cells(c, n, qx, qy, qz, ox, oy, oz, nb);
        double dU = info->U_new - info->U_old;
        double lnA = -c->beta * (dU + pressure * dV) + (double)(n + 1) * delta;
        info->lnA = lnA;
        ret = (lnA >= 0.0) || (lco_log(lco_u01(o[1])) <= lnA);
    }
    if (ret == 1) {
        memcpy(px, qx, sizeof(double) * (size_t)n);
        memcpy(py, qy, sizeof(double) * (size_t)n);
        memcpy(pz, qz, sizeof(double) * (size_t)n);
        box[0] = nb[0]; box[1] = nb[1]; box[2] = nb[2];
    }
    info->accepted = ret == 1;
    free(qx); free(qy); free(qz);
    return ret;
}

/* ------------------------------------------------------------------------ */
/* order parameter (compute_liquid_crystal_order_parameters,                 */
/* MCnptColloid.c:2117-2218), double precision, true largest eigenvalue      */
/* ------------------------------------------------------------------------ */

void lco_order_parameter(int n, const double *ox, const double *oy, const double *oz, double Q[6], double *P2,
                         double director[3])
{
    double s[6] = {0, 0, 0, 0, 0, 0}; /* xx xy xz yy yz zz */
    for (int i = 0; i < n; i++) {
        s[0] += ox[i] * ox[i];
        s[1] += ox[i] * oy[i];
        s[2] += ox[i] * oz[i];
        s[3] += oy[i] * oy[i];
        s[4] += oy[i] * oz[i];
        s[5] += oz[i] * oz[i];
    }
    double inv = 1.0 / (double)n;
    Q[0] = s[0] * inv - 1.0 / 3.0;
    Q[1] = s[1] * inv;
    Q[2] = s[2] * inv;
    Q[3] = s[3] * inv - 1.0 / 3.0;
    Q[4] = s[4] * inv;
    Q[5] = s[5] * inv - 1.0 / 3.0;
    double a[3][3] = {{Q[0], Q[1], Q[2]}, {Q[1], Q[3], Q[4]}, {Q[2], Q[4], Q[5]}};
    double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    /* cyclic Jacobi rotations (Golub & Van Loan, Algorithm 8.4.3) */
    for (int sweep = 0; sweep < 50; sweep++) {
        double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (off < 1e-40) break;
        for (int p = 0; p < 2; p++)
            for (int q = p + 1; q < 3; q++) {
                if (a[p][q] == 0.0) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < 3; k++) { /* A <- A J */
                    double akp = a[k][p], akq = a[k][q];
                    a[k][p] = cs * akp - sn * akq;
                    a[k][q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < 3; k++) { /* A <- J^T A */
                    double apk = a[p][k], aqk = a[q][k];
                    a[p][k] = cs * apk - sn * aqk;
                    a[q][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    double vkp = v[k][p], vkq = v[k][q];
                    v[k][p] = cs * vkp - sn * vkq;
                    v[k][q] = sn * vkp + cs * vkq;
                }
            }
    }
    int im = 0;
    for (int i = 1; i < 3; i++)
        if (a[i][i] > a[im][im]) im = i;
    *P2 = 1.5 * a[im][im];
    director[0] = v[0][im];
    director[1] = v[1][im];
    director[2] = v[2][im];
}
