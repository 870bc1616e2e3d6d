/*
 * lcmc_run.c - a C host over include/lcmc.h: the reference's serial cycle loop
 * (MCnptColloid.c:887-1061) with the Monte Carlo path in liblcmc.so.
 *
 *   lcmc_run <parametersFile.txt> <output directory>
 *
 * It is what a maintainer's MCnptColloid.c main becomes once
 * attempt_monte_carlo_move's loop is replaced (the C binding shown in
 * INTEGRATION.md), written out in full so that the header is compiled and
 * driven from C.  One sweep is num_particles attempts, where a reference cycle
 * is one attempt, so intervals given in cycles become ceil(interval / N)
 * sweeps (at least 1), and the run lasts total_mc_sweeps sweeps (or
 * ceil(total_mc_cycles / N) when that key is 0).  Files and intervals follow
 * the Python driver run_simulation (mc.py) line for line, so both write the
 * same bytes:
 *   start        initial_configuration_type 0: <dir>/fortSphere.1
 *                (read_initial_configuration; exact with its sidecar),
 *                2: the lattice (get_initial_config);
 *   every configuration_save_interval
 *                a status line on stdout (print_intermedio), a snapshot
 *                appended to Configuraciones.dat (print_Trayectoria) and
 *                fortSphere.1 rewritten (backup_restart_file);
 *   every statistics_print_interval
 *                P2 and running averages of E/N, rho and P2
 *                (compute_liquid_crystal_order_parameters,
 *                update_running_averages);
 *   at the end   qmga_mcnvtGB.cnf (print_Qmga), Histograma_Movimientos.dat
 *                (accepted moves per particle id) and fortSphere.1.
 * Every library call's status is checked; a failure prints the library's
 * message and exits 1 (the reference's exit(1)).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lcmc.h"

static lcmc_ctx *g_ctx = NULL;

static void check(int rc, const char *what)
{
    if (rc == LCMC_OK) return;
    char msg[512];
    lcmc_last_error(g_ctx, msg, sizeof(msg));
    fprintf(stderr, "lcmc_run: %s: %s (%s)\n", what, lcmc_strerror(rc), msg);
    if (g_ctx) lcmc_destroy(g_ctx);
    exit(1);
}

static void path_in(char *buf, size_t len, const char *dir, const char *name)
{
    snprintf(buf, len, "%s/%s", dir, name);
}

static int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: lcmc_run <parametersFile.txt> <output directory>\n");
        return 2;
    }
    const char *dir = argv[2];
    char path[4096];
    lcmc_params prm;
    check(lcmc_params_defaults(&prm), "lcmc_params_defaults");
    check(lcmc_params_load(argv[1], &prm), "lcmc_params_load"); /* load_initial_conditions */
    const int n = prm.num_particles;
    const int sweeps = prm.total_mc_sweeps > 0 ? prm.total_mc_sweeps : ceil_div(prm.total_mc_cycles, n);
    int save_every = ceil_div(prm.configuration_save_interval, n);
    int stats_every = ceil_div(prm.statistics_print_interval, n);
    if (save_every < 1) save_every = 1;
    if (stats_every < 1) stats_every = 1;

    check(lcmc_create(&prm, &g_ctx), "lcmc_create");
    if (prm.initial_configuration_type == 0) {
        path_in(path, sizeof(path), dir, "fortSphere.1");
        check(lcmc_load_restart(g_ctx, 0, path), "lcmc_load_restart");
    } else if (prm.initial_configuration_type == 2) {
        check(lcmc_init_config(g_ctx, 0), "lcmc_init_config");
    } else {
        check(LCMC_EPARAM, "initial_configuration_type 1 (random placement) is not provided");
    }

    double *x = malloc(sizeof(double) * 6 * (size_t)n);
    long long *hist = calloc((size_t)n, sizeof(long long));
    unsigned char *out = malloc((size_t)n);
    if (!x || !hist || !out) check(LCMC_ENOMEM, "host allocation");
    double *px = x, *py = x + n, *pz = x + 2 * (size_t)n, *ox = x + 3 * (size_t)n, *oy = x + 4 * (size_t)n,
           *oz = x + 5 * (size_t)n;
    double box[3];
    double avgE = 0.0, avgRho = 0.0, avgP2 = 0.0, P2 = 0.0;
    int navg = 0, first = 1;
    lcmc_stats st;
    for (int sweep = 1; sweep <= sweeps; sweep++) {
        check(lcmc_sweep(g_ctx, 1), "lcmc_sweep");
        check(lcmc_last_outcomes(g_ctx, 0, out, n), "lcmc_last_outcomes");
        for (int i = 0; i < n; i++) hist[i] += out[i] == 1;
        if (sweep % stats_every == 0) {
            double Q[6], dir3[3];
            check(lcmc_get_stats(g_ctx, 0, &st), "lcmc_get_stats");
            check(lcmc_order_parameter(g_ctx, 0, Q, &P2, dir3), "lcmc_order_parameter");
            const double V = st.box[0] * st.box[1] * st.box[2];
            avgE += st.energy / n;
            avgRho += n / V;
            avgP2 += P2;
            navg++;
        }
        if (sweep % save_every == 0) {
            check(lcmc_get_stats(g_ctx, 0, &st), "lcmc_get_stats");
            const int k = navg > 0 ? navg : 1;
            printf("sweep %d: E/N %.6f <E/N> %.6f P2 %.4f <P2> %.4f <rho> %.5f acceptance %.4f\n", sweep, st.energy / n,
                   avgE / k, P2, avgP2 / k, avgRho / k, (double)st.accepted / (double)(st.attempted > 0 ? st.attempted : 1));
            check(lcmc_download(g_ctx, 0, px, py, pz, ox, oy, oz, n, box), "lcmc_download");
            path_in(path, sizeof(path), dir, "Configuraciones.dat");
            check(lcmc_write_trajectory(path, !first, n, px, py, pz, ox, oy, oz, box), "lcmc_write_trajectory");
            first = 0;
            path_in(path, sizeof(path), dir, "fortSphere.1");
            check(lcmc_save_restart(g_ctx, 0, path), "lcmc_save_restart");
        }
    }
    check(lcmc_download(g_ctx, 0, px, py, pz, ox, oy, oz, n, box), "lcmc_download");
    path_in(path, sizeof(path), dir, "qmga_mcnvtGB.cnf");
    check(lcmc_write_qmga(path, 0, n, px, py, pz, ox, oy, oz, box), "lcmc_write_qmga");
    path_in(path, sizeof(path), dir, "Histograma_Movimientos.dat");
    FILE *f = fopen(path, "w");
    if (!f) check(LCMC_ENOFILE, "Histograma_Movimientos.dat");
    for (int i = 0; i < n; i++) fprintf(f, "%d       %lld\n", i, hist[i]);
    fclose(f);
    path_in(path, sizeof(path), dir, "fortSphere.1");
    check(lcmc_save_restart(g_ctx, 0, path), "lcmc_save_restart");
    check(lcmc_get_stats(g_ctx, 0, &st), "lcmc_get_stats");
    const int k = navg > 0 ? navg : 1;
    printf("done: %d sweeps, <E/N> %.6f <rho> %.5f <P2> %.4f\n", sweeps, avgE / k, avgRho / k, avgP2 / k);
    free(x);
    free(hist);
    free(out);
    const int rc = lcmc_destroy(g_ctx);
    g_ctx = NULL;
    check(rc, "lcmc_destroy");
    return 0;
}
