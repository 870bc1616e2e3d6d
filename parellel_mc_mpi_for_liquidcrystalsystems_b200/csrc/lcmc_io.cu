// lcmc_io.cu - the reference's configuration files (host code) and an exact
// restart of a context.
//
// Text formats, byte for byte as the reference writes them:
//   fortSphere.1         esc_fort1 / backup_restart_file (MCnptColloid.c:3193-3230):
//                        "%d %15.8lf x4\n" header (N, box, colloid radius), then per
//                        particle four lines of three "%15.8lf": position, zeros,
//                        orientation, zeros; read back as read_initial_configuration
//                        (2786-2831) reads it
//   Configuraciones.dat  print_Trayectoria (3081-3107): N, box, then one line of six
//                        "%5.7lf" separated by " \t " per particle; append = option 1
//   qmga_mcnvtGB.cnf     print_Qmga (3110-3158): N, box (three lines), "0 0", then
//                        twelve "%15.8lf" per particle (position relative to the box
//                        centre, zeros, orientation, zeros) and " 0 0"
// The text keeps 8 decimals; lcmc_save_restart adds a binary sidecar
// (<path>.lcmc) with the exact FP64 state, box, running energy and the sweep
// counter of the counter-based random streams, so a run resumed from it makes
// exactly the decisions the uninterrupted run makes.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lcmc.h"

namespace {

int write_fort1_file(const char *path, int n, const double *px, const double *py, const double *pz, const double *ox,
                     const double *oy, const double *oz, const double box[3], double colloid_radius)
{
    FILE *f = fopen(path, "w");
    if (!f) return LCMC_ENOFILE;
    fprintf(f, "%d %15.8lf %15.8lf %15.8lf %15.8lf\n", n, box[0], box[1], box[2], colloid_radius);
    for (int i = 0; i < n; i++) {
        fprintf(f, "%15.8lf %15.8lf %15.8lf\n", px[i], py[i], pz[i]);
        fprintf(f, "%15.8lf %15.8lf %15.8lf\n", 0.0, 0.0, 0.0);
        fprintf(f, "%15.8lf %15.8lf %15.8lf\n", ox[i], oy[i], oz[i]);
        fprintf(f, "%15.8lf %15.8lf %15.8lf\n", 0.0, 0.0, 0.0);
    }
    return fclose(f) == 0 ? LCMC_OK : LCMC_ENOFILE;
}

const char SIDE_MAGIC[8] = {'L', 'C', 'M', 'C', 'R', 'S', 'T', '1'};

} // namespace

extern "C" int lcmc_write_fort1(const char *path, int n, const double *px, const double *py, const double *pz,
                                const double *ox, const double *oy, const double *oz, const double box[3],
                                double colloid_radius)
{
    if (!path || n < 0 || (n > 0 && (!px || !py || !pz || !ox || !oy || !oz)) || !box) return LCMC_EINVAL;
    return write_fort1_file(path, n, px, py, pz, ox, oy, oz, box, colloid_radius);
}

extern "C" int lcmc_read_fort1(const char *path, int n_max, double *px, double *py, double *pz, double *ox,
                               double *oy, double *oz, double box[3], double *colloid_radius, int *n_read)
{
    if (!path || n_max < 0 || !box || !colloid_radius || !n_read) return LCMC_EINVAL;
    FILE *f = fopen(path, "r");
    if (!f) return LCMC_ENOFILE;
    int n = 0;
    if (fscanf(f, "%d %lf %lf %lf %lf", &n, &box[0], &box[1], &box[2], colloid_radius) != 5 || n < 0) {
        fclose(f);
        return LCMC_EPARAM;
    }
    *n_read = n;
    if (n > n_max) { // the reference reads the first num_particles of a larger file
        n = n_max;
    }
    double z;
    for (int i = 0; i < n; i++) {
        int got = fscanf(f, "%lf %lf %lf", &px[i], &py[i], &pz[i]);
        got += fscanf(f, "%lf %lf %lf", &z, &z, &z);
        got += fscanf(f, "%lf %lf %lf", &ox[i], &oy[i], &oz[i]);
        got += fscanf(f, "%lf %lf %lf", &z, &z, &z);
        if (got != 12) {
            fclose(f);
            return LCMC_EPARAM;
        }
    }
    fclose(f);
    return LCMC_OK;
}

extern "C" int lcmc_write_trajectory(const char *path, int append, int n, const double *px, const double *py,
                                     const double *pz, const double *ox, const double *oy, const double *oz,
                                     const double box[3])
{
    if (!path || n < 0 || !box) return LCMC_EINVAL;
    FILE *f = fopen(path, append ? "a" : "w");
    if (!f) return LCMC_ENOFILE;
    fprintf(f, "%d \n", n);
    fprintf(f, "%3.5lf %3.5lf %3.5lf \n", box[0], box[1], box[2]);
    for (int i = 0; i < n; i++)
        fprintf(f, "%5.7lf \t %5.7lf \t %5.7lf \t %5.7lf \t %5.7lf \t %5.7lf \n", px[i], py[i], pz[i], ox[i], oy[i],
                oz[i]);
    return fclose(f) == 0 ? LCMC_OK : LCMC_ENOFILE;
}

extern "C" int lcmc_write_qmga(const char *path, int append, int n, const double *px, const double *py,
                               const double *pz, const double *ox, const double *oy, const double *oz,
                               const double box[3])
{
    if (!path || n < 0 || !box) return LCMC_EINVAL;
    FILE *f = fopen(path, append ? "a" : "w");
    if (!f) return LCMC_ENOFILE;
    fprintf(f, "%d\n", n);
    fprintf(f, "%lf\n", box[0]);
    fprintf(f, "%lf\n", box[1]);
    fprintf(f, "%lf\n", box[2]);
    fprintf(f, "%lf %lf\n", 0.0, 0.0);
    // the reference's format string continues its lines with backslashes, so
    // each record carries the source's indentation between groups of three
    const std::string gaps(35, ' ');
    const char *gap = gaps.c_str();
    for (int i = 0; i < n; i++) {
        fprintf(f, "%15.8lf %15.8lf %15.8lf %s%15.8lf %15.8lf %15.8lf %s%15.8lf %15.8lf %15.8lf %s%15.8lf %15.8lf "
                   "%15.8lf 0 0\n",
                px[i] - 0.5 * box[0], py[i] - 0.5 * box[1], pz[i] - 0.5 * box[2], gap, 0.0, 0.0, 0.0, gap, ox[i],
                oy[i], oz[i], gap, 0.0, 0.0, 0.0);
    }
    return fclose(f) == 0 ? LCMC_OK : LCMC_ENOFILE;
}

// ---------------------------------------------------------------------------
// exact restart of one replica of a context
// ---------------------------------------------------------------------------
extern "C" int lcmc_save_restart(lcmc_ctx *ctx, int replica, const char *path)
{
    if (!ctx || !path) return LCMC_EINVAL;
    lcmc_stats st;
    int rc = lcmc_get_stats(ctx, replica, &st);
    if (rc) return rc;
    lcmc_params p;
    rc = lcmc_get_params(ctx, replica, &p);
    if (rc) return rc;
    const int n = p.num_particles;
    std::vector<double> a((size_t)6 * n);
    double box[3];
    rc = lcmc_download(ctx, replica, &a[0], &a[n], &a[2 * (size_t)n], &a[3 * (size_t)n], &a[4 * (size_t)n],
                       &a[5 * (size_t)n], n, box);
    if (rc) return rc;
    rc = write_fort1_file(path, n, &a[0], &a[n], &a[2 * (size_t)n], &a[3 * (size_t)n], &a[4 * (size_t)n],
                          &a[5 * (size_t)n], box, p.colloid_radius);
    if (rc) return rc;
    const std::string side = std::string(path) + ".lcmc";
    FILE *f = fopen(side.c_str(), "wb");
    if (!f) return LCMC_ENOFILE;
    const int64_t n64 = n, sweep = st.sweeps;
    const uint64_t seed = p.rng_seed;
    bool ok = fwrite(SIDE_MAGIC, 1, 8, f) == 8 && fwrite(&n64, 8, 1, f) == 1 && fwrite(&sweep, 8, 1, f) == 1 &&
              fwrite(&seed, 8, 1, f) == 1 && fwrite(&st.energy, 8, 1, f) == 1 && fwrite(box, 8, 3, f) == 3 &&
              fwrite(a.data(), 8, a.size(), f) == a.size();
    ok = (fclose(f) == 0) && ok;
    return ok ? LCMC_OK : LCMC_ENOFILE;
}

extern "C" int lcmc_load_restart(lcmc_ctx *ctx, int replica, const char *path)
{
    if (!ctx || !path) return LCMC_EINVAL;
    lcmc_params p;
    int rc = lcmc_get_params(ctx, replica, &p);
    if (rc) return rc;
    const int n = p.num_particles;
    std::vector<double> a((size_t)6 * n);
    double box[3], R = 0.0;
    const std::string side = std::string(path) + ".lcmc";
    FILE *f = fopen(side.c_str(), "rb");
    if (f) { // exact state and the position of the random streams
        char magic[8];
        int64_t n64 = 0, sweep = 0;
        uint64_t seed = 0;
        double energy = 0.0;
        bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, SIDE_MAGIC, 8) == 0 && fread(&n64, 8, 1, f) == 1 &&
                  n64 == n && fread(&sweep, 8, 1, f) == 1 && fread(&seed, 8, 1, f) == 1 &&
                  fread(&energy, 8, 1, f) == 1 && fread(box, 8, 3, f) == 3 && fread(a.data(), 8, a.size(), f) == a.size();
        fclose(f);
        if (!ok) return LCMC_EPARAM;
        if (seed != p.rng_seed) return LCMC_EPARAM; // the streams would differ
        rc = lcmc_upload_with_energy(ctx, replica, &a[0], &a[n], &a[2 * (size_t)n], &a[3 * (size_t)n],
                                     &a[4 * (size_t)n], &a[5 * (size_t)n], n, box, energy);
        if (rc) return rc;
        return lcmc_set_sweep_counter(ctx, replica, sweep);
    }
    int n_read = 0;
    rc = lcmc_read_fort1(path, n, &a[0], &a[n], &a[2 * (size_t)n], &a[3 * (size_t)n], &a[4 * (size_t)n],
                         &a[5 * (size_t)n], box, &R, &n_read);
    if (rc) return rc;
    if (n_read < n) return LCMC_EPARAM; // fewer particles than num_particles
    return lcmc_upload(ctx, replica, &a[0], &a[n], &a[2 * (size_t)n], &a[3 * (size_t)n], &a[4 * (size_t)n],
                       &a[5 * (size_t)n], n, box);
}
