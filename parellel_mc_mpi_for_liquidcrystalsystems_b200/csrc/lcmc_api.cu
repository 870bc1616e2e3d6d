// lcmc_api.cu - host side of liblcmc.so: the C ABI declared in include/lcmc.h.
//
// Owns the device buffers of a batch of replicas, enqueues the per-sweep
// kernels (rebin, 8 colour phases, optional volume move, finalize) on one
// stream and replays them as CUDA graphs (one per buffer parity).
#include <cuda_runtime.h>

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/lcmc.h"
#include "lcmc_internal.h"
#include "lcmc_launch.h"
#include "lcmc_rng.cuh"

using namespace lcmc;

static thread_local std::string g_create_error;

constexpr int kMaxGroups = 8;
constexpr int kGroups = 2; // replica groups of a batch of 8 or more replicas (2, 4 and 8 timed alike)

struct lcmc_ctx {
    int R = 0;
    int ntot = 0, ctot = 0;
    std::vector<lcmc_params> params;
    std::vector<Replica> rep; // host copy of the static part
    cudaStream_t stream = nullptr;
    int device = 0, sms = 148;
    // device buffers
    Replica *d_rep = nullptr;
    DevStats *d_stats = nullptr;
    int *d_act_off = nullptr, *d_p2r = nullptr;
    double *d_x[2][6] = {{nullptr}};
    int *d_id[2] = {nullptr, nullptr};
    int *d_cid = nullptr, *d_rank = nullptr, *d_perm = nullptr, *d_scid = nullptr;
    int *d_cell_count = nullptr, *d_cell_start = nullptr, *d_block_sums = nullptr, *d_flag = nullptr;
    double *d_cell_e0 = nullptr, *d_cell_e1 = nullptr;
    int *d_cell_n0 = nullptr, *d_cell_n1 = nullptr;
    unsigned long long *d_cell_pairs = nullptr, *d_cell_cands = nullptr;
    double *d_cell_abs = nullptr;
    int *d_cell_fp64 = nullptr;
    int *d_p2c = nullptr, *d_resc_count = nullptr, *d_resc_list = nullptr;
    int nphase = 8; // colour phases per sweep (LCMC_MAX_COLOURS with a fine-grid replica)
    // Replica groups of a batch: the colour phases of each group run on their
    // own stream (a branch of the sweep graph between the rebin and the
    // statistics), so the phases of different groups overlap instead of all
    // replicas waiting for the slowest cell of every phase.
    int ngroup = 1;
    int grp_lo[kMaxGroups] = {}, grp_hi[kMaxGroups] = {};
    cudaStream_t side[kMaxGroups] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kMaxGroups] = {};
    unsigned char *d_outcome = nullptr;
    double *d_rec_dE = nullptr, *d_rec_lu = nullptr; // move records (lcmc_record_moves)
    std::vector<unsigned long long> sweeps; // host mirror of every replica's sweep counter
    double *d_pe0 = nullptr, *d_pe1 = nullptr;
    int *d_phard = nullptr;
    double *d_red = nullptr;
    double *d_red_part = nullptr; // chunk partial sums
    int red_nchunk = 1;
    double *d_trial_d[8] = {nullptr}; // tnx tny tnz tux tuy tuz tdU tlu
    float *d_trial_f[3] = {nullptr};  // tdx tdy tdz
    unsigned char *d_thard = nullptr;
    float4 *d_cl4 = nullptr;
    float2 *d_cl2 = nullptr;
    // surrogate, recordings
    unsigned long long *d_feat_acc = nullptr;
    float *d_feat_f = nullptr;
    int rec_cap = 0;
    int *d_rec_count = nullptr;
    float *d_rec_x = nullptr, *d_rec_y = nullptr;
    int hist_cap = 0;
    double *d_hist = nullptr;
    lcmc_mlp *mlp = nullptr;
    bool any_da = false;     // an NPT replica uses the learned surrogate
    bool any_screen = false; // an NPT replica uses the FP32-pair screen
    int cur = 0;
    bool uploaded_all = false;
    std::vector<char> uploaded;
    // kernels
    int kernel_override = -1;
    int fast_variant = 0;
    int need_amax = 0; // active-cell capacity the capacity rule asks for
    int need_min = 0;  // the smallest capacity lcmc_autotune may try: mean + 3 standard deviations of a cell's count
    int tuned_class = -1; // capacity class lcmc_autotune chose (kept while it holds the rule's capacity)
    bool checks_off = false; // no periodic energy checks (autotune trials)
    int grid_elem = 0, grid_exact = 0, grid_fast = 0, grid_energy = 0, grid_screen = 0;
    bool any_fast = false, any_exact = false, any_npt = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool timed = false;
    std::string err;
};

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

static int set_err(lcmc_ctx *c, int code, const char *msg)
{
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

#define CUDA_TRY(ctx, call)                                                                                           \
    do {                                                                                                              \
        cudaError_t e_ = (call);                                                                                      \
        if (e_ != cudaSuccess) {                                                                                      \
            char b_[256];                                                                                             \
            snprintf(b_, sizeof(b_), "%s: %s", #call, cudaGetErrorString(e_));                                        \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? LCMC_ENOMEM : LCMC_ECUDA, b_);                      \
        }                                                                                                             \
    } while (0)

extern "C" const char *lcmc_strerror(int code)
{
    switch (code) {
    case LCMC_OK: return "ok";
    case LCMC_EINVAL: return "invalid argument";
    case LCMC_ENOFILE: return "file cannot be opened";
    case LCMC_EPARAM: return "missing or unparsable parameter";
    case LCMC_ECUDA: return "CUDA error";
    case LCMC_ENOMEM: return "out of memory";
    case LCMC_ECELLCAP: return "cell or stencil above kernel capacity";
    case LCMC_ENUMERIC: return "non-finite energy";
    case LCMC_EBOX: return "box too small for the cutoff";
    case LCMC_ENODEV: return "no CUDA device";
    case LCMC_EOVERLAP: return "particle inside the colloid";
    case LCMC_ETIMEOUT: return "bounded wait gave up";
    case LCMC_EDRIFT: return "running energy out of tolerance at an FP64 energy check";
    default: return "unknown error";
    }
}

extern "C" int lcmc_last_error(const lcmc_ctx *ctx, char *buf, size_t len)
{
    if (!buf || len == 0) return LCMC_EINVAL;
    const std::string &s = ctx ? ctx->err : g_create_error;
    snprintf(buf, len, "%s", s.c_str());
    return LCMC_OK;
}

extern "C" int lcmc_abi_version(void) { return LCMC_ABI_VERSION; }

// ---------------------------------------------------------------------------
// parameters (load_initial_conditions, MCnptColloid.c:3933-4133)
// ---------------------------------------------------------------------------

static const char *kRefKeys[23] = {
    "mc_ensemble_type", "num_particles", "system_density", "system_temperature", "system_pressure",
    "gb_sigma_sidetoside", "gb_epsilon0", "gb_kappa", "gb_kappa_prime", "gb_mu_exponent", "gb_nu_exponent",
    "max_displacement", "max_rotation", "initial_configuration_type", "cutoff_radius", "verlet_radius",
    "total_mc_cycles", "configuration_save_interval", "statistics_print_interval", "colloid_wall_option",
    "colloid_interaction_epsilon", "colloid_interaction_amplitude", "colloid_radius"};

extern "C" int lcmc_params_defaults(lcmc_params *p)
{
    if (!p) return LCMC_EINVAL;
    memset(p, 0, sizeof(*p));
    p->mc_ensemble_type = LCMC_NVT;
    p->num_particles = 1000;
    p->system_density = 0.30;
    p->system_temperature = 1.0;
    p->system_pressure = 2.0;
    p->gb_sigma_sidetoside = 1.0;
    p->gb_epsilon0 = 1.0;
    p->gb_kappa = 3.0;
    p->gb_kappa_prime = 5.0;
    p->gb_mu_exponent = 2.0;
    p->gb_nu_exponent = 1.0;
    p->max_displacement = 0.1f;
    p->max_rotation = 0.1f;
    p->initial_configuration_type = 2;
    p->cutoff_radius = 4.0;
    p->verlet_radius = 4.8;
    p->total_mc_cycles = 1000;
    p->configuration_save_interval = 100;
    p->statistics_print_interval = 100;
    p->colloid_wall_option = 0;
    p->colloid_interaction_epsilon = 15.0;
    p->colloid_interaction_amplitude = 1.5;
    p->colloid_radius = 0.0;
    p->rng_seed = 12345u;
    p->total_mc_sweeps = 0;
    p->cell_capacity = 0;
    p->npt_max_dlnV = 0.01;
    p->volume_moves_per_sweep = 1;
    p->precision_mode = LCMC_PREC_FP32;
    p->init_orientation_cone_deg = 180.0;
    return LCMC_OK;
}

extern "C" int lcmc_params_load(const char *path, lcmc_params *p)
{
    if (!path || !p) return LCMC_EINVAL;
    FILE *f = fopen(path, "r");
    if (!f) return set_err(nullptr, LCMC_ENOFILE, "cannot open parameter file");
    char line[256], name[256], value[256];
    int seen[23] = {0};
    // read_next_parameter grammar (MCnptColloid.c:3894-3910)
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '\n' || line[0] == '#' || line[0] == '\0') continue;
        value[0] = '\0';
        if (sscanf(line, "%255s %255[^\n]", name, value) < 1) continue;
        int k = -1;
        for (int i = 0; i < 23; i++)
            if (strcmp(name, kRefKeys[i]) == 0) k = i;
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
                unsigned long long s = 0;
                ok = sscanf(value, "%llu", &s);
                p->rng_seed = s;
            } else if (strcmp(name, "total_mc_sweeps") == 0) ok = sscanf(value, "%d", &p->total_mc_sweeps);
            else if (strcmp(name, "cell_capacity") == 0) ok = sscanf(value, "%d", &p->cell_capacity);
            else if (strcmp(name, "npt_max_dlnV") == 0) ok = sscanf(value, "%lf", &p->npt_max_dlnV);
            else if (strcmp(name, "volume_moves_per_sweep") == 0) ok = sscanf(value, "%d", &p->volume_moves_per_sweep);
            else if (strcmp(name, "precision_mode") == 0) {
                if (strncmp(value, "fp32", 4) == 0) p->precision_mode = LCMC_PREC_FP32;
                else if (strncmp(value, "fp64", 4) == 0) p->precision_mode = LCMC_PREC_FP64;
                else ok = sscanf(value, "%d", &p->precision_mode);
            } else if (strcmp(name, "init_orientation_cone_deg") == 0)
                ok = sscanf(value, "%lf", &p->init_orientation_cone_deg);
            else if (strcmp(name, "energy_check_interval") == 0) ok = sscanf(value, "%d", &p->energy_check_interval);
            else if (strcmp(name, "energy_check_tolerance") == 0)
                ok = sscanf(value, "%lf", &p->energy_check_tolerance);
            else if (strcmp(name, "init_lattice") == 0) ok = sscanf(value, "%d", &p->init_lattice);
            else if (strcmp(name, "cell_grid") == 0) ok = sscanf(value, "%d", &p->cell_grid);
            break; // other keys: ignored, as the reference only warns (MCnptColloid.c:4093)
        }
        if (ok != 1) {
            fclose(f);
            char b[300];
            snprintf(b, sizeof(b), "cannot parse value of '%s'", name);
            return set_err(nullptr, LCMC_EPARAM, b);
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
    if (p->n_read != 23) return set_err(nullptr, LCMC_EPARAM, "not all 23 parameters were read");
    return LCMC_OK;
}

// get_system_const (MCnptColloid.c:2752-2783) with chi after kappa^2.
static void make_consts(const lcmc_params &p, GBConsts &k)
{
    memset(&k, 0, sizeof(k));
    k.beta = 1.0 / p.system_temperature;
    k.four_eps0 = 4.0 * p.gb_epsilon0;
    k.rc = p.cutoff_radius;
    k.rc2 = p.cutoff_radius * p.cutoff_radius;
    k.sigma0 = p.gb_sigma_sidetoside;
    double sigma_ee = p.gb_sigma_sidetoside * p.gb_kappa;
    double k_imu = pow(p.gb_kappa_prime, 1.0 / p.gb_mu_exponent);
    double kappa_sq = p.gb_kappa * p.gb_kappa;
    k.chi = (kappa_sq - 1.0) / (kappa_sq + 1.0);
    k.chi_sq = k.chi * k.chi;
    k.chi_prime = (k_imu - 1.0) / (k_imu + 1.0);
    k.mu = p.gb_mu_exponent;
    k.nu = p.gb_nu_exponent;
    k.kappa_prime = p.gb_kappa_prime;
    k.coll_R = p.colloid_radius;
    k.coll_cutoff = 4.0 * sigma_ee;
    k.coll_on = p.colloid_wall_option == 1;
    k.max_disp = (double)p.max_displacement;
    k.max_rot = (double)p.max_rotation;
    k.mu_code = p.gb_mu_exponent == 1.0 ? 1 : (p.gb_mu_exponent == 2.0 ? 2 : 0);
    k.nu_code = p.gb_nu_exponent == 1.0 ? 1 : (p.gb_nu_exponent == 2.0 ? 2 : 0);
    k.f_rc2 = (float)k.rc2;
    k.f_chi = (float)k.chi;
    k.f_chi_sq = (float)k.chi_sq;
    k.f_chip = (float)k.chi_prime;
    k.f_chip_sq = (float)(k.chi_prime * k.chi_prime);
    k.f_sigma0 = (float)k.sigma0;
    k.f_4eps0 = (float)k.four_eps0;
    k.f_half_chi = (float)(0.5 * k.chi);
    k.f_half_chip = (float)(0.5 * k.chi_prime);
    // 25 (4 eps0) = 100 eps0: an FP32 term of that size has a rounding error
    // of at most ~0.02 eps0 (1.9e-4 relative); larger terms (overlaps) are
    // evaluated in FP64
    k.f_big = (float)(25.0 * k.four_eps0);
}

static double min_cell_width(const lcmc_params &p)
{
    double w = p.cutoff_radius + (double)p.max_displacement;
    if (p.mc_ensemble_type == LCMC_NPT) w *= 1.0 + p.npt_max_dlnV;
    return w;
}

static int grid_dim_host(double L, double wmin, bool fine)
{
    int m = (int)floor(L / wmin);
    return m >= 2 ? ((fine && m >= 3) ? m : m - (m & 1)) : 1;
}

// ---------------------------------------------------------------------------
// initial configuration (initialize_cubic_lattice_positions, MCnptColloid.c:2920-3033)
// ---------------------------------------------------------------------------

static double box_length(const lcmc_params &p)
{
    const double pi = 3.1415926535898; // MCnptColloid.c:10
    double vcol = (4. / 3.) * pi * pow(p.colloid_radius, 3);
    double V = (p.num_particles / p.system_density) + vcol; // MCnptColloid.c:2935
    return pow(V, 1.0 / 3.0);
}

// Box V = N/rho + V_colloid; smallest n_s^3 lattice whose sites outside the
// colloid hold N; spacing L/n_s without the reference's clamp to sigma_ee
// (MCnptColloid.c:2957-2963 pushes sites outside the box when dense); sites
// with |r - C|^2 <= R^2 skipped when R > 0; orientations uniform on the sphere
// (Marsaglia, seeded) or uniform on the cap within init_orientation_cone_deg
// of +z.
extern "C" int lcmc_lattice(const lcmc_params *pp, int replica, double *px, double *py, double *pz, double *ox,
                            double *oy, double *oz, double box[3])
{
    if (!pp || !px || !py || !pz || !ox || !oy || !oz || !box) return LCMC_EINVAL;
    const lcmc_params &p = *pp;
    const double pi = 3.1415926535898;
    const int n = p.num_particles;
    if (n <= 0 || p.system_density <= 0.0) return LCMC_EINVAL;
    const double R = p.colloid_radius;
    const double L = box_length(p);
    box[0] = box[1] = box[2] = L;
    const double C = 0.5 * L;
    auto inside = [&](double x, double y, double z) {
        double d[3] = {C - x, C - y, C - z};
        for (int a = 0; a < 3; a++) {
            if (d[a] > 0.5 * L) d[a] -= L;
            else if (d[a] < -0.5 * L) d[a] += L;
        }
        double xs = d[0] * d[0], ys = d[1] * d[1], zs = d[2] * d[2];
        double r2 = xs + ys + zs;
        return R > 0.0 && r2 <= R * R;
    };
    uint32_t key[2];
    if (p.init_lattice == 1) {
        // body-centred tetragonal: layers c = L / floor(L / (1.05 sigma_ee)) apart
        // along z, square sites a = L / n_a apart in x, y, the second site of
        // each cell at (a/2, a/2, c/2); the smallest n_a whose sites outside
        // the colloid hold N, and the surplus sites left empty evenly over the
        // site order (site s is kept when floor((s+1) N / S) > floor(s N / S))
        const double cz = 1.05 * p.gb_sigma_sidetoside * p.gb_kappa;
        const long long nz = std::max(1LL, (long long)floor(L / cz));
        const double c = L / (double)nz;
        auto site = [&](long long s, long long na, double *x, double *y, double *z) {
            const double a = L / (double)na;
            const long long b = s & 1, q = s >> 1;
            const long long ix = q % na, iy = (q / na) % na, iz = q / (na * na);
            *x = ((double)ix + 0.5 * (double)b) * a;
            *y = ((double)iy + 0.5 * (double)b) * a;
            *z = ((double)iz + 0.5 * (double)b) * c;
        };
        long long na = 1;
        std::vector<long long> freeidx;
        for (;; na++) {
            freeidx.clear();
            const long long S = 2 * na * na * nz;
            for (long long s = 0; s < S; s++) {
                double x, y, z;
                site(s, na, &x, &y, &z);
                if (!inside(x, y, z)) freeidx.push_back(s);
            }
            if ((long long)freeidx.size() >= n) break;
        }
        const long long F = (long long)freeidx.size();
        int i = 0;
        for (long long f = 0; f < F && i < n; f++) {
            if ((f + 1) * n / F == f * n / F) continue;
            site(freeidx[f], na, &px[i], &py[i], &pz[i]);
            i++;
        }
    } else {
        int ns = 2;
        for (;; ns++) {
            long long free_sites = 0;
            double d = L / (double)ns;
            for (long long s = 0; s < (long long)ns * ns * ns; s++) {
                double x = (double)(s % ns) * d, y = (double)((s / ns) % ns) * d,
                       z = (double)(s / ((long long)ns * ns)) * d;
                if (!inside(x, y, z)) free_sites++;
            }
            if (free_sites >= n) break;
        }
        const double delta = L / (double)ns;
        long long site = 0;
        for (int i = 0; i < n; i++) {
            double x, y, z;
            for (;;) {
                long long ix = site % ns, iy = (site / ns) % ns, iz = site / ((long long)ns * ns);
                site++;
                x = (double)ix * delta;
                y = (double)iy * delta;
                z = (double)iz * delta;
                if (!inside(x, y, z)) break;
            }
            px[i] = x;
            py[i] = y;
            pz[i] = z;
        }
    }
    (void)replica;
    seed_key(p.rng_seed, key);
    const double cone = p.init_orientation_cone_deg;
    const double cmin = cos(cone * (pi / 180.0));
    for (int i = 0; i < n; i++) {
        if (cone >= 180.0) {
            double v[3];
            sphere_point(key, (uint32_t)i, INIT_SWEEP, v);
            ox[i] = v[0];
            oy[i] = v[1];
            oz[i] = v[2];
        } else {
            U4 o = draw(key, (uint32_t)i, INIT_SWEEP, TAG_INIT);
            double ct = 1.0 - u01(o.x) * (1.0 - cmin);
            double st = sqrt(1.0 - ct * ct);
            double ph = 2.0 * pi * u01(o.y);
            ox[i] = st * cos(ph);
            oy[i] = st * sin(ph);
            oz[i] = ct;
        }
    }
    return LCMC_OK;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

static DevView view(const lcmc_ctx *c, int parity)
{
    DevView v;
    memset(&v, 0, sizeof(v));
    v.R = c->R;
    v.ntot = c->ntot;
    v.ctot = c->ctot;
    v.rep = c->d_rep;
    v.stats = c->d_stats;
    v.act_off = c->d_act_off;
    v.p2r = c->d_p2r;
    const int a = parity, b = parity ^ 1;
    v.px = c->d_x[a][0];
    v.py = c->d_x[a][1];
    v.pz = c->d_x[a][2];
    v.ox = c->d_x[a][3];
    v.oy = c->d_x[a][4];
    v.oz = c->d_x[a][5];
    v.id = c->d_id[a];
    v.qx = c->d_x[b][0];
    v.qy = c->d_x[b][1];
    v.qz = c->d_x[b][2];
    v.qux = c->d_x[b][3];
    v.quy = c->d_x[b][4];
    v.quz = c->d_x[b][5];
    v.qid = c->d_id[b];
    v.cid = c->d_cid;
    v.scid = c->d_scid;
    v.rank = c->d_rank;
    v.perm = c->d_perm;
    v.cell_count = c->d_cell_count;
    v.cell_start = c->d_cell_start;
    v.block_sums = c->d_block_sums;
    v.cell_e0 = c->d_cell_e0;
    v.cell_e1 = c->d_cell_e1;
    v.cell_n0 = c->d_cell_n0;
    v.cell_n1 = c->d_cell_n1;
    v.cell_pairs = c->d_cell_pairs;
    v.cell_cands = c->d_cell_cands;
    v.cell_abs = c->d_cell_abs;
    v.cell_fp64 = c->d_cell_fp64;
    v.p2c = c->d_p2c;
    v.resc_count = c->d_resc_count;
    v.nphase = c->nphase;
    v.r_lo = 0;
    v.r_hi = c->R;
    v.ngroup = c->ngroup;
    v.resc_list = c->d_resc_list;
    v.rec_dE = c->d_rec_dE;
    v.rec_lu = c->d_rec_lu;
    v.outcome = c->d_outcome;
    v.scratch_d = c->d_red;
    v.red_part = c->d_red_part;
    v.red_nchunk = c->red_nchunk;
    v.tnx = c->d_trial_d[0];
    v.tny = c->d_trial_d[1];
    v.tnz = c->d_trial_d[2];
    v.tux = c->d_trial_d[3];
    v.tuy = c->d_trial_d[4];
    v.tuz = c->d_trial_d[5];
    v.tdU = c->d_trial_d[6];
    v.tlu = c->d_trial_d[7];
    v.tdx = c->d_trial_f[0];
    v.tdy = c->d_trial_f[1];
    v.tdz = c->d_trial_f[2];
    v.thard = c->d_thard;
    v.cl4 = c->d_cl4;
    v.cl2 = c->d_cl2;
    v.feat_acc = c->d_feat_acc;
    v.feat_f = c->d_feat_f;
    v.rec_cap = c->rec_cap;
    v.rec_count = c->d_rec_count;
    v.rec_x = c->d_rec_x;
    v.rec_y = c->d_rec_y;
    v.hist_cap = c->hist_cap;
    v.hist = c->d_hist;
    return v;
}

static void free_ctx(lcmc_ctx *c)
{
    if (!c) return;
    for (int i = 0; i < 2; i++)
        if (c->graph[i]) cudaGraphExecDestroy(c->graph[i]);
    for (int i = 0; i < 5; i++)
        if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (int g = 0; g < kMaxGroups; g++) {
        if (c->side[g]) cudaStreamDestroy(c->side[g]);
        if (c->ev_join[g]) cudaEventDestroy(c->ev_join[g]);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    void *ptrs[] = {c->d_rep, c->d_stats, c->d_act_off, c->d_p2r, c->d_id[0], c->d_id[1], c->d_cid, c->d_rank,
                    c->d_perm, c->d_scid, c->d_cell_count, c->d_cell_start, c->d_block_sums, c->d_flag, c->d_cell_e0,
                    c->d_cell_e1, c->d_cell_n0, c->d_cell_n1, c->d_cell_pairs, c->d_cell_cands, c->d_outcome,
                    c->d_pe0, c->d_pe1, c->d_phard, c->d_red, c->d_red_part, c->d_cell_abs, c->d_cell_fp64,
                    c->d_rec_dE, c->d_rec_lu, c->d_p2c, c->d_resc_count, c->d_resc_list};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int k = 0; k < 8; k++)
        if (c->d_trial_d[k]) cudaFree(c->d_trial_d[k]);
    for (int k = 0; k < 3; k++)
        if (c->d_trial_f[k]) cudaFree(c->d_trial_f[k]);
    if (c->d_thard) cudaFree(c->d_thard);
    if (c->d_cl4) cudaFree(c->d_cl4);
    if (c->d_cl2) cudaFree(c->d_cl2);
    void *more[] = {c->d_feat_acc, c->d_feat_f, c->d_rec_count, c->d_rec_x, c->d_rec_y, c->d_hist};
    for (void *p : more)
        if (p) cudaFree(p);
    for (int a = 0; a < 2; a++)
        for (int k = 0; k < 6; k++)
            if (c->d_x[a][k]) cudaFree(c->d_x[a][k]);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

template <typename T>
static cudaError_t dalloc(T **p, size_t n)
{
    return cudaMalloc((void **)p, sizeof(T) * (n > 0 ? n : 1));
}

static void invalidate_graphs(lcmc_ctx *c)
{
    for (int i = 0; i < 2; i++)
        if (c->graph[i]) {
            cudaGraphExecDestroy(c->graph[i]);
            c->graph[i] = nullptr;
        }
}

// Active-cell capacity the FP32 kernel needs for a system in a cubic box of
// side L: the caller's cell_capacity when given; else the mean occupancy m
// plus four standard deviations of a cell's count plus 4, with the variance
// m S: S = 1 (Poisson) for a gas (rho* <= 0.15), 0.3 for a dense liquid
// (rho* >= 0.25, whose counts fluctuate far less), linear between.  NPT
// systems, whose box may compress far below its creation volume, take at
// least the middle class.  A cell above the capacity (a lattice start's
// fullest cells, a rare fluctuation) is attempted in FP64 by the hand-over
// kernel.
// mean occupancy of a cell and the standard deviation of its count (variance
// m S: S = 1, Poisson, for a gas, rho* <= 0.15; 0.3 for a dense liquid,
// rho* >= 0.25, whose counts fluctuate far less; linear between)
static void cell_count_stats(const lcmc_params &p, double L, double wmin, double *mean, double *sd)
{
    const int nc = grid_dim_host(L, wmin, p.cell_grid == 1);
    const double rho = p.num_particles / (L * L * L);
    const double wcell = L / (double)nc;
    const double S = rho >= 0.25 ? 0.3 : (rho <= 0.15 ? 1.0 : 1.0 - 0.7 * (rho - 0.15) / 0.10);
    *mean = rho * wcell * wcell * wcell;
    *sd = std::sqrt(*mean * S);
}

static int capacity_rule(const lcmc_params &p, double L, double wmin, bool npt)
{
    if (p.cell_capacity > 0) return p.cell_capacity;
    double mean, sd;
    cell_count_stats(p, L, wmin, &mean, &sd);
    // a cell above the capacity is attempted in FP64 (correct, only slower),
    // so the rule sizes for the liquid, not for the lattice start's fullest
    // cells or rare fluctuations: 4 standard deviations, + 4.  NPT systems
    // get no larger class by default (the classes with more CTAs per SM are
    // the faster ones): a box that compresses far below its creation volume
    // fills its cells beyond the rule, and its over-full cells are attempted
    // in FP64; cell_capacity or lcmc_autotune chooses a larger class
    (void)npt;
    return (int)std::ceil(mean + 4.0 * sd + 4.0);
}

// The smallest capacity the autotuner tries: mean + 3 standard deviations of a
// cell's count (the caller's cell_capacity when given).  A class between this
// and the rule's capacity hands a few more cells to the FP64 kernel per sweep,
// which the timed trials weigh against its higher occupancy.
static int capacity_floor(const lcmc_params &p, double L, double wmin)
{
    if (p.cell_capacity > 0) return p.cell_capacity;
    double mean, sd;
    cell_count_stats(p, L, wmin, &mean, &sd);
    return (int)std::ceil(mean + 3.0 * sd);
}

// the smallest capacity class that holds `want` (else the largest)
static int capacity_class(int want)
{
    int cls = fast_variant_count() - 1;
    for (int v = fast_variant_count() - 1; v >= 0; v--)
        if (fast_variant(v).amax >= want) cls = v;
    return cls;
}

extern "C" int lcmc_cell_capacity(const lcmc_params *p, int *capacity, int *class_capacity)
{
    if (!p || !capacity || !class_capacity || p->num_particles <= 0 || !(p->system_density > 0.0)) return LCMC_EINVAL;
    const double L = box_length(*p);
    *capacity = capacity_rule(*p, L, min_cell_width(*p), p->mc_ensemble_type == LCMC_NPT);
    *class_capacity = fast_variant(capacity_class(*capacity)).amax;
    return LCMC_OK;
}

// Per-replica fields that follow from the kernel choice: the FP32 kernel's
// cell capacity (cells above it are attempted in FP64) and the automatic
// tolerance of the periodic energy check.
static void set_caps(lcmc_ctx *c)
{
    const int amax = fast_variant(c->fast_variant >> 1).amax;
    for (int r = 0; r < c->R; r++) {
        Replica &rp = c->rep[r];
        const lcmc_params &p = c->params[r];
        rp.cap = p.cell_capacity > 0 ? std::min(p.cell_capacity, amax) : amax;
        rp.check_tol = p.energy_check_tolerance > 0.0 ? p.energy_check_tolerance : (rp.kernel == 1 ? 1e-4 : 1e-9);
    }
}

// The fields set_caps and choose_kernels write, into the device table.
static int push_kernel_fields(lcmc_ctx *c)
{
    for (int r = 0; r < c->R; r++) {
        char *base = (char *)c->d_rep + sizeof(Replica) * r;
        const Replica &rp = c->rep[r];
        CUDA_TRY(c, cudaMemcpyAsync(base + offsetof(Replica, kernel), &rp.kernel, sizeof(int), cudaMemcpyHostToDevice,
                                    c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(base + offsetof(Replica, cap), &rp.cap, sizeof(int), cudaMemcpyHostToDevice,
                                    c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(base + offsetof(Replica, check_tol), &rp.check_tol, sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return LCMC_OK;
}

// Kernel selection: FP32 kernel for precision_mode fp32 (boxes with >= 4
// cells per axis; smaller boxes run the FP64 kernel), FP64 kernel otherwise.
static void choose_kernels(lcmc_ctx *c)
{
    c->any_fast = c->any_exact = c->any_npt = false;
    int need_amax = 0, need_min = 0;
    bool spec21 = true; // every system has mu = 2, nu = 1, sigma0 = 1
    for (int r = 0; r < c->R; r++) {
        Replica &rp = c->rep[r];
        const lcmc_params &p = c->params[r];
        int kern = c->kernel_override >= 0 ? c->kernel_override : (p.precision_mode == LCMC_PREC_FP32 ? 1 : 0);
        // an FP32 system whose cells the capacity rule puts above the largest
        // class (wide cells of a small box, or a gas) runs on the FP64 kernel,
        // which has no cell capacity, unless the caller chose the kernel or set
        // cell_capacity
        if (kern == 1 && c->kernel_override < 0 && p.cell_capacity <= 0 &&
            capacity_rule(p, rp.L[0], rp.wmin, rp.ensemble == 2) > fast_variant(fast_variant_count() - 1).amax)
            kern = 0;
        rp.kernel = kern;
        int nc = grid_dim_host(rp.L[0], rp.wmin, rp.fine);
        if (kern == 1) {
            c->any_fast = true;
            if (nc < 6) c->any_exact = true; // NPT boxes near the 4-cell threshold may switch
            const int want = capacity_rule(p, rp.L[0], rp.wmin, rp.ensemble == 2);
            if (want > need_amax) need_amax = want;
            need_min = std::max(need_min, capacity_floor(p, rp.L[0], rp.wmin));
        } else {
            c->any_exact = true;
        }
        if (rp.ensemble == 2) c->any_npt = true;
        spec21 = spec21 && p.gb_mu_exponent == 2.0 && p.gb_nu_exponent == 1.0 && p.gb_sigma_sidetoside == 1.0;
    }
    c->need_amax = need_amax;
    c->need_min = need_min;
    int cls = capacity_class(need_amax);
    if (c->tuned_class >= 0 && fast_variant(c->tuned_class).amax >= need_min) cls = c->tuned_class;
    c->fast_variant = 2 * cls + (spec21 ? 1 : 0);
    set_caps(c);
}

static int upload_replica_table(lcmc_ctx *c)
{
    CUDA_TRY(c, cudaMemcpyAsync(c->d_rep, c->rep.data(), sizeof(Replica) * c->R, cudaMemcpyHostToDevice, c->stream));
    return LCMC_OK;
}

extern "C" int lcmc_create_batch(const lcmc_params *params, int n, lcmc_ctx **out)
{
    if (!params || n <= 0 || !out) return set_err(nullptr, LCMC_EINVAL, "bad arguments");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(nullptr, LCMC_ENODEV, "no CUDA device");
    }
    lcmc_ctx *c = new lcmc_ctx();
    c->R = n;
    c->params.assign(params, params + n);
    c->rep.resize(n);
    c->uploaded.assign(n, 0);
    cudaGetDevice(&c->device);
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    int poff = 0, coff = 0;
    for (int r = 0; r < n; r++) {
        const lcmc_params &p = params[r];
        if (p.num_particles <= 0 || p.system_density <= 0.0 || p.system_temperature <= 0.0 || p.cutoff_radius <= 0.0) {
            free_ctx(c);
            return set_err(nullptr, LCMC_EINVAL, "bad parameters");
        }
        Replica &rp = c->rep[r];
        memset(&rp, 0, sizeof(rp));
        rp.n = p.num_particles;
        rp.p_off = poff;
        rp.ensemble = p.mc_ensemble_type == LCMC_NPT ? 2 : 1;
        rp.pressure = p.system_pressure;
        rp.dlnv_max = rp.ensemble == 2 && p.volume_moves_per_sweep > 0 ? p.npt_max_dlnV : 0.0;
        rp.wmin = min_cell_width(p);
        rp.fine = p.cell_grid == 1 ? 1 : 0;
        if (rp.fine) c->nphase = LCMC_MAX_COLOURS;
        rp.d_cap = (double)p.max_displacement;
        rp.vol_cells = 1;
        rp.min_thick = (double)(float)std::min(p.gb_sigma_sidetoside * p.gb_kappa, p.gb_sigma_sidetoside);
        seed_key(p.rng_seed, rp.key);
        make_consts(p, rp.k);
        rp.check_every = p.energy_check_interval > 0 ? p.energy_check_interval : 0;
        rp.check_tol = p.energy_check_tolerance; // 0: set by choose_kernels from the kernel
        const double L = box_length(p);
        rp.L[0] = rp.L[1] = rp.L[2] = L;
        if (L < 2.0 * p.cutoff_radius) {
            free_ctx(c);
            return set_err(nullptr, LCMC_EBOX, "box shorter than twice the cutoff");
        }
        // cell grid capacity: NVT boxes keep their size; NPT boxes may grow (then cells stay wider)
        double Lmax = rp.ensemble == 2 ? 1.25 * L : L;
        rp.nc_max = grid_dim_host(Lmax, rp.wmin, rp.fine);
        rp.cell_off = coff;
        rp.sweep = 0ull;
        poff += rp.n;
        coff += rp.nc_max * rp.nc_max * rp.nc_max;
    }
    c->ntot = poff;
    c->ctot = coff;
#define ALLOC(ptr, cnt)                                                                                               \
    do {                                                                                                              \
        cudaError_t e_ = dalloc(&(ptr), (size_t)(cnt));                                                               \
        if (e_ != cudaSuccess) {                                                                                      \
            cudaGetLastError();                                                                                       \
            free_ctx(c);                                                                                              \
            return set_err(nullptr, LCMC_ENOMEM, "device allocation failed");                                         \
        }                                                                                                             \
    } while (0)
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        free_ctx(c);
        return set_err(nullptr, LCMC_ECUDA, "stream creation failed");
    }
    for (int i = 0; i < 5; i++)
        if (cudaEventCreate(&c->ev[i]) != cudaSuccess) {
            free_ctx(c);
            return set_err(nullptr, LCMC_ECUDA, "event creation failed");
        }
    // replica groups: batches of 8 or more replicas get kGroups contiguous
    // groups of about equal particle counts (at least two replicas each)
    c->ngroup = n >= 8 ? std::min(kGroups, n / 2) : 1;
    {
        long long total = 0, acc = 0;
        for (int r = 0; r < n; r++) total += params[r].num_particles;
        int g = 0;
        c->grp_lo[0] = 0;
        for (int r = 0; r < n && g < c->ngroup - 1; r++) {
            acc += params[r].num_particles;
            // close group g once it holds its share, leaving a replica for every later group
            if (acc * c->ngroup >= total * (g + 1) && n - (r + 1) >= c->ngroup - (g + 1)) {
                c->grp_hi[g] = r + 1;
                c->grp_lo[++g] = r + 1;
            }
        }
        c->ngroup = g + 1;
        c->grp_hi[g] = n;
    }
    if (c->ngroup > 1) {
        if (cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
            free_ctx(c);
            return set_err(nullptr, LCMC_ECUDA, "event creation failed");
        }
        for (int g = 1; g < c->ngroup; g++)
            if (cudaStreamCreateWithFlags(&c->side[g], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->ev_join[g], cudaEventDisableTiming) != cudaSuccess) {
                free_ctx(c);
                return set_err(nullptr, LCMC_ECUDA, "stream creation failed");
            }
    }
    ALLOC(c->d_rep, n);
    ALLOC(c->d_stats, n);
    ALLOC(c->d_act_off, c->nphase * (n + 1));
    ALLOC(c->d_p2r, c->ntot);
    for (int a = 0; a < 2; a++) {
        for (int k = 0; k < 6; k++) ALLOC(c->d_x[a][k], c->ntot);
        ALLOC(c->d_id[a], c->ntot);
    }
    ALLOC(c->d_cid, c->ntot);
    ALLOC(c->d_rank, c->ntot);
    ALLOC(c->d_perm, c->ntot);
    ALLOC(c->d_scid, c->ntot);
    ALLOC(c->d_cell_count, c->ctot);
    ALLOC(c->d_cell_start, c->ctot + 1);
    ALLOC(c->d_block_sums, 4096);
    ALLOC(c->d_flag, 1);
    ALLOC(c->d_cell_e0, c->ctot);
    ALLOC(c->d_cell_e1, c->ctot);
    ALLOC(c->d_cell_n0, c->ctot);
    ALLOC(c->d_cell_n1, c->ctot);
    ALLOC(c->d_cell_pairs, c->ctot);
    ALLOC(c->d_cell_cands, c->ctot);
    ALLOC(c->d_cell_abs, c->ctot);
    ALLOC(c->d_cell_fp64, c->ctot);
    ALLOC(c->d_p2c, c->ctot);
    ALLOC(c->d_resc_count, c->nphase * c->ngroup);
    ALLOC(c->d_resc_list, (size_t)c->nphase * c->ngroup * c->ctot);
    ALLOC(c->d_outcome, c->ntot);
    ALLOC(c->d_pe0, c->ntot);
    ALLOC(c->d_pe1, c->ntot);
    ALLOC(c->d_phard, c->ntot);
    ALLOC(c->d_red, 16 * n + 16);
    {
        int nmax = 1; // largest count a chunked sum covers: particles or cells of a replica
        for (int r = 0; r < n; r++)
            nmax = std::max(nmax, std::max(params[r].num_particles, c->rep[r].nc_max * c->rep[r].nc_max * c->rep[r].nc_max));
        c->red_nchunk = (nmax + LCMC_RED_CHUNK - 1) / LCMC_RED_CHUNK;
    }
    ALLOC(c->d_red_part, (size_t)n * c->red_nchunk * LCMC_RED_K);
    for (int k = 0; k < 8; k++) ALLOC(c->d_trial_d[k], c->ntot);
    for (int k = 0; k < 3; k++) ALLOC(c->d_trial_f[k], c->ntot);
    ALLOC(c->d_thard, c->ntot);
    ALLOC(c->d_cl4, c->ntot);
    ALLOC(c->d_cl2, c->ntot);
    ALLOC(c->d_feat_acc, (size_t)n * 512 * 7);
    ALLOC(c->d_feat_f, (size_t)n * LCMC_FEAT);
#undef ALLOC
    if ((c->ctot + 4095) / 4096 > 4096) {
        free_ctx(c);
        return set_err(nullptr, LCMC_EINVAL, "cell grid too large");
    }
    std::vector<int> p2r(c->ntot);
    for (int r = 0; r < n; r++)
        for (int i = 0; i < c->rep[r].n; i++) p2r[c->rep[r].p_off + i] = r;
    cudaMemcpy(c->d_p2r, p2r.data(), sizeof(int) * c->ntot, cudaMemcpyHostToDevice);
    std::vector<int> p2c(c->ctot);
    for (int r = 0; r < n; r++)
        for (int i = 0; i < c->rep[r].nc_max * c->rep[r].nc_max * c->rep[r].nc_max; i++) p2c[c->rep[r].cell_off + i] = r;
    cudaMemcpy(c->d_p2c, p2c.data(), sizeof(int) * c->ctot, cudaMemcpyHostToDevice);
    cudaMemset(c->d_resc_count, 0, sizeof(int) * c->nphase * c->ngroup);
    cudaMemset(c->d_stats, 0, sizeof(DevStats) * n);
    cudaMemset(c->d_outcome, 0, c->ntot);
    cudaMemset(c->d_cell_e0, 0, sizeof(double) * c->ctot);
    cudaMemset(c->d_cell_n0, 0, sizeof(int) * c->ctot);
    cudaMemset(c->d_cell_n1, 0, sizeof(int) * c->ctot);
    cudaMemset(c->d_cell_pairs, 0, sizeof(unsigned long long) * c->ctot);
    cudaMemset(c->d_cell_cands, 0, sizeof(unsigned long long) * c->ctot);
    cudaMemset(c->d_cell_abs, 0, sizeof(double) * c->ctot);
    cudaMemset(c->d_cell_fp64, 0, sizeof(int) * c->ctot);
    c->sweeps.assign(n, 0ull);
    choose_kernels(c);
    c->grid_elem = 4 * c->sms;
    c->grid_exact = 4 * c->sms;
    c->grid_energy = energy_exact_blocks_per_sm() * c->sms;
    c->grid_screen = screen_blocks_per_sm() * c->sms;
    c->grid_fast = fast_blocks_per_sm(c->fast_variant) * c->sms;
    rescue_init();
    int rc = upload_replica_table(c);
    if (rc) {
        free_ctx(c);
        return rc;
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        free_ctx(c);
        return set_err(nullptr, LCMC_ECUDA, "initialisation failed");
    }
    *out = c;
    return LCMC_OK;
}

extern "C" int lcmc_create(const lcmc_params *p, lcmc_ctx **out) { return lcmc_create_batch(p, 1, out); }

extern "C" int lcmc_destroy(lcmc_ctx *ctx)
{
    if (!ctx) return LCMC_EINVAL;
    cudaStreamSynchronize(ctx->stream);
    free_ctx(ctx);
    return LCMC_OK;
}

extern "C" int lcmc_num_replicas(const lcmc_ctx *ctx) { return ctx ? ctx->R : 0; }

// Re-run the kernel choice on the replicas' current boxes (read back from the
// device: NPT volume moves change them) and push the fields it sets.
static int rechoose_kernels(lcmc_ctx *c)
{
    std::vector<Replica> dev(c->R);
    CUDA_TRY(c, cudaMemcpyAsync(dev.data(), c->d_rep, sizeof(Replica) * c->R, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (int r = 0; r < c->R; r++)
        for (int a = 0; a < 3; a++) c->rep[r].L[a] = dev[r].L[a];
    const int old_variant = c->fast_variant;
    const bool old_fast = c->any_fast, old_exact = c->any_exact;
    choose_kernels(c);
    int rc = push_kernel_fields(c);
    if (rc) return rc;
    c->grid_fast = fast_blocks_per_sm(c->fast_variant) * c->sms;
    if (old_variant != c->fast_variant || old_fast != c->any_fast || old_exact != c->any_exact) invalidate_graphs(c);
    return LCMC_OK;
}

extern "C" int lcmc_set_kernel(lcmc_ctx *ctx, int kernel)
{
    if (!ctx || kernel < -1 || kernel > 1) return LCMC_EINVAL;
    ctx->kernel_override = kernel;
    int rc = rechoose_kernels(ctx);
    if (rc) return rc;
    invalidate_graphs(ctx);
    return LCMC_OK;
}

// ---------------------------------------------------------------------------
// sweeps
// ---------------------------------------------------------------------------

// Rebin into the other buffer: afterwards the current buffer is cur ^ 1.
static void enqueue_rebin(lcmc_ctx *c, int parity) { launch_rebin(view(c, parity), c->stream, c->grid_elem); }

// One sweep; the event records become event nodes of the captured graph and
// time its parts on the device (lcmc_last_sweep_timing).
static void enqueue_sweep(lcmc_ctx *c, int parity)
{
    // cudaEventRecordExternal: captured as event-record nodes (timestamps), not
    // as internal dependencies
    cudaEventRecordWithFlags(c->ev[0], c->stream, cudaEventRecordExternal);
    enqueue_rebin(c, parity);
    cudaEventRecordWithFlags(c->ev[1], c->stream, cudaEventRecordExternal);
    DevView v = view(c, parity ^ 1);
    if (c->ngroup > 1) cudaEventRecord(c->ev_fork, c->stream);
    for (int g = 0; g < c->ngroup; g++) {
        // group g's phases: its replicas' cells, its own hand-over lists, its own stream
        DevView vg = v;
        vg.r_lo = c->grp_lo[g];
        vg.r_hi = c->grp_hi[g];
        vg.resc_count = c->d_resc_count + (size_t)g * c->nphase;
        vg.resc_list = c->d_resc_list + (size_t)g * c->nphase * c->ctot;
        cudaStream_t sg = g == 0 ? c->stream : c->side[g];
        if (g > 0) cudaStreamWaitEvent(sg, c->ev_fork, 0);
        for (int ci = 0; ci < c->nphase; ci++) {
            if (c->any_exact) launch_phase_exact(vg, sg, ci, c->grid_exact);
            if (c->any_fast) {
                launch_phase_fast(c->fast_variant, vg, sg, ci, c->grid_fast);
                launch_phase_rescue(c->fast_variant & 1, vg, sg, ci, c->sms);
            }
        }
        if (g > 0) cudaEventRecord(c->ev_join[g], sg);
    }
    for (int g = 1; g < c->ngroup; g++) cudaStreamWaitEvent(c->stream, c->ev_join[g], 0);
    cudaEventRecordWithFlags(c->ev[2], c->stream, cudaEventRecordExternal);
    launch_sweep_stats(v, c->stream);
    if (c->any_npt) {
        launch_volume_propose(v, c->stream);
        if (c->any_da || c->rec_cap > 0)
            launch_features(v, c->stream, c->any_da ? mlp_input(c->mlp) : nullptr, c->any_da ? mlp_ld(c->mlp) : 0,
                            c->grid_elem);
        if (c->any_screen) launch_screen(v, c->stream, c->d_pe0, c->d_pe1, c->d_phard, c->grid_screen, c->fast_variant & 1);
        if (c->any_da) {
            const int B = (2 * c->R + 127) / 128 * 128;
            const float *y = mlp_forward_device(c->mlp, B, c->stream);
            launch_da_stage1(v, c->stream, y);
        }
        launch_volume_finish(v, c->stream, c->d_pe0, c->d_pe1, c->d_phard, c->grid_energy);
    }
    cudaEventRecordWithFlags(c->ev[3], c->stream, cudaEventRecordExternal);
    launch_sweep_advance(v, c->stream);
    if (c->hist_cap > 0) launch_hist_record(v, c->stream);
    cudaEventRecordWithFlags(c->ev[4], c->stream, cudaEventRecordExternal);
}

static int check_flags(lcmc_ctx *c)
{
    std::vector<DevStats> st(c->R);
    CUDA_TRY(c, cudaMemcpyAsync(st.data(), c->d_stats, sizeof(DevStats) * c->R, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    int f = 0;
    for (auto &s : st) f |= s.flags;
    if (f & (F_CELLCAP | F_STENCILCAP | F_LISTCAP)) return set_err(c, LCMC_ECELLCAP, "cell capacity exceeded");
    if (f & F_NONFINITE) return set_err(c, LCMC_ENUMERIC, "non-finite energy change");
    if (f & F_DRIFT) {
        char b[200];
        for (int r = 0; r < c->R; r++)
            if (st[r].flags & F_DRIFT) {
                snprintf(b, sizeof(b), "replica %d: running energy off the FP64 recompute by %.6g (tolerance %.6g)", r,
                         st[r].drift, st[r].drift_bound);
                break;
            }
        return set_err(c, LCMC_EDRIFT, b);
    }
    return LCMC_OK;
}

// FP64 energy check of the replicas marked in the check kernel (all = every
// replica; else those whose sweep counter is a multiple of their
// energy_check_interval): rebin, FP64 total energy, compare and reset.
static void enqueue_energy_check(lcmc_ctx *c, int all)
{
    enqueue_rebin(c, c->cur);
    c->cur ^= 1;
    DevView v = view(c, c->cur);
    launch_energy_exact(v, c->stream, c->d_pe0, c->d_pe1, c->d_phard, 0, c->grid_energy);
    launch_energy_check(v, c->stream, c->d_pe0, all);
}

static bool check_due(const lcmc_ctx *c)
{
    for (int r = 0; r < c->R; r++) {
        const int every = c->rep[r].check_every;
        if (every > 0 && c->sweeps[r] % (unsigned long long)every == 0ull) return true;
    }
    return false;
}

extern "C" int lcmc_energy_check(lcmc_ctx *ctx)
{
    if (!ctx) return LCMC_EINVAL;
    for (int r = 0; r < ctx->R; r++)
        if (!ctx->uploaded[r]) return set_err(ctx, LCMC_EINVAL, "replica has no configuration (upload or init first)");
    enqueue_energy_check(ctx, 1);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaGetLastError());
    return check_flags(ctx);
}

extern "C" int lcmc_clear_error_flags(lcmc_ctx *ctx)
{
    if (!ctx) return LCMC_EINVAL;
    for (int r = 0; r < ctx->R; r++) {
        const int zero = 0;
        CUDA_TRY(ctx, cudaMemcpyAsync((char *)ctx->d_stats + sizeof(DevStats) * r + offsetof(DevStats, flags), &zero,
                                      sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    }
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->err.clear();
    return LCMC_OK;
}

extern "C" int lcmc_record_moves(lcmc_ctx *ctx, int on)
{
    if (!ctx) return LCMC_EINVAL;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (on && !ctx->d_rec_dE) {
        CUDA_TRY(ctx, dalloc(&ctx->d_rec_dE, ctx->ntot));
        CUDA_TRY(ctx, dalloc(&ctx->d_rec_lu, ctx->ntot));
        CUDA_TRY(ctx, cudaMemset(ctx->d_rec_dE, 0, sizeof(double) * ctx->ntot));
        CUDA_TRY(ctx, cudaMemset(ctx->d_rec_lu, 0, sizeof(double) * ctx->ntot));
    } else if (!on && ctx->d_rec_dE) {
        cudaFree(ctx->d_rec_dE);
        cudaFree(ctx->d_rec_lu);
        ctx->d_rec_dE = ctx->d_rec_lu = nullptr;
    }
    invalidate_graphs(ctx); // the view the graphs captured changed
    return LCMC_OK;
}

extern "C" int lcmc_get_move_records(lcmc_ctx *ctx, int replica, double *dE, double *log_u, int n)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !dE || !log_u || n != ctx->rep[replica].n) return LCMC_EINVAL;
    if (!ctx->d_rec_dE) return set_err(ctx, LCMC_EINVAL, "move recording is off (lcmc_record_moves)");
    const size_t off = (size_t)ctx->rep[replica].p_off;
    CUDA_TRY(ctx, cudaMemcpyAsync(dE, ctx->d_rec_dE + off, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(log_u, ctx->d_rec_lu + off, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LCMC_OK;
}

extern "C" int lcmc_sweep(lcmc_ctx *ctx, int n_sweeps)
{
    if (!ctx || n_sweeps < 0) return LCMC_EINVAL;
    for (int r = 0; r < ctx->R; r++)
        if (!ctx->uploaded[r]) return set_err(ctx, LCMC_EINVAL, "replica has no configuration (upload or init first)");
    for (int s = 0; s < n_sweeps; s++) {
        const int par = ctx->cur;
        if (!ctx->graph[par]) {
            cudaGraph_t g;
            CUDA_TRY(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            enqueue_sweep(ctx, par);
            CUDA_TRY(ctx, cudaStreamEndCapture(ctx->stream, &g));
            cudaError_t e = cudaGraphInstantiate(&ctx->graph[par], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                ctx->graph[par] = nullptr;
                return set_err(ctx, LCMC_ECUDA, cudaGetErrorString(e));
            }
        }
        CUDA_TRY(ctx, cudaGraphLaunch(ctx->graph[par], ctx->stream));
        ctx->cur = par ^ 1;
        ctx->timed = true;
        for (int r = 0; r < ctx->R; r++) ctx->sweeps[r]++;
        if (!ctx->checks_off && check_due(ctx)) enqueue_energy_check(ctx, 0);
    }
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaGetLastError());
    return check_flags(ctx);
}

extern "C" int lcmc_pair_terms(const lcmc_params *p, int n, const double *d, const double *ei, const double *ej,
                               double *out32, double *out64)
{
    if (!p || n < 0 || !d || !ei || !ej || !out32 || !out64) return LCMC_EINVAL;
    if (n == 0) return LCMC_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(nullptr, LCMC_ENODEV, "no CUDA device");
    }
    GBConsts k;
    make_consts(*p, k);
    double *buf = nullptr;
    const size_t b = sizeof(double) * (size_t)n;
    if (cudaMalloc(&buf, 11 * b) != cudaSuccess) return set_err(nullptr, LCMC_ENOMEM, "device allocation failed");
    double *dd = buf, *de = buf + 3 * (size_t)n, *dj = buf + 6 * (size_t)n, *o32 = buf + 9 * (size_t)n,
           *o64 = buf + 10 * (size_t)n;
    cudaMemcpy(dd, d, 3 * b, cudaMemcpyHostToDevice);
    cudaMemcpy(de, ei, 3 * b, cudaMemcpyHostToDevice);
    cudaMemcpy(dj, ej, 3 * b, cudaMemcpyHostToDevice);
    launch_pair_terms32(k, n, dd, de, dj, o32, 0);
    launch_pair_terms64(k, n, dd, de, dj, o64, 0);
    cudaMemcpy(out32, o32, b, cudaMemcpyDeviceToHost);
    cudaError_t e = cudaMemcpy(out64, o64, b, cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) return set_err(nullptr, LCMC_ECUDA, cudaGetErrorString(e));
    return LCMC_OK;
}

// Allocation-free total energy: no counterpart in the reference; for callers
// that must not let this library allocate device memory (see lcmc.h).  Makes
// no cudaMalloc/cudaFree call; scratch is the fixed area in lcmc_noalloc.cu.
extern "C" int lcmc_total_energy_noalloc(const lcmc_params *p, int n, const double *d_px, const double *d_py,
                                         const double *d_pz, const double *d_ox, const double *d_oy,
                                         const double *d_oz, const double box[3], double *d_energy, void *stream)
{
    if (!p || n < 0 || !box || !d_energy || (n > 0 && (!d_px || !d_py || !d_pz || !d_ox || !d_oy || !d_oz)))
        return set_err(nullptr, LCMC_EINVAL, "bad arguments");
    if (p->cutoff_radius <= 0.0) return set_err(nullptr, LCMC_EINVAL, "cutoff_radius must be positive");
    GBConsts k;
    make_consts(*p, k);
    char msg[256] = {0};
    int rc = total_energy_noalloc(k, n, d_px, d_py, d_pz, d_ox, d_oy, d_oz, box, d_energy, (cudaStream_t)stream, msg,
                                  sizeof(msg));
    if (rc) return set_err(nullptr, rc, msg);
    return LCMC_OK;
}

extern "C" int lcmc_get_stream(lcmc_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return LCMC_EINVAL;
    *stream = (void *)ctx->stream;
    return LCMC_OK;
}

extern "C" int lcmc_kernels_per_sweep(lcmc_ctx *ctx)
{
    if (!ctx) return LCMC_EINVAL;
    // rebin: setup, bin, 3 scan, scatter, sort, gather; phases, per replica group (FP32: with the FP64 hand-over
    // kernel); statistics: chunk sums, sums; volume: propose,
    // energy, chunk sums, accept, scale; surrogate: 2 feature kernels, 2 GEMMs + 3 small kernels, stage 1;
    // recording; history: chunk sums, rows; sweep counter
    int n = 8 + ctx->ngroup * ctx->nphase * ((int)ctx->any_exact + 2 * (int)ctx->any_fast) + 5 * (int)ctx->any_npt + 3;
    if (ctx->any_npt && (ctx->any_da || ctx->rec_cap > 0)) n += 2;
    if (ctx->any_npt && ctx->any_da) n += 6;
    if (ctx->any_npt && ctx->any_screen) n += 3; // screen energies, chunk sums, stage 1
    if (ctx->any_npt && ctx->rec_cap > 0) n += 1;
    if (ctx->hist_cap > 0) n += 2;
    return n;
}

static int push_replica_fields(lcmc_ctx *c, int r)
{
    Replica &rp = c->rep[r];
    char *base = (char *)c->d_rep + sizeof(Replica) * r;
    CUDA_TRY(c, cudaMemcpyAsync(base + offsetof(Replica, da_on), &rp.da_on, sizeof(int), cudaMemcpyHostToDevice,
                                c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(base + offsetof(Replica, da_kind), &rp.da_kind, sizeof(int), cudaMemcpyHostToDevice,
                                c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(base + offsetof(Replica, da_scale), &rp.da_scale, sizeof(double),
                                cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return LCMC_OK;
}

extern "C" int lcmc_set_surrogate(lcmc_ctx *ctx, lcmc_mlp *m, double target_scale)
{
    if (!ctx) return LCMC_EINVAL;
    if (m && (mlp_n_in(m) != LCMC_FEAT || mlp_bmax(m) < 2 * ctx->R))
        return set_err(ctx, LCMC_EINVAL, "surrogate needs 4097 inputs and a batch of at least 2 x replicas");
    ctx->mlp = m;
    ctx->any_da = false;
    ctx->any_screen = false; // one screen at a time
    for (int r = 0; r < ctx->R; r++) {
        Replica &rp = ctx->rep[r];
        rp.da_on = (m && rp.ensemble == 2) ? 1 : 0;
        rp.da_kind = rp.da_on ? 1 : 0;
        rp.da_scale = target_scale;
        ctx->any_da = ctx->any_da || rp.da_on;
        int rc = push_replica_fields(ctx, r);
        if (rc) return rc;
    }
    invalidate_graphs(ctx);
    return LCMC_OK;
}

extern "C" int lcmc_set_fp32_screen(lcmc_ctx *ctx, int on)
{
    if (!ctx) return LCMC_EINVAL;
    ctx->mlp = nullptr; // one screen at a time
    ctx->any_da = false;
    ctx->any_screen = false;
    for (int r = 0; r < ctx->R; r++) {
        Replica &rp = ctx->rep[r];
        rp.da_on = (on && rp.ensemble == 2 && rp.kernel == 1) ? 1 : 0;
        rp.da_kind = rp.da_on ? 2 : 0;
        ctx->any_screen = ctx->any_screen || rp.da_on;
        int rc = push_replica_fields(ctx, r);
        if (rc) return rc;
    }
    invalidate_graphs(ctx);
    return LCMC_OK;
}

extern "C" int lcmc_record_volume_samples(lcmc_ctx *ctx, int capacity)
{
    if (!ctx || capacity < 0) return LCMC_EINVAL;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->d_rec_x) cudaFree(ctx->d_rec_x);
    if (ctx->d_rec_y) cudaFree(ctx->d_rec_y);
    if (ctx->d_rec_count) cudaFree(ctx->d_rec_count);
    ctx->d_rec_x = nullptr;
    ctx->d_rec_y = nullptr;
    ctx->d_rec_count = nullptr;
    ctx->rec_cap = 0;
    if (capacity > 0) {
        CUDA_TRY(ctx, cudaMalloc(&ctx->d_rec_x, sizeof(float) * (size_t)capacity * LCMC_FEAT));
        CUDA_TRY(ctx, cudaMalloc(&ctx->d_rec_y, sizeof(float) * (size_t)capacity));
        CUDA_TRY(ctx, cudaMalloc(&ctx->d_rec_count, sizeof(int)));
        CUDA_TRY(ctx, cudaMemset(ctx->d_rec_count, 0, sizeof(int)));
        ctx->rec_cap = capacity;
    }
    invalidate_graphs(ctx);
    return LCMC_OK;
}

extern "C" int lcmc_get_volume_samples(lcmc_ctx *ctx, float *x, float *y, int max_n)
{
    if (!ctx || max_n < 0) return LCMC_EINVAL;
    if (!ctx->rec_cap) return 0;
    int n = 0;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(&n, ctx->d_rec_count, sizeof(int), cudaMemcpyDeviceToHost));
    if (n > ctx->rec_cap) n = ctx->rec_cap;
    if (n > max_n) n = max_n;
    if (n > 0 && x) CUDA_TRY(ctx, cudaMemcpy(x, ctx->d_rec_x, sizeof(float) * (size_t)n * LCMC_FEAT, cudaMemcpyDeviceToHost));
    if (n > 0 && y) CUDA_TRY(ctx, cudaMemcpy(y, ctx->d_rec_y, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
    return n;
}

extern "C" int lcmc_record_history(lcmc_ctx *ctx, int capacity)
{
    if (!ctx || capacity < 0) return LCMC_EINVAL;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->d_hist) cudaFree(ctx->d_hist);
    ctx->d_hist = nullptr;
    ctx->hist_cap = 0;
    if (capacity > 0) {
        CUDA_TRY(ctx, cudaMalloc(&ctx->d_hist, sizeof(double) * 9 * (size_t)capacity * ctx->R));
        CUDA_TRY(ctx, cudaMemset(ctx->d_hist, 0xFF, sizeof(double) * 9 * (size_t)capacity * ctx->R));
        ctx->hist_cap = capacity;
    }
    invalidate_graphs(ctx);
    return LCMC_OK;
}

extern "C" int lcmc_get_history(lcmc_ctx *ctx, int replica, double *rows, int max_rows)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !rows || max_rows < 0) return LCMC_EINVAL;
    if (!ctx->hist_cap) return 0;
    std::vector<double> h((size_t)9 * ctx->hist_cap);
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(h.data(), ctx->d_hist + (size_t)9 * ctx->hist_cap * replica,
                             sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
    // rows in sweep order; unwritten rows hold NaN (0xFF bytes)
    std::vector<std::pair<double, int>> order;
    for (int i = 0; i < ctx->hist_cap; i++)
        if (h[(size_t)9 * i] == h[(size_t)9 * i]) order.push_back({h[(size_t)9 * i], i});
    std::sort(order.begin(), order.end());
    int n = (int)order.size() < max_rows ? (int)order.size() : max_rows;
    for (int k = 0; k < n; k++) memcpy(rows + (size_t)9 * k, &h[(size_t)9 * order[k].second], 9 * sizeof(double));
    return n;
}

extern "C" int lcmc_set_adaptive_step(lcmc_ctx *ctx, int on)
{
    if (!ctx) return LCMC_EINVAL;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int r = 0; r < ctx->R; r++) {
        Replica rp;
        char *base = (char *)ctx->d_rep + sizeof(Replica) * r;
        CUDA_TRY(ctx, cudaMemcpy(&rp, base, sizeof(Replica), cudaMemcpyDeviceToHost));
        rp.adapt_on = on ? 1 : 0;
        rp.adapt_att = 0ull;
        rp.adapt_acc = 0ull;
        CUDA_TRY(ctx, cudaMemcpy(base + offsetof(Replica, adapt_on), &rp.adapt_on,
                                 offsetof(Replica, d_cap) - offsetof(Replica, adapt_on), cudaMemcpyHostToDevice));
        ctx->rep[r].adapt_on = rp.adapt_on;
    }
    return LCMC_OK;
}

extern "C" int lcmc_get_step(lcmc_ctx *ctx, int replica, double *max_displacement, double *max_rotation)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !max_displacement || !max_rotation) return LCMC_EINVAL;
    GBConsts k;
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(ctx, cudaMemcpy(&k, (char *)ctx->d_rep + sizeof(Replica) * replica + offsetof(Replica, k),
                             sizeof(GBConsts), cudaMemcpyDeviceToHost));
    *max_displacement = k.max_disp;
    *max_rotation = k.max_rot;
    return LCMC_OK;
}

extern "C" int lcmc_get_params(lcmc_ctx *ctx, int replica, lcmc_params *out)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !out) return LCMC_EINVAL;
    *out = ctx->params[replica];
    return LCMC_OK;
}

extern "C" int lcmc_set_sweep_counter(lcmc_ctx *ctx, int replica, int64_t sweep)
{
    if (!ctx || replica < 0 || replica >= ctx->R || sweep < 0) return LCMC_EINVAL;
    Replica &rp = ctx->rep[replica];
    rp.sweep = (unsigned long long)sweep;
    ctx->sweeps[replica] = rp.sweep;
    CUDA_TRY(ctx, cudaMemcpyAsync((char *)ctx->d_rep + sizeof(Replica) * replica + offsetof(Replica, sweep), &rp.sweep,
                                  sizeof(rp.sweep), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LCMC_OK;
}

extern "C" int lcmc_last_sweep_timing(lcmc_ctx *ctx, double ms[4])
{
    if (!ctx || !ms) return LCMC_EINVAL;
    if (!ctx->timed) return set_err(ctx, LCMC_EINVAL, "no sweep has run yet");
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < 4; i++) {
        float t = 0.0f;
        CUDA_TRY(ctx, cudaEventElapsedTime(&t, ctx->ev[i], ctx->ev[i + 1]));
        ms[i] = t;
    }
    return LCMC_OK;
}

// Rebin (no sweep) and recompute the FP64 total energy of every replica with
// the FP64 kernel; resets the running energies.
static int recompute_energy(lcmc_ctx *c, int replica_only)
{
    enqueue_rebin(c, c->cur);
    c->cur ^= 1;
    DevView v = view(c, c->cur);
    launch_energy_exact(v, c->stream, c->d_pe0, c->d_pe1, c->d_phard, 0, c->grid_energy);
    launch_energy_reduce(v, c->stream, c->d_pe0, replica_only);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    CUDA_TRY(c, cudaGetLastError());
    return LCMC_OK;
}

extern "C" int lcmc_total_energy(lcmc_ctx *ctx, int replica, int precision, double *energy)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !energy) return LCMC_EINVAL;
    (void)precision; // pair terms of the recompute always run in FP64 (B200 FP64 rate is ample here)
    int rc = recompute_energy(ctx, replica);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaMemcpy(energy, ctx->d_red + replica, sizeof(double), cudaMemcpyDeviceToHost));
    return LCMC_OK;
}

// Stage the caller's arrays in the rebin's spare buffer, check them on the
// device, and only then copy them over the replica's current slots: a rejected
// upload leaves the context's state as it was.
static int upload_state(lcmc_ctx *ctx, int replica, const double *px, const double *py, const double *pz,
                        const double *ox, const double *oy, const double *oz, int n, const double box[3])
{
    if (!ctx || replica < 0 || replica >= ctx->R || !px || !py || !pz || !ox || !oy || !oz || !box)
        return LCMC_EINVAL;
    Replica &rp = ctx->rep[replica];
    if (n != rp.n) return set_err(ctx, LCMC_EINVAL, "particle count differs from num_particles");
    const double rc = ctx->params[replica].cutoff_radius;
    for (int a = 0; a < 3; a++)
        if (!(box[a] >= 2.0 * rc)) return set_err(ctx, LCMC_EBOX, "box shorter than twice the cutoff");
    const double R = ctx->params[replica].colloid_radius;
    const int off = rp.p_off, cur = ctx->cur, spare = cur ^ 1;
    const double *src[6] = {px, py, pz, ox, oy, oz};
    const double *stage[6];
    for (int k = 0; k < 6; k++) {
        CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_x[spare][k] + off, src[k], sizeof(double) * n, cudaMemcpyHostToDevice,
                                      ctx->stream));
        stage[k] = ctx->d_x[spare][k] + off;
    }
    CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
    launch_validate_upload(stage, ctx->d_id[spare] + off, n, box, R * R, ctx->d_flag, ctx->stream, ctx->grid_elem);
    int flag = 0;
    CUDA_TRY(ctx, cudaMemcpyAsync(&flag, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (flag & 1) return set_err(ctx, LCMC_EINVAL, "particle outside the box");
    if (flag & 2) return set_err(ctx, LCMC_EOVERLAP, "particle inside the colloid");
    if (flag & 4) return set_err(ctx, LCMC_EINVAL, "zero or non-finite orientation");
    for (int k = 0; k < 6; k++)
        CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_x[cur][k] + off, stage[k], sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->d_id[cur] + off, ctx->d_id[spare] + off, sizeof(int) * n,
                                  cudaMemcpyDeviceToDevice, ctx->stream));
    for (int a = 0; a < 3; a++) rp.L[a] = box[a];
    // box (dynamic field) into the device table
    CUDA_TRY(ctx, cudaMemcpyAsync((char *)ctx->d_rep + sizeof(Replica) * replica + offsetof(Replica, L), rp.L,
                                  sizeof(double) * 3, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->uploaded[replica] = 1;
    // the kernel choice and the FP32 kernel's capacity follow the new box
    return rechoose_kernels(ctx);
}

extern "C" int lcmc_upload(lcmc_ctx *ctx, int replica, const double *px, const double *py, const double *pz,
                           const double *ox, const double *oy, const double *oz, int n, const double box[3])
{
    int rc = upload_state(ctx, replica, px, py, pz, ox, oy, oz, n, box);
    if (rc) return rc;
    bool all = true;
    for (int r = 0; r < ctx->R; r++) all = all && ctx->uploaded[r];
    if (!all) return LCMC_OK; // energies are computed once every replica holds a configuration
    int e = recompute_energy(ctx, -1);
    if (e) return e;
    // zero the drift of the first recompute
    std::vector<DevStats> st(ctx->R);
    CUDA_TRY(ctx, cudaMemcpy(st.data(), ctx->d_stats, sizeof(DevStats) * ctx->R, cudaMemcpyDeviceToHost));
    for (auto &s : st) s.drift = 0.0;
    CUDA_TRY(ctx, cudaMemcpy(ctx->d_stats, st.data(), sizeof(DevStats) * ctx->R, cudaMemcpyHostToDevice));
    return LCMC_OK;
}

extern "C" int lcmc_upload_with_energy(lcmc_ctx *ctx, int replica, const double *px, const double *py,
                                       const double *pz, const double *ox, const double *oy, const double *oz, int n,
                                       const double box[3], double energy)
{
    if (!ctx || replica < 0 || replica >= ctx->R) return LCMC_EINVAL;
    if (!std::isfinite(energy)) return set_err(ctx, LCMC_EINVAL, "non-finite energy");
    int rc = upload_state(ctx, replica, px, py, pz, ox, oy, oz, n, box);
    if (rc) return rc;
    // the caller's running energy replaces the recompute (no drift recorded)
    const size_t base = sizeof(DevStats) * replica;
    const double zero = 0.0;
    CUDA_TRY(ctx, cudaMemcpyAsync((char *)ctx->d_stats + base + offsetof(DevStats, energy), &energy, sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync((char *)ctx->d_stats + base + offsetof(DevStats, drift), &zero, sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LCMC_OK;
}

extern "C" int lcmc_init_config(lcmc_ctx *ctx, int replica)
{
    if (!ctx || replica < 0 || replica >= ctx->R) return LCMC_EINVAL;
    const lcmc_params &p = ctx->params[replica];
    const int n = p.num_particles;
    std::vector<double> a(6 * (size_t)n);
    double box[3];
    int rc = lcmc_lattice(&p, replica, &a[0], &a[n], &a[2 * n], &a[3 * n], &a[4 * n], &a[5 * n], box);
    if (rc) return rc;
    return lcmc_upload(ctx, replica, &a[0], &a[n], &a[2 * n], &a[3 * n], &a[4 * n], &a[5 * n], n, box);
}

extern "C" int lcmc_download(lcmc_ctx *ctx, int replica, double *px, double *py, double *pz, double *ox, double *oy,
                             double *oz, int n, double box[3])
{
    if (!ctx || replica < 0 || replica >= ctx->R || !px || !py || !pz || !ox || !oy || !oz) return LCMC_EINVAL;
    const Replica &rp = ctx->rep[replica];
    if (n != rp.n) return LCMC_EINVAL;
    DevView v = view(ctx, ctx->cur);
    launch_to_id_order(v, ctx->stream, replica, ctx->grid_elem);
    double *dst[6] = {px, py, pz, ox, oy, oz};
    const int other = ctx->cur ^ 1;
    for (int k = 0; k < 6; k++)
        CUDA_TRY(ctx, cudaMemcpyAsync(dst[k], ctx->d_x[other][k] + rp.p_off, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                      ctx->stream));
    if (box)
        CUDA_TRY(ctx, cudaMemcpyAsync(box, (char *)ctx->d_rep + sizeof(Replica) * replica + offsetof(Replica, L),
                                      sizeof(double) * 3, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LCMC_OK;
}

extern "C" int lcmc_get_stats(lcmc_ctx *ctx, int replica, lcmc_stats *out)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !out) return LCMC_EINVAL;
    DevStats s;
    Replica rp;
    CUDA_TRY(ctx, cudaMemcpyAsync(&s, ctx->d_stats + replica, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaMemcpyAsync(&rp, ctx->d_rep + replica, sizeof(rp), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    memset(out, 0, sizeof(*out));
    out->sweeps = (int64_t)rp.sweep;
    out->attempted = (int64_t)s.attempted;
    out->accepted = (int64_t)s.accepted;
    out->hardcore_rejected = (int64_t)s.hard;
    out->volume_attempted = (int64_t)s.vol_att;
    out->volume_accepted = (int64_t)s.vol_acc;
    out->energy = s.energy;
    out->box[0] = rp.L[0];
    out->box[1] = rp.L[1];
    out->box[2] = rp.L[2];
    out->last_recompute = s.last_recompute;
    out->drift = s.drift;
    out->pairs_in_cutoff = (int64_t)s.pairs;
    out->stencil_candidates = (int64_t)s.cands;
    out->error_flags = s.flags;
    out->volume_stage1_rejected = (int64_t)s.vol_s1rej;
    out->kernel = rp.use_fast;
    out->fp64_cells = (int64_t)s.fp64_cells;
    out->overcap_cells = (int64_t)s.overcap_cells;
    out->energy_checks = (int64_t)s.checks;
    out->drift_breaches = (int64_t)s.breaches;
    out->drift_bound = s.drift_bound;
    out->abs_dE_since_check = s.abs_dE;
    return LCMC_OK;
}

extern "C" int lcmc_last_outcomes(lcmc_ctx *ctx, int replica, unsigned char *out, int n)
{
    if (!ctx || replica < 0 || replica >= ctx->R || !out || n != ctx->rep[replica].n) return LCMC_EINVAL;
    CUDA_TRY(ctx, cudaMemcpyAsync(out, ctx->d_outcome + ctx->rep[replica].p_off, (size_t)n, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LCMC_OK;
}

// Q = <u u> - I/3, P2 = 1.5 lambda_max and its eigenvector (cyclic Jacobi,
// Golub & Van Loan Alg. 8.4.3) - the reference's float Jacobi and its
// largest-eigenvalue search (which starts at index 1, MCnptColloid.c:1890)
// are replaced.
extern "C" int lcmc_order_parameter(lcmc_ctx *ctx, int replica, double Q[6], double *P2, double director[3])
{
    if (!ctx || replica < 0 || replica >= ctx->R) return LCMC_EINVAL;
    DevView v = view(ctx, ctx->cur);
    launch_order_sums(v, ctx->stream, replica, ctx->d_red + 8 * ctx->R);
    double s[6];
    CUDA_TRY(ctx, cudaMemcpyAsync(s, ctx->d_red + 8 * ctx->R, sizeof(s), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    const double inv = 1.0 / (double)ctx->rep[replica].n;
    double q[6] = {s[0] * inv - 1.0 / 3.0, s[1] * inv, s[2] * inv, s[3] * inv - 1.0 / 3.0, s[4] * inv,
                   s[5] * inv - 1.0 / 3.0};
    double a[3][3] = {{q[0], q[1], q[2]}, {q[1], q[3], q[4]}, {q[2], q[4], q[5]}};
    double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int sweep = 0; sweep < 50; sweep++) {
        double offd = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        if (offd < 1e-40) break;
        for (int pp = 0; pp < 2; pp++)
            for (int qq = pp + 1; qq < 3; qq++) {
                if (a[pp][qq] == 0.0) continue;
                double th = (a[qq][qq] - a[pp][pp]) / (2.0 * a[pp][qq]);
                double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
                double cs = 1.0 / sqrt(t * t + 1.0), sn = t * cs;
                for (int k = 0; k < 3; k++) {
                    double akp = a[k][pp], akq = a[k][qq];
                    a[k][pp] = cs * akp - sn * akq;
                    a[k][qq] = sn * akp + cs * akq;
                }
                for (int k = 0; k < 3; k++) {
                    double apk = a[pp][k], aqk = a[qq][k];
                    a[pp][k] = cs * apk - sn * aqk;
                    a[qq][k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < 3; k++) {
                    double vkp = V[k][pp], vkq = V[k][qq];
                    V[k][pp] = cs * vkp - sn * vkq;
                    V[k][qq] = sn * vkp + cs * vkq;
                }
            }
    }
    int im = 0;
    for (int i = 1; i < 3; i++)
        if (a[i][i] > a[im][im]) im = i;
    if (Q)
        for (int k = 0; k < 6; k++) Q[k] = q[k];
    if (P2) *P2 = 1.5 * a[im][im];
    if (director) {
        director[0] = V[0][im];
        director[1] = V[1][im];
        director[2] = V[2][im];
    }
    return LCMC_OK;
}

// ---------------------------------------------------------------------------
// autotuner (no reference counterpart): measured choice of the FP32 phase
// kernel's capacity class and of the kernel for the volume move's energies
// ---------------------------------------------------------------------------

namespace {

struct TuneChoice {
    int variant_class; // index into the phase-kernel capacity classes
    int vol_cells;     // 1: per-cell volume-energy kernel, 0: per-particle kernel
};

// The workload signature a cached choice is valid for: device, replica layout
// and every replica's size, ensemble, kernel, grid capacity and screen.
std::string tune_key(const lcmc_ctx *c)
{
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) prop.name[0] = 0;
    std::string k = std::string(prop.name) + "|sms=" + std::to_string(c->sms) + "|R=" + std::to_string(c->R);
    for (int r = 0; r < c->R; r++) {
        const Replica &rp = c->rep[r];
        const lcmc_params &p = c->params[r];
        char b[160];
        snprintf(b, sizeof(b), "|%d,%d,%d,%d,%d,%.3g,%d", rp.n, rp.ensemble, rp.kernel, rp.nc_max, rp.da_kind,
                 p.system_density, p.cell_capacity);
        k += b;
    }
    for (char &ch : k)
        if (ch == '\t' || ch == '\n') ch = ' ';
    return k;
}

bool tune_cache_read(const char *path, const std::string &key, TuneChoice &ch, double &ms)
{
    if (!path) return false;
    FILE *f = fopen(path, "r");
    if (!f) return false;
    char line[8192];
    bool found = false;
    while (fgets(line, sizeof(line), f)) {
        char *tab = strchr(line, '\t');
        if (!tab) continue;
        *tab = 0;
        if (key != line) continue;
        int a = 0, b = 0;
        double m = 0.0;
        if (sscanf(tab + 1, "%d\t%d\t%lf", &a, &b, &m) == 3 && a >= 0 && a < fast_variant_count() && (b == 0 || b == 1)) {
            ch.variant_class = a;
            ch.vol_cells = b;
            ms = m;
            found = true; // the last entry for a key wins
        }
    }
    fclose(f);
    return found;
}

void tune_cache_append(const char *path, const std::string &key, const TuneChoice &ch, double ms)
{
    if (!path) return;
    FILE *f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "%s\t%d\t%d\t%.6f\n", key.c_str(), ch.variant_class, ch.vol_cells, ms);
    fclose(f);
}

} // namespace

static int apply_tuning(lcmc_ctx *c, const TuneChoice &ch)
{
    c->fast_variant = 2 * ch.variant_class + (c->fast_variant & 1);
    c->tuned_class = ch.variant_class;
    set_caps(c);
    int prc = push_kernel_fields(c);
    if (prc) return prc;
    c->grid_fast = fast_blocks_per_sm(c->fast_variant) * c->sms;
    for (int r = 0; r < c->R; r++) {
        Replica &rp = c->rep[r];
        rp.vol_cells = ch.vol_cells;
        CUDA_TRY(c, cudaMemcpyAsync((char *)c->d_rep + sizeof(Replica) * r + offsetof(Replica, vol_cells), &rp.vol_cells,
                                    sizeof(int), cudaMemcpyHostToDevice, c->stream));
    }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    invalidate_graphs(c);
    return LCMC_OK;
}

extern "C" int lcmc_autotune(lcmc_ctx *ctx, int sweeps, const char *cache_path, lcmc_tuning *out)
{
    if (!ctx || sweeps < 1) return LCMC_EINVAL;
    for (int r = 0; r < ctx->R; r++)
        if (!ctx->uploaded[r]) return set_err(ctx, LCMC_EINVAL, "replica has no configuration (upload or init first)");
    if (ctx->hist_cap > 0 || ctx->rec_cap > 0)
        return set_err(ctx, LCMC_EINVAL, "autotune before recording history or volume samples");
    const std::string key = tune_key(ctx);
    TuneChoice best{ctx->fast_variant >> 1, 1};
    double best_ms = 0.0;
    lcmc_tuning res;
    memset(&res, 0, sizeof(res));
    if (tune_cache_read(cache_path, key, best, best_ms)) {
        int rc = apply_tuning(ctx, best);
        if (rc) return rc;
        res.from_cache = 1;
    } else {
        // candidates: every capacity class the capacity rule allows, each volume-energy kernel that applies
        std::vector<TuneChoice> cand;
        bool npt4 = false; // an NPT replica on the per-cell volume kernel's grid (>= 4 cells per axis)
        for (int r = 0; r < ctx->R; r++)
            npt4 = npt4 || (ctx->rep[r].ensemble == 2 && grid_dim_host(ctx->rep[r].L[0], ctx->rep[r].wmin, ctx->rep[r].fine) >= 4);
        for (int v = 0; v < fast_variant_count(); v++) {
            if (!ctx->any_fast && v != (ctx->fast_variant >> 1)) continue;
            // classes below mean + 3 standard deviations of a cell's count are not tried (the largest always is)
            if (ctx->any_fast && fast_variant(v).amax < ctx->need_min && v != fast_variant_count() - 1) continue;
            cand.push_back({v, 1});
            if (npt4) cand.push_back({v, 0});
        }
        // snapshot: the current state buffer, ids, replica table, statistics, outcomes
        const int cur = ctx->cur;
        const size_t n = (size_t)ctx->ntot;
        double *sx = nullptr;
        int *sid = nullptr;
        Replica *srep = nullptr;
        DevStats *sst = nullptr;
        unsigned char *sout = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        auto release = [&]() {
            cudaFree(sx);
            cudaFree(sid);
            cudaFree(srep);
            cudaFree(sst);
            cudaFree(sout);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        };
        if (cudaMalloc(&sx, sizeof(double) * 6 * n) != cudaSuccess || cudaMalloc(&sid, sizeof(int) * n) != cudaSuccess ||
            cudaMalloc(&srep, sizeof(Replica) * ctx->R) != cudaSuccess ||
            cudaMalloc(&sst, sizeof(DevStats) * ctx->R) != cudaSuccess || cudaMalloc(&sout, n) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            release();
            cudaGetLastError();
            return set_err(ctx, LCMC_ENOMEM, "autotune snapshot");
        }
        auto copy_state = [&](bool save) -> cudaError_t {
            cudaError_t e = cudaSuccess;
            for (int k = 0; k < 6 && e == cudaSuccess; k++)
                e = save ? cudaMemcpyAsync(sx + k * n, ctx->d_x[cur][k], sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                           ctx->stream)
                         : cudaMemcpyAsync(ctx->d_x[cur][k], sx + k * n, sizeof(double) * n, cudaMemcpyDeviceToDevice,
                                           ctx->stream);
            if (e == cudaSuccess)
                e = save ? cudaMemcpyAsync(sid, ctx->d_id[cur], sizeof(int) * n, cudaMemcpyDeviceToDevice, ctx->stream)
                         : cudaMemcpyAsync(ctx->d_id[cur], sid, sizeof(int) * n, cudaMemcpyDeviceToDevice, ctx->stream);
            if (e == cudaSuccess)
                e = save ? cudaMemcpyAsync(srep, ctx->d_rep, sizeof(Replica) * ctx->R, cudaMemcpyDeviceToDevice,
                                           ctx->stream)
                         : cudaMemcpyAsync(ctx->d_rep, srep, sizeof(Replica) * ctx->R, cudaMemcpyDeviceToDevice,
                                           ctx->stream);
            if (e == cudaSuccess)
                e = save ? cudaMemcpyAsync(sst, ctx->d_stats, sizeof(DevStats) * ctx->R, cudaMemcpyDeviceToDevice,
                                           ctx->stream)
                         : cudaMemcpyAsync(ctx->d_stats, sst, sizeof(DevStats) * ctx->R, cudaMemcpyDeviceToDevice,
                                           ctx->stream);
            if (e == cudaSuccess)
                e = save ? cudaMemcpyAsync(sout, ctx->d_outcome, n, cudaMemcpyDeviceToDevice, ctx->stream)
                         : cudaMemcpyAsync(ctx->d_outcome, sout, n, cudaMemcpyDeviceToDevice, ctx->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
            if (!save) ctx->cur = cur;
            return e;
        };
        if (copy_state(true) != cudaSuccess) {
            release();
            return set_err(ctx, LCMC_ECUDA, "autotune snapshot");
        }
        const std::vector<unsigned long long> saved_sweeps = ctx->sweeps;
        ctx->checks_off = true;
        best_ms = -1.0;
        int rc = LCMC_OK;
        for (const TuneChoice &ch : cand) {
            rc = apply_tuning(ctx, ch);
            if (rc) break;
            rc = lcmc_sweep(ctx, 1); // warm-up: captures the graph
            double ms = -1.0;
            if (rc == LCMC_OK) {
                cudaEventRecord(e0, ctx->stream);
                rc = lcmc_sweep(ctx, sweeps);
                cudaEventRecord(e1, ctx->stream);
                float t = 0.0f;
                if (rc == LCMC_OK && cudaEventSynchronize(e1) == cudaSuccess &&
                    cudaEventElapsedTime(&t, e0, e1) == cudaSuccess)
                    ms = t / sweeps;
            }
            res.trials++;
            ctx->sweeps = saved_sweeps;
            if (copy_state(false) != cudaSuccess) {
                ctx->checks_off = false;
                release();
                return set_err(ctx, LCMC_ECUDA, "autotune restore");
            }
            if (rc == LCMC_ECELLCAP) rc = LCMC_OK; // this class is too small for the configuration
            if (rc) break;
            if (ms > 0.0 && (best_ms < 0.0 || ms < best_ms)) {
                best_ms = ms;
                best = ch;
            }
        }
        release();
        ctx->checks_off = false;
        if (rc) return rc;
        if (best_ms < 0.0) return set_err(ctx, LCMC_ECELLCAP, "no candidate ran");
        rc = apply_tuning(ctx, best);
        if (rc) return rc;
        tune_cache_append(cache_path, key, best, best_ms);
    }
    res.capacity = fast_variant(best.variant_class).amax;
    res.volume_by_cell = best.vol_cells;
    res.ms_per_sweep = best_ms;
    if (out) *out = res;
    ctx->err.clear();
    return LCMC_OK;
}
