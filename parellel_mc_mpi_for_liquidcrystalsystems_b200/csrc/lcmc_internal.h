// lcmc_internal.h - data shared by the host side and the kernels.
#pragma once
#include <stdint.h>

namespace lcmc {

// Derived constants of one system (get_system_const, MCnptColloid.c:2752-2783,
// with chi computed after kappa^2).  FP64, plus FP32 copies for the FP32 kernel.
struct GBConsts {
    double beta, four_eps0, rc, rc2, sigma0, chi, chi_sq, chi_prime, mu, nu, kappa_prime;
    double coll_R, coll_cutoff, max_disp, max_rot;
    int coll_on;
    int mu_code, nu_code; // 1 or 2: exact integer power; 0: general pow
    float f_rc2, f_chi, f_chi_sq, f_chip, f_chip_sq, f_sigma0, f_4eps0, f_half_chi, f_half_chip;
};

// One replica (system).  Static fields are set by the host at create time;
// dynamic fields are rewritten on the device every sweep.
struct Replica {
    int n;        // particles
    int p_off;    // first particle slot in the concatenated arrays
    int cell_off; // first cell slot
    int nc_max;   // cells per axis allocated (nc_max^3 cells)
    int ensemble; // 1 NVT, 2 NPT
    int kernel;   // 0 FP64 kernel, 1 FP32 kernel
    int npt_energy_fp64;
    uint32_t key[2];
    double pressure, dlnv_max, wmin;
    GBConsts k;
    // dynamic
    double L[3];
    int nc[3];
    double w[3];
    double shift[3];
    int perm[8];
    unsigned long long sweep;
    int use_fast;  // this sweep runs the FP32 kernel (needs >= 4 cells per axis)
    // volume move of this sweep
    double vol_delta, vol_lambda, vol_U_old, vol_U_new;
    int vol_state; // 0 none, 1 accepted, 2 rejected, 3 hard-core reject, 4 rejected by the surrogate (stage 1)
    // delayed acceptance with the learned surrogate
    int da_on;         // a stage-1 screen is set for this replica
    int da_kind;       // 1 the learned surrogate, 2 the FP32-pair energy change
    // adaptive step (equilibration only): block counters, the cell grid's cap
    // on the displacement (creation value) and min(sigma_ee, sigma_ss)
    int adapt_on;
    unsigned long long adapt_att, adapt_acc;
    double d_cap, min_thick;
    int vol_stage1;    // this sweep: 0 rejected by the screen, 1 no screen, 2 passed the screen
    double da_scale;   // surrogate output -> dU / N
    double vol_dU_sur; // surrogate dU of this sweep's move
    int vol_cells;     // 1: the volume move's exact energies by the per-cell kernel (>= 4 cells per axis)
};

constexpr int LCMC_FEAT = 8 * 512 + 1; // surrogate input: 8 channels x 8^3 cells + delta ln V

// Per-replica counters kept on the device.
struct DevStats {
    unsigned long long attempted, accepted, hard, vol_att, vol_acc, pairs, cands, vol_s1rej;
    double energy, last_recompute, drift;
    int flags;
    int pad;
};

// error flag bits (mirrors LCMC_F_* in lcmc.h)
constexpr int F_CELLCAP = 1, F_STENCILCAP = 2, F_LISTCAP = 4, F_NONFINITE = 8, F_GRIDCAP = 16;

// Launch view of the device buffers, passed by value to every kernel.
// particles per chunk of the two-level reductions (sums over a replica)
constexpr int LCMC_RED_CHUNK = 4096;

struct DevView {
    int R;              // replicas
    int ntot;           // particles, all replicas
    int ctot;           // cells allocated, all replicas
    Replica *rep;       // [R]
    DevStats *stats;    // [R]
    int *act_off;       // [8 * (R + 1)] active-cell prefix per phase
    int *p2r;           // [ntot] replica of each particle slot
    // particle state, cell-sorted (current buffer)
    double *px, *py, *pz, *ox, *oy, *oz;
    int *id;            // local particle id
    // the other buffer (rebin target)
    double *qx, *qy, *qz, *qux, *quy, *quz;
    int *qid;
    int *cid;           // [ntot] cell of each particle (pre-rebin order)
    int *scid;          // [ntot] cell of each slot of the current (sorted) buffer
    int *rank;          // [ntot] arrival rank inside its cell
    int *perm;          // [ntot] gather permutation
    int *cell_count;    // [ctot]
    int *cell_start;    // [ctot + 1]
    int *block_sums;    // scan scratch
    double *cell_e0, *cell_e1; // per-cell FP64 sums (sweep dE / energies)
    int *cell_n0, *cell_n1;    // per-cell counts (accepted / hard-core)
    unsigned long long *cell_pairs, *cell_cands;
    unsigned char *outcome;    // [ntot] by particle slot of id: 0/1/2
    double *scratch_d;         // [R * 8] small reductions
    double *red_part;          // [R x red_nchunk x 6] per-chunk partial sums
    int red_nchunk;            // chunks of LCMC_RED_CHUNK particles per replica (largest replica)
    // this sweep's trial moves, by sorted slot (FP32 kernel systems)
    double *tnx, *tny, *tnz;   // new position, wrapped
    double *tux, *tuy, *tuz;   // new orientation, normalised
    double *tdU;               // colloid-term change
    double *tlu;               // log of the Metropolis draw
    float *tdx, *tdy, *tdz;    // displacement
    unsigned char *thard;      // 1 = colloid hard-core reject
    // FP32 copy of the state of FP32-kernel systems, relative to each particle's
    // own cell origin: (x, y, z, ux) and (uy, uz), unit orientation; written by
    // the gather, kept current by the phase write-back
    float4 *cl4;
    float2 *cl2;
    // surrogate features and recordings
    unsigned long long *feat_acc; // [R x 512 x 7] pooled sums, fixed point 2^-32
    float *feat_f;             // [R x LCMC_FEAT] features of the current configuration
    int rec_cap;               // sample ring capacity (0 = off)
    int *rec_count;
    float *rec_x, *rec_y;      // [rec_cap x LCMC_FEAT], [rec_cap]
    int hist_cap;              // per-sweep history capacity (0 = off)
    double *hist;              // [R x hist_cap x 9]
};

} // namespace lcmc
