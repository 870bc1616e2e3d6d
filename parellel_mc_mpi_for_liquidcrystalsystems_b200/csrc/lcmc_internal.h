// lcmc_internal.h - data shared by the host side and the kernels.
#pragma once
#include <stdint.h>

namespace lcmc {

// Most colour phases of a sweep: 3 colours per axis on odd cell counts (fine grid).
constexpr int LCMC_MAX_COLOURS = 27;

// Cells of colour b along an axis of nc cells with k colours, and the index
// of the j-th of them.  k = 2 (even nc, or a single cell): cells b, b + 2, ...
// k = 3 (odd nc >= 3, fine grid), nc = 3q + r: colour i mod 3 for i < 3q, then
// r = 1: cell 3q takes colour 1; r = 2: cells 3q, 3q + 1 take colours 0, 1.
// Neighbouring cells (the periodic seam included) never share a colour, and
// the colours hold q or q + 1 cells each, so the phases stay balanced.
__host__ __device__ __forceinline__ int axis_colour_count(int nc, int k, int b)
{
    if (k != 3) return (nc - b + 1) / 2;
    const int q = nc / 3, r = nc - 3 * q;
    return q + ((r >= 1 && b == 1) ? 1 : 0) + ((r == 2 && b == 0) ? 1 : 0);
}
__host__ __device__ __forceinline__ int axis_colour_cell(int nc, int k, int b, int j)
{
    if (k != 3) return 2 * j + b;
    const int q = nc / 3, r = nc - 3 * q;
    return j < q ? b + 3 * j : 3 * q + (r == 2 ? b : 0);
}

// Derived constants of one system (get_system_const, MCnptColloid.c:2752-2783,
// with chi computed after kappa^2).  FP64, plus FP32 copies for the FP32 kernel.
struct GBConsts {
    double beta, four_eps0, rc, rc2, sigma0, chi, chi_sq, chi_prime, mu, nu, kappa_prime;
    double coll_R, coll_cutoff, max_disp, max_rot;
    int coll_on;
    int mu_code, nu_code; // 1 or 2: exact integer power; 0: general pow
    float f_rc2, f_chi, f_chi_sq, f_chip, f_chip_sq, f_sigma0, f_4eps0, f_half_chi, f_half_chip;
    // FP32 kernel: a cell with any pair term above f_big in magnitude (or the
    // overlap clamp, or a non-finite term) is attempted in FP64 instead
    float f_big;
};

// One replica (system).  Static fields are set by the host at create time;
// dynamic fields are rewritten on the device every sweep.
struct Replica {
    int n;        // particles
    int p_off;    // first particle slot in the concatenated arrays
    int cell_off; // first cell slot
    int nc_max;   // cells per axis allocated (nc_max^3 cells)
    int fine;     // cell grid: 0 even counts per axis (8 colours), 1 any count (odd: 3 colours on that axis)
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
    int kc[3];      // colours per axis: 2 (even count, or 1 cell), 3 (odd count >= 3, fine grid only)
    int ncol;       // colours this sweep: kc[0] kc[1] kc[2]
    int perm[LCMC_MAX_COLOURS]; // colour of each phase (-1: phase empty for this replica)
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
    int cap;           // FP32 kernel: cells holding more particles are attempted in FP64 (the caller's
                       // cell_capacity, else the kernel class's capacity)
    // periodic FP64 energy check: every check_every sweeps (0 = off), tolerance
    // check_tol relative to max(|E|, N 4 eps0) + sum of |dE| accepted since the last check
    int check_every;
    double check_tol;
};

constexpr int LCMC_FEAT = 8 * 512 + 1; // surrogate input: 8 channels x 8^3 cells + delta ln V

// Per-replica counters kept on the device.
struct DevStats {
    unsigned long long attempted, accepted, hard, vol_att, vol_acc, pairs, cands, vol_s1rej;
    double energy, last_recompute, drift;
    int flags;
    int pad;
    unsigned long long fp64_cells;   // FP32-kernel cells attempted in FP64 (large terms or capacity)
    unsigned long long overcap_cells; // of which: above the cell, stencil or list capacity
    unsigned long long checks, breaches; // periodic energy checks run / out of tolerance
    double abs_dE;                   // sum of |dE| of accepted moves since the last check
    double drift_bound;              // tolerance of the last check
};

// error flag bits (mirrors LCMC_F_* in lcmc.h)
constexpr int F_CELLCAP = 1, F_STENCILCAP = 2, F_LISTCAP = 4, F_NONFINITE = 8, F_GRIDCAP = 16, F_DRIFT = 32;

// Launch view of the device buffers, passed by value to every kernel.
// particles per chunk of the two-level reductions (sums over a replica)
constexpr int LCMC_RED_CHUNK = 4096;
// values per chunk in red_part (sums of up to LCMC_RED_K quantities at once)
constexpr int LCMC_RED_K = 8;

struct DevView {
    int R;              // replicas
    int ntot;           // particles, all replicas
    int ctot;           // cells allocated, all replicas
    Replica *rep;       // [R]
    DevStats *stats;    // [R]
    int *act_off;       // [nphase * (R + 1)] active-cell prefix per phase
    int nphase;         // colour phases per sweep: 8, or LCMC_MAX_COLOURS with a fine-grid replica
    int r_lo, r_hi;     // replicas whose cells the phase kernels attempt (a group of a batch: [r_lo, r_hi))
    int ngroup;         // replica groups (resc_count/resc_list hold one set of phases per group)
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
    double *cell_abs;          // per cell: sum of |dE| of the accepted moves
    int *p2c;                  // [ctot] replica of each cell slot
    int *resc_count;           // [nphase] cells the FP32 kernel handed over to the FP64 kernel, per colour phase
                               // (per group: a group's view points at its own nphase counts and lists)
    int *resc_list;            // [nphase x ctot] their codes: cell * 4 + mode (1 large term, 2 capacity)
    int *cell_fp64;            // per cell: 0 FP32, 1 attempted in FP64 (large term), 2 (capacity)
    unsigned char *outcome;    // [ntot] by particle slot of id: 0/1/2
    double *rec_dE, *rec_lu;   // [ntot] by particle slot of id: dE and log u of the last sweep (null: off)
    double *scratch_d;         // [R * 8] small reductions
    double *red_part;          // [R x red_nchunk x LCMC_RED_K] per-chunk partial sums
    int red_nchunk;            // chunks of LCMC_RED_CHUNK particles per replica (largest replica)
    // this sweep's trial moves, by sorted slot (FP32 kernel systems)
    double *tnx, *tny, *tnz;   // new position, wrapped
    double *tux, *tuy, *tuz;   // new orientation, normalised
    double *tdU;               // colloid-term change
    double *tlu;               // log of the Metropolis draw
    float *tdx, *tdy, *tdz;    // displacement
    unsigned char *thard;      // 0 evaluate, 1 colloid hard-core reject, 3 leaves its cell (rejected)
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
