// lcmc_trial.cuh - the trial move of one particle (translation + rotation).
#pragma once
#include "lcmc_gb.cuh"
#include "lcmc_internal.h"
#include "lcmc_rng.cuh"

namespace lcmc {

// Coordinate relative to a cell origin o, folded by whole periods into the
// window of the stencil cell it belongs to (centre cexp = (d + 1/2) w
// for stencil offset d).  A stored coordinate may lie on either side of the
// shifted periodic seam (cells that straddle it, or particles that crossed it
// earlier in the sweep); the fold is exact because every particle stays within
// w/2 + max_displacement/2 of its cell centre and w <= L/4.
__device__ __forceinline__ double fold_rel(double x, double o, double cexp, double L, double invL)
{
    const double r = x - o;
    return r - L * rint((r - cexp) * invL);
}

// Checkerboard rule for detailed balance: a trial translation that carries a
// particle out of the cell it was binned into at the start of the sweep is
// rejected without an energy evaluation.  Within a sweep the cell of every
// particle then stays fixed, so the cells' contents and the order of the
// attempts do not depend on the moves made (a move that crossed a cell face
// would change both, and the sweep would no longer leave the Boltzmann
// distribution invariant); the random grid shift of every sweep keeps the
// chain ergodic.  The same rule as parallel hard-particle MC on GPUs
// (Anderson et al., J. Comput. Phys. 254 (2013) 27).  The reference's
// random-sequential schedule (MCnptColloid.c:2474-2598) needs no such rule.
// (cx, cy, cz): the cell; ro: the position at the sweep's start; dsp: the
// unwrapped displacement.  Rounded operations throughout, so every kernel and
// the CPU oracle decide alike.
__device__ __forceinline__ bool leaves_cell(const Replica &p, int cx, int cy, int cz, const double ro[3],
                                            const double dsp[3])
{
    const int c[3] = {cx, cy, cz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double o = __dadd_rn(p.shift[a], __dmul_rn((double)c[a], p.w[a]));
        const double r = __dsub_rn(ro[a], o);
        const double k = rint(__dmul_rn(__dsub_rn(r, __dmul_rn(0.5, p.w[a])), __ddiv_rn(1.0, p.L[a])));
        const double rel = __dsub_rn(r, __dmul_rn(p.L[a], k));
        const double nr = __dadd_rn(rel, dsp[a]);
        if (!(nr >= 0.0 && nr < p.w[a])) return true;
    }
    return false;
}

// FP32 unit orientation of an FP64 orientation, with explicitly rounded FP64
// operations (no contraction into FMA, whatever the file's flags), so every
// kernel that forms it gets the same bits: the FP32 state copy written by the
// gather and by the phase write-back, read by the FP32-pair volume screen.
__device__ __forceinline__ void unit_f32(double x, double y, double z, float &ux, float &uy, float &uz)
{
    const double n2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
    const double in = __ddiv_rn(1.0, __dsqrt_rn(n2));
    ux = (float)__dmul_rn(x, in);
    uy = (float)__dmul_rn(y, in);
    uz = (float)__dmul_rn(z, in);
}

// apply_pbc (MCnptColloid.c:2420-2430): a single +-L fold per axis.
__device__ __forceinline__ void apply_pbc(double r[3], const double L[3])
{
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (r[a] > L[a]) r[a] -= L[a];
        else if (r[a] < 0.0) r[a] += L[a];
    }
}

// Trial move of attempt_monte_carlo_move (MCnptColloid.c:2502-2551) with
// Philox draws in place of rand():
//   r' = r + d (u - 1/2) per axis (d = max_displacement, full width), wrapped;
//   colloid hard core: reject without energy evaluation if |r' - C|^2 <= R^2;
//   u' = normalise(u + max_rotation v), v a Marsaglia point on the sphere;
//        the old orientation is kept if |u + max_rotation v|^2 <= 1e-12.
// Returns 0 on a hard-core reject (en = eo then).  dsp receives the
// unwrapped displacement, *u_acc the Metropolis draw.
__device__ __forceinline__ int make_trial(const Replica &p, uint32_t id, const double ro[3], const double eo[3],
                                          double rn[3], double en[3], double dsp[3], double *u_acc)
{
    U4 m = draw(p.key, id, p.sweep, TAG_MOVE);
    const double d = p.k.max_disp;
    dsp[0] = d * (u01(m.x) - 0.5);
    dsp[1] = d * (u01(m.y) - 0.5);
    dsp[2] = d * (u01(m.z) - 0.5);
    rn[0] = ro[0] + dsp[0];
    rn[1] = ro[1] + dsp[1];
    rn[2] = ro[2] + dsp[2];
    *u_acc = u01(m.w);
    apply_pbc(rn, p.L);
    en[0] = eo[0];
    en[1] = eo[1];
    en[2] = eo[2];
    double c[3];
    double r2 = dist_fold(rn[0], rn[1], rn[2], 0.5 * p.L[0], 0.5 * p.L[1], 0.5 * p.L[2], p.L, c);
    if (!(r2 > p.k.coll_R * p.k.coll_R)) return 0;
    double v[3];
    sphere_point(p.key, id, p.sweep, v);
    const double a = p.k.max_rot;
    en[0] = a * v[0] + eo[0];
    en[1] = a * v[1] + eo[1];
    en[2] = a * v[2] + eo[2];
    double n2 = en[0] * en[0] + en[1] * en[1] + en[2] * en[2];
    if (n2 <= 1e-12) {
        en[0] = eo[0];
        en[1] = eo[1];
        en[2] = eo[2];
    } else {
        double nr = __dsqrt_rn(n2);
        en[0] /= nr;
        en[1] /= nr;
        en[2] /= nr;
    }
    return 1;
}

} // namespace lcmc
