// lcmc_gb.cuh - Gay-Berne pair and colloid-rod terms for the kernels.
#pragma once
#include "lcmc_internal.h"

namespace lcmc {

// ---------------------------------------------------------------------------
// FP64, reference order of operations (g_omega + pij_GB, MCnptColloid.c:2607-
// 2681, per-pair preamble of GBij_PosMod, 1573-1591).  Compiled without FMA
// contraction in the FP64 kernel so that it matches the CPU oracle bit for bit.
// ---------------------------------------------------------------------------

__device__ __forceinline__ double ipow_d(double x, int code, double e)
{
    return code == 1 ? x : (code == 2 ? x * x : pow(x, e));
}

__device__ __forceinline__ double g_omega_d(double eiej, double amasb2, double amenb2, double omega)
{
    double ome = omega * eiej;
    double gmas = amasb2 / (1.0 + ome);
    double gmen = amenb2 / (1.0 - ome);
    return 1.0 - 0.50 * omega * (gmas + gmen);
}

// One-fold minimum image of d = r_j - r_i (compute_distance_sq, MCnptColloid.c:2690-2721).
__device__ __forceinline__ double dist_fold(double xi, double yi, double zi, double xj, double yj, double zj,
                                            const double L[3], double d[3])
{
    // rounded operations throughout, so the result is the same in every
    // translation unit whatever its contraction setting
    d[0] = __dsub_rn(xj, xi);
    d[1] = __dsub_rn(yj, yi);
    d[2] = __dsub_rn(zj, zi);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double h = __dmul_rn(0.5, L[a]);
        if (d[a] > h) d[a] = __dsub_rn(d[a], L[a]);
        else if (d[a] < -h) d[a] = __dadd_rn(d[a], L[a]);
    }
    const double xs = __dmul_rn(d[0], d[0]), ys = __dmul_rn(d[1], d[1]), zs = __dmul_rn(d[2], d[2]);
    return __dadd_rn(__dadd_rn(xs, ys), zs);
}

// Pair term for r^2 < rc^2 (the caller tests the cutoff), orientations of any norm.
__device__ __forceinline__ double pair_exact(const GBConsts &k, double r2, const double dr[3], const double ei[3],
                                             const double ej[3])
{
    double rij = __dsqrt_rn(r2);
    double irij = 1.0 / rij;
    double ei2 = ei[0] * ei[0] + ei[1] * ei[1] + ei[2] * ei[2];
    double ej2 = ej[0] * ej[0] + ej[1] * ej[1] + ej[2] * ej[2];
    double iei = 1.0 / __dsqrt_rn(ei2), iej = 1.0 / __dsqrt_rn(ej2);
    double eiej = iei * iej * (ei[0] * ej[0] + ei[1] * ej[1] + ei[2] * ej[2]);
    double eirij = irij * iei * (dr[0] * ei[0] + dr[1] * ei[1] + dr[2] * ei[2]);
    double ejrij = irij * iej * (dr[0] * ej[0] + dr[1] * ej[1] + dr[2] * ej[2]);
    double amasb = eirij + ejrij, amenb = eirij - ejrij;
    double amab2 = amasb * amasb, ameb2 = amenb * amenb;
    double eps1 = 1.0 / __dsqrt_rn(1.0 - k.chi_sq * eiej * eiej);
    double ctep1 = ipow_d(eps1, k.nu_code, k.nu);
    double eps2 = g_omega_d(eiej, amab2, ameb2, k.chi_prime);
    double ctep2 = ipow_d(eps2, k.mu_code, k.mu);
    double s_chi = g_omega_d(eiej, amab2, ameb2, k.chi);
    double sigma = k.sigma0 / __dsqrt_rn(s_chi);
    double distreal = (rij - sigma + k.sigma0);
    if (distreal < 0.001) return 1000000000.0; // MCnptColloid.c:2670
    double erre = k.sigma0 / distreal;
    double erre2 = erre * erre;
    double erre6 = erre2 * erre2 * erre2;
    double epsil = ctep1 * ctep2;
    return k.four_eps0 * epsil * erre6 * (erre6 - 1.0);
}

// FP64 pair term for total energies (tot_ene and the NPT volume move): the
// function of pair_exact with fewer divisions and square roots (reciprocal
// square roots; the two fractions of each g_omega over one denominator,
//   g(w) = 1 - (w/2) [s+^2 (1 - w c) + s-^2 (1 + w c)] / (1 - w^2 c^2)),
// 3 divisions and 5 reciprocal square roots in place of 10 divisions and 5
// square roots.  A few ulp from pair_exact, so totals agree with it to about
// 1e-15 relative, not bit for bit.
__device__ __forceinline__ double pair_energy64(const GBConsts &k, double r2, const double dr[3], const double ei[3],
                                                const double ej[3])
{
    const double irij = rsqrt(r2);
    const double rij = r2 * irij;
    const double iei = rsqrt(ei[0] * ei[0] + ei[1] * ei[1] + ei[2] * ei[2]);
    const double iej = rsqrt(ej[0] * ej[0] + ej[1] * ej[1] + ej[2] * ej[2]);
    const double c = iei * iej * (ei[0] * ej[0] + ei[1] * ej[1] + ei[2] * ej[2]);
    const double a = irij * iei * (dr[0] * ei[0] + dr[1] * ei[1] + dr[2] * ei[2]);
    const double b = irij * iej * (dr[0] * ej[0] + dr[1] * ej[1] + dr[2] * ej[2]);
    const double sp2 = (a + b) * (a + b), sm2 = (a - b) * (a - b);
    const double eps1 = rsqrt(1.0 - k.chi_sq * c * c);
    const double ctep1 = ipow_d(eps1, k.nu_code, k.nu);
    const double wp = k.chi_prime * c, wc = k.chi * c;
    const double eps2 = 1.0 - 0.5 * k.chi_prime * (sp2 * (1.0 - wp) + sm2 * (1.0 + wp)) / (1.0 - wp * wp);
    const double ctep2 = ipow_d(eps2, k.mu_code, k.mu);
    const double s_chi = 1.0 - 0.5 * k.chi * (sp2 * (1.0 - wc) + sm2 * (1.0 + wc)) / (1.0 - wc * wc);
    const double distreal = rij - k.sigma0 * rsqrt(s_chi) + k.sigma0;
    if (distreal < 0.001) return 1000000000.0; // MCnptColloid.c:2670
    const double erre = k.sigma0 / distreal;
    const double erre2 = erre * erre;
    const double erre6 = erre2 * erre2 * erre2;
    return k.four_eps0 * (ctep1 * ctep2) * erre6 * (erre6 - 1.0);
}

// pair_energy64 for mu = 2, nu = 1, sigma0 = 1 (no general powers): the FP32
// kernel's FP64 fallback for cells with overlapping pairs.
__device__ __forceinline__ double pair_energy64_21(const GBConsts &k, double r2, const double dr[3], const double ei[3],
                                                   const double ej[3])
{
    const double irij = rsqrt(r2);
    const double rij = r2 * irij;
    const double iei = rsqrt(ei[0] * ei[0] + ei[1] * ei[1] + ei[2] * ei[2]);
    const double iej = rsqrt(ej[0] * ej[0] + ej[1] * ej[1] + ej[2] * ej[2]);
    const double c = iei * iej * (ei[0] * ej[0] + ei[1] * ej[1] + ei[2] * ej[2]);
    const double a = irij * iei * (dr[0] * ei[0] + dr[1] * ei[1] + dr[2] * ei[2]);
    const double b = irij * iej * (dr[0] * ej[0] + dr[1] * ej[1] + dr[2] * ej[2]);
    const double sp2 = (a + b) * (a + b), sm2 = (a - b) * (a - b);
    const double eps1 = rsqrt(1.0 - k.chi_sq * c * c);
    const double wp = k.chi_prime * c, wc = k.chi * c;
    const double eps2 = 1.0 - 0.5 * k.chi_prime * (sp2 * (1.0 - wp) + sm2 * (1.0 + wp)) / (1.0 - wp * wp);
    const double s_chi = 1.0 - 0.5 * k.chi * (sp2 * (1.0 - wc) + sm2 * (1.0 + wc)) / (1.0 - wc * wc);
    const double distreal = rij - rsqrt(s_chi) + 1.0;
    if (distreal < 0.001) return 1000000000.0; // MCnptColloid.c:2670
    const double erre = 1.0 / distreal;
    const double erre2 = erre * erre;
    const double erre6 = erre2 * erre2 * erre2;
    return k.four_eps0 * (eps1 * eps2 * eps2) * erre6 * (erre6 - 1.0);
}

// GBCollRod (MCnptColloid.c:1758-1854): colloid of radius R at the box centre.
__device__ __forceinline__ double colloid_rod(const GBConsts &k, const double ri[3], const double ei[3],
                                              const double L[3])
{
    double C[3] = {0.5 * L[0], 0.5 * L[1], 0.5 * L[2]};
    double d[3];
    double d_nc = __dsqrt_rn(dist_fold(ri[0], ri[1], ri[2], C[0], C[1], C[2], L, d));
    double dij = d_nc - k.coll_R;
    if (d_nc <= 1e-12) return 1.0e8;
    if (dij > k.coll_cutoff) return 0.0;
    double px = ri[0] - C[0], py = ri[1] - C[1], pz = ri[2] - C[2];
    double rhx = px / d_nc, rhy = py / d_nc, rhz = pz / d_nc;
    double ct = rhx * ei[0] + rhy * ei[1] + rhz * ei[2];
    if (ct > 1.0) ct = 1.0;
    if (ct < -1.0) ct = -1.0;
    double sin2 = 1.0 - ct * ct;
    double s0 = k.sigma0;
    double denom = 1.0 - k.chi, numer = 1.0 - k.chi * sin2;
    if (denom <= 0.0) denom = 1e-12;
    if (numer <= 1e-12) numer = 1e-12;
    double sigma_CR = s0 * __dsqrt_rn(numer / denom);
    double denom_eps = 1.0 - k.chi_prime * sin2, numer_eps = 1.0 - k.chi_prime;
    if (denom_eps <= 1e-12) denom_eps = 1e-12;
    double eps_CR = k.kappa_prime * ipow_d(numer_eps / denom_eps, k.mu_code, k.mu);
    double x = dij - sigma_CR + s0;
    if (x <= 1e-10) return 1.0e8;
    double s3 = s0 * s0 * s0, s9 = s3 * s3 * s3;
    double x2 = x * x, x3 = x2 * x, x8 = x3 * x3 * x2, x9 = x8 * x;
    double term1 = s9 / (45.0 * x9);
    double term2 = s3 / (6.0 * x3);
    double term3 = s9 / (40.0 * d_nc * x8);
    double term4 = s3 / (4.0 * d_nc * x2);
    return eps_CR * (term1 - term2 - term3 + term4);
}

// ---------------------------------------------------------------------------
// FP32 pair term for the FP32 kernel.  Unit orientations (normalised when a
// move is accepted), d = r_j - r_i already unwrapped, r^2 given.  The two
// g_omega terms share one denominator:
//   g(w) = 1 - (w/2) [(s^2 + d^2) - w c (s^2 - d^2)] / (1 - w^2 c^2)
// with s, d = (e_i.r +- e_j.r)/r and c = e_i.e_j; 1/(1 - chi^2 c^2) = eps1^2.
// mu = 2 and nu = 1 are specialised (the general case uses powf).
// ---------------------------------------------------------------------------
struct FastK {
    float rc2, chi, chi_sq, chip, chip_sq, sigma0, four_eps0, half_chi, half_chip;
    float big; // largest pair-term magnitude the FP32 kernel keeps (larger: the cell runs in FP64)
    int mu_code, nu_code;
    float mu, nu;
};

// mu = 2, nu = 1, sigma0 = 1 (the Gay-Berne parametrisation of every workload
// here), without the general branches.
__device__ __forceinline__ float pair_fast_21(const FastK &k, float dx, float dy, float dz, float r2, float eix,
                                              float eiy, float eiz, float ejx, float ejy, float ejz)
{
    float ir = rsqrtf(r2);
    float r = r2 * ir;
    float a = (dx * eix + dy * eiy + dz * eiz) * ir;
    float b = (dx * ejx + dy * ejy + dz * ejz) * ir;
    float c = eix * ejx + eiy * ejy + eiz * ejz;
    float s = a + b, d = a - b;
    float s2 = s * s, d2 = d * d;
    float sp = s2 + d2, sm = s2 - d2;
    float c2 = c * c;
    float eps1 = rsqrtf(1.0f - k.chi_sq * c2);
    float s_chi = 1.0f - k.half_chi * (sp - k.chi * c * sm) * (eps1 * eps1);
    float inv2 = __fdividef(1.0f, 1.0f - k.chip_sq * c2);
    float eps2 = 1.0f - k.half_chip * (sp - k.chip * c * sm) * inv2;
    float dr = r - rsqrtf(s_chi) + 1.0f;
    float R = __fdividef(1.0f, dr);
    float R2 = R * R;
    float R6 = R2 * R2 * R2;
    float v = k.four_eps0 * (eps1 * eps2 * eps2) * R6 * (R6 - 1.0f);
    return dr < 0.001f ? 1.0e9f : v;
}

// FP32 constants of a system for the FP32 pair term.
__device__ __forceinline__ FastK fast_consts(const GBConsts &k)
{
    FastK K;
    K.rc2 = k.f_rc2;
    K.chi = k.f_chi;
    K.chi_sq = k.f_chi_sq;
    K.chip = k.f_chip;
    K.chip_sq = k.f_chip_sq;
    K.sigma0 = k.f_sigma0;
    K.four_eps0 = k.f_4eps0;
    K.half_chi = k.f_half_chi;
    K.half_chip = k.f_half_chip;
    K.big = k.f_big;
    K.mu_code = k.mu_code;
    K.nu_code = k.nu_code;
    K.mu = (float)k.mu;
    K.nu = (float)k.nu;
    return K;
}

template <bool SPEC21>
__device__ __forceinline__ float pair_fast_t(const FastK &k, float dx, float dy, float dz, float r2, float eix,
                                             float eiy, float eiz, float ejx, float ejy, float ejz);

__device__ __forceinline__ float pair_fast(const FastK &k, float dx, float dy, float dz, float r2, float eix,
                                           float eiy, float eiz, float ejx, float ejy, float ejz)
{
    float ir = rsqrtf(r2);
    float r = r2 * ir;
    float a = (dx * eix + dy * eiy + dz * eiz) * ir;
    float b = (dx * ejx + dy * ejy + dz * ejz) * ir;
    float c = eix * ejx + eiy * ejy + eiz * ejz;
    float s = a + b, d = a - b;
    float s2 = s * s, d2 = d * d;
    float sp = s2 + d2, sm = s2 - d2;
    float c2 = c * c;
    float eps1 = rsqrtf(1.0f - k.chi_sq * c2);
    float inv1 = eps1 * eps1;
    float s_chi = 1.0f - k.half_chi * (sp - k.chi * c * sm) * inv1;
    float inv2 = __fdividef(1.0f, 1.0f - k.chip_sq * c2);
    float eps2 = 1.0f - k.half_chip * (sp - k.chip * c * sm) * inv2;
    float e1 = k.nu_code == 1 ? eps1 : (k.nu_code == 2 ? eps1 * eps1 : __powf(eps1, k.nu));
    float e2 = k.mu_code == 2 ? eps2 * eps2 : (k.mu_code == 1 ? eps2 : __powf(eps2, k.mu));
    float sigma = k.sigma0 * rsqrtf(s_chi);
    float dr = r - sigma + k.sigma0;
    float R = __fdividef(k.sigma0, dr);
    float R2 = R * R;
    float R6 = R2 * R2 * R2;
    float v = k.four_eps0 * (e1 * e2) * R6 * (R6 - 1.0f);
    return dr < 0.001f ? 1.0e9f : v;
}

} // namespace lcmc

namespace lcmc {
template <>
__device__ __forceinline__ float pair_fast_t<true>(const FastK &k, float dx, float dy, float dz, float r2, float eix,
                                                   float eiy, float eiz, float ejx, float ejy, float ejz)
{
    return pair_fast_21(k, dx, dy, dz, r2, eix, eiy, eiz, ejx, ejy, ejz);
}
template <>
__device__ __forceinline__ float pair_fast_t<false>(const FastK &k, float dx, float dy, float dz, float r2, float eix,
                                                    float eiy, float eiz, float ejx, float ejy, float ejz)
{
    return pair_fast(k, dx, dy, dz, r2, eix, eiy, eiz, ejx, ejy, ejz);
}
} // namespace lcmc
