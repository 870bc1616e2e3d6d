// lcmc_rng.cuh - counter-based random draws shared by host and device code.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11) replaces the reference's libc rand() (seeded by time(0),
// MCnptColloid.c:440, 800) so that every draw is a pure function of
// (seed, replica, sweep, particle id, purpose): host and device, and any launch
// order, see the same numbers.
//
// Counter layout: {particle id | SWEEP_ID, sweep lo, sweep hi, tag}.
// Arithmetic here is plain IEEE double (+ - * / sqrt); translation units that
// must be bit-identical to the host are compiled without contraction.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define LCMC_HD __host__ __device__ __forceinline__
#else
#define LCMC_HD inline
#endif

namespace lcmc {

constexpr uint32_t TAG_MOVE = 0u;      // 3 displacement draws + 1 acceptance draw
constexpr uint32_t TAG_SPHERE = 1u;    // 1..16: Marsaglia pairs, two per call
constexpr uint32_t TAG_SHIFT = 0x100u; // per-sweep grid shift
constexpr uint32_t TAG_COLOUR = 0x101u;// per-sweep colour order (two calls)
constexpr uint32_t TAG_VOLUME = 0x103u;// per-sweep volume move
constexpr uint32_t TAG_COLOUR_EXT = 0x110u; // 0x110..0x114: colour order beyond 8 colours (fine grid)
constexpr uint32_t TAG_INIT = 0x200u;  // initial orientations (cone mode)
constexpr uint32_t SWEEP_ID = 0xFFFFFFFFu;
constexpr uint64_t INIT_SWEEP = 0xFFFFFFFFFFFFFFFFull;

struct U4 {
    uint32_t x, y, z, w;
};

LCMC_HD U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
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
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
    }
    return U4{c0, c1, c2, c3};
}

LCMC_HD U4 draw(const uint32_t key[2], uint32_t id, uint64_t sweep, uint32_t tag)
{
    return philox4x32_10(id, (uint32_t)sweep, (uint32_t)(sweep >> 32), tag, key[0], key[1]);
}

// uniform on (0, 1): (x + 1/2) 2^-32, exact in double
LCMC_HD double u01(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

// Philox key of a system: its rng_seed alone, so that a system reproduces the
// same trajectory whether it runs alone or as one replica of a batch (the
// batch caller gives every replica its own seed).
LCMC_HD void seed_key(uint64_t seed, uint32_t key[2])
{
    key[0] = (uint32_t)seed;
    key[1] = (uint32_t)(seed >> 32);
}

// Natural log on (0, 1], written for this library so that host and device
// agree bit for bit: u = m 2^e, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(t)
// with t = (m - 1)/(m + 1), odd Taylor series of atanh to t^21, ln 2 split in
// a 32-bit head (e * head exact) and a tail.  |error| < 3e-16 relative.
LCMC_HD double log_unit(double u)
{
    // exponent/mantissa split of a positive normal double by its bits
    union {
        double d;
        uint64_t b;
    } v;
    v.d = u;
    int e = (int)((v.b >> 52) & 0x7FF) - 1022;
    v.b = (v.b & 0x800FFFFFFFFFFFFFull) | 0x3FE0000000000000ull; // m in [0.5, 1)
    double m = v.d;
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

// e^x - 1 for |x| <= 1.5: Taylor series to x^30 in nested form.
LCMC_HD double expm1_small(double x)
{
    double s = 1.0;
    for (int k = 30; k >= 2; k--) s = 1.0 + s * x / (double)k;
    return x * s;
}

// Marsaglia (1972) point on the unit sphere, the method of the reference's
// pto_ransphr (MCnptColloid.c:3050-3078), in double, from Philox pairs.
LCMC_HD void sphere_point(const uint32_t key[2], uint32_t id, uint64_t sweep, double v[3])
{
    for (int t = 0; t < 32; t++) {
        U4 o = draw(key, id, sweep, TAG_SPHERE + (uint32_t)(t >> 1));
        uint32_t a = (t & 1) ? o.z : o.x;
        uint32_t b = (t & 1) ? o.w : o.y;
        double x1 = 1.0 - 2.0 * u01(a);
        double x2 = 1.0 - 2.0 * u01(b);
        double s = x1 * x1 + x2 * x2;
        if (s < 1.0) {
#ifdef __CUDA_ARCH__
            double q = __dsqrt_rn(1.0 - s);
#else
            double q = sqrt(1.0 - s);
#endif
            v[0] = 2.0 * x1 * q;
            v[1] = 2.0 * x2 * q;
            v[2] = 1.0 - 2.0 * s;
            return;
        }
    }
    v[0] = 0.0;
    v[1] = 0.0;
    v[2] = 1.0;
}

} // namespace lcmc
