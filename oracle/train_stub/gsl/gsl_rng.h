// Stand-in for the GSL random number generators the reference's training
// library uses (gsl_rng_mt19937 and gsl_rng_taus with gsl_rng_alloc / set /
// get / uniform / uniform_int / free), written for this project and used
// ONLY to compile the reference's nnp-train into the test oracle.  The two
// generators are restated from their published algorithms:
//  * MT19937: M. Matsumoto and T. Nishimura, ACM TOMACS 8 (1998) 3-30, with
//    the authors' 2002 initialisation; seed 0 means 4357 (GSL's default).
//  * taus: P. L'Ecuyer, Math. Comp. 65 (1996) 203-213, the three-component
//    combined Tausworthe generator; components seeded by s -> 69069 s mod
//    2^32 (seed 0 means 1) and six outputs discarded.
// uniform() = get() / 2^32; uniform_int(n) bins the range into n bins of
// floor((2^32 - 1) / n) outputs and redraws past the last full bin.
#ifndef N2P2B200_GSL_RNG_STUB_H
#define N2P2B200_GSL_RNG_STUB_H

#include <cstddef>
#include <stdexcept>

struct gsl_rng_type
{
    const char* name;
    int         kind;   // 0 mt19937, 1 taus
};

struct gsl_rng
{
    const gsl_rng_type* type;
    unsigned long       mt[624];
    int                 mti;
    unsigned long       s1, s2, s3;
};

static const gsl_rng_type n2p2b200_gsl_mt19937 = {"mt19937", 0};
static const gsl_rng_type n2p2b200_gsl_taus = {"taus", 1};
static const gsl_rng_type* gsl_rng_mt19937 = &n2p2b200_gsl_mt19937;
static const gsl_rng_type* gsl_rng_taus = &n2p2b200_gsl_taus;

inline unsigned long n2p2b200_taus_get(gsl_rng* r)
{
    const unsigned long M = 0xffffffffUL;
    r->s1 = (((r->s1 & 4294967294UL) << 12) & M) ^ ((((r->s1 << 13) & M) ^ r->s1) >> 19);
    r->s2 = (((r->s2 & 4294967288UL) << 4) & M) ^ ((((r->s2 << 2) & M) ^ r->s2) >> 25);
    r->s3 = (((r->s3 & 4294967280UL) << 17) & M) ^ ((((r->s3 << 3) & M) ^ r->s3) >> 11);
    return r->s1 ^ r->s2 ^ r->s3;
}

inline unsigned long n2p2b200_mt_get(gsl_rng* r)
{
    const int N = 624, K = 397;
    if (r->mti >= N)
    {
        for (int i = 0; i < N; ++i)
        {
            const unsigned long y = (r->mt[i] & 0x80000000UL) | (r->mt[(i + 1) % N] & 0x7fffffffUL);
            r->mt[i] = r->mt[(i + K) % N] ^ (y >> 1) ^ ((y & 1UL) ? 0x9908b0dfUL : 0UL);
        }
        r->mti = 0;
    }
    unsigned long y = r->mt[r->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680UL;
    y ^= (y << 15) & 0xefc60000UL;
    y ^= y >> 18;
    return y & 0xffffffffUL;
}

inline void gsl_rng_set(gsl_rng* r, unsigned long s)
{
    if (r->type->kind == 0)
    {
        if (s == 0) s = 4357;
        r->mt[0] = s & 0xffffffffUL;
        for (int i = 1; i < 624; ++i)
            r->mt[i] = (1812433253UL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (unsigned long)i) & 0xffffffffUL;
        r->mti = 624;
    }
    else
    {
        if (s == 0) s = 1;
        r->s1 = (69069UL * s) & 0xffffffffUL;
        r->s2 = (69069UL * r->s1) & 0xffffffffUL;
        r->s3 = (69069UL * r->s2) & 0xffffffffUL;
        for (int k = 0; k < 6; ++k) n2p2b200_taus_get(r);
    }
}

inline gsl_rng* gsl_rng_alloc(const gsl_rng_type* t)
{
    gsl_rng* r = new gsl_rng();
    r->type = t;
    gsl_rng_set(r, 0);
    return r;
}

inline void gsl_rng_free(gsl_rng* r) { delete r; }

inline unsigned long gsl_rng_get(const gsl_rng* r)
{
    gsl_rng* m = const_cast<gsl_rng*>(r);
    return r->type->kind == 0 ? n2p2b200_mt_get(m) : n2p2b200_taus_get(m);
}

inline double gsl_rng_uniform(const gsl_rng* r) { return gsl_rng_get(r) / 4294967296.0; }

inline unsigned long gsl_rng_uniform_int(const gsl_rng* r, unsigned long n)
{
    const unsigned long range = 0xffffffffUL;
    if (n == 0 || n > range) throw std::runtime_error("gsl stub: invalid n");
    const unsigned long scale = range / n;
    unsigned long k;
    do k = gsl_rng_get(r) / scale;
    while (k >= n);
    return k;
}

#endif
