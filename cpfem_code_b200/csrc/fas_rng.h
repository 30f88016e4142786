/*
 * fas_rng.h -- counter-based uniform deviate for the twin trigger.
 *
 * The reference draws RANDOM_NUMBER in sequential Gauss-point order inside
 * SLPINI (src/fasolt/crys-cons.f90:169), which no parallel code can
 * reproduce.  Here the deviate is a pure function of (seed, GP, increment,
 * global Newton iteration, CPSTRS iteration, slip system), built from the
 * SplitMix64 finaliser (Steele, Lea & Flood, "Fast splittable pseudorandom
 * number generators", OOPSLA 2014).  For twinprob in {0, 1} the trigger is
 * deterministic and identical to the reference, because RANDOM_NUMBER and
 * this deviate both lie in [0, 1).
 */
#ifndef FAS_RNG_H
#define FAS_RNG_H

#include "fas_flops.h"

FAS_HD unsigned long long fas_mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

FAS_HD double fas_twin_u01(unsigned long long seed, int gp, int inc, int nit,
                           int cpit, int sys)
{
    unsigned long long k = fas_mix64(seed ^ fas_mix64((unsigned long long)gp));
    unsigned long long c = ((unsigned long long)(unsigned)inc << 40)
                         ^ ((unsigned long long)(unsigned)nit << 24)
                         ^ ((unsigned long long)(unsigned)cpit << 8)
                         ^ (unsigned long long)(unsigned)sys;
    k = fas_mix64(k ^ c);
    return (double)(k >> 11) * (1.0 / 9007199254740992.0);
}

#endif /* FAS_RNG_H */
