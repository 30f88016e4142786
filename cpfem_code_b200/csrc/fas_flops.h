/*
 * fas_flops.h -- algorithmic operation counts of the crystal-plasticity
 * Gauss-point update (DSTRSS -> CPSTRS -> SLPINI / SLPFTA / PLASTC).
 *
 * Both the device kernels and the CPU checker accumulate these formulas from
 * their own iteration counts and active-set sizes, so equal totals also show
 * that both took the same iteration path.  Convention: every add, subtract,
 * multiply, divide, compare-free sqrt/exp/log/pow counts as one operation;
 * a multiply-add counts as two.  Transcendentals are therefore counted once,
 * so the figure is a lower bound on the FP64 pipe work.  Every formula is an
 * integer, so sums of them are exact in double precision whatever the
 * order or contraction of the arithmetic.
 */
#ifndef FAS_FLOPS_H
#define FAS_FLOPS_H

#ifdef __CUDACC__
#define FAS_HD __host__ __device__ __forceinline__
#else
#define FAS_HD inline
#endif

/* LU without pivoting of an n x n matrix (FACTOR, crys-cons.f90:244-269):
 * sum over pivots of (n-1-k) divisions and (n-1-k)^2 multiply-adds. */
FAS_HD double fas_ops_lu(int n)
{
    const long long m = n > 0 ? n - 1 : 0;
    return (double)(m * (m + 1) / 2 + m * (m + 1) * (2 * m + 1) / 3);
}
/* forward + back substitution (SOLVER, crys-cons.f90:283-309). */
FAS_HD double fas_ops_solve(int n) { return (double)(2LL * n * n - n); }

/* Work done once per plastic GP update outside the outer loop:
 * ELASTC (21 entries x 18 products/sums), TENS_ROT, CTMATRX/BTMATRX (ns
 * systems x 36), ECHROT (6 ns + 30), the 6 solves of chi = djac^-1 and the
 * symmetrisation. */
FAS_HD double fas_ops_cp_fixed(int ns)
{
    return 21.0 * 60.0 + 60.0 + 21.0 + 36.0 * ns + (6.0 * ns + 30.0)
         + 6.0 * fas_ops_solve(6) + 36.0 + 2.0 * 18.0;
}

/* One inner (SLPFTA) Newton iteration on nsa active of ns systems:
 * PLASTC (3 transcendentals + 8 ops per system, 4 ns^2 hardening products,
 * nsa^2 log-hardening entries), completion of ah, LU, residual (6 per active
 * incl. pow/log), its norm, the solve and the exponential update. */
FAS_HD double fas_ops_inner(int ns, int nsa)
{
    return (11.0 * ns + 4.0 * ns * ns + 3.0 * nsa * nsa)
         + (2.0 * nsa * nsa + nsa) + fas_ops_lu(nsa)
         + 6.0 * nsa + 2.0 * nsa + fas_ops_solve(nsa) + 4.0 * nsa;
}

/* One outer (CPSTRS) iteration excluding its inner iterations: resolved
 * shear (12 ns), SLPINI (6 ns), two SCALE_IT passes (4 ns), the final PLASTC
 * and X completion, plastic strain (12 ns), strain error (84), LU of X,
 * djac = b X^-1 b^T (6 solves + 36 dots of nsa), + S, 6x6 LU + solve,
 * two von Mises measures and the damped update. */
FAS_HD double fas_ops_outer(int ns, int nsa)
{
    return 12.0 * ns + 6.0 * ns + 4.0 * ns
         + (11.0 * ns + 4.0 * ns * ns + 3.0 * nsa * nsa) + (3.0 * nsa * nsa + 3.0 * nsa)
         + 12.0 * ns + 84.0 + fas_ops_lu(nsa)
         + 6.0 * fas_ops_solve(nsa) + 36.0 * 2.0 * nsa + 36.0
         + fas_ops_lu(6) + fas_ops_solve(6) + 2.0 * 18.0 + 14.0;
}

/* Elastic-branch update: ELASTC, TENS_ROT, the 6x6 inverse and chi*de. */
FAS_HD double fas_ops_elastic(void)
{
    return 21.0 * 60.0 + 60.0 + fas_ops_lu(6) + 6.0 * fas_ops_solve(6) + 72.0;
}

#endif /* FAS_FLOPS_H */
