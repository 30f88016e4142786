// fas_device.cuh -- device routines of the crystal-plasticity Gauss-point
// update and the brick kinematics, in FP64, one thread per Gauss point.
//
// Each function restates one routine of gabortimar/CPFEM_code src/fasolt
// (cited per function).  The module-global scratch of FAS_CPL
// (fas-com-mod.f90:62-66: tau, gam, s0, s1, ah, isa, nsa, b, rot, wks) is
// private per thread here (struct CpScratch), which is what makes the
// Gauss-point loop parallel.  NS is the compile-time bound on slip systems
// of the instantiation (12 for FCC, 32 for HCP sets, 60 = maxss).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fas_flops.h"
#include "fas_rng.h"

namespace fasdev {

constexpr int MAXSS = 60;

// Material tables on the device (FAS_CPL, fas-com-mod.f90:68-78), FP64.
struct DevMat {
    int nmatl;
    int ns[12];
    double amax[12];            // MAXVAL(ampar(1,1:ns)) per material (SLPFTA conv)
    const double *e;            // [nmatl][9]
    const double *ssang;        // [nmatl][60]
    const double *ab, *an;      // [nmatl][60][3]
    const double *ampar;        // [nmatl][60][6]
    const double *sm;           // [nmatl][60*60], sm[i*ns+j] = smatrx(i,j)
    int twinlim;
    double twinprob;
    int tld, sld;               // per-material strides: systems of the per-system tables
                                // (MAXSS) and entries of sm (MAXSS^2); smaller in a
                                // shared-memory copy (stage_tables)
    int stage_t;                // > 0: constitutive kernels copy the tables into shared
                                // memory at this system stride (FAS_SMEM_TABLES builds)
};

struct DevCtrl {
    double toler, alpha, afactor, efix, smale, smalr;
    int maxit;
    int tangent;                // 1: consistent tangent at the converged stress
    unsigned long long seed;
    const int *nit_dev;         // set in a graph-launched NRITER: the Newton
                                // iteration number is *nit_dev + 1
};

// Gauss-point state, structure of arrays: field[k * ngps + g].
struct DevGp {
    int ngps, ldsv, ldsl;
    double *eps, *dep, *st, *ep, *ds, *de, *rt, *dr, *sv, *dsv, *srate, *cumslip;
    int *timestwinned, *twinsys;
    int *tflag;                 // set to 1 when any GP triggers a twin
    int *cp_iters;              // diagnostics of the last pass
    double *erepmd, *ops;
};

#ifndef FAS_SMEM_TABLES
#define FAS_SMEM_TABLES 0
#endif
#if FAS_SMEM_TABLES
// the tables may sit in shared memory: a generic load
__device__ __forceinline__ double ld_ro(const double *p) { return *p; }
#else
__device__ __forceinline__ double ld_ro(const double *p) { return __ldg(p); }
#endif

// Doubles of the shared-memory copy of nmatl materials' tables at a stride
// of t systems: e, ssang, ab, an, ampar and sm.
__host__ __device__ inline int staged_doubles(int nmatl, int t) { return nmatl * (9 + t * (13 + t)); }

// Copies the tables into shared memory (every thread of the CTA takes part;
// call before any thread leaves) and returns M with its pointers and strides
// on the copy.
__device__ __forceinline__ DevMat stage_tables(const DevMat &M, double *s)
{
    const int nm = M.nmatl, t = M.stage_t;
    double *e = s, *ss = e + 9 * nm, *ab = ss + nm * t, *an = ab + 3 * nm * t, *amp = an + 3 * nm * t,
           *sm = amp + 6 * nm * t;
    for (int i = threadIdx.x; i < 9 * nm; i += blockDim.x) e[i] = M.e[i];
    for (int i = threadIdx.x; i < nm * t; i += blockDim.x) ss[i] = M.ssang[(i / t) * MAXSS + i % t];
    for (int i = threadIdx.x; i < 3 * nm * t; i += blockDim.x) {
        const int m = i / (3 * t), r = i % (3 * t);
        ab[i] = M.ab[(size_t)m * MAXSS * 3 + r];
        an[i] = M.an[(size_t)m * MAXSS * 3 + r];
    }
    for (int i = threadIdx.x; i < 6 * nm * t; i += blockDim.x)
        amp[i] = M.ampar[(size_t)(i / (6 * t)) * MAXSS * 6 + i % (6 * t)];
    for (int i = threadIdx.x; i < nm * t * t; i += blockDim.x)
        sm[i] = M.sm[(size_t)(i / (t * t)) * MAXSS * MAXSS + i % (t * t)];
    __syncthreads();
    DevMat S = M;
    S.e = e;
    S.ssang = ss;
    S.ab = ab;
    S.an = an;
    S.ampar = amp;
    S.sm = sm;
    S.tld = t;
    S.sld = t * t;
    return S;
}

// FJ2VOM, src/fasolt/Sig_eps.f90:217-241
__device__ __forceinline__ double fj2vom(bool stress, const double *x)
{
    const double amult = stress ? 6.0 : 1.5;
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3;
        sum = sum + (x[i] - x[j]) * (x[i] - x[j]) + amult * x[i + 3] * x[i + 3];
    }
    return sqrt(sum / 4.5);
}

// SPOWER, src/fasolt/crys-cons.f90:210-230: signed power with clamps.
__device__ __forceinline__ double spower(double a, double b)
{
    const double aa = fabs(a);
    if (aa < 1.e-35) return 0.0;
    double sparg = b * log(aa);
    sparg = sparg < -80.0 ? -80.0 : (sparg > 80.0 ? 80.0 : sparg);
    return copysign(exp(sparg), a);
}

// FACTOR, src/fasolt/crys-cons.f90:244-269 (LU, no pivoting); w[i*LD+j].
template <int LD>
__device__ __forceinline__ int lu_factor(int n, double *w)
{
    for (int k = 0; k < n - 1; ++k) {
        const double pk = w[k * LD + k];
        if (pk == 0.0) return 1;
        for (int i = k + 1; i < n; ++i) {
            const double l = w[i * LD + k] / pk;
            w[i * LD + k] = l;
            for (int j = k + 1; j < n; ++j) w[i * LD + j] = w[i * LD + j] - l * w[k * LD + j];
        }
    }
    return w[(n - 1) * LD + (n - 1)] == 0.0 ? 1 : 0;
}

// SOLVER, src/fasolt/crys-cons.f90:283-309
template <int LD>
__device__ __forceinline__ void lu_solve(int n, const double *w, double *x)
{
    for (int i = 1; i < n; ++i) {
        double xi = x[i];
        for (int j = 0; j < i; ++j) xi = xi - w[i * LD + j] * x[j];
        x[i] = xi;
    }
    x[n - 1] = x[n - 1] / w[(n - 1) * LD + (n - 1)];
    for (int i = n - 2; i >= 0; --i) {
        double xi = x[i];
        for (int j = i + 1; j < n; ++j) xi = xi - w[i * LD + j] * x[j];
        x[i] = xi / w[i * LD + i];
    }
}

// The same factorisation and solve for an n x n matrix stored with row
// stride n (the active-set matrices: only nsa x nsa of them are live, and a
// packed copy touches far fewer cache lines than a fixed stride).
__device__ __forceinline__ int lu_factor_n(int n, double *w)
{
    for (int k = 0; k < n - 1; ++k) {
        const double pk = w[k * n + k];
        if (pk == 0.0) return 1;
        for (int i = k + 1; i < n; ++i) {
            const double l = w[i * n + k] / pk;
            w[i * n + k] = l;
            for (int j = k + 1; j < n; ++j) w[i * n + j] = w[i * n + j] - l * w[k * n + j];
        }
    }
    return w[(n - 1) * n + (n - 1)] == 0.0 ? 1 : 0;
}
__device__ __forceinline__ void lu_solve_n(int n, const double *w, double *x)
{
    for (int i = 1; i < n; ++i) {
        double xi = x[i];
        for (int j = 0; j < i; ++j) xi = xi - w[i * n + j] * x[j];
        x[i] = xi;
    }
    x[n - 1] = x[n - 1] / w[(n - 1) * n + (n - 1)];
    for (int i = n - 2; i >= 0; --i) {
        double xi = x[i];
        for (int j = i + 1; j < n; ++j) xi = xi - w[i * n + j] * x[j];
        x[i] = xi / w[i * n + i];
    }
}

// CTMATRX, src/fasolt/crys_math.f90:25-62 (a[i][j] = a(i+1,j+1)).
__device__ __forceinline__ void ctmatrx(double ph1, double phi, double ph2, double a[3][3],
                                        double aug[3])
{
    double s1, c1, s2, c2, s, c;
    sincos(ph1, &s1, &c1);
    sincos(ph2, &s2, &c2);
    sincos(phi, &s, &c);
    const double c1c2 = c1 * c2, s1s2 = s1 * s2, c1s2 = c1 * s2, s1c2 = s1 * c2;
    a[0][0] = c1c2 - s1s2 * c;
    a[1][0] = -c1s2 - s1c2 * c;
    a[2][0] = s1 * s;
    a[0][1] = s1c2 + c1s2 * c;
    a[1][1] = -s1s2 + c1c2 * c;
    a[2][1] = -c1 * s;
    a[0][2] = s2 * s;
    a[1][2] = c2 * s;
    a[2][2] = c;
    aug[0] = s2;
    aug[1] = c2;
    aug[2] = s;
}

// ELASTC, src/fasolt/ela-plas.f90:12-86: compliance of the rotated crystal
// with engineering shears; e = S11,S22,S33,S23,S31,S12,S44,S55,S66.
__device__ __forceinline__ void elastc(const double *e, double ph1, double phi, double ph2,
                                       double S[6][6])
{
    double a0[3][3], aug[3], a[3][3];
    ctmatrx(ph1, phi, ph2, a0, aug);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a[i][j] = a0[j][i];
    double ev[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) ev[k] = ld_ro(e + k);
    const int pi[6] = {0, 1, 2, 1, 2, 0}, pj[6] = {0, 1, 2, 2, 0, 1};
#pragma unroll
    for (int I = 0; I < 6; ++I) {
        const int i = pi[I], j = pj[I];
        const double mult = I < 3 ? 1.0 : 2.0;
#pragma unroll
        for (int J = I; J < 6; ++J) {
            const int k = pi[J], l = pj[J];
            const double t1 = a[i][0] * a[j][0] * a[k][0] * a[l][0] * ev[0] +
                              a[i][1] * a[j][1] * a[k][1] * a[l][1] * ev[1] +
                              a[i][2] * a[j][2] * a[k][2] * a[l][2] * ev[2];
            const double t2 = a[i][1] * a[j][1] * a[k][2] * a[l][2] * ev[3] +
                              a[i][2] * a[j][2] * a[k][1] * a[l][1] * ev[3] +
                              a[i][2] * a[j][2] * a[k][0] * a[l][0] * ev[4] +
                              a[i][0] * a[j][0] * a[k][2] * a[l][2] * ev[4] +
                              a[i][0] * a[j][0] * a[k][1] * a[l][1] * ev[5] +
                              a[i][1] * a[j][1] * a[k][0] * a[l][0] * ev[5];
            const double t3 = a[i][1] * a[j][2] * a[k][1] * a[l][2] * ev[6] +
                              a[i][2] * a[j][1] * a[k][2] * a[l][1] * ev[6] +
                              a[i][2] * a[j][0] * a[k][2] * a[l][0] * ev[7] +
                              a[i][0] * a[j][2] * a[k][0] * a[l][2] * ev[7] +
                              a[i][0] * a[j][1] * a[k][0] * a[l][1] * ev[8] +
                              a[i][1] * a[j][0] * a[k][1] * a[l][0] * ev[8];
            S[I][J] = mult * (t1 + t2 + 0.5 * t3);
        }
    }
#pragma unroll
    for (int I = 0; I < 5; ++I)
#pragma unroll
        for (int J = I + 1; J < 6; ++J) S[J][I] = S[I][J];
}

// TENS_ROT, src/fasolt/Sig_eps.f90:166-202: R^T a R for the small spin r.
__device__ __forceinline__ void tens_rot(const double r[3], const double a[6], double b[6])
{
    double rot[3][3], old[3][3], tmp[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        old[i][i] = a[i];
        old[j][k] = a[i + 3];
        old[k][j] = a[i + 3];
        rot[j][k] = r[i];
        rot[k][j] = -r[i];
        rot[i][i] = sqrt(1.0 - r[j] * r[j] - r[k] * r[k]);
    }
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int q = 0; q < 3; ++q)
            tmp[p][q] = old[p][0] * rot[0][q] + old[p][1] * rot[1][q] + old[p][2] * rot[2][q];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        b[i] = rot[0][i] * tmp[0][i] + rot[1][i] * tmp[1][i] + rot[2][i] * tmp[2][i];
        b[i + 3] = rot[0][j] * tmp[0][k] + rot[1][j] * tmp[1][k] + rot[2][j] * tmp[2][k];
    }
}

// SHAPE_12 + INVERT_3, src/fasolt/Shapef.f90:32-86,499-537.
// xn[i][k] node i coordinate k; returns weight, fills dndx[i][k].
__device__ __forceinline__ double shape12(const double xn[8][3], double dndx[8][3])
{
    // dN/dxi at the centre: +-1/8 with the sign of the local node offset
    const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    const double sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    const double sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    double jac[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double a = 0.0, b = 0.0, c = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            a = a + (0.125 * sx[i]) * xn[i][k];
            b = b + (0.125 * sy[i]) * xn[i][k];
            c = c + (0.125 * sz[i]) * xn[i][k];
        }
        jac[0][k] = a;
        jac[1][k] = b;
        jac[2][k] = c;
    }
    double inv[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int ia = (i + 1) % 3, ib = (ia + 1) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int ja = (j + 1) % 3, jb = (ja + 1) % 3;
            inv[j][i] = jac[ia][ja] * jac[ib][jb] - jac[ia][jb] * jac[ib][ja];
        }
    }
    const double det = inv[0][0] * jac[0][0] + inv[0][1] * jac[1][0] + inv[0][2] * jac[2][0];
    if (det != 0.0) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) inv[i][j] = inv[i][j] / det;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k)
            dndx[i][k] = inv[k][0] * (0.125 * sx[i]) + inv[k][1] * (0.125 * sy[i]) +
                         inv[k][2] * (0.125 * sz[i]);
    return 8.0 * det;
}

// INVERT_3, src/fasolt/Shapef.f90:499-537: inv = jac^-1 (cofactors / det),
// returns det (inv left as the cofactors when det == 0).
__device__ __forceinline__ double invert3(const double jac[3][3], double inv[3][3])
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int ia = (i + 1) % 3, ib = (ia + 1) % 3;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int ja = (j + 1) % 3, jb = (ja + 1) % 3;
            inv[j][i] = jac[ia][ja] * jac[ib][jb] - jac[ia][jb] * jac[ib][ja];
        }
    }
    const double det = inv[0][0] * jac[0][0] + inv[0][1] * jac[1][0] + inv[0][2] * jac[2][0];
    if (det != 0.0) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) inv[i][j] = inv[i][j] / det;
    }
    return det;
}

// DSTRNS (src/fasolt/Sig_eps.f90:25-61) from the displacement gradient
// g[a][b] = sum_i sfd(a,i) dxl(b,i).  Returns 0, 905 or 906.
__device__ __forceinline__ int dstrns_grad(const double g[3][3], double smalr, double smale, double del[6],
                                           double r[3], double &deff)
{
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        del[i] = g[i][i];
        del[i + 3] = g[k][j] + g[j][k];
        r[i] = (g[k][j] - g[j][k]) / 2.0;
        sum = sum + r[i] * r[i];
    }
    deff = fj2vom(false, del);
    if (sum > smalr) return 905;
    if (deff > smale) return 906;
    return 0;
}

// DSTRNS, src/fasolt/Sig_eps.f90:25-61.  Returns 0, 905 or 906.
__device__ __forceinline__ int dstrns(const double sfd[8][3], const double dxl[8][3],
                                      double smalr, double smale, double del[6], double r[3],
                                      double &deff)
{
    double g[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
#pragma unroll
            for (int i = 0; i < 8; ++i) s = s + sfd[i][a] * dxl[i][b];
            g[a][b] = s;
        }
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        del[i] = g[i][i];
        del[i + 3] = g[k][j] + g[j][k];
        r[i] = (g[k][j] - g[j][k]) / 2.0;
        sum = sum + r[i] * r[i];
    }
    deff = fj2vom(false, del);
    if (sum > smalr) return 905;
    if (deff > smale) return 906;
    return 0;
}

// Per-thread copy of the FAS_CPL scratch.
template <int NS> struct CpScratch {
    int ns, nsa, mc;
    int isa[NS];
    double tau[NS], gam[NS], s0[NS], s1[NS], am[NS];
    double b[NS][6], rot[NS][3];
    double ah[NS * NS];
};

// BTMATRX, src/fasolt/crys_math.f90:75-115
template <int NS>
__device__ __forceinline__ void btmatrx(const DevMat &M, const double a[3][3], CpScratch<NS> &w)
{
    const double *ab = M.ab + (size_t)w.mc * M.tld * 3;
    const double *an = M.an + (size_t)w.mc * M.tld * 3;
    for (int i = 0; i < w.ns; ++i) {
        double d0 = ld_ro(ab + 3 * i), d1 = ld_ro(ab + 3 * i + 1), d2 = ld_ro(ab + 3 * i + 2);
        double n0 = ld_ro(an + 3 * i), n1 = ld_ro(an + 3 * i + 1), n2 = ld_ro(an + 3 * i + 2);
        double sdr[3], spn[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            sdr[j] = a[0][j] * d0 + a[1][j] * d1 + a[2][j] * d2;
            spn[j] = a[0][j] * n0 + a[1][j] * n1 + a[2][j] * n2;
        }
        w.b[i][0] = sdr[0] * spn[0];
        w.b[i][1] = sdr[1] * spn[1];
        w.b[i][2] = sdr[2] * spn[2];
        w.b[i][3] = sdr[1] * spn[2] + sdr[2] * spn[1];
        w.b[i][4] = sdr[2] * spn[0] + sdr[0] * spn[2];
        w.b[i][5] = sdr[0] * spn[1] + sdr[1] * spn[0];
        w.rot[i][0] = (sdr[1] * spn[2] - sdr[2] * spn[1]) / 2.0;
        w.rot[i][1] = (sdr[2] * spn[0] - sdr[0] * spn[2]) / 2.0;
        w.rot[i][2] = (sdr[0] * spn[1] - sdr[1] * spn[0]) / 2.0;
    }
}

// x^y with the two exponents hardening laws use most taken exactly: x^0 = 1
// (A6 = 0: a rate-independent saturation stress) and x^1 = x (A4 = 1: Voce).
__device__ __forceinline__ double pow_exact01(double x, double y)
{
    if (y == 0.0) return 1.0;
    if (y == 1.0) return x;
    return pow(x, y);
}

// PLASTC, src/fasolt/ela-plas.f90:110-201: s1 and the log-hardening matrix
// of the active systems (ah(i,j) = sgn(gam_j) h_ij / s1_i).  Kept out of
// line: SLPFTA calls it in and after its loop, and one copy of its code
// spares the instruction cache.
template <int NS>
__device__ __noinline__ void plastc(const DevMat &M, CpScratch<NS> &w, double dt)
{
    const int ns = w.ns;
    const double *amp = M.ampar + (size_t)w.mc * M.tld * 6;
    const double *sm = M.sm + (size_t)w.mc * M.sld;
    double sumss = 0.0;
    for (int i = 0; i < ns; ++i) sumss = sumss + fabs(w.gam[i]);
    double gradh[NS];
    for (int i = 0; i < ns; ++i) {
        const double sst = ld_ro(amp + 6 * i + 4) * pow_exact01(sumss / dt, ld_ro(amp + 6 * i + 5));
        double arg = (sst != 0.0) ? 1.0 - (w.s0[i] / sst) : 0.0;
        if (arg < 0.0) arg = 0.0;
        gradh[i] = ld_ro(amp + 6 * i + 2) +
                   ld_ro(amp + 6 * i + 1) * copysign(pow_exact01(fabs(arg), ld_ro(amp + 6 * i + 3)), arg);
    }
    for (int i = 0; i < ns; ++i) {
        double s = w.s0[i];
        for (int j = 0; j < ns; ++j) s = s + (ld_ro(sm + i * ns + j) * gradh[j]) * fabs(w.gam[j]);
        w.s1[i] = s;
    }
    for (int i = 0; i < w.nsa; ++i) {
        const int is = w.isa[i];
        const double inv_s1 = w.s1[is];
        for (int j = 0; j < w.nsa; ++j) {
            const int js = w.isa[j];
            const double g = w.gam[js];
            w.ah[i * w.nsa + j] = fabs(g) > 1.e-14
                                   ? (copysign(1.0, g) * (ld_ro(sm + is * ns + js) * gradh[js])) / inv_s1
                                   : 0.0;
        }
    }
}

// SLPINI, src/fasolt/crys-cons.f90:143-197: predictor slips, twin trigger,
// active set.
template <int NS>
__device__ __forceinline__ void slpini(const DevMat &M, CpScratch<NS> &w, const DevGp &G,
                                       const DevCtrl &C, int g, double dt, int inc, int nit,
                                       int cpit, int &twinsys, int timestwinned)
{
    const double *amp = M.ampar + (size_t)w.mc * M.tld * 6;
    const double *ssang = M.ssang + (size_t)w.mc * M.tld;
    double gammax = 0.0;
    for (int i = 0; i < w.ns; ++i) {
        w.am[i] = ld_ro(amp + 6 * i);
        const double sa = ld_ro(ssang + i);
        double gi;
        if (fabs(sa) > 1.5) {
            gi = 0.0;
            if (w.tau[i] > w.s0[i] && timestwinned != M.twinlim && twinsys == 0) {
                const double u = fas_twin_u01(C.seed, g, inc, nit, cpit, i);
                if (u < M.twinprob) {
                    twinsys = i + 1;
                    *G.tflag = 1;
                }
            }
        } else if (sa * w.tau[i] / w.s0[i] < 0.0) {
            gi = 0.0;
        } else {
            gi = dt * spower(w.tau[i] / w.s0[i], 1.0 / w.am[i]);
        }
        w.gam[i] = gi;
        if (fabs(gi) > gammax) gammax = fabs(gi);
    }
    const double cutoff = 1.e-6 * gammax;
    int nsa = 0;
    for (int i = 0; i < w.ns; ++i) {
        if (fabs(w.gam[i]) < cutoff) w.gam[i] = 0.0;
        else w.isa[nsa++] = i;
    }
    w.nsa = nsa;
}

// SCALE_IT, src/fasolt/Cpstrs.f90:187-230 (amax starts from am(1), the
// first system, as the reference writes it).
template <int NS>
__device__ __forceinline__ void scale_it(CpScratch<NS> &w, double s[6], double gamcap,
                                         double afactor)
{
    double amax = w.am[0];
    double gammax = fabs(w.gam[w.isa[0]]);
    for (int i = 1; i < w.nsa; ++i) {
        const int ii = w.isa[i];
        if (fabs(w.gam[ii]) > gammax) {
            gammax = fabs(w.gam[ii]);
            amax = w.am[ii];
        }
    }
    if (gammax > gamcap) {
        const double scale = gamcap / gammax;
        double smult = spower(0.9 * scale, afactor * amax);
        if (smult == 0.0) smult = 0.004 / amax;
#pragma unroll
        for (int i = 0; i < 6; ++i) s[i] = smult * s[i];
        for (int i = 0; i < w.ns; ++i) {
            w.gam[i] = scale * w.gam[i];
            w.tau[i] = smult * w.tau[i];
        }
    }
}

// SLPFTA, src/fasolt/crys-cons.f90:24-128: Newton on log(gamma) of the
// active systems; leaves X (the visco-plastic matrix) in ah.
template <int NS>
__device__ __forceinline__ int slpfta(const DevMat &M, CpScratch<NS> &w, const DevCtrl &C,
                                      double dt, int &ninner)
{
    const double conv = C.toler * M.amax[w.mc];
    const int n = w.nsa;
    double errtau[NS];
    double tauerr = 0.0;
    int iter = 0;
    bool l_iter = true;
    while (l_iter) {
        ++iter;
        plastc(M, w, dt);
        for (int i = 0; i < n; ++i) {
            const double gamn = w.gam[w.isa[i]];
            for (int j = 0; j < n; ++j) w.ah[j * n + i] = gamn * w.ah[j * n + i];
            w.ah[i * n + i] = w.ah[i * n + i] + w.am[w.isa[i]];
        }
        if (lu_factor_n(n, w.ah)) { ninner = iter; return 910; }
        for (int i = 0; i < n; ++i) {
            const int ii = w.isa[i];
            const double taufg = w.s1[ii] * spower(w.gam[ii] / dt, w.am[ii]);
            errtau[i] = (w.tau[ii] * taufg > 0.0) ? log(w.tau[ii] / taufg) : 0.0;
        }
        tauerr = 0.0;
        for (int i = 0; i < n; ++i) tauerr = tauerr + errtau[i] * errtau[i];
        tauerr = sqrt(tauerr);
        lu_solve_n(n, w.ah, errtau);
        double errmax = 0.0;
        for (int i = 0; i < n; ++i)
            if (fabs(errtau[i]) > errmax) errmax = fabs(errtau[i]);
        const double scale = errmax > 5.0 ? 5.0 / errmax : 1.0;
        for (int i = 0; i < n; ++i) {
            const int ii = w.isa[i];
            w.gam[ii] = w.gam[ii] * exp(scale * errtau[i]);
        }
        l_iter = (iter < C.maxit) && (tauerr > conv);
    }
    ninner = iter;
    if (tauerr > 0.5) return 987;
    plastc(M, w, dt);
    for (int i = 0; i < n; ++i) {
        const int ii = w.isa[i];
        for (int j = 0; j < n; ++j) w.ah[j * n + i] = w.tau[w.isa[j]] * w.ah[j * n + i];
        const double g = w.gam[ii];
        w.ah[i * n + i] = w.ah[i * n + i] +
                           (fabs(g) > 1.e-12 ? w.am[ii] * w.tau[ii] / g : w.am[ii] / 1.e-12);
    }
    return 0;
}

// ECHROT, src/fasolt/crys_math.f90:137-167
template <int NS>
__device__ __forceinline__ void echrot(const CpScratch<NS> &w, const double a[3][3],
                                       const double aug[3], const double r[3], double &dp1,
                                       double &dph, double &dp2)
{
    double rtn[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double s = 0.0;
        for (int i = 0; i < w.ns; ++i) s = s + w.rot[i][k] * w.gam[i];
        rtn[k] = s - r[k];
    }
    double rx[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) rx[k] = a[k][0] * rtn[0] + a[k][1] * rtn[1] + a[k][2] * rtn[2];
    dp1 = fabs(aug[2]) < 1.e-5 ? rtn[2] : (aug[0] * rx[0] + aug[1] * rx[1]) / aug[2];
    dph = aug[1] * rx[0] - aug[0] * rx[1];
    dp2 = rx[2] - dp1 * a[2][2];
}

// Results of one DSTRSS call that the callers store.
struct GpOut {
    double t[6];         // new stress
    double chi[6][6];    // tangent (symmetrised in the plastic branch)
    double deff;         // effective plastic strain increment
};

// CPSTRS (src/fasolt/Cpstrs.f90:34-172) inside DSTRSS
// (src/fasolt/Sig_eps.f90:84-151).  Reads sv/dsv of GP g, updates dsv,
// srate and the twin flag, returns 0 or a FAFERR code.
template <int NS>
__device__ int dstrss(const DevMat &M, const DevCtrl &C, const DevGp &G, int g, int iel,
                      const double de[6], const double r[3], const double st[6], double ds[6],
                      double dt, int inc, int nit, GpOut &o)
{
    const int mc = (iel < 0 ? -iel : iel) - 1;
    const int ng = G.ngps;
    const double ph1 = G.sv[g] + G.dsv[g];
    const double phi = G.sv[ng + g] + G.dsv[ng + g];
    const double ph2 = G.sv[2 * ng + g] + G.dsv[2 * ng + g];
    double S[6][6];
    elastc(M.e + 9 * mc, ph1, phi, ph2, S);
    double t[6];
    tens_rot(r, st, t);
    double s[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = t[i] + ds[i];
    const double sinit = fj2vom(true, s);
    const double einit = fj2vom(false, de);
    G.erepmd[g] = 0.0;
    if (iel > 0 && sinit > 0.0 && einit > 0.0) {
        CpScratch<NS> w;
        w.mc = mc;
        w.ns = M.ns[mc];
        for (int i = 0; i < w.ns; ++i) w.s0[i] = G.sv[(3 + i) * ng + g];
        const double gamcap = 6.0 * fj2vom(false, de);
        double a[3][3], aug[3];
        ctmatrx(ph1, phi, ph2, a, aug);
        btmatrx<NS>(M, a, w);
        int twinsys = G.twinsys[g];
        const int timestwinned = G.timestwinned[g];
        double ops = fas_ops_cp_fixed(w.ns);
        double djac[6][6], erreps[6], epl[6];
        double erepmd = 0.0;
        int iter = 0, rc = 0;
        bool l_iter = true;
        while (l_iter) {
            ++iter;
            for (int i = 0; i < w.ns; ++i)
                w.tau[i] = w.b[i][0] * s[0] + w.b[i][1] * s[1] + w.b[i][2] * s[2] +
                           w.b[i][3] * s[3] + w.b[i][4] * s[4] + w.b[i][5] * s[5];
            slpini<NS>(M, w, G, C, g, dt, inc, nit, iter, twinsys, timestwinned);
            scale_it<NS>(w, s, gamcap, C.afactor);
            int ninner = 0;
            rc = slpfta<NS>(M, w, C, dt, ninner);
            ops += ninner * fas_ops_inner(w.ns, w.nsa) + fas_ops_outer(w.ns, w.nsa);
            if (rc) break;
            scale_it<NS>(w, s, gamcap, C.afactor);
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                double acc = 0.0;
                for (int i = 0; i < w.ns; ++i) acc = acc + w.b[i][k] * w.gam[i];
                epl[k] = acc;
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c < 6; ++c) acc = acc + S[k][c] * (s[c] - t[c]);
                erreps[k] = de[k] - epl[k] - acc;
            }
            const int n = w.nsa;
            if (lu_factor_n(n, w.ah)) { rc = 910; break; }
            // djac = b_a X^-1 b_a^T: one solve per column j
            for (int j = 0; j < 6; ++j) {
                double wk[NS];
                for (int k = 0; k < n; ++k) wk[k] = w.b[w.isa[k]][j];
                lu_solve_n(n, w.ah, wk);
                for (int i = 0; i < 6; ++i) {
                    double sum = 0.0;
                    for (int k = 0; k < n; ++k) sum = sum + w.b[w.isa[k]][i] * wk[k];
                    djac[i][j] = sum + S[i][j];
                }
            }
            if (lu_factor<6>(6, &djac[0][0])) { rc = 910; break; }
            lu_solve<6>(6, &djac[0][0], erreps);
            erepmd = fj2vom(true, erreps) / fj2vom(true, s);
            const double scale = 1.0 / (1.0 + C.alpha * erepmd);
#pragma unroll
            for (int i = 0; i < 6; ++i) s[i] = s[i] + scale * erreps[i];
            l_iter = (iter < C.maxit) && (erepmd > C.toler);
        }
        G.cp_iters[g] = iter;
        G.ops[g] = ops;
        G.twinsys[g] = twinsys;
        if (rc) return rc;
        for (int i = 0; i < w.ns; ++i) G.srate[i * ng + g] = fabs(w.gam[i] / dt);
        G.erepmd[g] = erepmd;
        double dp1, dph, dp2;
        echrot<NS>(w, a, aug, r, dp1, dph, dp2);
        G.dsv[g] = dp1;
        G.dsv[ng + g] = dph;
        G.dsv[2 * ng + g] = dp2;
        for (int i = 0; i < w.ns; ++i) G.dsv[(3 + i) * ng + g] = w.s1[i] - w.s0[i];
#pragma unroll
        for (int i = 0; i < 6; ++i) o.t[i] = s[i];
        o.deff = fj2vom(false, epl);
        if (C.tangent) {
            // the consistent tangent: (B X^-1 B^T + S)^-1 of the local
            // system at the converged stress -- its slip stresses, and the
            // slips and hardening that satisfy the flow rule there (SLPFTA
            // from the last slips, same active set) -- instead of the
            // Jacobian of the last iterate.  The outputs above are kept.
            for (int i = 0; i < w.ns; ++i)
                w.tau[i] = w.b[i][0] * s[0] + w.b[i][1] * s[1] + w.b[i][2] * s[2] +
                           w.b[i][3] * s[3] + w.b[i][4] * s[4] + w.b[i][5] * s[5];
            int ninner = 0;
            rc = slpfta<NS>(M, w, C, dt, ninner);
            if (rc) return rc;
            const int n = w.nsa;
            if (lu_factor_n(n, w.ah)) return 910;
            for (int j = 0; j < 6; ++j) {
                double wk[NS];
                for (int k = 0; k < n; ++k) wk[k] = w.b[w.isa[k]][j];
                lu_solve_n(n, w.ah, wk);
                for (int i = 0; i < 6; ++i) {
                    double sum = 0.0;
                    for (int k = 0; k < n; ++k) sum = sum + w.b[w.isa[k]][i] * wk[k];
                    djac[i][j] = sum + S[i][j];
                }
            }
            if (lu_factor<6>(6, &djac[0][0])) return 910;
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double e6[6] = {0, 0, 0, 0, 0, 0};
            e6[i] = 1.0;
            lu_solve<6>(6, &djac[0][0], e6);
#pragma unroll
            for (int j = 0; j < 6; ++j) o.chi[j][i] = e6[j];
        }
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j) {
                const double d = (o.chi[i][j] + o.chi[j][i]) / 2.0;
                o.chi[i][j] = d;
                o.chi[j][i] = d;
            }
    } else {
        o.deff = 0.0;
        G.cp_iters[g] = 0;
        G.ops[g] = fas_ops_elastic();
        lu_factor<6>(6, &S[0][0]);
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double e6[6] = {0, 0, 0, 0, 0, 0};
            e6[i] = 1.0;
            lu_solve<6>(6, &S[0][0], e6);
#pragma unroll
            for (int j = 0; j < 6; ++j) o.chi[j][i] = e6[j];
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < 6; ++c) acc = acc + o.chi[i][c] * de[c];
            o.t[i] = acc;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) ds[i] = o.t[i] - st[i];
    return 0;
}

}  // namespace fasdev
