// fas_device_warp.cuh -- warp-cooperative Gauss-point update (DSTRSS /
// CPSTRS / SLPINI / SLPFTA / PLASTC) for sm_100a: one warp per Gauss point,
// lane i owns slip system i (ns <= 32).
//
// The same algorithm as fas_device.cuh, restated for a warp: per-system
// quantities live in one lane's registers; the active-set matrices of
// SLPFTA and CPSTRS (ah, X) are stored one row per lane (row k = k-th active
// system), the 6x6 Jacobian one row per lane 0..5; LU factorisation without
// pivoting and the triangular solves broadcast the pivot row / solved
// unknown with shuffles.  Sums over systems are warp butterflies, so they
// round differently from a sequential sum (about 1e-16 relative); every
// other operation is in the reference's order.  No per-thread scratch goes to
// local memory.
#pragma once

#include "fas_device.cuh"

namespace fasdev {
namespace wc {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ double wsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
__device__ __forceinline__ double wmax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
__device__ __forceinline__ double bc(double v, int src) { return __shfl_sync(FULL, v, src); }
__device__ __forceinline__ int bci(int v, int src) { return __shfl_sync(FULL, v, src); }

// position of the n-th (0-based) set bit of m
__device__ __forceinline__ int nth_set(unsigned m, int n)
{
    for (int i = 0; i < n; ++i) m &= m - 1;
    return __ffs(m) - 1;
}

// LU without pivoting (FACTOR, crys-cons.f90:244-269) of an n x n matrix
// stored one row per lane (lane k holds row k in a[0..N-1]).  Returns 1 (in
// every lane) on a zero pivot.
template <int N>
__device__ __forceinline__ int lu_rows(int n, int lane, double (&a)[N])
{
    for (int k = 0; k < n - 1; ++k) {
        double pk = 0.0;
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (j == k) pk = bc(a[j], k);
        if (pk == 0.0) return 1;
        double l = 0.0;
#pragma unroll
        for (int j = 0; j < N; ++j)
            if (j == k) l = a[j] / pk;
        const bool below = lane > k && lane < n;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            if (j < n) {
                const double pkj = bc(a[j], k);
                if (j == k) {
                    if (below) a[j] = l;
                } else if (j > k && below) {
                    a[j] = a[j] - l * pkj;
                }
            }
        }
    }
    double d = 0.0;
#pragma unroll
    for (int j = 0; j < N; ++j)
        if (j == n - 1) d = bc(a[j], n - 1);
    return d == 0.0 ? 1 : 0;
}

// SOLVER (crys-cons.f90:283-309) with the LU rows in lanes; x is the
// right-hand side component of row `lane` on entry and the solution on exit.
template <int N>
__device__ __forceinline__ double solve_rows(int n, int lane, const double (&a)[N], double x)
{
    // forward: x_i -= L_ij x_j for j < i
    for (int j = 0; j < n - 1; ++j) {
        const double xj = bc(x, j);
        double lij = 0.0;
#pragma unroll
        for (int c = 0; c < N; ++c)
            if (c == j) lij = a[c];
        if (lane > j && lane < n) x = x - lij * xj;
    }
    // back: x_i = (x_i - sum_{j>i} U_ij x_j) / U_ii, rows from the last up;
    // the solved unknowns are kept so each row sums them in ascending j,
    // the reference's order
    double xall[N];
#pragma unroll
    for (int c = 0; c < N; ++c) xall[c] = 0.0;
    for (int j = n - 1; j >= 0; --j) {
        if (lane == j) {
            double xi = x;
#pragma unroll
            for (int c = 0; c < N; ++c)
                if (c > j && c < n) xi = xi - a[c] * xall[c];
            double ujj = 0.0;
#pragma unroll
            for (int c = 0; c < N; ++c)
                if (c == j) ujj = a[c];
            x = xi / ujj;
        }
        const double xj = bc(x, j);
#pragma unroll
        for (int c = 0; c < N; ++c)
            if (c == j) xall[c] = xj;
    }
    return x;
}

// Row `r` (< 6) of the rotated compliance (ELASTC, ela-plas.f90:34-83):
// entry (r, c) is the reference's upper-triangle formula at (min, max).
__device__ __forceinline__ void elastc_row(const double *e, const double a0[3][3], int r, double row[6])
{
    double a[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) a[i][j] = a0[j][i];
    double ev[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) ev[k] = ld_ro(e + k);
    const int pi[6] = {0, 1, 2, 1, 2, 0}, pj[6] = {0, 1, 2, 2, 0, 1};
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const int I = r < c ? r : c, J = r < c ? c : r;
        const int i = pi[I], j = pj[I], k = pi[J], l = pj[J];
        const double mult = I < 3 ? 1.0 : 2.0;
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
        row[c] = mult * (t1 + t2 + 0.5 * t3);
    }
}

// Per-lane (per slip system) data of one Gauss point.
struct Sys {
    bool on;                 // lane < ns
    double b[6], rot[3];
    double tau, gam, s0, s1, am, gradh, ssang;
    double A2, A3, A4, A5, A6;
};

// PLASTC (ela-plas.f90:110-201) for the lane's system: s1 and gradh; the
// sum over j of smatrx(i,j) gradh_j |gam_j| runs in the reference's order.
__device__ __forceinline__ void plastc_sys(Sys &y, const double *smrow, int ns, double dt)
{
    const double sumss = wsum(y.on ? fabs(y.gam) : 0.0);
    double gh = 0.0;
    if (y.on) {
        const double sst = y.A5 * pow_exact01(sumss / dt, y.A6);
        double arg = (sst != 0.0) ? 1.0 - (y.s0 / sst) : 0.0;
        if (arg < 0.0) arg = 0.0;
        gh = y.A3 + y.A2 * copysign(pow_exact01(fabs(arg), y.A4), arg);
    }
    y.gradh = gh;
    double s = y.s0;
    for (int j = 0; j < ns; ++j) {
        const double gj = bc(gh, j);
        const double agj = bc(fabs(y.gam), j);
        if (y.on) s = s + (ld_ro(smrow + j) * gj) * agj;
    }
    y.s1 = s;
}

// Row k (lane k < nsa) of PLASTC's log-hardening matrix for the active
// systems (ik = isa(k) in lane k): ah(k,j) = sgn(gam_j) smatrx(isa_k, isa_j)
// gradh_j / s1(isa_k).
template <int NA>
__device__ __forceinline__ void ah_row(const Sys &y, const double *sm, int ns, int ik, int nsa,
                                       int lane, double (&row)[NA])
{
    const double s1k = bc(y.s1, ik);
#pragma unroll
    for (int j = 0; j < NA; ++j) {
        if (j < nsa) {
            const int ij = bci(ik, j);
            const double gj = bc(y.gam, ij);
            const double hj = bc(y.gradh, ij);
            double v = 0.0;
            if (lane < nsa && fabs(gj) > 1.e-14)
                v = (copysign(1.0, gj) * (ld_ro(sm + ik * ns + ij) * hj)) / s1k;
            row[j] = v;
        } else {
            row[j] = 0.0;
        }
    }
}

// Results of one warp DSTRSS: the new stress and deff in every lane, row
// `lane` of the tangent in lanes 0..5.
struct GpOutW {
    double t[6];
    double deff;
    double chirow[6];
};

// Lane r (< 6) of the symmetric part of a 6x6 matrix held one row per lane.
__device__ __forceinline__ void symmetrise_rows(int lane, double row[6])
{
    double col[6];   // col[c] = m(c, lane), the transpose row
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        col[c] = 0.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const double v = bc(row[j], c);   // m(c, j)
            if (j == lane) col[c] = v;
        }
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) row[c] = (row[c] + col[c]) / 2.0;
}

// DSTRSS (Sig_eps.f90:84-151) with CPSTRS (Cpstrs.f90:34-172) for GP g,
// executed by one whole warp.  Every lane returns the same code.
// NA bounds the number of active systems (and slip systems) of any material.
template <int NA>
__device__ int dstrss_wc(const DevMat &M, const DevCtrl &C, const DevGp &G, int g, int iel,
                         const double de[6], const double r[3], const double st[6], double ds[6],
                         double dt, int inc, int nit, GpOutW &o)
{
    const int lane = threadIdx.x & 31;
    const int mc = (iel < 0 ? -iel : iel) - 1;
    const int ng = G.ngps;
    const double ph1 = G.sv[g] + G.dsv[g];
    const double phi = G.sv[ng + g] + G.dsv[ng + g];
    const double ph2 = G.sv[2 * ng + g] + G.dsv[2 * ng + g];
    double a[3][3], aug[3];
    ctmatrx(ph1, phi, ph2, a, aug);
    double Srow[6];                       // row `lane` of the compliance (lanes < 6)
    elastc_row(M.e + 9 * mc, a, lane < 6 ? lane : 0, Srow);
    double t[6];
    tens_rot(r, st, t);
    double s[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) s[i] = t[i] + ds[i];
    const double sinit = fj2vom(true, s);
    const double einit = fj2vom(false, de);
    double *chirow = o.chirow;            // row `lane` of chi (lanes < 6)
    if (lane == 0) G.erepmd[g] = 0.0;
    if (iel > 0 && sinit > 0.0 && einit > 0.0) {
        const int ns = M.ns[mc];
        Sys y;
        y.on = lane < ns;
        const int li = y.on ? lane : 0;
        {
            const double *ab = M.ab + ((size_t)mc * MAXSS + li) * 3;
            const double *an = M.an + ((size_t)mc * MAXSS + li) * 3;
            const double d0 = ld_ro(ab), d1 = ld_ro(ab + 1), d2 = ld_ro(ab + 2);
            const double n0 = ld_ro(an), n1 = ld_ro(an + 1), n2 = ld_ro(an + 2);
            double sdr[3], spn[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                sdr[j] = a[0][j] * d0 + a[1][j] * d1 + a[2][j] * d2;
                spn[j] = a[0][j] * n0 + a[1][j] * n1 + a[2][j] * n2;
            }
            y.b[0] = sdr[0] * spn[0];
            y.b[1] = sdr[1] * spn[1];
            y.b[2] = sdr[2] * spn[2];
            y.b[3] = sdr[1] * spn[2] + sdr[2] * spn[1];
            y.b[4] = sdr[2] * spn[0] + sdr[0] * spn[2];
            y.b[5] = sdr[0] * spn[1] + sdr[1] * spn[0];
            y.rot[0] = (sdr[1] * spn[2] - sdr[2] * spn[1]) / 2.0;
            y.rot[1] = (sdr[2] * spn[0] - sdr[0] * spn[2]) / 2.0;
            y.rot[2] = (sdr[0] * spn[1] - sdr[1] * spn[0]) / 2.0;
            if (!y.on) {
#pragma unroll
                for (int k = 0; k < 6; ++k) y.b[k] = 0.0;
#pragma unroll
                for (int k = 0; k < 3; ++k) y.rot[k] = 0.0;
            }
            const double *amp = M.ampar + ((size_t)mc * MAXSS + li) * 6;
            y.am = ld_ro(amp);
            y.A2 = ld_ro(amp + 1);
            y.A3 = ld_ro(amp + 2);
            y.A4 = ld_ro(amp + 3);
            y.A5 = ld_ro(amp + 4);
            y.A6 = ld_ro(amp + 5);
            y.ssang = ld_ro(M.ssang + (size_t)mc * MAXSS + li);
            y.s0 = y.on ? G.sv[(3 + lane) * ng + g] : 0.0;
            y.s1 = y.s0;
            y.gam = 0.0;
            y.tau = 0.0;
        }
        const double *sm = M.sm + (size_t)mc * MAXSS * MAXSS;
        const double *smrow = sm + (size_t)li * ns;
        const double am1 = bc(y.am, 0);
        const double gamcap = 6.0 * fj2vom(false, de);
        int twinsys = G.twinsys[g];
        const int timestwinned = G.timestwinned[g];
        double ops = fas_ops_cp_fixed(ns);
        double erreps[6], epl[6], djrow[6];
        double X[NA];
        double erepmd = 0.0;
        int iter = 0, rc = 0, nsa = 0, ik = 0;
        bool act = false;          // this lane's system is in the active set
        bool l_iter = true;
        while (l_iter) {
            ++iter;
            // resolved shear stress
            y.tau = y.b[0] * s[0] + y.b[1] * s[1] + y.b[2] * s[2] + y.b[3] * s[3] + y.b[4] * s[4] +
                    y.b[5] * s[5];
            // SLPINI (crys-cons.f90:143-197)
            {
                double gi = 0.0;
                bool cand = false;
                if (y.on) {
                    if (fabs(y.ssang) > 1.5) {
                        cand = y.tau > y.s0 && timestwinned != M.twinlim && twinsys == 0 &&
                               fas_twin_u01(C.seed, g, inc, nit, iter, lane) < M.twinprob;
                    } else if (y.ssang * y.tau / y.s0 < 0.0) {
                        gi = 0.0;
                    } else {
                        gi = dt * spower(y.tau / y.s0, 1.0 / y.am);
                    }
                }
                const unsigned tw = __ballot_sync(FULL, cand);
                if (tw) {
                    twinsys = __ffs(tw);
                    if (lane == 0) *G.tflag = 1;
                }
                y.gam = gi;
                const double gammax = wmax(y.on ? fabs(gi) : 0.0);
                const double cutoff = 1.e-6 * gammax;
                act = y.on && !(fabs(y.gam) < cutoff);
                if (y.on && !act) y.gam = 0.0;
                const unsigned amask = __ballot_sync(FULL, act);
                nsa = __popc(amask);
                ik = lane < nsa ? nth_set(amask, lane) : 0;
            }
            // SCALE_IT (Cpstrs.f90:187-230): the largest active |gam|; amax
            // starts from am(1) and changes only on a strictly larger value
            auto scale_it = [&]() {
                const int i0 = bci(ik, 0);
                const double g0 = fabs(bc(y.gam, i0));
                const double gmaxw = wmax(y.on && lane != i0 && fabs(y.gam) > 0.0 ? fabs(y.gam) : 0.0);
                // among actives after the first, the first lane attaining a
                // value strictly above the running maximum wins; that is the
                // first lane attaining the overall maximum when it exceeds g0
                double amax = am1, gammax = g0;
                if (gmaxw > g0) {
                    const unsigned hit = __ballot_sync(FULL, y.on && lane != i0 && fabs(y.gam) == gmaxw &&
                                                                 (fabs(y.gam) > 0.0));
                    const int w = __ffs(hit) - 1;
                    amax = bc(y.am, w);
                    gammax = gmaxw;
                }
                if (gammax > gamcap) {
                    const double scale = gamcap / gammax;
                    double smult = spower(0.9 * scale, C.afactor * amax);
                    if (smult == 0.0) smult = 0.004 / amax;
#pragma unroll
                    for (int i = 0; i < 6; ++i) s[i] = smult * s[i];
                    y.gam = scale * y.gam;
                    y.tau = smult * y.tau;
                }
            };
            scale_it();
            // SLPFTA (crys-cons.f90:24-128)
            int ninner = 0;
            {
                const double conv = C.toler * M.amax[mc];
                double tauerr = 0.0;
                int it2 = 0;
                bool li2 = true;
                while (li2) {
                    ++it2;
                    plastc_sys(y, smrow, ns, dt);
                    ah_row<NA>(y, sm, ns, ik, nsa, lane, X);
                    // column j scaled by gam(isa_j), + am on the diagonal
                    const double amk = bc(y.am, ik);
#pragma unroll
                    for (int j = 0; j < NA; ++j) {
                        if (j < nsa) {
                            const double gj = bc(y.gam, bci(ik, j));
                            X[j] = gj * X[j];
                            if (j == lane) X[j] = X[j] + amk;
                        }
                    }
                    if (lu_rows<NA>(nsa, lane, X)) { rc = 910; break; }
                    double et = 0.0;
                    {
                        const double tk = bc(y.tau, ik), s1k = bc(y.s1, ik), gk = bc(y.gam, ik);
                        if (lane < nsa) {
                            const double taufg = s1k * spower(gk / dt, amk);
                            et = (tk * taufg > 0.0) ? log(tk / taufg) : 0.0;
                        }
                    }
                    tauerr = sqrt(wsum(et * et));
                    et = solve_rows<NA>(nsa, lane, X, et);
                    const double errmax = wmax(lane < nsa ? fabs(et) : 0.0);
                    const double scale = errmax > 5.0 ? 5.0 / errmax : 1.0;
                    // back to the system lanes: active system isa(k) takes entry k
                    double dk = 0.0;
                    for (int k = 0; k < nsa; ++k) {
                        const double ek = bc(et, k);
                        if (lane == bci(ik, k)) dk = ek;
                    }
                    if (act) y.gam = y.gam * exp(scale * dk);
                    li2 = (it2 < C.maxit) && (tauerr > conv);
                }
                ninner = it2;
                if (!rc && tauerr > 0.5) rc = 987;
                if (!rc) {
                    plastc_sys(y, smrow, ns, dt);
                    ah_row<NA>(y, sm, ns, ik, nsa, lane, X);
                    const double tk = bc(y.tau, ik), amk = bc(y.am, ik), gk = bc(y.gam, ik);
#pragma unroll
                    for (int j = 0; j < NA; ++j) {
                        if (j < nsa) {
                            X[j] = tk * X[j];
                            if (j == lane)
                                X[j] = X[j] + (fabs(gk) > 1.e-12 ? amk * tk / gk : amk / 1.e-12);
                        }
                    }
                }
            }
            ops += ninner * fas_ops_inner(ns, nsa) + fas_ops_outer(ns, nsa);
            if (rc) break;
            scale_it();
            // plastic strain and strain error (Cpstrs.f90:96-98)
#pragma unroll
            for (int k = 0; k < 6; ++k) epl[k] = wsum(y.b[k] * y.gam);
            {
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c < 6; ++c) acc = acc + Srow[c] * (s[c] - t[c]);
                double dek = 0.0, eplk = 0.0;
#pragma unroll
                for (int k = 0; k < 6; ++k)
                    if (k == lane) {
                        dek = de[k];
                        eplk = epl[k];
                    }
                erreps[0] = dek - eplk - acc;   // this lane's component (lanes < 6)
            }
            if (lu_rows<NA>(nsa, lane, X)) { rc = 910; break; }
            // djac = b_a X^-1 b_a^T + S, row `lane` (lanes < 6)
            {
                double bk[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) bk[k] = bc(y.b[k], ik);
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    double wk = solve_rows<NA>(nsa, lane, X, lane < nsa ? bk[j] : 0.0);
                    double sum_i[6];
#pragma unroll
                    for (int i = 0; i < 6; ++i) sum_i[i] = wsum(lane < nsa ? bk[i] * wk : 0.0);
                    double mine = 0.0;
#pragma unroll
                    for (int i = 0; i < 6; ++i)
                        if (i == lane) mine = sum_i[i];
                    djrow[j] = mine + Srow[j];
                }
            }
            {
                double D6[6];
#pragma unroll
                for (int j = 0; j < 6; ++j) D6[j] = djrow[j];
                if (lu_rows<6>(6, lane, D6)) { rc = 910; break; }
                double e = solve_rows<6>(6, lane, D6, erreps[0]);
#pragma unroll
                for (int k = 0; k < 6; ++k) erreps[k] = bc(e, k);
                erepmd = fj2vom(true, erreps) / fj2vom(true, s);
                const double scale = 1.0 / (1.0 + C.alpha * erepmd);
#pragma unroll
                for (int i = 0; i < 6; ++i) s[i] = s[i] + scale * erreps[i];
#pragma unroll
                for (int j = 0; j < 6; ++j) djrow[j] = D6[j];   // keep the factors
            }
            l_iter = (iter < C.maxit) && (erepmd > C.toler);
        }
        if (lane == 0) {
            G.cp_iters[g] = iter;
            G.ops[g] = ops;
            G.twinsys[g] = twinsys;
        }
        if (rc) return rc;
        if (y.on) G.srate[lane * ng + g] = fabs(y.gam / dt);
        if (lane == 0) G.erepmd[g] = erepmd;
        // ECHROT (crys_math.f90:137-167)
        {
            double rtn[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) rtn[k] = wsum(y.rot[k] * y.gam) - r[k];
            double rx[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) rx[k] = a[k][0] * rtn[0] + a[k][1] * rtn[1] + a[k][2] * rtn[2];
            const double dp1 = fabs(aug[2]) < 1.e-5 ? rtn[2] : (aug[0] * rx[0] + aug[1] * rx[1]) / aug[2];
            const double dph = aug[1] * rx[0] - aug[0] * rx[1];
            const double dp2 = rx[2] - dp1 * a[2][2];
            if (lane == 0) {
                G.dsv[g] = dp1;
                G.dsv[ng + g] = dph;
                G.dsv[2 * ng + g] = dp2;
            }
        }
        // chi = djac^-1 from the last factors, one unit solve per column
#pragma unroll
        for (int i = 0; i < 6; ++i) chirow[i] = solve_rows<6>(6, lane, djrow, lane == i ? 1.0 : 0.0);
        if (y.on) G.dsv[(3 + lane) * ng + g] = y.s1 - y.s0;
#pragma unroll
        for (int i = 0; i < 6; ++i) o.t[i] = s[i];
        o.deff = fj2vom(false, epl);
        symmetrise_rows(lane, chirow);
    } else {
        o.deff = 0.0;
        if (lane == 0) {
            G.cp_iters[g] = 0;
            G.ops[g] = fas_ops_elastic();
        }
        double D6[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) D6[j] = Srow[j];
        lu_rows<6>(6, lane, D6);
#pragma unroll
        for (int i = 0; i < 6; ++i) chirow[i] = solve_rows<6>(6, lane, D6, lane == i ? 1.0 : 0.0);
        // t = chi de, row `lane`, then to every lane
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) acc = acc + chirow[c] * de[c];
#pragma unroll
        for (int i = 0; i < 6; ++i) o.t[i] = bc(acc, i);
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) ds[i] = o.t[i] - st[i];
    return 0;
}

}  // namespace wc
}  // namespace fasdev
