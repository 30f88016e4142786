// Adjoint of the constitutive update along the Gauss points' strain
// histories (no counterpart in the reference, which has no derivatives).
//
// Replay.  Every GP runs DSTRSS (dstrss<NS>, the code of the increments)
// through a recorded history of strain increments de_n, spins r_n and time
// steps dt_n, from the stress st and the state sv (Euler angles, slip
// resistances) it holds, and commits each increment as UPDATE_GPTV does
// (src/fasolt/Fasolt3.f90:254-284): st <- the new stress, sv <- sv + dsv.
// Each increment starts as the first Newton iteration of an increment does:
// dsv = 0 (orientation and slip resistances of the start of the increment)
// and a stress guess, here the elastic predictor S^-1 de, so that CPSTRS
// runs.  Twin systems carry no slip in CPSTRS; a twin that triggers is
// flagged but not reoriented within a replay.
//
// Objective.  J = sum_g w_g (q^T e_g q - y_g)^2 / 2 over the lattice strain
// e_g = S(phi_g) st_g of the final state (ELASEPS, src/csvmkr/data_out.f90:
// 263-361, engineering shears) along a scattering direction q.  The caller
// chooses the weights, e.g. 1 / count for the GPs of an orientation bin and
// 0 elsewhere; they are constants of the derivative.
//
// Derivative.  At every increment the converged local system of CPSTRS
// (src/fasolt/Cpstrs.f90:34-172, crys-cons.f90:24-128),
//     R_s = de - sum_a b_a g_a - S (s - t)                  = 0   (6 rows)
//     R_a = ln|tau_a| - ln s1_a - m_a ln(|g_a| / dt)       = 0   (each active system a)
// with tau = b^T s, t = TENS_ROT(r, st) and PLASTC's s1(g, s0), fixes the
// stress s and the active slips g as functions of the increment's input
// state z = (st, s0, phi) and of the hardening parameters p.  Its outputs
// are Y = (s, s1, phi + ECHROT(g, phi, r)).  For an adjoint Ybar of the
// outputs, the implicit function theorem gives
//     (dR/dx)^T lambda = (dY/dx)^T Ybar,
//     zbar = (dY/dz)^T Ybar - (dR/dz)^T lambda,   pbar += (dY/dp)^T Ybar - (dR/dp)^T lambda.
// The partial derivatives are the columns of one forward-mode dual pass of
// R and Y per input.  p shifts ampar(k, i) of every system i of the GP's
// material by the same amount, for k = 1 (rate exponent m), 2 (h0), 3 and
// 5 (saturation stress).  The elastic branch of DSTRSS has no local
// system; its output stress S^-1 de depends on phi only.
//
// Reverse sweep.  Checkpoints hold the state at the start of every
// segment of chk increments.  The reverse kernel takes the segments from
// the last.  The forward sweep has recorded the last segment: each
// increment's input state and converged system, in a per-GP record buffer.
// Every earlier segment is recomputed from its checkpoint (the forward
// sweep's code, so the same converged states) into that buffer.  Each
// segment is then swept backwards.
#pragma once

#include "fas_device.cuh"

namespace fasdev {

// ------------------------------------------------------------ dual numbers
// Value and one directional derivative.
struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double x) : v(x), d(0.0) {}
    __host__ __device__ Dual(double x, double y) : v(x), d(y) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual dsin(Dual a) { return Dual(sin(a.v), cos(a.v) * a.d); }
__device__ __forceinline__ Dual dcos(Dual a) { return Dual(cos(a.v), -sin(a.v) * a.d); }
__device__ __forceinline__ Dual dlog(Dual a) { return Dual(log(a.v), a.d / a.v); }
__device__ __forceinline__ Dual dexp(Dual a)
{
    const double e = exp(a.v);
    return Dual(e, e * a.d);
}
__device__ __forceinline__ Dual dsqrt(Dual a)
{
    const double r = sqrt(a.v);
    return Dual(r, a.d / (2.0 * r));
}
__device__ __forceinline__ Dual dfabs(Dual a) { return a.v < 0.0 ? -a : a; }
// x^y for x >= 0 with PLASTC's exact x^0 = 1 and x^1 = x
__device__ __forceinline__ Dual dpow01(Dual x, double y)
{
    if (y == 0.0) return Dual(1.0);
    if (y == 1.0) return x;
    if (x.v <= 0.0) return Dual(0.0);
    return dexp(y * dlog(x));
}

// ------------------------------------------- the reference's maps, in duals
// CTMATRX (src/fasolt/crys_math.f90:25-62)
__device__ __forceinline__ void ctmatrx_d(const Dual ph[3], Dual a[3][3], Dual aug[3])
{
    const Dual s1 = dsin(ph[0]), c1 = dcos(ph[0]), s2 = dsin(ph[2]), c2 = dcos(ph[2]);
    const Dual s = dsin(ph[1]), c = dcos(ph[1]);
    a[0][0] = c1 * c2 - s1 * s2 * c;
    a[1][0] = -(c1 * s2) - s1 * c2 * c;
    a[2][0] = s1 * s;
    a[0][1] = s1 * c2 + c1 * s2 * c;
    a[1][1] = -(s1 * s2) + c1 * c2 * c;
    a[2][1] = -(c1 * s);
    a[0][2] = s2 * s;
    a[1][2] = c2 * s;
    a[2][2] = c;
    aug[0] = s2;
    aug[1] = c2;
    aug[2] = s;
}

// ELASTC (src/fasolt/ela-plas.f90:12-86) from CTMATRX's a
__device__ __forceinline__ void elastc_d(const double *e, const Dual a0[3][3], Dual S[6][6])
{
    Dual a[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = a0[j][i];
    const int pi[6] = {0, 1, 2, 1, 2, 0}, pj[6] = {0, 1, 2, 2, 0, 1};
    for (int I = 0; I < 6; ++I) {
        const int i = pi[I], j = pj[I];
        const double mult = I < 3 ? 1.0 : 2.0;
        for (int J = I; J < 6; ++J) {
            const int k = pi[J], l = pj[J];
            const Dual t1 = a[i][0] * a[j][0] * a[k][0] * a[l][0] * e[0] +
                            a[i][1] * a[j][1] * a[k][1] * a[l][1] * e[1] +
                            a[i][2] * a[j][2] * a[k][2] * a[l][2] * e[2];
            const Dual t2 = (a[i][1] * a[j][1] * a[k][2] * a[l][2] + a[i][2] * a[j][2] * a[k][1] * a[l][1]) * e[3] +
                            (a[i][2] * a[j][2] * a[k][0] * a[l][0] + a[i][0] * a[j][0] * a[k][2] * a[l][2]) * e[4] +
                            (a[i][0] * a[j][0] * a[k][1] * a[l][1] + a[i][1] * a[j][1] * a[k][0] * a[l][0]) * e[5];
            const Dual t3 = (a[i][1] * a[j][2] * a[k][1] * a[l][2] + a[i][2] * a[j][1] * a[k][2] * a[l][1]) * e[6] +
                            (a[i][2] * a[j][0] * a[k][2] * a[l][0] + a[i][0] * a[j][2] * a[k][0] * a[l][2]) * e[7] +
                            (a[i][0] * a[j][1] * a[k][0] * a[l][1] + a[i][1] * a[j][0] * a[k][1] * a[l][0]) * e[8];
            S[I][J] = mult * (t1 + t2 + 0.5 * t3);
        }
    }
    for (int I = 0; I < 5; ++I)
        for (int J = I + 1; J < 6; ++J) S[J][I] = S[I][J];
}

// TENS_ROT (src/fasolt/Sig_eps.f90:166-202) of a dual tensor by a fixed spin
__device__ __forceinline__ void tens_rot_d(const double r[3], const Dual a[6], Dual b[6])
{
    double rot[3][3];
    Dual old[3][3], tmp[3][3];
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        old[i][i] = a[i];
        old[j][k] = a[i + 3];
        old[k][j] = a[i + 3];
        rot[j][k] = r[i];
        rot[k][j] = -r[i];
        rot[i][i] = sqrt(1.0 - r[j] * r[j] - r[k] * r[k]);
    }
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q)
            tmp[p][q] = old[p][0] * rot[0][q] + old[p][1] * rot[1][q] + old[p][2] * rot[2][q];
    for (int i = 0; i < 3; ++i) {
        const int j = (i + 1) % 3, k = (j + 1) % 3;
        b[i] = rot[0][i] * tmp[0][i] + rot[1][i] * tmp[1][i] + rot[2][i] * tmp[2][i];
        b[i + 3] = rot[0][j] * tmp[0][k] + rot[1][j] * tmp[1][k] + rot[2][j] * tmp[2][k];
    }
}

// The ampar(k) entries the parameter adjoint covers (1-based k = 1, 2, 3, 5).
constexpr int ADJ_NP = 4;
__host__ __device__ constexpr int adj_ampar_index(int j) { return j < 3 ? j : 4; }

// Inputs of one increment's local system, as dual numbers.
template <int NS> struct AdjIn {
    Dual st[6], s0[NS], ph[3];   // state at the start of the increment
    Dual s[6], g[NS];            // converged stress, signed slips (0 off the active set)
    Dual p[ADJ_NP];              // shifts of ampar(1), (2), (3), (5)
};

// Orientation values of one increment: CTMATRX's a and aug, ELASTC's S,
// and the rotated slip direction and plane normal of every active system
// (isa order).  Only the dual passes that perturb the Euler angles need
// their derivatives; the others take these values.
template <int NS> struct AdjOrient {
    double a[3][3], aug[3], S[6][6], sdr[NS][3], spn[NS][3];
};

template <int NS>
__device__ void adj_orient(const DevMat &M, int mc, int nsa, const int *isa, const double ph[3],
                           AdjOrient<NS> &o)
{
    ctmatrx(ph[0], ph[1], ph[2], o.a, o.aug);
    elastc(M.e + 9 * mc, ph[0], ph[1], ph[2], o.S);
    const double *ab = M.ab + (size_t)mc * MAXSS * 3;
    const double *an = M.an + (size_t)mc * MAXSS * 3;
    for (int q = 0; q < nsa; ++q) {
        const int i = isa[q];
        for (int j = 0; j < 3; ++j) {
            o.sdr[q][j] = o.a[0][j] * ab[3 * i] + o.a[1][j] * ab[3 * i + 1] + o.a[2][j] * ab[3 * i + 2];
            o.spn[q][j] = o.a[0][j] * an[3 * i] + o.a[1][j] * an[3 * i + 1] + o.a[2][j] * an[3 * i + 2];
        }
    }
}

// Residuals R (6 strain rows, then the active systems in isa order) and
// outputs Y (stress, slip resistances, Euler angles) of one increment.
// With `oc` the orientation values come from it (their derivatives are
// zero); without, they are formed from in.ph in dual arithmetic.
template <int NS>
__device__ void adj_eval(const DevMat &M, int mc, int ns, bool plastic, int nsa, const int *isa,
                         const double de[6], const double r[3], double dt, const AdjIn<NS> &in,
                         const AdjOrient<NS> *oc, Dual *R, Dual *Y)
{
    Dual a[3][3], aug[3], S[6][6];
    if (oc) {
        for (int i = 0; i < 3; ++i) {
            aug[i] = Dual(oc->aug[i]);
            for (int j = 0; j < 3; ++j) a[i][j] = Dual(oc->a[i][j]);
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) S[i][j] = Dual(oc->S[i][j]);
    } else {
        ctmatrx_d(in.ph, a, aug);
        elastc_d(M.e + 9 * mc, a, S);
    }
    if (!plastic) {
        // DSTRSS's elastic branch: new stress S^-1 de (Sig_eps.f90:137-145)
        double Sv[6][6], y[6];
        for (int i = 0; i < 6; ++i) {
            y[i] = de[i];
            for (int j = 0; j < 6; ++j) Sv[i][j] = S[i][j].v;
        }
        lu_factor<6>(6, &Sv[0][0]);
        lu_solve<6>(6, &Sv[0][0], y);
        double dy[6];
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
            for (int j = 0; j < 6; ++j) acc += S[i][j].d * y[j];
            dy[i] = -acc;
        }
        lu_solve<6>(6, &Sv[0][0], dy);
        for (int i = 0; i < 6; ++i) Y[i] = Dual(y[i], dy[i]);
        for (int i = 0; i < ns; ++i) Y[6 + i] = in.s0[i];
        for (int k = 0; k < 3; ++k) Y[6 + ns + k] = in.ph[k];
        return;
    }
    const double *amp = M.ampar + (size_t)mc * MAXSS * 6;
    const double *sm = M.sm + (size_t)mc * MAXSS * MAXSS;
    const double *ab = M.ab + (size_t)mc * MAXSS * 3;
    const double *an = M.an + (size_t)mc * MAXSS * 3;
    Dual t[6];
    tens_rot_d(r, in.st, t);
    // PLASTC (ela-plas.f90:110-201): s1 = s0 + smatrx diag(gradh) |g|
    Dual sumss(0.0);
    for (int i = 0; i < ns; ++i) sumss = sumss + dfabs(in.g[i]);
    Dual gradh[NS];
    for (int i = 0; i < ns; ++i) {
        const Dual A2 = Dual(amp[6 * i + 1]) + in.p[1], A3 = Dual(amp[6 * i + 2]) + in.p[2];
        const Dual A5 = Dual(amp[6 * i + 4]) + in.p[3];
        const Dual sst = A5 * dpow01(sumss / Dual(dt), amp[6 * i + 5]);
        Dual arg = sst.v != 0.0 ? Dual(1.0) - in.s0[i] / sst : Dual(0.0);
        if (arg.v < 0.0) arg = Dual(0.0);
        gradh[i] = A3 + A2 * dpow01(arg, amp[6 * i + 3]);
    }
    Dual s1[NS];
    for (int i = 0; i < ns; ++i) {
        Dual acc = in.s0[i];
        for (int j = 0; j < ns; ++j)
            if (in.g[j].v != 0.0) acc = acc + (sm[i * ns + j] * gradh[j]) * dfabs(in.g[j]);
        s1[i] = acc;
    }
    // BTMATRX (crys_math.f90:75-115) of the active systems; residuals
    Dual eps_p[6], rtn[3];
    for (int k = 0; k < 6; ++k) eps_p[k] = Dual(0.0);
    for (int k = 0; k < 3; ++k) rtn[k] = Dual(-r[k]);
    for (int q = 0; q < nsa; ++q) {
        const int i = isa[q];
        Dual sdr[3], spn[3];
        for (int j = 0; j < 3; ++j) {
            if (oc) {
                sdr[j] = Dual(oc->sdr[q][j]);
                spn[j] = Dual(oc->spn[q][j]);
            } else {
                sdr[j] = a[0][j] * ab[3 * i] + a[1][j] * ab[3 * i + 1] + a[2][j] * ab[3 * i + 2];
                spn[j] = a[0][j] * an[3 * i] + a[1][j] * an[3 * i + 1] + a[2][j] * an[3 * i + 2];
            }
        }
        Dual b[6];
        b[0] = sdr[0] * spn[0];
        b[1] = sdr[1] * spn[1];
        b[2] = sdr[2] * spn[2];
        b[3] = sdr[1] * spn[2] + sdr[2] * spn[1];
        b[4] = sdr[2] * spn[0] + sdr[0] * spn[2];
        b[5] = sdr[0] * spn[1] + sdr[1] * spn[0];
        Dual tau(0.0);
        for (int k = 0; k < 6; ++k) {
            tau = tau + b[k] * in.s[k];
            eps_p[k] = eps_p[k] + b[k] * in.g[i];
        }
        rtn[0] = rtn[0] + 0.5 * (sdr[1] * spn[2] - sdr[2] * spn[1]) * in.g[i];
        rtn[1] = rtn[1] + 0.5 * (sdr[2] * spn[0] - sdr[0] * spn[2]) * in.g[i];
        rtn[2] = rtn[2] + 0.5 * (sdr[0] * spn[1] - sdr[1] * spn[0]) * in.g[i];
        const Dual m = Dual(amp[6 * i]) + in.p[0];
        R[6 + q] = dlog(dfabs(tau)) - dlog(s1[i]) - m * dlog(dfabs(in.g[i]) / Dual(dt));
    }
    for (int k = 0; k < 6; ++k) {
        Dual acc = Dual(de[k]) - eps_p[k];
        for (int c = 0; c < 6; ++c) acc = acc - S[k][c] * (in.s[c] - t[c]);
        R[k] = acc;
    }
    for (int k = 0; k < 6; ++k) Y[k] = in.s[k];
    for (int i = 0; i < ns; ++i) Y[6 + i] = s1[i];
    // ECHROT (crys_math.f90:137-167)
    Dual rx[3];
    for (int k = 0; k < 3; ++k) rx[k] = a[k][0] * rtn[0] + a[k][1] * rtn[1] + a[k][2] * rtn[2];
    const Dual dp1 = fabs(aug[2].v) < 1.e-5 ? rtn[2] : (aug[0] * rx[0] + aug[1] * rx[1]) / aug[2];
    const Dual dph = aug[1] * rx[0] - aug[0] * rx[1];
    const Dual dp2 = rx[2] - dp1 * a[2][2];
    Y[6 + ns] = in.ph[0] + dp1;
    Y[6 + ns + 1] = in.ph[1] + dph;
    Y[6 + ns + 2] = in.ph[2] + dp2;
}

// Gaussian elimination with partial pivoting, A (n x n, row stride n)
// overwritten; x holds the right-hand side and receives the solution.
// Returns 1 for a zero pivot.
__device__ __forceinline__ int adj_solve(int n, double *A, double *x)
{
    for (int k = 0; k < n; ++k) {
        int piv = k;
        double best = fabs(A[k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[i * n + k]) > best) {
                best = fabs(A[i * n + k]);
                piv = i;
            }
        if (best == 0.0) return 1;
        if (piv != k) {
            for (int j = 0; j < n; ++j) {
                const double tmp = A[k * n + j];
                A[k * n + j] = A[piv * n + j];
                A[piv * n + j] = tmp;
            }
            const double tmp = x[k];
            x[k] = x[piv];
            x[piv] = tmp;
        }
        for (int i = k + 1; i < n; ++i) {
            const double l = A[i * n + k] / A[k * n + k];
            for (int j = k; j < n; ++j) A[i * n + j] -= l * A[k * n + j];
            x[i] -= l * x[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double acc = x[i];
        for (int j = i + 1; j < n; ++j) acc -= A[i * n + j] * x[j];
        x[i] = acc / A[i * n + i];
    }
    return 0;
}

// One increment backwards: ybar (adjoint of the outputs: stress 6, slip
// resistances ns, Euler angles 3) becomes the adjoint of the increment's
// input state; pbar accumulates the parameter adjoint.  zst/zs0/zph are
// the input state, xs/xg the converged stress and signed slips.
template <int NS>
__device__ int adj_step(const DevMat &M, int mc, int ns, bool plastic, const double de[6], const double r[3],
                        double dt, const double zst[6], const double *zs0, const double zph[3],
                        const double xs[6], const double *xg, double *ybar, double pbar[ADJ_NP])
{
    constexpr int NX = 6 + NS;
    int isa[NS], nsa = 0;
    if (plastic)
        for (int i = 0; i < ns; ++i)
            if (xg[i] != 0.0) isa[nsa++] = i;
    const int nx = plastic ? 6 + nsa : 0, ny = 9 + ns;
    AdjIn<NS> in;
    for (int k = 0; k < 6; ++k) {
        in.st[k] = Dual(zst[k]);
        in.s[k] = Dual(xs[k]);
    }
    for (int i = 0; i < ns; ++i) {
        in.s0[i] = Dual(zs0[i]);
        in.g[i] = Dual(xg[i]);
    }
    for (int k = 0; k < 3; ++k) in.ph[k] = Dual(zph[k]);
    for (int k = 0; k < ADJ_NP; ++k) in.p[k] = Dual(0.0);
    Dual R[NX], Y[NX + 3];
    double A[NX * NX], lam[NX];
    AdjOrient<NS> oc;
    adj_orient<NS>(M, mc, nsa, isa, zph, oc);
    // x passes: columns of dR/dx, and (dY/dx)^T ybar
    for (int j = 0; j < nx; ++j) {
        Dual &xj = j < 6 ? in.s[j] : in.g[isa[j - 6]];
        xj.d = 1.0;
        adj_eval<NS>(M, mc, ns, plastic, nsa, isa, de, r, dt, in, &oc, R, Y);
        xj.d = 0.0;
        double acc = 0.0;
        for (int i = 0; i < ny; ++i) acc += ybar[i] * Y[i].d;
        lam[j] = acc;
        for (int i = 0; i < nx; ++i) A[j * nx + i] = R[i].d;   // row j of (dR/dx)^T
    }
    if (nx > 0 && adj_solve(nx, A, lam)) return 910;
    // z and p passes
    double zbar[NX + 3];
    const int nz = 9 + ns;
    for (int j = 0; j < nz + ADJ_NP; ++j) {
        Dual &v = j < 6 ? in.st[j] : j < 6 + ns ? in.s0[j - 6] : j < nz ? in.ph[j - 6 - ns] : in.p[j - nz];
        v.d = 1.0;
        const bool euler = j >= 6 + ns && j < nz;   // only these passes move the orientation
        adj_eval<NS>(M, mc, ns, plastic, nsa, isa, de, r, dt, in, euler ? nullptr : &oc, R, Y);
        v.d = 0.0;
        double acc = 0.0;
        for (int i = 0; i < ny; ++i) acc += ybar[i] * Y[i].d;
        for (int i = 0; i < nx; ++i) acc -= lam[i] * R[i].d;
        if (j < nz) zbar[j] = acc;
        else pbar[j - nz] += acc;
    }
    for (int j = 0; j < nz; ++j) ybar[j] = zbar[j];
    return 0;
}

// Lattice strain along q of stress st at orientation ph, e = S(ph) st,
// q^T e q with engineering shears.
__device__ __forceinline__ Dual lattice_q(const double *e9, const Dual st[6], const Dual ph[3], const double q[3])
{
    Dual a[3][3], aug[3], S[6][6];
    ctmatrx_d(ph, a, aug);
    elastc_d(e9, a, S);
    const double qq[6] = {q[0] * q[0], q[1] * q[1], q[2] * q[2], q[1] * q[2], q[2] * q[0], q[0] * q[1]};
    Dual acc(0.0);
    for (int i = 0; i < 6; ++i) {
        Dual ei(0.0);
        for (int c = 0; c < 6; ++c) ei = ei + S[i][c] * st[c];
        acc = acc + qq[i] * ei;
    }
    return acc;
}

// The objective's share of one GP and its adjoint on the final state
// (ybar: stress 6, slip resistances ns (zero), Euler angles 3).
__device__ __forceinline__ double objective_seed(const double *e9, int ns, const double st[6], const double ph[3],
                                                 const double q[3], double w, double y, double *eq,
                                                 double *ybar)
{
    Dual dst[6], dph[3];
    for (int k = 0; k < 6; ++k) dst[k] = Dual(st[k]);
    for (int k = 0; k < 3; ++k) dph[k] = Dual(ph[k]);
    const double e = lattice_q(e9, dst, dph, q).v;
    *eq = e;
    const double f = w * (e - y);
    for (int j = 0; j < 9; ++j) {
        Dual &v = j < 6 ? dst[j] : dph[j - 6];
        v.d = 1.0;
        const double de = lattice_q(e9, dst, dph, q).d;
        v.d = 0.0;
        ybar[j < 6 ? j : 6 + ns + (j - 6)] = f * de;
    }
    for (int i = 0; i < ns; ++i) ybar[6 + i] = 0.0;
    return 0.5 * w * (e - y) * (e - y);
}

// ------------------------------------------------------------ the replay
// The history and objective of a replay.  de: de(6, ngps, ninc), dr:
// dr(3, ngps, ninc), dt: dt(ninc), w / y: per GP.
struct ReplayDev {
    const double *de, *dr, *dt, *w, *y;
    double q[3];
    int ninc, chk;
    int zs;          // stride (in rows of ngps) of one state record: 9 + the widest ns
};

// One replayed increment of GP g (above): DSTRSS from st and the state in
// G.sv, then the commit.  st becomes the new stress, G.sv the new state;
// xg receives the signed converged slips (|g| = srate dt, the sign of
// tau = b^T s) and `plastic` whether CPSTRS ran.  Returns 0 or a FAFERR code.
template <int NS>
__device__ int replay_step(const DevMat &M, const DevCtrl &C, const DevGp &G, int g, int iel, int ns,
                           const double de[6], const double r[3], double dt, int inc, double st[6],
                           double *xg, bool &plastic)
{
    const int ng = G.ngps;
    const int mc = (iel < 0 ? -iel : iel) - 1;
    for (int k = 0; k < 3 + ns; ++k) G.dsv[k * ng + g] = 0.0;
    const double ph1 = G.sv[g], phi = G.sv[ng + g], ph2 = G.sv[2 * ng + g];
    double S[6][6], ds[6];
    elastc(M.e + 9 * mc, ph1, phi, ph2, S);
    for (int k = 0; k < 6; ++k) ds[k] = de[k];
    if (lu_factor<6>(6, &S[0][0])) return 910;
    lu_solve<6>(6, &S[0][0], ds);
    GpOut o;
    const int rc = dstrss<NS>(M, C, G, g, iel, de, r, st, ds, dt, inc, 1, o);
    if (rc) return rc;
    plastic = G.cp_iters[g] > 0;
    if (plastic) {
        double a[3][3], aug[3];
        ctmatrx(ph1, phi, ph2, a, aug);
        const double *ab = M.ab + (size_t)mc * MAXSS * 3;
        const double *an = M.an + (size_t)mc * MAXSS * 3;
        for (int i = 0; i < ns; ++i) {
            const double sr = G.srate[i * ng + g];
            double sdr[3], spn[3];
            for (int j = 0; j < 3; ++j) {
                sdr[j] = a[0][j] * ab[3 * i] + a[1][j] * ab[3 * i + 1] + a[2][j] * ab[3 * i + 2];
                spn[j] = a[0][j] * an[3 * i] + a[1][j] * an[3 * i + 1] + a[2][j] * an[3 * i + 2];
            }
            const double tau = sdr[0] * spn[0] * o.t[0] + sdr[1] * spn[1] * o.t[1] + sdr[2] * spn[2] * o.t[2] +
                               (sdr[1] * spn[2] + sdr[2] * spn[1]) * o.t[3] +
                               (sdr[2] * spn[0] + sdr[0] * spn[2]) * o.t[4] +
                               (sdr[0] * spn[1] + sdr[1] * spn[0]) * o.t[5];
            xg[i] = sr > 0.0 ? copysign(sr * dt, tau) : 0.0;
        }
    } else {
        for (int i = 0; i < ns; ++i) xg[i] = 0.0;
    }
    for (int k = 0; k < 6; ++k) st[k] = o.t[k];
    for (int k = 0; k < 3 + ns; ++k) G.sv[k * ng + g] = G.sv[k * ng + g] + G.dsv[k * ng + g];
    return 0;
}

__device__ __forceinline__ void replay_load(const ReplayDev &H, int n, int g, int ng, double de[6], double r[3])
{
    const double *pe = H.de + ((size_t)n * ng + g) * 6;
    const double *pr = H.dr + ((size_t)n * ng + g) * 3;
    for (int k = 0; k < 6; ++k) de[k] = pe[k];
    for (int k = 0; k < 3; ++k) r[k] = pr[k];
}

// Forward sweep: G.sv holds the starting state (a copy of the handle's),
// st0 the starting stress ([6][ngps]).  Writes the checkpoints
// chk[(seg * zs + k) * ngps + g] (stress 6, Euler angles 3, slip
// resistances), the objective share Jg and the final lattice strain eq.
// With `rec` it also writes the last segment's records (the layout of
// k_replay_adj), so the reverse sweep need not recompute that segment;
// G.sv is left holding the final state.
template <int NS>
__global__ void __launch_bounds__(128) k_replay_fwd(DevMat M, DevCtrl C, DevGp G, const int *gp_iel,
                                                    const double *st0, ReplayDev H, double *chk, double *rec,
                                                    int rs, double *Jg, double *eq, unsigned long long *errkey)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int ng = G.ngps;
    if (g >= ng) return;
    const int iel = gp_iel[g], mc = (iel < 0 ? -iel : iel) - 1, ns = M.ns[mc];
    const int nlast = (H.ninc - 1) / H.chk * H.chk;   // first increment of the last segment
    double st[6], de[6], r[3], xg[NS];
    auto R = [&](int j, int k) -> double & { return rec[((size_t)j * rs + k) * ng + g]; };
    for (int k = 0; k < 6; ++k) st[k] = st0[k * ng + g];
    for (int n = 0; n < H.ninc; ++n) {
        if (n % H.chk == 0) {
            double *c = chk + (size_t)(n / H.chk) * H.zs * ng + g;
            for (int k = 0; k < 6; ++k) c[(size_t)k * ng] = st[k];
            for (int k = 0; k < 3 + ns; ++k) c[(size_t)(6 + k) * ng] = G.sv[k * ng + g];
        }
        const bool keep = rec && n >= nlast;
        const int j = n - nlast;
        if (keep) {
            for (int k = 0; k < 6; ++k) R(j, k) = st[k];
            for (int k = 0; k < 3 + ns; ++k) R(j, 6 + k) = G.sv[k * ng + g];
        }
        replay_load(H, n, g, ng, de, r);
        bool plastic = false;
        const int rc = replay_step<NS>(M, C, G, g, iel, ns, de, r, H.dt[n], n + 1, st, xg, plastic);
        if (rc) {
            atomicMin(errkey, ((unsigned long long)g << 16) | (unsigned long long)rc);
            return;
        }
        if (keep) {
            for (int k = 0; k < 6; ++k) R(j, H.zs + k) = st[k];
            for (int i = 0; i < ns; ++i) R(j, H.zs + 6 + i) = xg[i];
            R(j, H.zs + 6 + NS) = plastic ? 1.0 : 0.0;
        }
    }
    const double ph[3] = {G.sv[g], G.sv[ng + g], G.sv[2 * ng + g]};
    double ybar[9 + NS], e;
    Jg[g] = objective_seed(M.e + 9 * mc, ns, st, ph, H.q, H.w[g], H.y[g], &e, ybar);
    eq[g] = e;
}

// Reverse sweep (above), after k_replay_fwd with records.  rec holds chk
// increments of records per GP:
// record j at rec[(j * rs + k) * ngps + g], rs = zs + 6 + NS + 1 rows: input
// state (stress, Euler angles, slip resistances), converged stress,
// signed slips, branch.  Writes the adjoints of the starting stress
// g_st[6][ngps], of the starting state g_sv[zs - 6][ngps] (Euler angles,
// slip resistances) and of the parameters g_p[ADJ_NP][ngps].
template <int NS>
__global__ void __launch_bounds__(128) k_replay_adj(DevMat M, DevCtrl C, DevGp G, const int *gp_iel, ReplayDev H,
                                                    const double *chk, double *rec, int rs, double *Jg,
                                                    double *g_st, double *g_sv, double *g_p,
                                                    unsigned long long *errkey)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int ng = G.ngps;
    if (g >= ng) return;
    const int iel = gp_iel[g], mc = (iel < 0 ? -iel : iel) - 1, ns = M.ns[mc];
    const int nseg = (H.ninc + H.chk - 1) / H.chk;
    double ybar[9 + NS], pbar[ADJ_NP] = {0.0, 0.0, 0.0, 0.0};
    double st[6], de[6], r[3], xg[NS];
    auto R = [&](int j, int k) -> double & { return rec[((size_t)j * rs + k) * ng + g]; };
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int n0 = sg * H.chk, n1 = min(H.ninc, n0 + H.chk);
        if (sg == nseg - 1) {
            // recorded by the forward sweep, which left the final state in G.sv
            for (int k = 0; k < 6; ++k) st[k] = R(n1 - 1 - n0, H.zs + k);
        } else {
            const double *c = chk + (size_t)sg * H.zs * ng + g;
            for (int k = 0; k < 6; ++k) st[k] = c[(size_t)k * ng];
            for (int k = 0; k < 3 + ns; ++k) G.sv[k * ng + g] = c[(size_t)(6 + k) * ng];
        }
        for (int n = n0; n < n1 && sg < nseg - 1; ++n) {
            const int j = n - n0;
            for (int k = 0; k < 6; ++k) R(j, k) = st[k];
            for (int k = 0; k < 3 + ns; ++k) R(j, 6 + k) = G.sv[k * ng + g];
            replay_load(H, n, g, ng, de, r);
            bool plastic = false;
            const int rc = replay_step<NS>(M, C, G, g, iel, ns, de, r, H.dt[n], n + 1, st, xg, plastic);
            if (rc) {
                atomicMin(errkey, ((unsigned long long)g << 16) | (unsigned long long)rc);
                return;
            }
            for (int k = 0; k < 6; ++k) R(j, H.zs + k) = st[k];
            for (int i = 0; i < ns; ++i) R(j, H.zs + 6 + i) = xg[i];
            R(j, H.zs + 6 + NS) = plastic ? 1.0 : 0.0;
        }
        if (sg == nseg - 1) {
            const double ph[3] = {G.sv[g], G.sv[ng + g], G.sv[2 * ng + g]};
            double e;
            Jg[g] = objective_seed(M.e + 9 * mc, ns, st, ph, H.q, H.w[g], H.y[g], &e, ybar);
        }
        for (int n = n1 - 1; n >= n0; --n) {
            const int j = n - n0;
            double zst[6], zph[3], zs0[NS], xs[6];
            for (int k = 0; k < 6; ++k) {
                zst[k] = R(j, k);
                xs[k] = R(j, H.zs + k);
            }
            for (int k = 0; k < 3; ++k) zph[k] = R(j, 6 + k);
            for (int i = 0; i < ns; ++i) {
                zs0[i] = R(j, 9 + i);
                xg[i] = R(j, H.zs + 6 + i);
            }
            const bool plastic = R(j, H.zs + 6 + NS) != 0.0;
            replay_load(H, n, g, ng, de, r);
            // ybar is ordered (stress, slip resistances, Euler angles)
            const int rc = adj_step<NS>(M, mc, ns, plastic, de, r, H.dt[n], zst, zs0, zph, xs, xg, ybar, pbar);
            if (rc) {
                atomicMin(errkey, ((unsigned long long)g << 16) | (unsigned long long)rc);
                return;
            }
        }
    }
    for (int k = 0; k < 6; ++k) g_st[k * ng + g] = ybar[k];
    for (int k = 0; k < 3; ++k) g_sv[k * ng + g] = ybar[6 + ns + k];
    for (int i = 0; i < ns; ++i) g_sv[(3 + i) * ng + g] = ybar[6 + i];
    for (int k = 0; k < ADJ_NP; ++k) g_p[k * ng + g] = pbar[k];
}

}  // namespace fasdev
