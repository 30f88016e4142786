// fasolt_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never shipped
// on the product path).  CPU restatement of FASOLT3's per-increment hot path,
// following gabortimar/CPFEM_code src/fasolt/*.f90 routine by routine; each
// function cites the reference lines it restates.  Parity is unpinned by the
// reference itself (it has no tests or golden outputs, and no Fortran
// compiler exists here); physics known-answer tests pin this restatement.
//
// Templated on the arithmetic type R: double = the reference promoted to
// REAL(8) (the FP64 oracle), float = the FP32-faithful restatement.
// Internal arrays are 0-based; the descriptors carry the reference's 1-based,
// column-major module arrays.

#include "fasolt_oracle.h"
#include "../cpfem_code_b200/csrc/fas_flops.h"
#include "../cpfem_code_b200/csrc/fas_rng.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int MAXSS = FAS_MAXSS;   // maxss, fas-com-mod.f90:57
constexpr int SVLD = 63;           // maxsvs, fas-com-mod.f90:14

inline double rdv(const void *p, int rb, size_t i)
{
    return rb == 4 ? (double)((const float *)p)[i] : ((const double *)p)[i];
}
inline void wrv(void *p, int rb, size_t i, double v)
{
    if (rb == 4) ((float *)p)[i] = (float)v;
    else ((double *)p)[i] = v;
}

// ---------------------------------------------------------------- material
template <class R> struct Material {
    int ns = 0;
    R e[9];
    R ssang[MAXSS];
    R ab[MAXSS][3], an[MAXSS][3];
    R ampar[MAXSS][10];
    std::vector<R> sm;   // sm[i*ns+j] = smatrx(i,j)
};

// ---------------------------------------------------------------- problem
template <class R> struct Problem {
    int nlmnt = 0, nnod = 0, ngps = 0, ldn = 8;
    std::vector<int> le, lt, nd, np, ln, lg, ib, gp_iel;
    int nmatl = 0, nmpar = 0, twinlim = 0;
    R twinprob = 0;
    std::vector<Material<R>> mat;
    R toler, alpha, afactor, efix, smale, smalr;
    int maxit = 100, ninc1 = 0, nxs = 0, nfs = 0;
    std::vector<R> tiem, xspec, fspec;   // xspec[(inc*nxs+code)*15+k]
    unsigned long long seed = 0;
    // state
    int nsv = 0;
    bool have_state = false;
    std::vector<R> x, dx, fc, ddx, eps, dep, st, ep, ds, de, rt, dr, sv, dsv,
        srate, cumslip;
    std::vector<int> timestwinned, twinsys;
    int tflag = 0;
    // compact stiffness (SETPTA layout)
    int ld = 0;                     // entries per row: 1 + max off-diagonals
    std::vector<int> is;            // is[row*ld + k]; k=0 count, 1.. cols (0-based)
    std::vector<R> ss;              // ss[row*ld + k]; k=0 diagonal
    // SOR colouring
    std::vector<int> colour;
    int ncol = 0;
    std::vector<int> colour_order;  // nodes sorted by (colour, id)
    // diagnostics of the last constitutive pass
    std::vector<int> cp_iters;
    std::vector<R> erepmd_gp;
    std::vector<double> ops_gp;
    std::vector<R> chi_gp;          // chi[gp*36 + i + 6*j] = chi(i,j)
    R sumcpiter = 0;
    uint32_t mode = 0;
    int nthreads = 1;
    int last_mat = 1;               // mat_code left by the last DSTRSS call
};

// ================================================================ crystal math
// FJ2VOM, src/fasolt/Sig_eps.f90:217-241
template <class R> R fj2vom(bool stress, const R *x)
{
    const R amult = stress ? R(6.0) : R(1.5);
    R sum = 0;
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3;
        sum = sum + (x[i] - x[j]) * (x[i] - x[j]) + amult * x[i + 3] * x[i + 3];
    }
    return std::sqrt(sum / R(4.5));
}

// SPOWER, src/fasolt/crys-cons.f90:210-230
template <class R> R spower(R a, R b)
{
    R aa = std::fabs(a);
    if (aa < R(1.e-35)) return R(0);
    R sparg = b * std::log(aa);
    if (sparg < R(-80.0)) sparg = R(-80.0);
    if (sparg > R(80.0)) sparg = R(80.0);
    return std::copysign(std::exp(sparg), a);
}

// FACTOR, src/fasolt/crys-cons.f90:244-269.  w[i*ld+j] = w(i,j).
template <class R> int factor(int n, R *w, int ld)
{
    for (int k = 0; k < n - 1; ++k)
        for (int i = k + 1; i < n; ++i) {
            if (w[k * ld + k] == R(0)) return 1;
            w[i * ld + k] = w[i * ld + k] / w[k * ld + k];
            for (int j = k + 1; j < n; ++j)
                w[i * ld + j] = w[i * ld + j] - w[i * ld + k] * w[k * ld + j];
        }
    if (w[(n - 1) * ld + (n - 1)] == R(0)) return 1;
    return 0;
}

// SOLVER, src/fasolt/crys-cons.f90:283-309
template <class R> void solver(int n, const R *w, int ld, R *x)
{
    for (int i = 1; i < n; ++i)
        for (int j = 0; j < i; ++j) x[i] = x[i] - w[i * ld + j] * x[j];
    x[n - 1] = x[n - 1] / w[(n - 1) * ld + (n - 1)];
    for (int i = n - 2; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) x[i] = x[i] - w[i * ld + j] * x[j];
        x[i] = x[i] / w[i * ld + i];
    }
}

// CTMATRX, src/fasolt/crys_math.f90:25-62.  a[i][j] = a(i+1,j+1).
template <class R> void ctmatrx(R ph1, R phi, R ph2, R a[3][3], R aug[3])
{
    R c1 = std::cos(ph1), s1 = std::sin(ph1);
    R c2 = std::cos(ph2), s2 = std::sin(ph2);
    R c = std::cos(phi), s = std::sin(phi);
    R c1c2 = c1 * c2, s1s2 = s1 * s2, c1s2 = c1 * s2, s1c2 = s1 * c2;
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

// ELASTC, src/fasolt/ela-plas.f90:12-86: rotated compliance, engineering
// shears, from e(1:9) = S11,S22,S33,S23,S31,S12,S44,S55,S66.
template <class R> void elastc(const R e[9], R ph1, R phi, R ph2, R S[6][6])
{
    R a0[3][3], aug[3], a[3][3];
    ctmatrx(ph1, phi, ph2, a0, aug);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = a0[j][i];   // crystal -> specimen
    static const int pi[6] = {0, 1, 2, 1, 2, 0}, pj[6] = {0, 1, 2, 2, 0, 1};
    for (int is = 0; is < 6; ++is) {
        int i = pi[is], j = pj[is];
        R mult = is < 3 ? R(1.0) : R(2.0);
        for (int js = is; js < 6; ++js) {
            int k = pi[js], l = pj[js];
            R term1 = a[i][0] * a[j][0] * a[k][0] * a[l][0] * e[0]
                    + a[i][1] * a[j][1] * a[k][1] * a[l][1] * e[1]
                    + a[i][2] * a[j][2] * a[k][2] * a[l][2] * e[2];
            R term2 = a[i][1] * a[j][1] * a[k][2] * a[l][2] * e[3]
                    + a[i][2] * a[j][2] * a[k][1] * a[l][1] * e[3]
                    + a[i][2] * a[j][2] * a[k][0] * a[l][0] * e[4]
                    + a[i][0] * a[j][0] * a[k][2] * a[l][2] * e[4]
                    + a[i][0] * a[j][0] * a[k][1] * a[l][1] * e[5]
                    + a[i][1] * a[j][1] * a[k][0] * a[l][0] * e[5];
            R term3 = a[i][1] * a[j][2] * a[k][1] * a[l][2] * e[6]
                    + a[i][2] * a[j][1] * a[k][2] * a[l][1] * e[6]
                    + a[i][2] * a[j][0] * a[k][2] * a[l][0] * e[7]
                    + a[i][0] * a[j][2] * a[k][0] * a[l][2] * e[7]
                    + a[i][0] * a[j][1] * a[k][0] * a[l][1] * e[8]
                    + a[i][1] * a[j][0] * a[k][1] * a[l][0] * e[8];
            S[is][js] = mult * (term1 + term2 + R(0.5) * term3);
        }
    }
    for (int is = 0; is < 5; ++is)
        for (int js = is + 1; js < 6; ++js) S[js][is] = S[is][js];
}

// TENS_ROT, src/fasolt/Sig_eps.f90:166-202: R^T a R for small rotation r.
template <class R> void tens_rot(const R r[3], const R a[6], R b[6])
{
    R rot[3][3], old[3][3], tmp[3][3], nw[3][3];
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3, k = (j + 1) % 3;
        old[i][i] = a[i];
        old[j][k] = a[i + 3];
        old[k][j] = old[j][k];
        rot[j][k] = r[i];
        rot[k][j] = -r[i];
        rot[i][i] = std::sqrt(R(1.0) - r[j] * r[j] - r[k] * r[k]);
    }
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) {
            R s = 0;
            for (int c = 0; c < 3; ++c) s = s + old[p][c] * rot[c][q];
            tmp[p][q] = s;
        }
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) {
            R s = 0;
            for (int c = 0; c < 3; ++c) s = s + rot[c][p] * tmp[c][q];
            nw[p][q] = s;
        }
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3, k = (j + 1) % 3;
        b[i] = nw[i][i];
        b[i + 3] = nw[j][k];
    }
}

// INVERT_3, src/fasolt/Shapef.f90:499-537 (m[r][c] = matrix(r+1,c+1)).
template <class R> R invert3(R m[3][3])
{
    R loc[3][3];
    std::memcpy(loc, m, sizeof(loc));
    for (int i = 0; i < 3; ++i) {
        int ia = (i + 1) % 3, ib = (ia + 1) % 3;
        for (int j = 0; j < 3; ++j) {
            int ja = (j + 1) % 3, jb = (ja + 1) % 3;
            m[j][i] = loc[ia][ja] * loc[ib][jb] - loc[ia][jb] * loc[ib][ja];
        }
    }
    R det = m[0][0] * loc[0][0] + m[0][1] * loc[1][0] + m[0][2] * loc[2][0];
    if (det != R(0))
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) m[i][j] = m[i][j] / det;
    return det;
}

// SHAPE_12, src/fasolt/Shapef.f90:32-86: 8-node brick, one GP at the centre.
// xn[i][k] = xnode(k+1,i+1); dndx[i][k] = dndx(k+1,i+1).
template <class R> R shape12(const R xn[8][3], R dndx[8][3])
{
    static const R dn[3][8] = {
        {-0.125, 0.125, 0.125, -0.125, -0.125, 0.125, 0.125, -0.125},
        {-0.125, -0.125, 0.125, 0.125, -0.125, -0.125, 0.125, 0.125},
        {-0.125, -0.125, -0.125, -0.125, 0.125, 0.125, 0.125, 0.125}};
    R jac[3][3];
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
            R s = 0;
            for (int i = 0; i < 8; ++i) s = s + dn[j][i] * xn[i][k];
            jac[j][k] = s;
        }
    R w = invert3(jac);
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) {
            R s = 0;
            for (int j = 0; j < 3; ++j) s = s + jac[k][j] * dn[j][i];
            dndx[i][k] = s;
        }
    return R(8.0) * w;
}

// SHAPE_22, src/fasolt/Shapef.f90:210-342: 20-node brick, 8 Gauss points at
// (+-1/sqrt3)^3, GPs 1-4 anticlockwise from node 1 at zeta = -1/sqrt3, 5-8
// above them.  The reference tabulates the local derivatives of the
// serendipity functions at its GPs to 6 decimals; shape22_table() evaluates
// the same functions at the GP coordinate 0.57735 and rounds them to 6
// decimals, which reproduces all 480 entries of that table (with the exact
// 1/sqrt3, 24 entries would differ in the last digit).  Local node
// positions follow ADDEL_20NQ's order (corners 1,3,5,7
// and mid-sides 2,4,6,8 at zeta = -1, vertical mid-edges 9-12, the top
// face 13-20 like the bottom one).
struct Shape22Table {
    double dn[8][3][20];   // dn[g][j][i] = dndn(j+1, i+1, g+1)
};
inline const Shape22Table &shape22_table()
{
    static const Shape22Table t = [] {
        static const int loc[20][3] = {{-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {1, 0, -1}, {1, 1, -1},
                                       {0, 1, -1},   {-1, 1, -1}, {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0},
                                       {1, 1, 0},    {-1, 1, 0},  {-1, -1, 1}, {0, -1, 1},  {1, -1, 1},
                                       {1, 0, 1},    {1, 1, 1},   {0, 1, 1},   {-1, 1, 1},  {-1, 0, 1}};
        static const int gsign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                        {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
        const double a = 0.57735;
        Shape22Table t{};
        for (int g = 0; g < 8; ++g) {
            const double q[3] = {gsign[g][0] * a, gsign[g][1] * a, gsign[g][2] * a};
            for (int i = 0; i < 20; ++i) {
                const int *c = loc[i];
                double d[3];
                if (c[0] && c[1] && c[2]) {   // corner
                    const double f[3] = {1 + q[0] * c[0], 1 + q[1] * c[1], 1 + q[2] * c[2]};
                    const double sum = q[0] * c[0] + q[1] * c[1] + q[2] * c[2] - 2;
                    for (int j = 0; j < 3; ++j) {
                        const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
                        d[j] = 0.125 * c[j] * f[j1] * f[j2] * (sum + f[j]);
                    }
                } else {                       // mid-edge: the zero coordinate is the edge's
                    const int z = !c[0] ? 0 : (!c[1] ? 1 : 2);
                    const int z1 = (z + 1) % 3, z2 = (z + 2) % 3;
                    const double f1 = 1 + q[z1] * c[z1], f2 = 1 + q[z2] * c[z2], e = 1 - q[z] * q[z];
                    d[z] = 0.25 * (-2 * q[z]) * f1 * f2;
                    d[z1] = 0.25 * e * c[z1] * f2;
                    d[z2] = 0.25 * e * f1 * c[z2];
                }
                for (int j = 0; j < 3; ++j) t.dn[g][j][i] = std::round(d[j] * 1e6) / 1e6;
            }
        }
        return t;
    }();
    return t;
}

// SHAPE_21, src/fasolt/Shapef.f90:104-189: 10-node tetrahedron, 4 Gauss
// points.  Corner nodes 1, 3, 5, 10 carry volume coordinates L1..L4;
// mid-edge nodes 2 (1,3), 4 (3,5), 6 (1,5), 7 (1,10), 8 (3,10), 9 (5,10).
// GP g has L_g = (5 + 3 sqrt5)/20 and the other three (5 - sqrt5)/20.  The
// reference's three local directions are L4, L2 and L1 with L3 dependent:
// dndn(k) = dN/dL_p(k) - dN/dL3 for p = (4, 2, 1), its derivatives of
// L(2L-1) (corners) and 4 L_i L_j (mid-edges) rounded to 6 decimals as the
// reference tabulates them -- which reproduces every entry of that table.
// weight = -0.0416667 det(J).
struct Shape21Table {
    double dn[4][3][10];   // dn[g][j][i] = dndn(j+1, i+1, g+1)
};
inline const Shape21Table &shape21_table()
{
    static const Shape21Table t = [] {
        static const int corner[10] = {0, -1, 1, -1, 2, -1, -1, -1, -1, 3};   // node -> L index
        static const int mid[10][2] = {{-1, -1}, {0, 1}, {-1, -1}, {1, 2}, {-1, -1},
                                       {0, 2},   {0, 3}, {1, 3},   {2, 3}, {-1, -1}};
        static const int dir[3] = {3, 1, 0};
        const double r5 = std::sqrt(5.0), a = (5.0 + 3.0 * r5) / 20.0, b = (5.0 - r5) / 20.0;
        Shape21Table t{};
        for (int g = 0; g < 4; ++g) {
            double L[4] = {b, b, b, b};
            L[g] = a;
            auto dNdL = [&](int i, int p) {
                if (corner[i] >= 0) return corner[i] == p ? 4.0 * L[p] - 1.0 : 0.0;
                const int u = mid[i][0], v = mid[i][1];
                return p == u ? 4.0 * L[v] : (p == v ? 4.0 * L[u] : 0.0);
            };
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 10; ++i)
                    t.dn[g][j][i] = std::round((dNdL(i, dir[j]) - dNdL(i, 2)) * 1e6) / 1e6;
        }
        return t;
    }();
    return t;
}

// SHAPE_23, src/fasolt/Shapef.f90:360-485: 15-node pentahedron (wedge), 6
// Gauss points.  Base corners 1, 3, 5 and top corners 10, 12, 14 carry area
// coordinates L1..L3 at zeta = -1 / +1; mid-edge nodes 2 (1,3), 4 (3,5),
// 6 (5,1) on the base, 11, 13, 15 on the top, 7, 8, 9 on the vertical
// edges.  GP g < 3 sits at L_(g) = 2/3, the others 1/6, zeta = -1/sqrt3;
// GPs 4-6 above them at +1/sqrt3.  Local directions L1 and L2 (L3
// dependent) and zeta; the serendipity wedge functions' derivatives rounded
// to 6 decimals.  This reproduces 210 of the reference's 270 tabulated
// entries; the other 60 differ from it by one unit in the sixth decimal
// (rounding of the reference's own tabulation).  weight = det(J) / 6.
struct Shape23Table {
    double dn[6][3][15];
};
inline const Shape23Table &shape23_table()
{
    static const Shape23Table t = [] {
        // node -> (kind, a, b, side): kind 0 corner (L a), 1 mid-edge (L a,
        // L b), 2 vertical mid-edge (L a); side -1 base, +1 top
        static const int kind[15] = {0, 1, 0, 1, 0, 1, 2, 2, 2, 0, 1, 0, 1, 0, 1};
        static const int la[15] = {0, 0, 1, 1, 2, 2, 0, 1, 2, 0, 0, 1, 1, 2, 2};
        static const int lb[15] = {-1, 1, -1, 2, -1, 0, -1, -1, -1, -1, 1, -1, 2, -1, 0};
        static const int side[15] = {-1, -1, -1, -1, -1, -1, 0, 0, 0, 1, 1, 1, 1, 1, 1};
        Shape23Table t{};
        for (int g = 0; g < 6; ++g) {
            double L[3] = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
            L[g % 3] = 2.0 / 3.0;
            const double z = (g < 3 ? -1.0 : 1.0) / std::sqrt(3.0);
            auto dNdL = [&](int i, int p) {   // at fixed zeta
                const double s = side[i];
                if (kind[i] == 0)
                    return la[i] == p ? 0.5 * (4.0 * L[p] - 1.0) * (1.0 + s * z) - 0.5 * (1.0 - z * z) : 0.0;
                if (kind[i] == 1) {
                    const double f = 2.0 * (1.0 + s * z);
                    return p == la[i] ? f * L[lb[i]] : (p == lb[i] ? f * L[la[i]] : 0.0);
                }
                return la[i] == p ? 1.0 - z * z : 0.0;
            };
            auto dNdz = [&](int i) {
                const double s = side[i], La = L[la[i]];
                if (kind[i] == 0) return 0.5 * La * (2.0 * La - 1.0) * s + La * z;
                if (kind[i] == 1) return 2.0 * La * L[lb[i]] * s;
                return -2.0 * z * La;
            };
            for (int i = 0; i < 15; ++i) {
                t.dn[g][0][i] = std::round((dNdL(i, 0) - dNdL(i, 2)) * 1e6) / 1e6;
                t.dn[g][1][i] = std::round((dNdL(i, 1) - dNdL(i, 2)) * 1e6) / 1e6;
                t.dn[g][2][i] = std::round(dNdz(i) * 1e6) / 1e6;
            }
        }
        return t;
    }();
    return t;
}

// The Jacobian, its inverse and the global derivatives of an NN-node
// element from tabulated local derivatives dn[j][i] (j local direction);
// returns det(J).  The steps of SHAPE_21/22/23 after their tables.
template <class R, int NN> R shape_tab(const double dn_t[3][NN], const R xn[20][3], R dndx[20][3])
{
    R dn[3][NN];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < NN; ++i) dn[j][i] = (R)dn_t[j][i];
    R jac[3][3];
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
            R s = 0;
            for (int i = 0; i < NN; ++i) s = s + dn[j][i] * xn[i][k];
            jac[j][k] = s;
        }
    R w = invert3(jac);
    for (int i = 0; i < NN; ++i)
        for (int k = 0; k < 3; ++k) {
            R s = 0;
            for (int j = 0; j < 3; ++j) s = s + jac[k][j] * dn[j][i];
            dndx[i][k] = s;
        }
    return w;
}
template <class R> R shape21(int g, const R xn[20][3], R dndx[20][3])
{
    return R(-0.0416667) * shape_tab<R, 10>(shape21_table().dn[g], xn, dndx);
}
template <class R> R shape23(int g, const R xn[20][3], R dndx[20][3])
{
    return R(0.16666667) * shape_tab<R, 15>(shape23_table().dn[g], xn, dndx);
}

// xn[i][k] = xnode(k+1,i+1); dndx[i][k] = dndx(k+1,i+1); g is 0-based.
template <class R> R shape22(int g, const R xn[20][3], R dndx[20][3])
{
    const Shape22Table &t = shape22_table();
    R dn[3][20];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 20; ++i) dn[j][i] = (R)t.dn[g][j][i];
    R jac[3][3];
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 3; ++j) {
            R s = 0;
            for (int i = 0; i < 20; ++i) s = s + dn[j][i] * xn[i][k];
            jac[j][k] = s;
        }
    R w = invert3(jac);
    for (int i = 0; i < 20; ++i)
        for (int k = 0; k < 3; ++k) {
            R s = 0;
            for (int j = 0; j < 3; ++j) s = s + jac[k][j] * dn[j][i];
            dndx[i][k] = s;
        }
    return R(1.0) * w;
}

// ================================================================ constitutive
// Per-GP working set: the FAS_CPL module scratch (fas-com-mod.f90:62-66),
// made private to one Gauss-point update.
template <class R> struct CpWork {
    const Material<R> *m;
    int ns, nsa;
    int isa[MAXSS];
    R tau[MAXSS], gam[MAXSS], s0[MAXSS], s1[MAXSS], wks[MAXSS];
    R b[MAXSS][6], rot[MAXSS][3];
    R ah[MAXSS * MAXSS];   // ah[i*MAXSS+j] = ah(i+1,j+1)
    R am[MAXSS];           // CPSTRS's am (set by SLPINI)
};

// BTMATRX, src/fasolt/crys_math.f90:75-115
template <class R> void btmatrx(const R a[3][3], CpWork<R> &w)
{
    const Material<R> &m = *w.m;
    for (int i = 0; i < w.ns; ++i) {
        R sdr[3], spn[3];
        for (int j = 0; j < 3; ++j) {
            R s1 = 0, s2 = 0;
            for (int l = 0; l < 3; ++l) {
                s1 = s1 + a[l][j] * m.ab[i][l];
                s2 = s2 + a[l][j] * m.an[i][l];
            }
            sdr[j] = s1;
            spn[j] = s2;
        }
        w.b[i][0] = sdr[0] * spn[0];
        w.b[i][1] = sdr[1] * spn[1];
        w.b[i][2] = sdr[2] * spn[2];
        w.b[i][3] = sdr[1] * spn[2] + sdr[2] * spn[1];
        w.b[i][4] = sdr[2] * spn[0] + sdr[0] * spn[2];
        w.b[i][5] = sdr[0] * spn[1] + sdr[1] * spn[0];
        w.rot[i][0] = (sdr[1] * spn[2] - sdr[2] * spn[1]) / R(2.0);
        w.rot[i][1] = (sdr[2] * spn[0] - sdr[0] * spn[2]) / R(2.0);
        w.rot[i][2] = (sdr[0] * spn[1] - sdr[1] * spn[0]) / R(2.0);
    }
}

// PLASTC, src/fasolt/ela-plas.f90:110-201: slip resistances s1 and the
// log-hardening matrix of the active systems.  `am` receives ampar(1,:).
template <class R> void plastc(CpWork<R> &w, R dt, R *am)
{
    const Material<R> &m = *w.m;
    const int ns = w.ns;
    for (int i = 0; i < ns; ++i) am[i] = m.ampar[i][0];
    R sumss = 0;
    for (int i = 0; i < ns; ++i) sumss = sumss + std::fabs(w.gam[i]);
    R gradh[MAXSS];
    for (int i = 0; i < ns; ++i) {
        R sst = m.ampar[i][4] * std::pow(sumss / dt, m.ampar[i][5]);
        R arg = (sst != R(0)) ? R(1.0) - (w.s0[i] / sst) : R(0);
        if (arg < R(0)) arg = R(0);
        gradh[i] = m.ampar[i][2]
                 + m.ampar[i][1] * std::copysign(std::pow(std::fabs(arg), m.ampar[i][3]), arg);
    }
    // gradient(iss,jss) = smatrx(iss,jss)*grad_h(jss)
    for (int i = 0; i < ns; ++i) {
        R s = w.s0[i];
        for (int j = 0; j < ns; ++j) s = s + (m.sm[i * ns + j] * gradh[j]) * std::fabs(w.gam[j]);
        w.s1[i] = s;
    }
    for (int i = 0; i < w.nsa; ++i) {
        int is = w.isa[i];
        for (int j = 0; j < w.nsa; ++j) {
            int js = w.isa[j];
            if (std::fabs(w.gam[js]) > R(1.e-14)) {
                R sgn = w.gam[js] / std::fabs(w.gam[js]);
                w.ah[i * MAXSS + j] = sgn * (m.sm[is * ns + js] * gradh[js]) / w.s1[is];
            } else {
                w.ah[i * MAXSS + j] = R(0);
            }
        }
    }
}

// SLPINI, src/fasolt/crys-cons.f90:143-197
template <class R>
void slpini(Problem<R> &P, CpWork<R> &w, int jgp, R dt, int inc, int nit, int cpit)
{
    const Material<R> &m = *w.m;
    for (int i = 0; i < w.ns; ++i) w.am[i] = m.ampar[i][0];
    R gammax = 0;
    for (int i = 0; i < w.ns; ++i) {
        if (std::fabs(m.ssang[i]) > R(1.5)) {
            w.gam[i] = 0;
            if (w.tau[i] > w.s0[i] && P.timestwinned[jgp] != P.twinlim && P.twinsys[jgp] == 0) {
                double u = fas_twin_u01(P.seed, jgp, inc, nit, cpit, i);
                if (u < (double)P.twinprob) {
                    P.tflag = 1;
                    P.twinsys[jgp] = i + 1;
                }
            }
        } else if (m.ssang[i] * w.tau[i] / w.s0[i] < R(0)) {
            w.gam[i] = 0;
        } else {
            w.gam[i] = dt * spower(w.tau[i] / w.s0[i], R(1.0) / w.am[i]);
        }
        if (std::fabs(w.gam[i]) > gammax) gammax = std::fabs(w.gam[i]);
    }
    R cutoff = R(1.e-6) * gammax;
    w.nsa = 0;
    for (int i = 0; i < w.ns; ++i) {
        if (std::fabs(w.gam[i]) < cutoff) w.gam[i] = 0;
        else w.isa[w.nsa++] = i;
    }
}

// SCALE_IT, src/fasolt/Cpstrs.f90:187-230.  Note amax starts at am(1), the
// first system, not the first active one -- restated as written.
template <class R> void scale_it(Problem<R> &P, CpWork<R> &w, R s[6], R gamcap)
{
    R amax = w.am[0];
    R gammax = std::fabs(w.gam[w.isa[0]]);
    for (int i = 1; i < w.nsa; ++i) {
        int ii = w.isa[i];
        if (std::fabs(w.gam[ii]) > gammax) {
            gammax = std::fabs(w.gam[ii]);
            amax = w.am[ii];
        }
    }
    if (gammax > gamcap) {
        R scale = gamcap / gammax;
        R smult = spower(R(0.9) * scale, P.afactor * amax);
        if (smult == R(0)) smult = R(0.004) / amax;
        for (int i = 0; i < 6; ++i) s[i] = smult * s[i];
        for (int i = 0; i < w.ns; ++i) {
            w.gam[i] = scale * w.gam[i];
            w.tau[i] = smult * w.tau[i];
        }
    }
}

// SLPFTA, src/fasolt/crys-cons.f90:24-128.  Returns 0, 910 or 987.
template <class R> int slpfta(Problem<R> &P, CpWork<R> &w, R dt, int &ninner)
{
    const Material<R> &m = *w.m;
    R am[MAXSS];
    R amx = m.ampar[0][0];
    for (int i = 1; i < w.ns; ++i) amx = std::max(amx, m.ampar[i][0]);
    const R conv = P.toler * amx;
    const int n = w.nsa;
    R errtau[MAXSS];
    R tauerr = 0;
    int iter = 0;
    bool l_iter = true;
    ninner = 0;
    while (l_iter) {
        ++iter;
        plastc(w, dt, am);
        for (int i = 0; i < n; ++i) {
            R gamn = w.gam[w.isa[i]];
            for (int j = 0; j < n; ++j) w.ah[j * MAXSS + i] = gamn * w.ah[j * MAXSS + i];
            w.ah[i * MAXSS + i] = w.ah[i * MAXSS + i] + am[w.isa[i]];
        }
        if (factor(n, w.ah, MAXSS)) return 910;
        for (int i = 0; i < n; ++i) {
            int ii = w.isa[i];
            R taufg = w.s1[ii] * spower(w.gam[ii] / dt, am[ii]);
            if (w.tau[ii] * taufg > R(0)) errtau[i] = std::log(w.tau[ii] / taufg);
            else errtau[i] = 0;
        }
        tauerr = 0;
        for (int i = 0; i < n; ++i) tauerr = tauerr + errtau[i] * errtau[i];
        tauerr = std::sqrt(tauerr);
        solver(n, w.ah, MAXSS, errtau);
        R errmax = 0;
        for (int i = 0; i < n; ++i)
            if (std::fabs(errtau[i]) > errmax) errmax = std::fabs(errtau[i]);
        R scale = errmax > R(5.0) ? R(5.0) / errmax : R(1.0);
        for (int i = 0; i < n; ++i) {
            int ii = w.isa[i];
            w.gam[ii] = w.gam[ii] * std::exp(scale * errtau[i]);
        }
        l_iter = (iter < P.maxit) && (tauerr > conv);
    }
    ninner = iter;
    if (tauerr > R(0.5)) return 987;
    plastc(w, dt, am);
    for (int i = 0; i < n; ++i) {
        int ii = w.isa[i];
        for (int j = 0; j < n; ++j) {
            int jj = w.isa[j];
            w.ah[j * MAXSS + i] = w.tau[jj] * w.ah[j * MAXSS + i];
        }
        if (std::fabs(w.gam[ii]) > R(1.e-12))
            w.ah[i * MAXSS + i] = w.ah[i * MAXSS + i] + am[ii] * w.tau[ii] / w.gam[ii];
        else
            w.ah[i * MAXSS + i] = w.ah[i * MAXSS + i] + am[ii] / R(1.e-12);
    }
    return 0;
}

// ECHROT, src/fasolt/crys_math.f90:137-167
template <class R>
void echrot(const CpWork<R> &w, const R a[3][3], const R aug[3], const R r[3], R &dp1,
            R &dph, R &dp2)
{
    R rtn[3], rx[3];
    for (int k = 0; k < 3; ++k) {
        R s = 0;
        for (int i = 0; i < w.ns; ++i) s = s + w.rot[i][k] * w.gam[i];
        rtn[k] = s - r[k];
    }
    for (int k = 0; k < 3; ++k) {
        R s = 0;
        for (int c = 0; c < 3; ++c) s = s + a[k][c] * rtn[c];
        rx[k] = s;
    }
    if (std::fabs(aug[2]) < R(1.e-5)) dp1 = rtn[2];
    else dp1 = (aug[0] * rx[0] + aug[1] * rx[1]) / aug[2];
    dph = aug[1] * rx[0] - aug[0] * rx[1];
    dp2 = rx[2] - dp1 * a[2][2];
}

// CPSTRS, src/fasolt/Cpstrs.f90:34-172.  el_comp = S, del = strain
// increment, rl = spin, s in/out, t = start stress (current axes),
// epl out, chi out (chi[i][j]).  Returns 0 or a FAFERR code.
template <class R>
int cpstrs(Problem<R> &P, int jgp, const Material<R> &m, const R S[6][6], const R del[6],
           const R rl[3], R s[6], const R t[6], R epl[6], R chi[6][6], int inc, int nit)
{
    CpWork<R> w;
    w.m = &m;
    w.ns = m.ns;
    const R dt = P.tiem[inc - 1];
    R *sv = &P.sv[(size_t)jgp * SVLD];
    R *dsv = &P.dsv[(size_t)jgp * SVLD];
    R ph1 = sv[0] + dsv[0], phi = sv[1] + dsv[1], ph2 = sv[2] + dsv[2];
    for (int i = 0; i < w.ns; ++i) {
        w.s0[i] = sv[i + 3];
        w.s1[i] = w.s0[i] + dsv[i + 3];
    }
    R gamcap = R(6.0) * fj2vom(false, del);
    R a[3][3], aug[3];
    ctmatrx(ph1, phi, ph2, a, aug);
    btmatrx(a, w);

    double ops = fas_ops_cp_fixed(w.ns);
    R djac[6][6], erreps[6];
    R erepmd = 0;
    int iter = 0;
    bool l_iter = true;
    while (l_iter) {
        ++iter;
        for (int i = 0; i < w.ns; ++i) {
            R acc = 0;
            for (int k = 0; k < 6; ++k) acc = acc + w.b[i][k] * s[k];
            w.tau[i] = acc;
        }
        slpini(P, w, jgp, dt, inc, nit, iter);
        scale_it(P, w, s, gamcap);
        int ninner = 0;
        int rc = slpfta(P, w, dt, ninner);
        ops += ninner * fas_ops_inner(w.ns, w.nsa) + fas_ops_outer(w.ns, w.nsa);
        if (rc) {
            P.ops_gp[jgp] = ops;
            P.cp_iters[jgp] = iter;
            return rc;
        }
        scale_it(P, w, s, gamcap);
        for (int k = 0; k < 6; ++k) {
            R acc = 0;
            for (int i = 0; i < w.ns; ++i) acc = acc + w.b[i][k] * w.gam[i];
            epl[k] = acc;
        }
        for (int k = 0; k < 6; ++k) {
            R acc = 0;
            for (int c = 0; c < 6; ++c) acc = acc + S[k][c] * (s[c] - t[c]);
            erreps[k] = del[k] - epl[k] - acc;
        }
        const int n = w.nsa;
        if (factor(n, w.ah, MAXSS)) {
            P.ops_gp[jgp] = ops;
            P.cp_iters[jgp] = iter;
            return 910;
        }
        // djac(i,j) = b_a(i,:) X^-1 b_a(j,:)^T; one solve per column j gives
        // exactly the values of the reference's 36 identical solves.
        for (int j = 0; j < 6; ++j) {
            for (int k = 0; k < n; ++k) w.wks[k] = w.b[w.isa[k]][j];
            solver(n, w.ah, MAXSS, w.wks);
            for (int i = 0; i < 6; ++i) {
                R sum = 0;
                for (int k = 0; k < n; ++k) sum = sum + w.b[w.isa[k]][i] * w.wks[k];
                djac[i][j] = sum;
            }
        }
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) djac[i][j] = djac[i][j] + S[i][j];
        if (factor(6, &djac[0][0], 6)) {
            P.ops_gp[jgp] = ops;
            P.cp_iters[jgp] = iter;
            return 910;
        }
        solver(6, &djac[0][0], 6, erreps);
        erepmd = fj2vom(true, erreps) / fj2vom(true, s);
        R scale = R(1.0) / (R(1.0) + P.alpha * erepmd);
        for (int i = 0; i < 6; ++i) erreps[i] = scale * erreps[i];
        for (int i = 0; i < 6; ++i) s[i] = s[i] + erreps[i];
        l_iter = (iter < P.maxit) && (erepmd > P.toler);
    }
    R *sr = &P.srate[(size_t)jgp * MAXSS];
    for (int i = 0; i < w.ns; ++i) sr[i] = std::fabs(w.gam[i] / dt);
    P.erepmd_gp[jgp] = erepmd;
    P.cp_iters[jgp] = iter;
    R dp1, dph, dp2;
    echrot(w, a, aug, rl, dp1, dph, dp2);
    dsv[0] = dp1;
    dsv[1] = dph;
    dsv[2] = dp2;
    for (int i = 0; i < w.ns; ++i) dsv[i + 3] = w.s1[i] - w.s0[i];
    P.ops_gp[jgp] = ops;
    if (P.mode & FAS_MODE_TANGENT_CONSISTENT) {
        // the consistent tangent: (B X^-1 B^T + S)^-1 of the local system at
        // the converged stress -- its slip stresses, the slips and hardening
        // that satisfy the flow rule there (SLPFTA from the last slips, same
        // active set) -- instead of the Jacobian of the last iterate
        for (int i = 0; i < w.ns; ++i) {
            R acc = 0;
            for (int k = 0; k < 6; ++k) acc = acc + w.b[i][k] * s[k];
            w.tau[i] = acc;
        }
        int ninner = 0;
        int rc = slpfta(P, w, dt, ninner);
        if (rc) return rc;
        const int n = w.nsa;
        if (factor(n, w.ah, MAXSS)) return 910;
        for (int j = 0; j < 6; ++j) {
            for (int k = 0; k < n; ++k) w.wks[k] = w.b[w.isa[k]][j];
            solver(n, w.ah, MAXSS, w.wks);
            for (int i = 0; i < 6; ++i) {
                R sum = 0;
                for (int k = 0; k < n; ++k) sum = sum + w.b[w.isa[k]][i] * w.wks[k];
                djac[i][j] = sum + S[i][j];
            }
        }
        if (factor(6, &djac[0][0], 6)) return 910;
    }
    for (int i = 0; i < 6; ++i) {
        R e[6] = {0, 0, 0, 0, 0, 0};
        e[i] = R(1.0);
        solver(6, &djac[0][0], 6, e);
        for (int j = 0; j < 6; ++j) chi[j][i] = e[j];
    }
    return 0;
}

// DSTRSS, src/fasolt/Sig_eps.f90:84-151 (the `es` argument is unused there).
// ds in/out, t out (the new stress), chi out; deff out.
template <class R>
int dstrss(Problem<R> &P, int iel, int jgp, R &deff, const R de[6], const R st[6], R ds[6],
           R t[6], const R r[3], R chi[6][6], int inc, int nit)
{
    const int mc = std::abs(iel);
    const Material<R> &m = P.mat[mc - 1];
    const R *sv = &P.sv[(size_t)jgp * SVLD];
    const R *dsv = &P.dsv[(size_t)jgp * SVLD];
    R S[6][6];
    elastc(m.e, sv[0] + dsv[0], sv[1] + dsv[1], sv[2] + dsv[2], S);
    tens_rot(r, st, t);
    R s[6];
    for (int i = 0; i < 6; ++i) s[i] = t[i] + ds[i];
    R sinit = fj2vom(true, s);
    R einit = fj2vom(false, de);
    P.erepmd_gp[jgp] = 0;
    if (iel > 0 && sinit > R(0) && einit > R(0)) {
        R ep[6];
        int rc = cpstrs(P, jgp, m, S, de, r, s, t, ep, chi, inc, nit);
        if (rc) return rc;
        for (int i = 0; i < 6; ++i) t[i] = s[i];
        deff = fj2vom(false, ep);
        for (int i = 0; i < 6; ++i)
            for (int j = i; j < 6; ++j) {
                R d = (chi[i][j] + chi[j][i]) / R(2.0);
                chi[i][j] = d;
                chi[j][i] = d;
            }
    } else {
        deff = 0;
        P.cp_iters[jgp] = 0;
        P.ops_gp[jgp] = fas_ops_elastic();
        R Sf[6][6];
        std::memcpy(Sf, S, sizeof(Sf));
        factor(6, &Sf[0][0], 6);
        for (int i = 0; i < 6; ++i) {
            R e[6] = {0, 0, 0, 0, 0, 0};
            e[i] = R(1.0);
            solver(6, &Sf[0][0], 6, e);
            for (int j = 0; j < 6; ++j) chi[j][i] = e[j];
        }
        for (int i = 0; i < 6; ++i) {
            R acc = 0;
            for (int c = 0; c < 6; ++c) acc = acc + chi[i][c] * de[c];
            t[i] = acc;
        }
    }
    for (int i = 0; i < 6; ++i) ds[i] = t[i] - st[i];
    return 0;
}

// DSTRNS, src/fasolt/Sig_eps.f90:25-61.  sfd[i][a] = sfd(a+1,i+1),
// dxl[i][b] = dxl(b+1,i+1).  Returns 0, 905 or 906.
template <class R>
int dstrns(const Problem<R> &P, int npl, const R (*sfd)[3], const R (*dxl)[3], R del[6],
           R rl[3], R &deff)
{
    R g[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            R s = 0;
            for (int i = 0; i < npl; ++i) s = s + sfd[i][a] * dxl[i][b];
            g[a][b] = s;
        }
    R sum = 0;
    for (int i = 0; i < 3; ++i) {
        int j = (i + 1) % 3, k = (j + 1) % 3;
        del[i] = g[i][i];
        del[i + 3] = g[k][j] + g[j][k];
        rl[i] = (g[k][j] - g[j][k]) / R(2.0);
        sum = sum + rl[i] * rl[i];
    }
    deff = fj2vom(false, del);
    if (sum > P.smalr) return 905;
    if (deff > P.smale) return 906;
    return 0;
}

// Element stiffness block gaussm (Elvals.f90:132-220) for node pair (i,j):
// gm[r][c] = gaussm(r+1,c+1) before the weight is applied.  d = chi (only
// its upper triangle is read, exactly as the reference does).
template <class R>
void gaussm_block(const R ai[3], const R bj[3], const R d[6][6], const R s[6], R gm[3][3])
{
#define D(p, q) d[(p)-1][(q)-1]
#define S_(p) s[(p)-1]
    const R i1 = ai[0], i2 = ai[1], i3 = ai[2], j1 = bj[0], j2 = bj[1], j3 = bj[2];
    gm[0][0] = (i1 * j1 * (D(1, 1) - S_(1)) + i2 * j2 * (D(6, 6) - (S_(1) - S_(2)) / R(2.0)) +
                i3 * j3 * (D(5, 5) - (S_(1) - S_(3)) / R(2.0)) + i2 * j3 * (D(5, 6) + S_(4) / R(2.0)) +
                i3 * j1 * (D(1, 5)) + i1 * j2 * (D(1, 6)) + j2 * i3 * (D(5, 6) + S_(4) / R(2.0)) +
                j3 * i1 * (D(1, 5)) + j1 * i2 * (D(1, 6)));
    gm[1][0] = (i1 * j1 * (D(1, 6) - S_(6)) + i2 * j2 * (D(2, 6) - S_(6)) +
                i3 * j3 * (D(4, 5) - S_(6) / R(2.0)) + i2 * j3 * (D(2, 5) - S_(5) / R(4.0)) +
                i3 * j1 * (D(1, 4) - S_(4) / R(4.0)) + i1 * j2 * (D(6, 6) - (S_(1) + S_(2)) / R(4.0)) +
                j2 * i3 * (D(4, 6) - S_(5) / R(4.0)) + j3 * i1 * (D(5, 6) - S_(4) / R(4.0)) +
                j1 * i2 * (D(1, 2) - (S_(1) + S_(2)) / R(4.0)));
    gm[2][0] = (i1 * j1 * (D(1, 5) - S_(5)) + i2 * j2 * (D(4, 6) - S_(5) / R(2.0)) +
                i3 * j3 * (D(3, 5) - S_(5)) + i2 * j3 * (D(4, 5) - S_(6) / R(4.0)) +
                i3 * j1 * (D(1, 3) - (S_(1) + S_(3)) / R(4.0)) + i1 * j2 * (D(5, 6) - S_(4) / R(4.0)) +
                j2 * i3 * (D(3, 6) - S_(6) / R(4.0)) + j3 * i1 * (D(5, 5) - (S_(1) + S_(3)) / R(4.0)) +
                j1 * i2 * (D(1, 4) - S_(4) / R(4.0)));
    gm[0][1] = (j1 * i1 * (D(1, 6) - S_(6)) + j2 * i2 * (D(2, 6) - S_(6)) +
                j3 * i3 * (D(4, 5) - S_(6) / R(2.0)) + j2 * i3 * (D(2, 5) - S_(5) / R(4.0)) +
                j3 * i1 * (D(1, 4) - S_(4) / R(4.0)) + j1 * i2 * (D(6, 6) - (S_(1) + S_(2)) / R(4.0)) +
                i2 * j3 * (D(4, 6) - S_(5) / R(4.0)) + i3 * j1 * (D(5, 6) - S_(4) / R(4.0)) +
                i1 * j2 * (D(1, 2) - (S_(1) + S_(2)) / R(4.0)));
    gm[1][1] = (i1 * j1 * (D(6, 6) - (S_(2) - S_(1)) / R(2.0)) + i2 * j2 * (D(2, 2) - S_(2)) +
                i3 * j3 * (D(4, 4) - (S_(2) - S_(3)) / R(2.0)) + i2 * j3 * (D(2, 4)) +
                i3 * j1 * (D(4, 6) + S_(5) / R(2.0)) + i1 * j2 * (D(2, 6)) + j2 * i3 * (D(2, 4)) +
                j3 * i1 * (D(4, 6) + S_(5) / R(2.0)) + j1 * i2 * (D(2, 6)));
    gm[2][1] = (i1 * j1 * (D(5, 6) - S_(4) / R(2.0)) + i2 * j2 * (D(2, 4) - S_(4)) +
                i3 * j3 * (D(3, 4) - S_(4)) + i2 * j3 * (D(4, 4) - (S_(2) + S_(3)) / R(4.0)) +
                i3 * j1 * (D(3, 6) - S_(6) / R(4.0)) + i1 * j2 * (D(2, 5) - S_(5) / R(4.0)) +
                j2 * i3 * (D(2, 3) - (S_(2) + S_(3)) / R(4.0)) + j3 * i1 * (D(4, 5) - S_(6) / R(4.0)) +
                j1 * i2 * (D(4, 6) - S_(5) / R(4.0)));
    gm[0][2] = (j1 * i1 * (D(1, 5) - S_(5)) + j2 * i2 * (D(4, 6) - S_(5) / R(2.0)) +
                j3 * i3 * (D(3, 5) - S_(5)) + j2 * i3 * (D(4, 5) - S_(6) / R(4.0)) +
                j3 * i1 * (D(1, 3) - (S_(1) + S_(3)) / R(4.0)) + j1 * i2 * (D(5, 6) - S_(4) / R(4.0)) +
                i2 * j3 * (D(3, 6) - S_(6) / R(4.0)) + i3 * j1 * (D(5, 5) - (S_(1) + S_(3)) / R(4.0)) +
                i1 * j2 * (D(1, 4) - S_(4) / R(4.0)));
    gm[1][2] = (j1 * i1 * (D(5, 6) - S_(4) / R(2.0)) + j2 * i2 * (D(2, 4) - S_(4)) +
                j3 * i3 * (D(3, 4) - S_(4)) + j2 * i3 * (D(4, 4) - (S_(2) + S_(3)) / R(4.0)) +
                j3 * i1 * (D(3, 6) - S_(6) / R(4.0)) + j1 * i2 * (D(2, 5) - S_(5) / R(4.0)) +
                i2 * j3 * (D(2, 3) - (S_(2) + S_(3)) / R(4.0)) + i3 * j1 * (D(4, 5) - S_(6) / R(4.0)) +
                i1 * j2 * (D(4, 6) - S_(5) / R(4.0)));
    gm[2][2] = (i1 * j1 * (D(5, 5) - (S_(3) - S_(1)) / R(2.0)) +
                i2 * j2 * (D(4, 4) - (S_(3) - S_(2)) / R(2.0)) + i3 * j3 * (D(3, 3) - S_(3)) +
                i2 * j3 * (D(3, 4)) + i3 * j1 * (D(3, 5)) + i1 * j2 * (D(4, 5) + S_(6) / R(2.0)) +
                j2 * i3 * (D(3, 4)) + j3 * i1 * (D(3, 5)) + j1 * i2 * (D(4, 5) + S_(6) / R(2.0)));
#undef D
#undef S_
}

// ================================================================ assembly
// SETPTA, src/fasolt/Stif_sol.f90:98-149 (first-touch column order).  The
// reference appends, element by element, each new column of every row of the
// element in local DOF order; for one row that is the order of its elements
// (ascending) and their local DOFs, which is how it is built here -- one row
// at a time, with a stamp array instead of the reference's linear search.
template <class R> void setpta(Problem<R> &P)
{
    const int ndof = 3 * P.nnod;
    std::vector<int> ptr(P.nnod + 1, 0);
    for (int e = 0; e < P.nlmnt; ++e)
        for (int i = 0; i < P.nd[e]; ++i) ptr[P.ln[e * P.ldn + i] + 1]++;
    for (int n = 0; n < P.nnod; ++n) ptr[n + 1] += ptr[n];
    std::vector<int> adj(ptr[P.nnod]), fill(ptr.begin(), ptr.end() - 1);
    for (int e = 0; e < P.nlmnt; ++e)
        for (int i = 0; i < P.nd[e]; ++i) adj[fill[P.ln[e * P.ldn + i]]++] = e;
    std::vector<int> stamp(ndof, -1), cnt(ndof, 0);
    int mx = 0;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            P.ld = mx + 1;
            P.is.assign((size_t)ndof * P.ld, 0);
            P.ss.assign((size_t)ndof * P.ld, R(0));
            std::fill(stamp.begin(), stamp.end(), -1);
        }
        for (int row = 0; row < ndof; ++row) {
            const int n = row / 3;
            int c = 0;
            for (int k = ptr[n]; k < ptr[n + 1]; ++k) {
                const int e = adj[k];
                for (int i = 0; i < P.nd[e]; ++i)
                    for (int q = 0; q < 3; ++q) {
                        const int col = 3 * P.ln[e * P.ldn + i] + q;
                        if (col == row || stamp[col] == row) continue;
                        stamp[col] = row;
                        ++c;
                        if (pass == 1) P.is[(size_t)row * P.ld + c] = col;
                    }
            }
            if (pass == 0) mx = std::max(mx, c);
            else P.is[(size_t)row * P.ld] = c;
        }
    }
}

// Column slot of `col` in row `row` (the reference's linear search,
// Elvals.f90:250-257 / Bconds.f90:78-85).
template <class R> inline int slot_of(const Problem<R> &P, int row, int col)
{
    if (row == col) return 0;
    const int *r = &P.is[(size_t)row * P.ld];
    int k = 1;
    while (r[k] != col) ++k;
    return k;
}

// Greedy node colouring for the multicolour SOR.  Nodes are visited in
// ascending (z, y, x, id) order of their initial coordinates and take the
// smallest colour not used by any node that shares an element with them;
// on a structured brick mesh this is the 8-colour (i,j,k)-parity colouring.
// The device library computes the same colouring the same way.
template <class R> void colour_nodes(Problem<R> &P)
{
    const int nn = P.nnod;
    std::vector<int> order(nn);
    for (int i = 0; i < nn; ++i) order[i] = i;
    const std::vector<R> &x = P.x;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        for (int c = 2; c >= 0; --c) {
            double xa = (double)x[3 * a + c], xb = (double)x[3 * b + c];
            if (xa != xb) return xa < xb;
        }
        return a < b;
    });
    // node -> elements
    std::vector<int> cnt(nn + 1, 0);
    for (int e = 0; e < P.nlmnt; ++e)
        for (int i = 0; i < P.nd[e]; ++i) cnt[P.ln[e * P.ldn + i] + 1]++;
    for (int i = 0; i < nn; ++i) cnt[i + 1] += cnt[i];
    std::vector<int> adj(cnt[nn]);
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int e = 0; e < P.nlmnt; ++e)
        for (int i = 0; i < P.nd[e]; ++i) adj[fill[P.ln[e * P.ldn + i]]++] = e;
    P.colour.assign(nn, -1);
    P.ncol = 0;
    std::vector<int> used(64, -1);
    for (int n : order) {
        for (int k = cnt[n]; k < cnt[n + 1]; ++k) {
            int e = adj[k];
            for (int i = 0; i < P.nd[e]; ++i) {
                int m = P.ln[e * P.ldn + i];
                int c = P.colour[m];
                if (c >= 0) {
                    if (c >= (int)used.size()) used.resize(c + 1, -1);
                    used[c] = n;
                }
            }
        }
        int c = 0;
        while (c < (int)used.size() && used[c] == n) ++c;
        P.colour[n] = c;
        P.ncol = std::max(P.ncol, c + 1);
    }
    P.colour_order.resize(nn);
    for (int i = 0; i < nn; ++i) P.colour_order[i] = i;
    std::stable_sort(P.colour_order.begin(), P.colour_order.end(),
                     [&](int a, int b) { return P.colour[a] < P.colour[b]; });
}

// ELVALS, src/fasolt/Elvals.f90:11-275 (fc and ss zeroed first, as NRITER
// does at Stif_sol.f90:38-39).  Elements are evaluated in parallel when
// threads > 1 but scattered strictly in element order, so the sums are
// identical to the serial reference order.
template <class R> int elvals(Problem<R> &P, int inc, int nit)
{
    std::fill(P.fc.begin(), P.fc.end(), R(0));
    std::fill(P.ss.begin(), P.ss.end(), R(0));
    P.sumcpiter = 0;
    const int NE = P.nlmnt;
    const int CH = 2048;
    std::vector<R> esm_buf((size_t)CH * 3600), fl_buf((size_t)CH * 60);
    std::vector<int> rc_buf(CH);
    for (int e0 = 0; e0 < NE; e0 += CH) {
        const int e1 = std::min(NE, e0 + CH);
#pragma omp parallel for schedule(dynamic, 16) num_threads(P.nthreads) if (P.nthreads > 1)
        for (int e = e0; e < e1; ++e) {
            R *esm = &esm_buf[(size_t)(e - e0) * 3600];
            R *fl = &fl_buf[(size_t)(e - e0) * 60];
            rc_buf[e - e0] = 0;
            const int iel = P.le[e], itp = P.lt[e], nn = P.nd[e];
            const int n3 = 3 * nn;
            for (int i = 0; i < n3 * n3; ++i) esm[i] = 0;
            for (int i = 0; i < n3; ++i) fl[i] = 0;
            R xl[20][3], dxl[20][3];
            for (int i = 0; i < nn; ++i) {
                int ks = 3 * P.ln[e * P.ldn + i];
                for (int j = 0; j < 3; ++j) {
                    xl[i][j] = P.x[ks + j];
                    dxl[i][j] = P.dx[ks + j];
                }
            }
            if (itp < 9) {   // tie element (Elvals.f90:62-77), esm(r,c) -> esm[r*n3+c]
                auto put = [&](int r, int c, R v) { esm[(r - 1) * n3 + (c - 1)] = v; };
                if (itp <= 3) {
                    put(itp, itp, P.efix);
                    put(itp, itp + 3, -P.efix);
                } else {
                    int ii = 1 + (itp - 3) % 3;
                    put(ii, ii, P.efix);
                    put(ii, ii + 3, -P.efix);
                    ii = 1 + ii % 3;
                    put(ii, ii, P.efix);
                    put(ii, ii + 3, -P.efix);
                }
                continue;
            }
            // lt == 12 (one GP) or 22 (eight GPs); checked at create.  The GP
            // loop of Elvals.f90:82-236: forces and stiffness accumulate GP by GP.
            const int ng = P.np[e];
            for (int ig = 0; ig < ng; ++ig) {
                R sfd[20][3];
                R weight = itp == 12   ? shape12(reinterpret_cast<const R(*)[3]>(xl), reinterpret_cast<R(*)[3]>(sfd))
                           : itp == 21 ? shape21(ig, xl, sfd)
                           : itp == 23 ? shape23(ig, xl, sfd)
                                       : shape22(ig, xl, sfd);
                if (weight < R(1.e-7)) { rc_buf[e - e0] = 920; break; }
                const int j = P.lg[(size_t)e * 8 + ig];
                R del[6], r[3], defl;
                int rc = dstrns(P, nn, sfd, dxl, del, r, defl);
                if (rc) { rc_buf[e - e0] = rc; break; }
                R stl[6], dsl[6], s[6], d[6][6];
                for (int k = 0; k < 6; ++k) {
                    stl[k] = P.st[(size_t)j * 6 + k];
                    dsl[k] = P.ds[(size_t)j * 6 + k];
                }
                rc = dstrss(P, iel, j, defl, del, stl, dsl, s, r, d, inc, nit);
                if (rc) { rc_buf[e - e0] = rc; break; }
                P.dep[j] = defl;
                for (int k = 0; k < 6; ++k) {
                    P.de[(size_t)j * 6 + k] = del[k];
                    P.ds[(size_t)j * 6 + k] = dsl[k];
                }
                for (int k = 0; k < 3; ++k) P.dr[(size_t)j * 3 + k] = r[k];
                R *chi = &P.chi_gp[(size_t)j * 36];
                for (int a2 = 0; a2 < 6; ++a2)
                    for (int b2 = 0; b2 < 6; ++b2) chi[a2 + 6 * b2] = d[a2][b2];
                for (int i = 0; i < nn; ++i) {
                    fl[3 * i + 0] = fl[3 * i + 0] + weight * (s[0] * sfd[i][0] + s[5] * sfd[i][1] + s[4] * sfd[i][2]);
                    fl[3 * i + 1] = fl[3 * i + 1] + weight * (s[1] * sfd[i][1] + s[3] * sfd[i][2] + s[5] * sfd[i][0]);
                    fl[3 * i + 2] = fl[3 * i + 2] + weight * (s[2] * sfd[i][2] + s[4] * sfd[i][0] + s[3] * sfd[i][1]);
                }
                for (int i = 0; i < nn; ++i)
                    for (int jn = 0; jn < nn; ++jn) {
                        R gm[3][3];
                        gaussm_block(sfd[i], sfd[jn], d, s, gm);
                        for (int a2 = 0; a2 < 3; ++a2)
                            for (int b2 = 0; b2 < 3; ++b2)
                                esm[(3 * i + a2) * n3 + 3 * jn + b2] =
                                    esm[(3 * i + a2) * n3 + 3 * jn + b2] + weight * gm[a2][b2];
                    }
            }
        }
        // serial scatter in element order; the first error (in element order)
        // stops the pass like FAFERR's STOP
        for (int e = e0; e < e1; ++e) {
            if (rc_buf[e - e0]) return rc_buf[e - e0];
            const R *esm = &esm_buf[(size_t)(e - e0) * 3600];
            const R *fl = &fl_buf[(size_t)(e - e0) * 60];
            const int nn = P.nd[e], n3 = 3 * nn;
            int in2[60];
            for (int i = 0; i < nn; ++i)
                for (int c = 0; c < 3; ++c) in2[3 * i + c] = 3 * P.ln[e * P.ldn + i] + c;
            for (int i = 0; i < n3; ++i) {
                int ii = in2[i];
                for (int jj = 0; jj < n3; ++jj) {
                    int k = slot_of(P, ii, in2[jj]);
                    R &dst = P.ss[(size_t)ii * P.ld + k];
                    dst = dst + esm[i * n3 + jj];
                }
            }
            for (int i = 0; i < nn; ++i) {
                int k = 3 * P.ln[e * P.ldn + i];
                for (int c = 0; c < 3; ++c) P.fc[k + c] = P.fc[k + c] + fl[3 * i + c];
            }
            if (P.lt[e] >= 9) {
                for (int ig = 0; ig < P.np[e]; ++ig)
                    P.sumcpiter = P.sumcpiter + P.erepmd_gp[P.lg[(size_t)e * 8 + ig]];
                P.last_mat = std::abs(P.le[e]);
            }
        }
    }
    return 0;
}

// SUVALS, src/fasolt/Bconds.f90:19-113
template <class R> int suvals(Problem<R> &P, int inc)
{
    static const int point[3][3] = {{0, 1, 3}, {1, 2, 4}, {3, 4, 5}};
    const int ndof = 3 * P.nnod;
    for (int i = 0; i < ndof; ++i) P.ddx[i] = P.fc[i];
    for (int n = 0; n < P.nnod; ++n) {
        const int ibc = P.ib[n];
        if (ibc < 100) continue;
        const int idof = 3 * n;
        const int ikin = (ibc / 100) % 100;
        if (ikin > 0) {
            if (ikin > P.nxs) return FAS_E_ARG;
            const R *xs = &P.xspec[((size_t)(inc - 1) * P.nxs + (ikin - 1)) * 15];
            R xspec[3];
            if (ikin < 50) {
                xspec[0] = xs[6];
                xspec[1] = xs[10];
                xspec[2] = xs[14];
            } else {
                R dsp[3][3];
                int l = 6;
                for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k) dsp[j][k] = xs[l++];
                for (int j = 0; j < 3; ++j) {
                    R acc = 0;
                    for (int k = 0; k < 3; ++k) acc = acc + dsp[j][k] * (P.x[idof + k] + P.dx[idof + k]);
                    xspec[j] = acc;
                }
            }
            for (int i = 0; i < 3; ++i) {
                const int row = idof + i;
                for (int j = 0; j < 3; ++j) {
                    int k = slot_of(P, row, idof + j);
                    R &dst = P.ss[(size_t)row * P.ld + k];
                    dst = dst + (P.efix * xs[point[i][j]]);
                }
                R sum = 0;
                for (int j = 0; j < 3; ++j)
                    sum = sum + P.efix * xs[point[i][j]] * (P.dx[idof + j] - xspec[j]);
                P.ddx[row] = P.ddx[row] + sum;
            }
        }
        const int ispf = (ibc / 10000) % 100;
        if (ispf > 0) {
            if (ispf > P.nfs) return FAS_E_ARG;
            const R *fs = &P.fspec[((size_t)(inc - 1) * P.nfs + (ispf - 1)) * 3];
            for (int i = 0; i < 3; ++i) P.ddx[idof + i] = P.ddx[idof + i] + fs[i];
        }
    }
    return 0;
}

// One SOR row update (Stif_sol.f90:189-197).
template <class R> inline R sor_row(Problem<R> &P, const std::vector<R> &y, int i)
{
    const int *ir = &P.is[(size_t)i * P.ld];
    const R *sr = &P.ss[(size_t)i * P.ld];
    R sum = 0;
    const int cnt = ir[0];
    for (int j = 1; j <= cnt; ++j) sum = sum + sr[j] * P.ddx[ir[j]];
    sum = (y[i] - sum) / sr[0];
    R old = P.ddx[i];
    R nw = old + R(1.2) * (sum - old);
    P.ddx[i] = nw;
    return nw;
}

// FACSLS, src/fasolt/Stif_sol.f90:161-215.  Natural DOF order when
// FAS_MODE_SOR_NATURAL is set, otherwise the multicolour node order of the
// device path (colours ascending, nodes ascending, then x, y, z).
template <class R> int facsls(Problem<R> &P, int maxitl, int *sweeps, double *error)
{
    const int m = 3 * P.nnod;
    const R tolerl = P.toler * P.toler;
    std::vector<R> y(P.ddx.begin(), P.ddx.begin() + m), old(m);
    std::fill(P.ddx.begin(), P.ddx.begin() + m, R(0));
    for (int i = 0; i < m; ++i)
        if (std::fabs(P.ss[(size_t)i * P.ld]) == R(0)) return 903;
    const bool natural = (P.mode & FAS_MODE_SOR_NATURAL) != 0;
    bool conv = false;
    int iter = 0;
    R err = 0;
    while (!conv && iter < maxitl) {
        ++iter;
        std::copy(P.ddx.begin(), P.ddx.begin() + m, old.begin());
        if (natural) {
            for (int i = 0; i < m; ++i) sor_row(P, y, i);
        } else if (P.nthreads > 1) {
            int start = 0;
            for (int c = 0; c < P.ncol; ++c) {
                int end = start;
                while (end < P.nnod && P.colour[P.colour_order[end]] == c) ++end;
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
                for (int q = start; q < end; ++q) {
                    int n = P.colour_order[q];
                    for (int c3 = 0; c3 < 3; ++c3) sor_row(P, y, 3 * n + c3);
                }
                start = end;
            }
        } else {
            for (int q = 0; q < P.nnod; ++q) {
                int n = P.colour_order[q];
                for (int c3 = 0; c3 < 3; ++c3) sor_row(P, y, 3 * n + c3);
            }
        }
        R num = 0, den = 0;
        for (int i = 0; i < m; ++i) {
            R d = P.ddx[i] - old[i];
            num = num + d * d;
        }
        for (int i = 0; i < m; ++i) den = den + P.ddx[i] * P.ddx[i];
        err = num / den;
        conv = err < tolerl;
    }
    if (sweeps) *sweeps = iter;
    if (error) *error = (double)err;
    if (err > R(10.0) * tolerl) return 904;
    return 0;
}

// One pass of NRITER's loop body (src/fasolt/Stif_sol.f90:32-77): ELVALS,
// SUVALS, the residual norm, FACSLS, the damping factor and the correction.
// *more = the reference's loop condition for another pass.
template <class R> int nr_step(Problem<R> &P, int inc, int nit, fas_iter_report *r, bool *more)
{
    const int ndof = 3 * P.nnod;
    int rc = elvals(P, inc, nit);
    if (rc) return rc;
    rc = suvals(P, inc);
    if (rc) return rc;
    R sfc = 0;
    for (int i = 0; i < P.nnod; ++i)
        if (P.ib[i] < 10)
            sfc = sfc + P.ddx[3 * i] * P.ddx[3 * i] + P.ddx[3 * i + 1] * P.ddx[3 * i + 1] +
                  P.ddx[3 * i + 2] * P.ddx[3 * i + 2];
    sfc = std::sqrt(sfc);
    int sweeps = 0;
    double serr = 0;
    rc = facsls(P, 1000, &sweeps, &serr);
    if (rc) return rc;
    R a = 0, b = 0;
    for (int i = 0; i < ndof; ++i) a = a + P.dx[i] * P.dx[i];
    for (int i = 0; i < ndof; ++i) b = b + P.ddx[i] * P.ddx[i];
    R errdx = std::sqrt(a), erddx = std::sqrt(b);
    R sdx = errdx == R(0) ? P.toler : erddx / errdx;
    R alp2 = R(1.0) / (R(1.0) + P.alpha * sdx);
    R cperr = P.sumcpiter / (R)P.ngps;
    if (r) {
        r->nit = nit;
        r->sor_sweeps = sweeps;
        r->sdx = sdx;
        r->sfc = sfc;
        r->cp_err = cperr;
        r->alp2 = alp2;
        r->sor_error = serr;
    }
    for (int i = 0; i < ndof; ++i) {
        R xc = alp2 * P.ddx[i];
        P.x[i] = P.x[i] - xc;
        P.dx[i] = P.dx[i] - xc;
    }
    if (more) *more = (sdx >= P.toler) && (nit < P.maxit);
    return 0;
}

template <class R> void nr_finish(Problem<R> &P, int inc);

// NRITER, src/fasolt/Stif_sol.f90:10-88 (ITEREP lines go to `rep`).
template <class R>
int nriter(Problem<R> &P, int inc, fas_iter_report *rep, int cap, int *n_rep)
{
    int nit = 0;
    bool l_conv = true;
    while (l_conv) {
        ++nit;
        if (n_rep) *n_rep = nit;
        fas_iter_report r;
        int rc = nr_step(P, inc, nit, &r, &l_conv);
        if (rc) return rc;
        if (rep && nit <= cap) rep[nit - 1] = r;
    }
    if (n_rep) *n_rep = nit;
    nr_finish(P, inc);
    return 0;
}

// NRITER's tail after its loop: cumslip over nss(mat_code) of the last
// material touched (Stif_sol.f90:80-84).
template <class R> void nr_finish(Problem<R> &P, int inc)
{
    const int nsc = P.mat[P.last_mat - 1].ns;
    const R tm = P.tiem[inc - 1];
    for (int g = 0; g < P.ngps; ++g)
        for (int k = 0; k < nsc; ++k)
            P.cumslip[(size_t)g * MAXSS + k] =
                P.cumslip[(size_t)g * MAXSS + k] + (P.srate[(size_t)g * MAXSS + k] * tm);
}

// UPDATE_GPTV, src/fasolt/Fasolt3.f90:254-284
template <class R> void update_gptv(Problem<R> &P)
{
    for (int i = 0; i < P.ngps; ++i) {
        P.eps[i] = P.eps[i] + P.dep[i];
        for (int j = 0; j < 3; ++j) P.rt[i * 3 + j] = P.rt[i * 3 + j] + P.dr[i * 3 + j];
        for (int j = 0; j < 6; ++j) {
            P.ep[i * 6 + j] = P.ep[i * 6 + j] + P.de[i * 6 + j];
            P.st[i * 6 + j] = P.st[i * 6 + j] + P.ds[i * 6 + j];
        }
        for (int j = 0; j < P.nsv; ++j)
            P.sv[(size_t)i * SVLD + j] = P.sv[(size_t)i * SVLD + j] + P.dsv[(size_t)i * SVLD + j];
    }
}

// DoReorient, src/fasolt/Fasolt3.f90:79-178.  Uses material 1's tables and
// pi = 3.14159, as the reference does.
template <class R> int reorient(Problem<R> &P, int inc, fas_twin_event *ev, int cap)
{
    int nev = 0;
    const Material<R> &m = P.mat[0];
    for (int j = 0; j < P.ngps; ++j) {
        if (P.twinsys[j] == 0) continue;
        const int i = P.twinsys[j] - 1;
        R *sv = &P.sv[(size_t)j * SVLD];
        R e1 = sv[0], e2 = sv[1], e3 = sv[2];
        R ang = m.ssang[i] * R(3.14159) / R(180.0);
        R c1 = std::cos(e1), c2 = std::cos(e2), c3 = std::cos(e3);
        R ss1 = std::sin(e1), s2 = std::sin(e2), s3 = std::sin(e3);
        R RM[3][3];
        RM[0][0] = c1 * c3 - c2 * ss1 * s3;
        RM[0][1] = -c1 * s3 - c2 * c3 * ss1;
        RM[0][2] = ss1 * s2;
        RM[1][0] = c3 * ss1 + c1 * c2 * s3;
        RM[1][1] = c1 * c2 * c3 - ss1 * s3;
        RM[1][2] = -c1 * s2;
        RM[2][0] = s2 * s3;
        RM[2][1] = c3 * s2;
        RM[2][2] = c2;
        R nv[3], dv[3];
        for (int a = 0; a < 3; ++a) {
            R sn = 0, sd = 0;
            for (int c = 0; c < 3; ++c) {
                sn = sn + RM[a][c] * m.an[i][c];
                sd = sd + RM[a][c] * m.ab[i][c];
            }
            nv[a] = sn;
            dv[a] = sd;
        }
        R u1 = nv[1] * dv[2] - nv[2] * dv[1];
        R u2 = nv[2] * dv[0] - nv[0] * dv[2];
        R u3 = nv[0] * dv[1] - nv[1] * dv[0];
        R c = std::cos(ang), s = std::sin(ang);
        R E[3][3];
        E[0][0] = c + u1 * u1 * (R(1.0) - c);
        E[0][1] = u1 * u2 * (R(1.0) - c) - u3 * s;
        E[0][2] = u1 * u3 * (R(1.0) - c) + u2 * s;
        E[1][0] = u1 * u2 * (R(1.0) - c) + u3 * s;
        E[1][1] = c + u2 * u2 * (R(1.0) - c);
        E[1][2] = u2 * u3 * (R(1.0) - c) - u1 * s;
        E[2][0] = u1 * u3 * (R(1.0) - c) - u2 * s;
        E[2][1] = u2 * u3 * (R(1.0) - c) + u1 * s;
        E[2][2] = c + u3 * u3 * (R(1.0) - c);
        R F[3][3];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                R acc = 0;
                for (int k = 0; k < 3; ++k) acc = acc + E[a][k] * RM[k][b];
                F[a][b] = acc;
            }
        R e1n = std::atan2(F[0][2], -F[1][2]);
        if (std::fabs(F[2][2]) > R(1.0)) F[2][2] = F[2][2] / std::fabs(F[2][2]);
        R e2n = std::acos(F[2][2]);
        R e3n = std::atan2(F[2][0], F[2][1]);
        sv[0] = e1n;
        sv[1] = e2n;
        sv[2] = e3n;
        if (ev && nev < cap) {
            fas_twin_event &t = ev[nev];
            t.inc = inc;
            t.gp = j + 1;
            t.sys = i + 1;
            t.pad = 0;
            t.euler_old[0] = e1; t.euler_old[1] = e2; t.euler_old[2] = e3;
            t.euler_new[0] = e1n; t.euler_new[1] = e2n; t.euler_new[2] = e3n;
        }
        ++nev;
        P.twinsys[j] = 0;
        P.timestwinned[j] = P.timestwinned[j] + 1;
    }
    return nev;
}

// ================================================================ set-up / IO
template <class R>
int create(Problem<R> &P, const fas_mesh_desc *M, const fas_matl_desc *T, const fas_ctrl_desc *C)
{
    if (!M || !T || !C) return FAS_E_ARG;
    if (M->nlmnt < 0 || M->nnod < 0 || M->ngps <= 0) return FAS_E_ARG;
    P.nlmnt = M->nlmnt;
    P.nnod = M->nnod;
    P.ngps = M->ngps;
    P.gp_iel.assign(P.ngps, 1);
    if (P.nlmnt > 0) {
        int ldn = 0;
        for (int e = 0; e < P.nlmnt; ++e) ldn = std::max(ldn, M->nd[e]);
        if (ldn > 20 || ldn > M->ld_ln) return FAS_E_ARG;
        P.ldn = std::max(ldn, 1);
        P.le.assign(M->le, M->le + P.nlmnt);
        P.lt.assign(M->lt, M->lt + P.nlmnt);
        P.nd.assign(M->nd, M->nd + P.nlmnt);
        P.np.assign(M->np, M->np + P.nlmnt);
        P.ln.assign((size_t)P.nlmnt * P.ldn, 0);
        P.lg.assign((size_t)P.nlmnt * 8, 0);
        for (int e = 0; e < P.nlmnt; ++e) {
            if (!(P.lt[e] == 12 || P.lt[e] == 21 || P.lt[e] == 22 || P.lt[e] == 23 || P.lt[e] < 9))
                return FAS_E_ELTYPE;
            if (P.lt[e] == 12 && (P.nd[e] != 8 || P.np[e] != 1)) return FAS_E_ARG;
            if (P.lt[e] == 21 && (P.nd[e] != 10 || P.np[e] != 4 || M->ld_lg < 4)) return FAS_E_ARG;
            if (P.lt[e] == 22 && (P.nd[e] != 20 || P.np[e] != 8 || M->ld_lg < 8)) return FAS_E_ARG;
            if (P.lt[e] == 23 && (P.nd[e] != 15 || P.np[e] != 6 || M->ld_lg < 6)) return FAS_E_ARG;
            for (int i = 0; i < P.nd[e]; ++i) {
                int id = M->ln[(size_t)e * M->ld_ln + i];
                if (id < 1 || id > P.nnod) return FAS_E_ARG;
                P.ln[(size_t)e * P.ldn + i] = id - 1;
            }
            if (P.np[e] < 0 || P.np[e] > 8) return FAS_E_ARG;
            for (int ig = 0; ig < P.np[e]; ++ig) {
                int g = M->lg[(size_t)e * M->ld_lg + ig];
                if (g < 1 || g > P.ngps) return FAS_E_ARG;
                P.lg[(size_t)e * 8 + ig] = g - 1;
                P.gp_iel[g - 1] = P.le[e];
            }
        }
        P.ib.assign(M->ib, M->ib + P.nnod);
    } else {
        for (int g = 0; g < P.ngps; ++g) P.gp_iel[g] = M->le[g];
    }
    // materials
    const int rb = T->real_bytes;
    if (rb != 4 && rb != 8) return FAS_E_ARG;
    P.nmatl = T->nmatl;
    P.nmpar = T->nmpar;
    if (P.nmatl < 1 || T->ld_ss < 1 || T->ld_ss > MAXSS) return FAS_E_ARG;
    P.twinlim = T->twinlim;
    P.twinprob = (R)T->twinprob;
    P.mat.resize(P.nmatl);
    const int L = T->ld_ss;
    for (int mc = 0; mc < P.nmatl; ++mc) {
        Material<R> &m = P.mat[mc];
        m.ns = T->nss[mc];
        if (m.ns < 1 || m.ns > L) return FAS_E_ARG;
        for (int k = 0; k < 9; ++k) m.e[k] = (R)rdv(T->e, rb, (size_t)mc * 9 + k);
        for (int i = 0; i < m.ns; ++i) {
            m.ssang[i] = (R)rdv(T->ssang, rb, (size_t)mc * L + i);
            for (int k = 0; k < 3; ++k) {
                m.ab[i][k] = (R)rdv(T->ab, rb, ((size_t)mc * L + i) * 3 + k);
                m.an[i][k] = (R)rdv(T->an, rb, ((size_t)mc * L + i) * 3 + k);
            }
            for (int k = 0; k < 10; ++k)
                m.ampar[i][k] = k < T->nmpar ? (R)rdv(T->ampar, rb, ((size_t)mc * L + i) * 10 + k) : R(0);
        }
        m.sm.assign((size_t)m.ns * m.ns, R(0));
        for (int i = 0; i < m.ns; ++i)
            for (int j = 0; j < m.ns; ++j)
                m.sm[(size_t)i * m.ns + j] =
                    (R)rdv(T->smatrx, rb, (size_t)mc * L * L + (size_t)j * L + i);
    }
    for (int e = 0; e < P.nlmnt; ++e)
        if (P.lt[e] >= 9 && (P.le[e] == 0 || std::abs(P.le[e]) > P.nmatl)) return FAS_E_ARG;
    // control
    const int cb = C->real_bytes;
    if (cb != 4 && cb != 8) return FAS_E_ARG;
    P.toler = (R)C->toler;
    P.alpha = (R)C->alpha;
    P.afactor = (R)C->afactor;
    P.efix = (R)C->efix;
    P.smale = (R)C->smale;
    P.smalr = (R)C->smalr;
    P.maxit = C->maxit;
    P.ninc1 = C->ninc1;
    P.nxs = C->nxs;
    P.nfs = C->nfs;
    P.seed = C->twin_seed;
    P.tiem.resize(P.ninc1);
    for (int i = 0; i < P.ninc1; ++i) P.tiem[i] = (R)rdv(C->tiem, cb, i);
    P.xspec.assign((size_t)P.ninc1 * std::max(P.nxs, 1) * 15, R(0));
    for (int i = 0; i < P.ninc1; ++i)
        for (int j = 0; j < P.nxs; ++j)
            for (int k = 0; k < 15; ++k)
                P.xspec[((size_t)i * P.nxs + j) * 15 + k] =
                    (R)rdv(C->x_spec, cb, ((size_t)i * C->ld_xs + j) * 15 + k);
    P.fspec.assign((size_t)P.ninc1 * std::max(P.nfs, 1) * 3, R(0));
    for (int i = 0; i < P.ninc1; ++i)
        for (int j = 0; j < P.nfs; ++j)
            for (int k = 0; k < 3; ++k)
                P.fspec[((size_t)i * P.nfs + j) * 3 + k] =
                    (R)rdv(C->f_spec, cb, ((size_t)i * C->ld_xs + j) * 3 + k);
    // state storage
    const size_t nd3 = 3 * (size_t)P.nnod, ng = P.ngps;
    P.x.assign(nd3, 0); P.dx.assign(nd3, 0); P.fc.assign(nd3, 0); P.ddx.assign(nd3, 0);
    P.eps.assign(ng, 0); P.dep.assign(ng, 0);
    P.st.assign(ng * 6, 0); P.ep.assign(ng * 6, 0); P.ds.assign(ng * 6, 0); P.de.assign(ng * 6, 0);
    P.rt.assign(ng * 3, 0); P.dr.assign(ng * 3, 0);
    P.sv.assign(ng * SVLD, 0); P.dsv.assign(ng * SVLD, 0);
    P.srate.assign(ng * MAXSS, 0); P.cumslip.assign(ng * MAXSS, 0);
    P.timestwinned.assign(ng, 0); P.twinsys.assign(ng, 0);
    P.cp_iters.assign(ng, 0); P.erepmd_gp.assign(ng, 0); P.ops_gp.assign(ng, 0);
    P.chi_gp.assign(ng * 36, 0);
    if (P.nlmnt > 0) setpta(P);
    return 0;
}

template <class R> int upload(Problem<R> &P, const fas_state_desc *S)
{
    if (!S || (S->real_bytes != 4 && S->real_bytes != 8)) return FAS_E_ARG;
    const int rb = S->real_bytes;
    if (S->nsv < 0 || S->nsv > SVLD || S->nsv > S->ld_sv) return FAS_E_ARG;
    P.nsv = S->nsv;
    const size_t nd3 = 3 * (size_t)P.nnod;
    auto vec = [&](std::vector<R> &dst, const void *src, size_t n) {
        if (src) for (size_t i = 0; i < n; ++i) dst[i] = (R)rdv(src, rb, i);
    };
    vec(P.x, S->x, nd3); vec(P.dx, S->dx, nd3); vec(P.fc, S->fc, nd3); vec(P.ddx, S->ddx, nd3);
    vec(P.eps, S->eps, P.ngps); vec(P.dep, S->dep, P.ngps);
    vec(P.st, S->st, 6 * (size_t)P.ngps); vec(P.ep, S->ep, 6 * (size_t)P.ngps);
    vec(P.ds, S->ds, 6 * (size_t)P.ngps); vec(P.de, S->de, 6 * (size_t)P.ngps);
    vec(P.rt, S->rt, 3 * (size_t)P.ngps); vec(P.dr, S->dr, 3 * (size_t)P.ngps);
    for (int g = 0; g < P.ngps; ++g)
        for (int k = 0; k < P.nsv; ++k) {
            if (S->sv) P.sv[(size_t)g * SVLD + k] = (R)rdv(S->sv, rb, (size_t)g * S->ld_sv + k);
            if (S->dsv) P.dsv[(size_t)g * SVLD + k] = (R)rdv(S->dsv, rb, (size_t)g * S->ld_sv + k);
        }
    if (S->timestwinned) std::copy(S->timestwinned, S->timestwinned + P.ngps, P.timestwinned.begin());
    if (S->twinsys) std::copy(S->twinsys, S->twinsys + P.ngps, P.twinsys.begin());
    const int ls = S->ld_slip;
    if ((S->srate || S->cumslip) && (ls < 1 || ls > MAXSS)) return FAS_E_ARG;
    for (int g = 0; g < P.ngps; ++g)
        for (int k = 0; k < ls; ++k) {
            if (S->srate) P.srate[(size_t)g * MAXSS + k] = (R)rdv(S->srate, rb, (size_t)g * ls + k);
            if (S->cumslip) P.cumslip[(size_t)g * MAXSS + k] = (R)rdv(S->cumslip, rb, (size_t)g * ls + k);
        }
    if (!P.have_state && P.nlmnt > 0) {
        if (!S->x) return FAS_E_STATE;
        colour_nodes(P);
    }
    P.have_state = true;
    return 0;
}

template <class R> int download(Problem<R> &P, const fas_state_desc *S)
{
    if (!S || (S->real_bytes != 4 && S->real_bytes != 8)) return FAS_E_ARG;
    const int rb = S->real_bytes;
    const size_t nd3 = 3 * (size_t)P.nnod;
    auto vec = [&](const std::vector<R> &src, void *dst, size_t n) {
        if (dst) for (size_t i = 0; i < n; ++i) wrv(dst, rb, i, (double)src[i]);
    };
    vec(P.x, S->x, nd3); vec(P.dx, S->dx, nd3); vec(P.fc, S->fc, nd3); vec(P.ddx, S->ddx, nd3);
    vec(P.eps, S->eps, P.ngps); vec(P.dep, S->dep, P.ngps);
    vec(P.st, S->st, 6 * (size_t)P.ngps); vec(P.ep, S->ep, 6 * (size_t)P.ngps);
    vec(P.ds, S->ds, 6 * (size_t)P.ngps); vec(P.de, S->de, 6 * (size_t)P.ngps);
    vec(P.rt, S->rt, 3 * (size_t)P.ngps); vec(P.dr, S->dr, 3 * (size_t)P.ngps);
    const int nsv = std::min(S->nsv, SVLD);
    for (int g = 0; g < P.ngps; ++g)
        for (int k = 0; k < nsv; ++k) {
            if (S->sv) wrv(S->sv, rb, (size_t)g * S->ld_sv + k, (double)P.sv[(size_t)g * SVLD + k]);
            if (S->dsv) wrv(S->dsv, rb, (size_t)g * S->ld_sv + k, (double)P.dsv[(size_t)g * SVLD + k]);
        }
    if (S->timestwinned) std::copy(P.timestwinned.begin(), P.timestwinned.end(), S->timestwinned);
    if (S->twinsys) std::copy(P.twinsys.begin(), P.twinsys.end(), S->twinsys);
    const int ls = std::min(S->ld_slip, MAXSS);
    for (int g = 0; g < P.ngps; ++g)
        for (int k = 0; k < ls; ++k) {
            if (S->srate) wrv(S->srate, rb, (size_t)g * S->ld_slip + k, (double)P.srate[(size_t)g * MAXSS + k]);
            if (S->cumslip) wrv(S->cumslip, rb, (size_t)g * S->ld_slip + k, (double)P.cumslip[(size_t)g * MAXSS + k]);
        }
    return 0;
}

// constitutive update of every GP from the stored de / dr (micro-benchmark)
template <class R> int constitutive(Problem<R> &P, int inc, int nit)
{
    std::vector<int> rc(P.ngps, 0);
#pragma omp parallel for schedule(dynamic, 64) num_threads(P.nthreads) if (P.nthreads > 1)
    for (int j = 0; j < P.ngps; ++j) {
        R de[6], st[6], ds[6], t[6], r[3], d[6][6], deff = 0;
        for (int k = 0; k < 6; ++k) {
            de[k] = P.de[(size_t)j * 6 + k];
            st[k] = P.st[(size_t)j * 6 + k];
            ds[k] = P.ds[(size_t)j * 6 + k];
        }
        for (int k = 0; k < 3; ++k) r[k] = P.dr[(size_t)j * 3 + k];
        int c = dstrss(P, P.gp_iel[j], j, deff, de, st, ds, t, r, d, inc, nit);
        rc[j] = c;
        if (c) continue;
        P.dep[j] = deff;
        for (int k = 0; k < 6; ++k) P.ds[(size_t)j * 6 + k] = ds[k];
        R *chi = &P.chi_gp[(size_t)j * 36];
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b) chi[a + 6 * b] = d[a][b];
    }
    P.sumcpiter = 0;
    for (int j = 0; j < P.ngps; ++j) {
        if (rc[j]) return rc[j];
        P.sumcpiter = P.sumcpiter + P.erepmd_gp[j];
    }
    return 0;
}

// Replay of Gauss-point strain histories (the checker of the GPU library's
// fas_gpu_adjoint_forward, which has no counterpart in the reference): per
// increment DSTRSS (src/fasolt/Sig_eps.f90:84-151) with dsv = 0 and the
// elastic predictor S^-1 de as the stress guess, then the commit of
// UPDATE_GPTV (src/fasolt/Fasolt3.f90:254-284).  Works on a copy of the
// problem; J and the final lattice strains q^T e q (ELASEPS,
// src/csvmkr/data_out.f90:263-361) as the GPU library defines them.
template <class R> int replay(const Problem<R> &P0, const fas_replay_desc *d, double *J, double *eq)
{
    if (!d || !d->de || !d->dr || !d->dt || !d->w || !d->y || d->ninc < 1) return FAS_E_ARG;
    if (!P0.have_state) return FAS_E_STATE;
    const double qn = std::sqrt(d->q[0] * d->q[0] + d->q[1] * d->q[1] + d->q[2] * d->q[2]);
    if (!(qn > 0.0)) return FAS_E_ARG;
    const double q[3] = {d->q[0] / qn, d->q[1] / qn, d->q[2] / qn};
    const double qq[6] = {q[0] * q[0], q[1] * q[1], q[2] * q[2], q[1] * q[2], q[2] * q[0], q[0] * q[1]};
    Problem<R> P = P0;
    P.tiem.assign(d->dt, d->dt + d->ninc);
    const size_t ng = P.ngps;
    double jsum = 0.0;
    for (size_t g = 0; g < ng; ++g) {
        const int iel = P.gp_iel[g];
        const Material<R> &m = P.mat[std::abs(iel) - 1];
        R st[6];
        for (int k = 0; k < 6; ++k) st[k] = P.st[g * 6 + k];
        R *sv = &P.sv[g * SVLD];
        R *dsv = &P.dsv[g * SVLD];
        for (int n = 0; n < d->ninc; ++n) {
            R de[6], r[3], ds[6], t[6], chi[6][6], S[6][6], deff = 0;
            for (int k = 0; k < 6; ++k) de[k] = (R)d->de[((size_t)n * ng + g) * 6 + k];
            for (int k = 0; k < 3; ++k) r[k] = (R)d->dr[((size_t)n * ng + g) * 3 + k];
            for (int k = 0; k < 3 + m.ns; ++k) dsv[k] = 0;
            elastc(m.e, sv[0], sv[1], sv[2], S);
            if (factor(6, &S[0][0], 6)) return 910;
            for (int k = 0; k < 6; ++k) ds[k] = de[k];
            solver(6, &S[0][0], 6, ds);
            const int rc = dstrss(P, iel, (int)g, deff, de, st, ds, t, r, chi, n + 1, 1);
            if (rc) return rc;
            for (int k = 0; k < 6; ++k) st[k] = t[k];
            for (int k = 0; k < 3 + m.ns; ++k) sv[k] = sv[k] + dsv[k];
        }
        R S[6][6];
        elastc(m.e, sv[0], sv[1], sv[2], S);
        double e = 0.0;
        for (int i = 0; i < 6; ++i) {
            double ei = 0.0;
            for (int c = 0; c < 6; ++c) ei += (double)S[i][c] * (double)st[c];
            e += qq[i] * ei;
        }
        if (eq) eq[g] = e;
        jsum += 0.5 * d->w[g] * (e - d->y[g]) * (e - d->y[g]);
    }
    if (J) *J = jsum;
    return 0;
}

struct AnyProblem {
    int rb;
    std::unique_ptr<Problem<double>> d;
    std::unique_ptr<Problem<float>> f;
};

}  // namespace

struct ora_problem {
    AnyProblem a;
};

#define DISPATCH(p, expr)                                   \
    do {                                                    \
        if (!(p)) return FAS_E_ARG;                         \
        if ((p)->a.rb == 8) { auto &P = *(p)->a.d; expr; } \
        else { auto &P = *(p)->a.f; expr; }                 \
    } while (0)

extern "C" {

int32_t ora_create(const fas_mesh_desc *mesh, const fas_matl_desc *matl,
                   const fas_ctrl_desc *ctrl, int32_t real_bytes, uint32_t mode,
                   ora_problem **out)
{
    if (!out || (real_bytes != 4 && real_bytes != 8)) return FAS_E_ARG;
    *out = nullptr;
    auto *p = new (std::nothrow) ora_problem;
    if (!p) return FAS_E_NOMEM;
    p->a.rb = real_bytes;
    int rc;
    if (real_bytes == 8) {
        p->a.d.reset(new Problem<double>);
        p->a.d->mode = mode;
        rc = create(*p->a.d, mesh, matl, ctrl);
    } else {
        p->a.f.reset(new Problem<float>);
        p->a.f->mode = mode;
        rc = create(*p->a.f, mesh, matl, ctrl);
    }
    if (rc) { delete p; return rc; }
    *out = p;
    return 0;
}

void ora_destroy(ora_problem *p) { delete p; }

int32_t ora_set_mode(ora_problem *p, uint32_t mode) { DISPATCH(p, P.mode = mode); return 0; }
int32_t ora_set_threads(ora_problem *p, int32_t n)
{
    DISPATCH(p, P.nthreads = n < 1 ? 1 : n);
    return 0;
}
int32_t ora_upload_state(ora_problem *p, const fas_state_desc *s) { DISPATCH(p, return upload(P, s)); }
int32_t ora_download_state(ora_problem *p, const fas_state_desc *s) { DISPATCH(p, return download(P, s)); }
int32_t ora_update_node(ora_problem *p)
{
    DISPATCH(p, {
        if (!P.have_state) return FAS_E_STATE;
        for (size_t i = 0; i < P.x.size(); ++i) P.x[i] = P.x[i] + P.dx[i];
    });
    return 0;
}
int32_t ora_elvals(ora_problem *p, int32_t inc, int32_t nit)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        if (inc < 1 || inc > P.ninc1) return FAS_E_ARG;
        return elvals(P, inc, nit);
    });
}
int32_t ora_suvals(ora_problem *p, int32_t inc)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        if (inc < 1 || inc > P.ninc1) return FAS_E_ARG;
        return suvals(P, inc);
    });
}
int32_t ora_facsls(ora_problem *p, int32_t *sweeps, double *error)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        return facsls(P, 1000, sweeps, error);
    });
}
int32_t ora_facsls_limited(ora_problem *p, int32_t max_sweeps, int32_t *sweeps, double *error)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        return facsls(P, max_sweeps, sweeps, error);
    });
}
int32_t ora_nriter(ora_problem *p, int32_t inc, fas_iter_report *rep, int32_t cap, int32_t *n_rep)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        if (inc < 1 || inc > P.ninc1) return FAS_E_ARG;
        return nriter(P, inc, rep, cap, n_rep);
    });
}
int32_t ora_nr_step(ora_problem *p, int32_t inc, int32_t nit, fas_iter_report *rep, int32_t *more)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        if (inc < 1 || inc > P.ninc1) return FAS_E_ARG;
        bool m = false;
        int rc = nr_step(P, inc, nit, rep, &m);
        if (more) *more = m ? 1 : 0;
        return rc;
    });
}
int32_t ora_nr_finish(ora_problem *p, int32_t inc)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        if (inc < 1 || inc > P.ninc1) return FAS_E_ARG;
        nr_finish(P, inc);
        return 0;
    });
}
int32_t ora_update_gptv(ora_problem *p)
{
    DISPATCH(p, {
        if (!P.have_state) return FAS_E_STATE;
        update_gptv(P);
    });
    return 0;
}
int32_t ora_reorient(ora_problem *p, int32_t inc, fas_twin_event *ev, int32_t cap, int32_t *n_ev)
{
    DISPATCH(p, {
        if (!P.have_state) return FAS_E_STATE;
        int n = reorient(P, inc, ev, cap);
        if (n_ev) *n_ev = n;
        P.tflag = 0;
    });
    return 0;
}
int32_t ora_increment(ora_problem *p, int32_t inc, fas_iter_report *rep, int32_t cap, int32_t *n_rep,
                      fas_twin_event *ev, int32_t ev_cap, int32_t *n_ev)
{
    int32_t rc = ora_update_node(p);
    if (rc) return rc;
    rc = ora_nriter(p, inc, rep, cap, n_rep);
    if (rc) return rc;
    rc = ora_update_gptv(p);
    if (rc) return rc;
    if (n_ev) *n_ev = 0;
    int any = 0;
    DISPATCH(p, any = P.tflag);
    if (any) rc = ora_reorient(p, inc, ev, ev_cap, n_ev);
    return rc;
}
int32_t ora_get_pattern(ora_problem *p, int32_t *is, int32_t ld_is)
{
    DISPATCH(p, {
        if (!is || P.nlmnt == 0) return FAS_E_ARG;
        if (ld_is < P.ld) return 955;
        const int ndof = 3 * P.nnod;
        for (int r = 0; r < ndof; ++r) {
            const int *src = &P.is[(size_t)r * P.ld];
            int32_t *dst = is + (size_t)r * ld_is;
            std::fill(dst, dst + ld_is, 0);
            dst[0] = src[0];
            for (int k = 1; k <= src[0]; ++k) dst[k] = src[k] + 1;
        }
    });
    return 0;
}
int32_t ora_get_stiffness(ora_problem *p, void *ss, int32_t ld_ss, int32_t rb)
{
    DISPATCH(p, {
        if (!ss || P.nlmnt == 0 || (rb != 4 && rb != 8)) return FAS_E_ARG;
        if (ld_ss < P.ld) return 955;
        const int ndof = 3 * P.nnod;
        for (int r = 0; r < ndof; ++r)
            for (int k = 0; k < ld_ss; ++k)
                wrv(ss, rb, (size_t)r * ld_ss + k, k < P.ld ? (double)P.ss[(size_t)r * P.ld + k] : 0.0);
    });
    return 0;
}
int32_t ora_get_colouring(ora_problem *p, int32_t *colour, int32_t *ncol)
{
    DISPATCH(p, {
        if (!P.have_state || P.nlmnt == 0) return FAS_E_STATE;
        if (colour) std::copy(P.colour.begin(), P.colour.end(), colour);
        if (ncol) *ncol = P.ncol;
    });
    return 0;
}
int32_t ora_constitutive(ora_problem *p, int32_t inc, int32_t nit)
{
    DISPATCH(p, {
        if (!P.have_state) return FAS_E_STATE;
        if (inc < 1 || inc > P.ninc1) return FAS_E_ARG;
        return constitutive(P, inc, nit);
    });
}
int32_t ora_get_tangent(ora_problem *p, void *chi, int32_t rb)
{
    DISPATCH(p, {
        if (!chi || (rb != 4 && rb != 8)) return FAS_E_ARG;
        for (size_t i = 0; i < P.chi_gp.size(); ++i) wrv(chi, rb, i, (double)P.chi_gp[i]);
    });
    return 0;
}
int32_t ora_get_cp_stats(ora_problem *p, int32_t *iters, double *erepmd)
{
    DISPATCH(p, {
        if (iters) std::copy(P.cp_iters.begin(), P.cp_iters.end(), iters);
        if (erepmd) for (int j = 0; j < P.ngps; ++j) erepmd[j] = (double)P.erepmd_gp[j];
    });
    return 0;
}
int32_t ora_get_cp_ops(ora_problem *p, double *ops)
{
    DISPATCH(p, {
        if (ops) std::copy(P.ops_gp.begin(), P.ops_gp.end(), ops);
    });
    return 0;
}

// ELASEPS, src/csvmkr/data_out.f90:263-361
int32_t ora_lattice_strain(ora_problem *p, double *out)
{
    DISPATCH(p, {
        if (!out) return FAS_E_ARG;
        for (int g = 0; g < P.ngps; ++g) {
            const auto &m = P.mat[std::abs(P.gp_iel[g]) - 1];
            const auto *sv = &P.sv[(size_t)g * SVLD];
            decltype(P.toler) S[6][6];
            elastc(m.e, sv[0], sv[1], sv[2], S);
            for (int i = 0; i < 6; ++i) {
                decltype(P.toler) acc = 0;
                for (int c = 0; c < 6; ++c) acc = acc + S[i][c] * P.st[(size_t)g * 6 + c];
                out[(size_t)g * 6 + i] = (double)acc;
            }
        }
    });
    return 0;
}

int32_t ora_adjoint_forward(ora_problem *p, const fas_replay_desc *d, double *J, double *eq)
{
    DISPATCH(p, return replay(P, d, J, eq));
}

double ora_spower(double a, double b) { return spower<double>(a, b); }
double ora_fj2vom(int32_t stress, const double *x6) { return fj2vom<double>(stress != 0, x6); }
int32_t ora_factor_solve(int32_t n, const double *a, double *x)
{
    std::vector<double> w((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) w[(size_t)i * n + j] = a[(size_t)j * n + i];
    if (factor<double>(n, w.data(), n)) return 910;
    solver<double>(n, w.data(), n, x);
    return 0;
}
void ora_ctmatrx(double ph1, double phi, double ph2, double *a9, double *aug3)
{
    double a[3][3];
    ctmatrx<double>(ph1, phi, ph2, a, aug3);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a9[i + 3 * j] = a[i][j];
}
void ora_elastc(const double *e9, const double *eu, double *s36)
{
    double S[6][6];
    elastc<double>(e9, eu[0], eu[1], eu[2], S);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) s36[i + 6 * j] = S[i][j];
}
void ora_tens_rot(const double *r3, const double *a6, double *b6) { tens_rot<double>(r3, a6, b6); }
double ora_shape12(const double *x38, double *d38)
{
    double xn[8][3], dn[8][3];
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) xn[i][k] = x38[k + 3 * i];
    double w = shape12<double>(xn, dn);
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) d38[k + 3 * i] = dn[i][k];
    return w;
}
double ora_shape22(int g, const double *x320, double *d320)
{
    if (g < 0 || g > 7) return 0.0;
    double xn[20][3], dn[20][3];
    for (int i = 0; i < 20; ++i)
        for (int k = 0; k < 3; ++k) xn[i][k] = x320[k + 3 * i];
    double w = shape22<double>(g, xn, dn);
    for (int i = 0; i < 20; ++i)
        for (int k = 0; k < 3; ++k) d320[k + 3 * i] = dn[i][k];
    return w;
}
// SHAPE_21 / SHAPE_22 / SHAPE_23 of element type lt for GP g (0-based):
// x[3*i + k] node coordinates, d[3*i + k] global derivatives; returns the
// GP weight (0 for an unknown type or GP).
double ora_shape_elem(int lt, int g, const double *x, double *d)
{
    const int nn = lt == 21 ? 10 : (lt == 22 ? 20 : (lt == 23 ? 15 : 0));
    const int ng = lt == 21 ? 4 : (lt == 22 ? 8 : (lt == 23 ? 6 : 0));
    if (!nn || g < 0 || g >= ng) return 0.0;
    double xn[20][3] = {}, dn[20][3] = {};
    for (int i = 0; i < nn; ++i)
        for (int k = 0; k < 3; ++k) xn[i][k] = x[k + 3 * i];
    const double w = lt == 21 ? shape21<double>(g, xn, dn) : (lt == 22 ? shape22<double>(g, xn, dn)
                                                                         : shape23<double>(g, xn, dn));
    for (int i = 0; i < nn; ++i)
        for (int k = 0; k < 3; ++k) d[k + 3 * i] = dn[i][k];
    return w;
}
// The local-derivative tables of SHAPE_21 ([4][3][10]) and SHAPE_23
// ([6][3][15]), dn[(g*3 + j)*nn + i].
void ora_shape21_table(double *dn)
{
    const Shape21Table &t = shape21_table();
    for (int g = 0; g < 4; ++g)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 10; ++i) dn[(g * 3 + j) * 10 + i] = t.dn[g][j][i];
}
void ora_shape23_table(double *dn)
{
    const Shape23Table &t = shape23_table();
    for (int g = 0; g < 6; ++g)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 15; ++i) dn[(g * 3 + j) * 15 + i] = t.dn[g][j][i];
}
void ora_shape22_table(double *dn)
{
    const Shape22Table &t = shape22_table();
    for (int g = 0; g < 8; ++g)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 20; ++i) dn[(g * 3 + j) * 20 + i] = t.dn[g][j][i];
}

}  // extern "C"
