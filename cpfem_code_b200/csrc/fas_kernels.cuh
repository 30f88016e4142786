// fas_kernels.cuh -- the sm_100a kernels of the increment hot path.
//
// Data layout in HBM (all FP64 unless noted):
//   * nodal vectors x, dx, fc, ddx, rhs: reference DOF order 3*node+comp;
//   * Gauss-point state: structure of arrays field[k * ngps + g];
//   * Gauss-point record rec[item * RecLayout<NN>::LEN + .] (item = element
//     for 8-node bricks, element*NPG + GP for the quadratic elements):
//     sfd (3 NN),
//     stress (6), weight, tangent upper triangle (21) -- written once per
//     Newton iteration by the element kernel, read by the row-gather
//     assembly;
//   * stiffness: block-ELL of 3x3 node blocks, rows permuted so each SOR
//     colour is a contiguous row range.  A row of S slots (27 for 8-node
//     bricks, 81 for the quadratic elements) holds brow_of(S) values, component-major:
//     blk[row*brow + (r*3+c)*S + slot], padded so FP64 and FP32 rows are
//     16-byte multiples as bulk copies need (244 and 732 values).  Slot 0 is
//     the diagonal block; bcol[row*crow + slot] is the column node and
//     bcol[row*crow + S] the row's slot count (crow = 28 or 84).
//
// Kernels: the element pass (k_elem, k_elemq, the opt-in warp variants),
// the work-sorted launch order of the constitutive kernels (k_work_*), the
// row-gather assembly with fused SUVALS (k_assemble), the SOR colour phase
// streamed by the bulk-copy engine (k_sor_colour_tma, launched with
// programmatic serialisation) and its stopping test (k_sor_check), the
// one-CTA solve of small meshes (k_sor_small), the FP32 refinement pieces,
// the increment commit, twin reorientation, ELASEPS and the exports.
#pragma once

#include <type_traits>

#include "fas_device.cuh"
#include "fas_device_warp.cuh"

namespace fasdev {

// Gauss-point record of an NN-node element: sfd (3 NN), stress (6),
// weight, pad, tangent upper triangle (21), pad.
template <int NN> struct RecLayout {
    static constexpr int S = 3 * NN, W = 3 * NN + 6, D = 3 * NN + 8, LEN = 3 * NN + 32;
};
constexpr int REC = RecLayout<8>::LEN;   // 56 doubles per 8-node element record
constexpr int REC_S = RecLayout<8>::S, REC_W = RecLayout<8>::W, REC_D = RecLayout<8>::D;
constexpr int SLOTS = 27;        // node blocks per row of an 8-node brick mesh
constexpr int SLOTS20 = 81;      // node blocks per row of a 20-node brick mesh
constexpr int MAXADJ = 64;       // elements per node the tables allow (bytes of a local-index word)

// block matrix addressing: a row of S slots holds 9 S values padded to a
// multiple of 4 (so FP64 and FP32 rows are both 16-byte multiples, as bulk
// copies need) and S column ids plus the slot count padded to a multiple of 4
__host__ __device__ constexpr int brow_of(int S) { return (S * 9 + 3) / 4 * 4; }
__host__ __device__ constexpr int crow_of(int S) { return (S + 1 + 3) / 4 * 4; }
constexpr int BROW = brow_of(SLOTS);   // 244
constexpr int CROW = crow_of(SLOTS);   // 28
static_assert(BROW == 244 && CROW == 28, "8-node row layout");

// upper-triangle index of chi(i,j), i <= j (0-based)
__host__ __device__ __forceinline__ int utri(int i, int j) { return i * 6 - (i * (i - 1)) / 2 + (j - i); }

struct MeshDev {
    int nlmnt, nnod;
    int nn, npg;         // nodes and Gauss points per element (8, 1 or 20, 8)
    const int *ln;       // [nn][nlmnt] 0-based node ids
    const int *gpe;      // [npg][nlmnt] 0-based GPs of the element
    const int *le;       // [nlmnt]
    const int *lt;       // [nlmnt] element type: the family's (12 or 22), or 1-6 for a tie
    const int *ib;       // [nnod]
    const int *ne_elem;  // [maxadj][nnod] adjacent elements, ascending
    const int *ne_loc;   // [maxadj][nnod] local index of the node in it
    const int *ne_cnt;   // [nnod]
};

struct BlockDev {
    int R;               // rows (= nnod)
    int slots, brow, crow;   // slots per row and the row lengths (brow_of, crow_of)
    const int *perm;     // row -> node
    const int *nslot;    // [R]
    const int *bcol;     // [R][crow] column node of each slot; [slots] = nslot
    const unsigned long long *bloc;   // [R][crow][nbw] byte k: local index of the column node
                                      // in the k-th adjacent element of the row node (0xFF: absent)
    int nbw;             // words of bloc per slot: ceil(elements per node / 8)
    double *blk;         // [R][brow]: value (r, c) of slot s at (r*3+c)*slots + s
    float *blk32;        // FP32 copy of blk (tuned mode), or null
    __host__ __device__ size_t si(int p, int s) const { return (size_t)p * crow + s; }
    __host__ __device__ size_t bi(int p, int s, int q) const { return (size_t)p * brow + (size_t)q * slots + s; }
};

// The items of a constitutive pass, entry t of the launch order (`order`,
// or the natural order when it is null).  With a device queue (`queue`
// non-null, a persistent grid) every warp takes the next 32 entries until
// the order is exhausted, so the work-sorted order is served heaviest first
// and no CTA slot idles behind one slow warp; otherwise thread t takes
// entry t.
template <typename F>
__device__ __forceinline__ void for_each_item(int n, const int *__restrict__ order, int *queue, F &&f)
{
    if (queue) {
        const int lane = threadIdx.x & 31;
        for (;;) {
            int base = 0;
            if (lane == 0) base = atomicAdd(queue, 32);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= n) return;
            const int t = base + lane;
            if (t < n) f(order ? order[t] : t);
        }
    }
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) f(order ? order[t] : t);
}

// ---------------------------------------------------------------- element pass
// ELVALS per element (src/fasolt/Elvals.f90:31-126): gather, SHAPE_12,
// DSTRNS, DSTRSS, store the GP increments and the element record.
template <int NS>
__global__ void __launch_bounds__(128) k_elem(MeshDev Mh, DevMat M, DevCtrl C, DevGp G,
                                              const double *__restrict__ x,
                                              const double *__restrict__ dx, double *rec,
                                              double dt, int inc, int nit,
                                              unsigned long long *errkey, const int *__restrict__ order,
                                              int *queue)
{
#if FAS_SMEM_TABLES
    extern __shared__ double s_tables[];
    if (M.stage_t > 0) M = stage_tables(M, s_tables);
#endif
    for_each_item(Mh.nlmnt, order, queue, [&](int e) {
        if (Mh.lt[e] < 9) return;   // tie element: no Gauss point
        const int ne = Mh.nlmnt;
        double xl[8][3], dxl[8][3];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int n = Mh.ln[a * ne + e];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xl[a][c] = x[3 * n + c];
                dxl[a][c] = dx[3 * n + c];
            }
        }
        double sfd[8][3];
        const double w = shape12(xl, sfd);
        if (w < 1.e-7) {
            atomicMin(errkey, ((unsigned long long)e << 16) | 920ull);
            return;
        }
        double del[6], r[3], defl;
        int rc = dstrns(sfd, dxl, C.smalr, C.smale, del, r, defl);
        if (rc) {
            atomicMin(errkey, ((unsigned long long)e << 16) | (unsigned long long)rc);
            return;
        }
        const int g = Mh.gpe[e];
        const int ng = G.ngps;
        double st[6], ds[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            st[k] = G.st[k * ng + g];
            ds[k] = G.ds[k * ng + g];
        }
        GpOut o;
        rc = dstrss<NS>(M, C, G, g, Mh.le[e], del, r, st, ds, dt, inc, C.nit_dev ? *C.nit_dev + 1 : nit, o);
        if (rc) {
            atomicMin(errkey, ((unsigned long long)e << 16) | (unsigned long long)rc);
            return;
        }
        G.dep[g] = o.deff;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            G.de[k * ng + g] = del[k];
            G.ds[k * ng + g] = ds[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) G.dr[k * ng + g] = r[k];
        double *R = rec + (size_t)e * REC;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) R[3 * a + c] = sfd[a][c];
#pragma unroll
        for (int k = 0; k < 6; ++k) R[REC_S + k] = o.t[k];
        R[REC_W] = w;
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j) R[REC_D + utri(i, j)] = o.chi[i][j];
    });
}

// ELVALS per Gauss point of the quadratic elements (src/fasolt/Elvals.f90:
// 82-126): 10-node tetrahedra with SHAPE_21 (NN 10, NPG 4,
// src/fasolt/Shapef.f90:104-189), 20-node bricks with SHAPE_22 (20, 8,
// :210-342) and 15-node wedges with SHAPE_23 (15, 6, :360-485); one thread
// per (element, GP).  dnt[(g*3 + j)*NN + i] = dndn(j+1, i+1, g+1) is the
// element type's tabulated local-derivative table and wfac its GP weight
// factor (-0.0416667, 1, 0.16666667).  The element's nodes are streamed
// twice -- the Jacobian, then sfd (written straight to the GP record) and
// the displacement gradient -- so no node array is held in registers.
// Errors are keyed by (element, GP) so the first one in the reference's
// loop order wins.
template <int NS, int NN, int NPG>
__global__ void __launch_bounds__(128) k_elemq(MeshDev Mh, DevMat M, DevCtrl C, DevGp G,
                                               const double *__restrict__ dnt, double wfac,
                                               const double *__restrict__ x,
                                               const double *__restrict__ dx, double *rec,
                                               double dt, int inc, int nit,
                                               unsigned long long *errkey, const int *__restrict__ order,
                                               int *queue)
{
#if FAS_SMEM_TABLES
    extern __shared__ double s_tables[];
    if (M.stage_t > 0) M = stage_tables(M, s_tables);
#endif
    using L = RecLayout<NN>;
    for_each_item(NPG * Mh.nlmnt, order, queue, [&](int t) {   // item e*NPG + gq
        const int e = t / NPG, gq = t - e * NPG;
        if (Mh.lt[e] < 9) return;   // tie element: no Gauss point
        const int ne = Mh.nlmnt;
        const unsigned long long key = (unsigned long long)t << 16;
        const double *dn = dnt + gq * 3 * NN;
        double jac[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int i = 0; i < NN; ++i) {
            const int n = Mh.ln[i * ne + e];
            const double d0 = __ldg(dn + i), d1 = __ldg(dn + NN + i), d2 = __ldg(dn + 2 * NN + i);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const double xk = x[3 * n + k];
                jac[0][k] = jac[0][k] + d0 * xk;
                jac[1][k] = jac[1][k] + d1 * xk;
                jac[2][k] = jac[2][k] + d2 * xk;
            }
        }
        double inv[3][3];
        const double w = wfac * invert3(jac, inv);
        if (w < 1.e-7) {
            atomicMin(errkey, key | 920ull);
            return;
        }
        double *R = rec + (size_t)t * L::LEN;
        double gr[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int i = 0; i < NN; ++i) {
            const int n = Mh.ln[i * ne + e];
            const double d0 = __ldg(dn + i), d1 = __ldg(dn + NN + i), d2 = __ldg(dn + 2 * NN + i);
            double sf[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                sf[k] = inv[k][0] * d0 + inv[k][1] * d1 + inv[k][2] * d2;
                R[3 * i + k] = sf[k];
            }
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const double u = dx[3 * n + b];
#pragma unroll
                for (int a = 0; a < 3; ++a) gr[a][b] = gr[a][b] + sf[a] * u;
            }
        }
        double del[6], r[3], defl;
        int rc = dstrns_grad(gr, C.smalr, C.smale, del, r, defl);
        if (rc) {
            atomicMin(errkey, key | (unsigned long long)rc);
            return;
        }
        const int g = Mh.gpe[gq * ne + e];
        const int ng = G.ngps;
        double st[6], ds[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            st[k] = G.st[k * ng + g];
            ds[k] = G.ds[k * ng + g];
        }
        GpOut o;
        rc = dstrss<NS>(M, C, G, g, Mh.le[e], del, r, st, ds, dt, inc, C.nit_dev ? *C.nit_dev + 1 : nit, o);
        if (rc) {
            atomicMin(errkey, key | (unsigned long long)rc);
            return;
        }
        G.dep[g] = o.deff;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            G.de[k * ng + g] = del[k];
            G.ds[k * ng + g] = ds[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) G.dr[k * ng + g] = r[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) R[L::S + k] = o.t[k];
        R[L::W] = w;
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = i; j < 6; ++j) R[L::D + utri(i, j)] = o.chi[i][j];
    });
}

// Work-sorted launch order for the constitutive kernels: items (elements or
// points) grouped by the operation count of their GP's last update, so the
// lanes of a warp take similar iteration counts and active-set sizes.  A
// counting sort in WORK_BINS bins of 512 counted operations; the order within
// a bin is whatever the atomics give, which no result depends on (every GP
// is updated independently, errors are reduced with atomicMin).
constexpr int WORK_BINS = 256;
__device__ __forceinline__ int work_bin(int g, const double *ops)
{
    if (g < 0) return 0;
    const double b = ops[g] * (1.0 / 512.0);
    return b < (double)(WORK_BINS - 1) ? (int)b : WORK_BINS - 1;
}
__global__ void k_work_hist(int n, const int *__restrict__ gp_of, const double *__restrict__ ops, int *hist)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    atomicAdd(&hist[work_bin(gp_of ? gp_of[i] : i, ops)], 1);
}
// Bin offsets: heaviest bin first (FAS_WORK_DESC, the default), so the
// tail of a pass holds the cheapest items, or lightest first.
#ifndef FAS_WORK_DESC
#define FAS_WORK_DESC 1
#endif
__global__ void __launch_bounds__(WORK_BINS) k_work_scan(int *hist)
{
    __shared__ int v[WORK_BINS];
    v[threadIdx.x] = hist[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < WORK_BINS; ++k) {
            const int b = FAS_WORK_DESC ? WORK_BINS - 1 - k : k;
            const int c = v[b];
            v[b] = acc;
            acc += c;
        }
    }
    __syncthreads();
    hist[threadIdx.x] = v[threadIdx.x];
}
__global__ void k_work_scatter(int n, const int *__restrict__ gp_of, const double *__restrict__ ops, int *offs,
                               int *order)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    order[atomicAdd(&offs[work_bin(gp_of ? gp_of[i] : i, ops)], 1)] = i;
}

// Constitutive update of independent points (no mesh): DSTRSS with the
// stored de / dr; the full tangent goes to chi[36][ngps] (column-major 6x6).
template <int NS>
__global__ void __launch_bounds__(128) k_points(DevMat M, DevCtrl C, DevGp G, const int *gp_iel,
                                                double *chi, double dt, int inc, int nit,
                                                unsigned long long *errkey, const int *__restrict__ order,
                                                int *queue)
{
#if FAS_SMEM_TABLES
    extern __shared__ double s_tables[];
    if (M.stage_t > 0) M = stage_tables(M, s_tables);
#endif
    for_each_item(G.ngps, order, queue, [&](int g) {
        const int ng = G.ngps;
        double de[6], r[3], st[6], ds[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            de[k] = G.de[k * ng + g];
            st[k] = G.st[k * ng + g];
            ds[k] = G.ds[k * ng + g];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) r[k] = G.dr[k * ng + g];
        GpOut o;
        const int rc = dstrss<NS>(M, C, G, g, gp_iel[g], de, r, st, ds, dt, inc, nit, o);
        if (rc) {
            atomicMin(errkey, ((unsigned long long)g << 16) | (unsigned long long)rc);
            return;
        }
        G.dep[g] = o.deff;
#pragma unroll
        for (int k = 0; k < 6; ++k) G.ds[k * ng + g] = ds[k];
#pragma unroll
        for (int i = 0; i < 6; ++i)
#pragma unroll
            for (int j = 0; j < 6; ++j) chi[(i + 6 * j) * (size_t)ng + g] = o.chi[i][j];
    });
}

// ---------------------------------------------------------------- warp-cooperative pass
// ELVALS per element with one warp per element: every lane forms the
// element kinematics (identical values), the warp runs dstrss_wc with lane i
// owning slip system i, and the lanes share out the stores.
template <int NA>
__global__ void __launch_bounds__(128) k_elem_wc(MeshDev Mh, DevMat M, DevCtrl C, DevGp G,
                                                 const double *__restrict__ x,
                                                 const double *__restrict__ dx, double *rec,
                                                 double dt, int inc, int nit,
                                                 unsigned long long *errkey)
{
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (e >= Mh.nlmnt) return;           // whole warps only
    if (Mh.lt[e] < 9) return;            // tie element: no Gauss point
    const int ne = Mh.nlmnt;
    double del[6], r[3], defl;
    double *R = rec + (size_t)e * REC;
    {
        double xl[8][3], dxl[8][3];
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            const int n = Mh.ln[a * ne + e];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                xl[a][c] = x[3 * n + c];
                dxl[a][c] = dx[3 * n + c];
            }
        }
        double sfd[8][3];
        const double w = shape12(xl, sfd);
        if (w < 1.e-7) {
            if (lane == 0) atomicMin(errkey, ((unsigned long long)e << 16) | 920ull);
            return;
        }
        const int rc = dstrns(sfd, dxl, C.smalr, C.smale, del, r, defl);
        if (rc) {
            if (lane == 0) atomicMin(errkey, ((unsigned long long)e << 16) | (unsigned long long)rc);
            return;
        }
        // record: lanes 0-23 shape derivatives, lane 30 the weight
        double v = 0.0;
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (lane == 3 * a + c) v = sfd[a][c];
        if (lane == REC_W) v = w;
        if (lane < 24 || lane == REC_W) R[lane] = v;
    }
    const int g = Mh.gpe[e];
    const int ng = G.ngps;
    double st[6], ds[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        st[k] = G.st[k * ng + g];
        ds[k] = G.ds[k * ng + g];
    }
    wc::GpOutW o;
    const int rc = wc::dstrss_wc<NA>(M, C, G, g, Mh.le[e], del, r, st, ds, dt, inc,
                                     C.nit_dev ? *C.nit_dev + 1 : nit, o);
    if (rc) {
        if (lane == 0) atomicMin(errkey, ((unsigned long long)e << 16) | (unsigned long long)rc);
        return;
    }
    if (lane == 0) G.dep[g] = o.deff;
    if (lane < 6) {
        double dk = 0.0, sk = 0.0, tk = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (k == lane) {
                dk = del[k];
                sk = ds[k];
                tk = o.t[k];
            }
        G.de[lane * ng + g] = dk;
        G.ds[lane * ng + g] = sk;
        R[REC_S + lane] = tk;
        // tangent upper triangle, row `lane`
#pragma unroll
        for (int j = 0; j < 6; ++j)
            if (j >= lane) R[REC_D + utri(lane, j)] = o.chirow[j];
    }
    if (lane < 3) {
        double rk = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (k == lane) rk = r[k];
        G.dr[lane * ng + g] = rk;
    }
}

// Independent points with one warp per point (the micro-benchmark path).
template <int NA>
__global__ void __launch_bounds__(128) k_points_wc(DevMat M, DevCtrl C, DevGp G, const int *gp_iel,
                                                   double *chi, double dt, int inc, int nit,
                                                   unsigned long long *errkey)
{
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= G.ngps) return;
    const int ng = G.ngps;
    double de[6], r[3], st[6], ds[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        de[k] = G.de[k * ng + g];
        st[k] = G.st[k * ng + g];
        ds[k] = G.ds[k * ng + g];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] = G.dr[k * ng + g];
    wc::GpOutW o;
    const int rc = wc::dstrss_wc<NA>(M, C, G, g, gp_iel[g], de, r, st, ds, dt, inc, nit, o);
    if (rc) {
        if (lane == 0) atomicMin(errkey, ((unsigned long long)g << 16) | (unsigned long long)rc);
        return;
    }
    if (lane == 0) G.dep[g] = o.deff;
    if (lane < 6) {
        double sk = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (k == lane) sk = ds[k];
        G.ds[lane * ng + g] = sk;
    }
    if (lane < 6) {   // row `lane` of the tangent, column-major 6x6 per point
#pragma unroll
        for (int j = 0; j < 6; ++j) chi[(size_t)(lane + 6 * j) * ng + g] = o.chirow[j];
    }
}

// gaussm (src/fasolt/Elvals.f90:132-220) for node pair (i, j) of one
// element: gm[r][c] = gaussm(r+1, c+1).  d is the tangent's upper
// triangle -- the only entries the reference reads.
__device__ __forceinline__ void gaussm_block(const double ai[3], const double bj[3],
                                             const double *d, const double s[6], double gm[9])
{
#define D(p, q) d[utri((p)-1, (q)-1)]
#define SS(p) s[(p)-1]
    const double i1 = ai[0], i2 = ai[1], i3 = ai[2], j1 = bj[0], j2 = bj[1], j3 = bj[2];
    gm[0] = (i1 * j1 * (D(1, 1) - SS(1)) + i2 * j2 * (D(6, 6) - (SS(1) - SS(2)) / 2.0) +
             i3 * j3 * (D(5, 5) - (SS(1) - SS(3)) / 2.0) + i2 * j3 * (D(5, 6) + SS(4) / 2.0) +
             i3 * j1 * (D(1, 5)) + i1 * j2 * (D(1, 6)) + j2 * i3 * (D(5, 6) + SS(4) / 2.0) +
             j3 * i1 * (D(1, 5)) + j1 * i2 * (D(1, 6)));
    gm[3] = (i1 * j1 * (D(1, 6) - SS(6)) + i2 * j2 * (D(2, 6) - SS(6)) +
             i3 * j3 * (D(4, 5) - SS(6) / 2.0) + i2 * j3 * (D(2, 5) - SS(5) / 4.0) +
             i3 * j1 * (D(1, 4) - SS(4) / 4.0) + i1 * j2 * (D(6, 6) - (SS(1) + SS(2)) / 4.0) +
             j2 * i3 * (D(4, 6) - SS(5) / 4.0) + j3 * i1 * (D(5, 6) - SS(4) / 4.0) +
             j1 * i2 * (D(1, 2) - (SS(1) + SS(2)) / 4.0));
    gm[6] = (i1 * j1 * (D(1, 5) - SS(5)) + i2 * j2 * (D(4, 6) - SS(5) / 2.0) +
             i3 * j3 * (D(3, 5) - SS(5)) + i2 * j3 * (D(4, 5) - SS(6) / 4.0) +
             i3 * j1 * (D(1, 3) - (SS(1) + SS(3)) / 4.0) + i1 * j2 * (D(5, 6) - SS(4) / 4.0) +
             j2 * i3 * (D(3, 6) - SS(6) / 4.0) + j3 * i1 * (D(5, 5) - (SS(1) + SS(3)) / 4.0) +
             j1 * i2 * (D(1, 4) - SS(4) / 4.0));
    gm[1] = (j1 * i1 * (D(1, 6) - SS(6)) + j2 * i2 * (D(2, 6) - SS(6)) +
             j3 * i3 * (D(4, 5) - SS(6) / 2.0) + j2 * i3 * (D(2, 5) - SS(5) / 4.0) +
             j3 * i1 * (D(1, 4) - SS(4) / 4.0) + j1 * i2 * (D(6, 6) - (SS(1) + SS(2)) / 4.0) +
             i2 * j3 * (D(4, 6) - SS(5) / 4.0) + i3 * j1 * (D(5, 6) - SS(4) / 4.0) +
             i1 * j2 * (D(1, 2) - (SS(1) + SS(2)) / 4.0));
    gm[4] = (i1 * j1 * (D(6, 6) - (SS(2) - SS(1)) / 2.0) + i2 * j2 * (D(2, 2) - SS(2)) +
             i3 * j3 * (D(4, 4) - (SS(2) - SS(3)) / 2.0) + i2 * j3 * (D(2, 4)) +
             i3 * j1 * (D(4, 6) + SS(5) / 2.0) + i1 * j2 * (D(2, 6)) + j2 * i3 * (D(2, 4)) +
             j3 * i1 * (D(4, 6) + SS(5) / 2.0) + j1 * i2 * (D(2, 6)));
    gm[7] = (i1 * j1 * (D(5, 6) - SS(4) / 2.0) + i2 * j2 * (D(2, 4) - SS(4)) +
             i3 * j3 * (D(3, 4) - SS(4)) + i2 * j3 * (D(4, 4) - (SS(2) + SS(3)) / 4.0) +
             i3 * j1 * (D(3, 6) - SS(6) / 4.0) + i1 * j2 * (D(2, 5) - SS(5) / 4.0) +
             j2 * i3 * (D(2, 3) - (SS(2) + SS(3)) / 4.0) + j3 * i1 * (D(4, 5) - SS(6) / 4.0) +
             j1 * i2 * (D(4, 6) - SS(5) / 4.0));
    gm[2] = (j1 * i1 * (D(1, 5) - SS(5)) + j2 * i2 * (D(4, 6) - SS(5) / 2.0) +
             j3 * i3 * (D(3, 5) - SS(5)) + j2 * i3 * (D(4, 5) - SS(6) / 4.0) +
             j3 * i1 * (D(1, 3) - (SS(1) + SS(3)) / 4.0) + j1 * i2 * (D(5, 6) - SS(4) / 4.0) +
             i2 * j3 * (D(3, 6) - SS(6) / 4.0) + i3 * j1 * (D(5, 5) - (SS(1) + SS(3)) / 4.0) +
             i1 * j2 * (D(1, 4) - SS(4) / 4.0));
    gm[5] = (j1 * i1 * (D(5, 6) - SS(4) / 2.0) + j2 * i2 * (D(2, 4) - SS(4)) +
             j3 * i3 * (D(3, 4) - SS(4)) + j2 * i3 * (D(4, 4) - (SS(2) + SS(3)) / 4.0) +
             j3 * i1 * (D(3, 6) - SS(6) / 4.0) + j1 * i2 * (D(2, 5) - SS(5) / 4.0) +
             i2 * j3 * (D(2, 3) - (SS(2) + SS(3)) / 4.0) + i3 * j1 * (D(4, 5) - SS(6) / 4.0) +
             i1 * j2 * (D(4, 6) - SS(5) / 4.0));
    gm[8] = (i1 * j1 * (D(5, 5) - (SS(3) - SS(1)) / 2.0) +
             i2 * j2 * (D(4, 4) - (SS(3) - SS(2)) / 2.0) + i3 * j3 * (D(3, 3) - SS(3)) +
             i2 * j3 * (D(3, 4)) + i3 * j1 * (D(3, 5)) + i1 * j2 * (D(4, 5) + SS(6) / 2.0) +
             j2 * i3 * (D(3, 4)) + j3 * i1 * (D(3, 5)) + j1 * i2 * (D(4, 5) + SS(6) / 2.0));
#undef D
#undef SS
}

// Penalty boundary condition of one node (SUVALS, src/fasolt/Bconds.f90:40-109)
// applied to its diagonal block D (row-major 3x3) and right-hand side f.
__device__ __forceinline__ int apply_bc(int ibc, int n, const double *x, const double *dx,
                                        const double *xspec, const double *fspec, int nxs,
                                        int nfs, double efix, double D[9], double f[3])
{
    if (ibc < 100) return 0;
    const int ikin = (ibc / 100) % 100;
    if (ikin > 0) {
        if (ikin > nxs) return 1;
        const double *xs = xspec + (size_t)(ikin - 1) * 15;
        double xsp[3];
        if (ikin < 50) {
            xsp[0] = xs[6];
            xsp[1] = xs[10];
            xsp[2] = xs[14];
        } else {
#pragma unroll
            for (int j = 0; j < 3; ++j)
                xsp[j] = xs[6 + 3 * j] * (x[3 * n] + dx[3 * n]) +
                         xs[7 + 3 * j] * (x[3 * n + 1] + dx[3 * n + 1]) +
                         xs[8 + 3 * j] * (x[3 * n + 2] + dx[3 * n + 2]);
        }
        const int point[3][3] = {{0, 1, 3}, {1, 2, 4}, {3, 4, 5}};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            double sum = 0.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double pen = efix * xs[point[i][j]];
                D[3 * i + j] = D[3 * i + j] + pen;
                sum = sum + pen * (dx[3 * n + j] - xsp[j]);
            }
            f[i] = f[i] + sum;
        }
    }
    const int ispf = (ibc / 10000) % 100;
    if (ispf > 0) {
        if (ispf > nfs) return 1;
        const double *fs = fspec + (size_t)(ispf - 1) * 3;
#pragma unroll
        for (int i = 0; i < 3; ++i) f[i] = f[i] + fs[i];
    }
    return 0;
}

// Row-gather assembly: thread (slot, row) sums, in ascending element order
// (the reference's scatter order, Elvals.f90:244-262), w * gaussm over the
// elements that hold both the row node and the slot's column node, and
// writes the 3x3 block once -- no atomics, no read-modify-write of the
// matrix.  The diagonal-slot thread also forms the nodal force
// (Elvals.f90:122-126,265-271) and, when `bc` is set, applies SUVALS.
template <int NN, int NPG>
__global__ void __launch_bounds__(256) k_assemble(MeshDev Mh, BlockDev B,
                                                  const double *__restrict__ rec,
                                                  const double *__restrict__ x,
                                                  const double *__restrict__ dx, double *fc,
                                                  double *ddx, const double *xspec,
                                                  const double *fspec, int nxs, int nfs,
                                                  double efix, int bc, int *bad_bc)
{
    using L = RecLayout<NN>;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int p = (int)(tid / B.slots);
    const int s = (int)(tid - (long long)p * B.slots);
    if (p >= B.R) return;
    if (s >= B.nslot[p]) return;
    const int n = B.perm[p];
    const unsigned long long *bl = B.bloc + B.si(p, s) * B.nbw;
    const int cnt = Mh.ne_cnt[n];
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double f[3] = {0, 0, 0};
    for (int k = 0; k < cnt; ++k) {
        const int b = (int)((bl[k >> 3] >> (8 * (k & 7))) & 0xFFull);
        if (b == 0xFF) continue;
        const int e = Mh.ne_elem[k * Mh.nnod + n];
        const int a = Mh.ne_loc[k * Mh.nnod + n];
        const int itp = Mh.lt[e];
        if (itp < 9) {
            // tie element (Elvals.f90:62-77): +efix on the tied DOFs of its
            // first node and -efix towards the same DOFs of its second, in
            // the first node's rows only; no force
            if (a == 0) {
                const double v = b == 0 ? efix : -efix;
                if (itp <= 3) {
                    acc[(itp - 1) * 4] = acc[(itp - 1) * 4] + v;
                } else {
                    const int i1 = (itp - 3) % 3, i2 = (i1 + 1) % 3;   // 0-based DOFs
                    acc[i1 * 4] = acc[i1 * 4] + v;
                    acc[i2 * 4] = acc[i2 * 4] + v;
                }
            }
            continue;
        }
        // the element's contribution, summed over its GPs first
        // (Elvals.f90:82-236), is added to the block in element order
        double ae[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double fe[3] = {0, 0, 0};
        for (int g = 0; g < NPG; ++g) {
            const double *Rr = rec + ((size_t)e * NPG + g) * L::LEN;
            double sa[3], sb[3], st[6], d[21];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                sa[c] = __ldg(Rr + 3 * a + c);
                sb[c] = __ldg(Rr + 3 * b + c);
            }
#pragma unroll
            for (int c = 0; c < 6; ++c) st[c] = __ldg(Rr + L::S + c);
            const double w = __ldg(Rr + L::W);
#pragma unroll
            for (int c = 0; c < 21; ++c) d[c] = __ldg(Rr + L::D + c);
            double gm[9];
            gaussm_block(sa, sb, d, st, gm);
            double *ta = NPG == 1 ? acc : ae;
            double *tf = NPG == 1 ? f : fe;
#pragma unroll
            for (int q = 0; q < 9; ++q) ta[q] = ta[q] + w * gm[q];
            if (s == 0) {
                tf[0] = tf[0] + w * (st[0] * sa[0] + st[5] * sa[1] + st[4] * sa[2]);
                tf[1] = tf[1] + w * (st[1] * sa[1] + st[3] * sa[2] + st[5] * sa[0]);
                tf[2] = tf[2] + w * (st[2] * sa[2] + st[4] * sa[0] + st[3] * sa[1]);
            }
        }
        if (NPG > 1) {
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] = acc[q] + ae[q];
            if (s == 0)
#pragma unroll
                for (int c = 0; c < 3; ++c) f[c] = f[c] + fe[c];
        }
    }
    if (s == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) fc[3 * n + c] = f[c];
        if (bc) {
            if (apply_bc(Mh.ib[n], n, x, dx, xspec, fspec, nxs, nfs, efix, acc, f)) *bad_bc = 1;
#pragma unroll
            for (int c = 0; c < 3; ++c) ddx[3 * n + c] = f[c];
        }
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) B.blk[B.bi(p, s, q)] = acc[q];
    if (B.blk32) {
#pragma unroll
        for (int q = 0; q < 9; ++q) B.blk32[B.bi(p, s, q)] = (float)acc[q];
    }
}

// Stand-alone SUVALS (src/fasolt/Bconds.f90:19-113): ddx = fc, then the
// penalty terms of every constrained node.
__global__ void k_suvals(MeshDev Mh, BlockDev B, const int *rowof, const double *x,
                         const double *dx, const double *fc, double *ddx, const double *xspec,
                         const double *fspec, int nxs, int nfs, double efix, int *bad_bc)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Mh.nnod) return;
    double f[3] = {fc[3 * n], fc[3 * n + 1], fc[3 * n + 2]};
    const int ibc = Mh.ib[n];
    if (ibc >= 100) {
        const int p = rowof[n];
        double D[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) D[q] = B.blk[B.bi(p, 0, q)];
        if (apply_bc(ibc, n, x, dx, xspec, fspec, nxs, nfs, efix, D, f)) *bad_bc = 1;
#pragma unroll
        for (int q = 0; q < 9; ++q) B.blk[B.bi(p, 0, q)] = D[q];
        if (B.blk32) {
#pragma unroll
            for (int q = 0; q < 9; ++q) B.blk32[B.bi(p, 0, q)] = (float)D[q];
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) ddx[3 * n + c] = f[c];
}

// ---------------------------------------------------------------- reductions
// Deterministic block sum of NV values per thread; block b writes
// part[v * nblk + b].
template <int NV>
__device__ __forceinline__ void block_sum_store(double v[NV], double *part, int nblk)
{
    __shared__ double red[NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < nw ? red[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) part[k * nblk + blockIdx.x] = t;
        }
    }
}

// Single-block final sum of NV partial vectors of length nblk.
template <int NV>
__global__ void __launch_bounds__(1024) k_final_sum(const double *part, int nblk, double *out)
{
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (int i = threadIdx.x; i < nblk; i += blockDim.x) t += part[k * nblk + i];
        v[k] = t;
    }
    __shared__ double red[NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = lane < nw ? red[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (lane == 0) out[k] = t;
        }
    }
}

// NRITER's norms (src/fasolt/Stif_sol.f90:46-51,56-58,65): sum of rhs^2
// over nodes with ib < 10, |dx|^2, |ddx|^2, and the CPSTRS error sum.
__global__ void __launch_bounds__(256) k_nr_norms(int nnod, int ngps, const int *ib,
                                                  const double *rhs, const double *dx,
                                                  const double *ddx, const double *erepmd,
                                                  double *part, int nblk)
{
    double v[4] = {0, 0, 0, 0};
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nnod; i += stride) {
        const double a = rhs[3 * i], b = rhs[3 * i + 1], c = rhs[3 * i + 2];
        if (ib[i] < 10) v[0] += a * a + b * b + c * c;
        const double d0 = dx[3 * i], d1 = dx[3 * i + 1], d2 = dx[3 * i + 2];
        v[1] += d0 * d0 + d1 * d1 + d2 * d2;
        const double e0 = ddx[3 * i], e1 = ddx[3 * i + 1], e2 = ddx[3 * i + 2];
        v[2] += e0 * e0 + e1 * e1 + e2 * e2;
    }
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngps; g += stride) v[3] += erepmd[g];
    block_sum_store<4>(v, part, nblk);
}

// ---------------------------------------------------------------- SOR
// FACSLS (src/fasolt/Stif_sol.f90:161-215) in multicolour node order: one
// launch per colour; each thread updates the x, y, z DOFs of one node with
// point SOR (omega = 1.2) and adds its share of |dx_sweep|^2 and |x|^2.
struct SorCtl {
    int conv;       // set once error < toler^2
    int sweeps;     // sweeps actually performed
    double err;     // error of the last sweep
    int fault;      // a bounded wait gave up
    int pad;
};

// Operands of one row for one lane: the lane's 3x3 block (slot = lane), the
// solution at the slot's column node, and (lane 0) the right-hand side.
// Slot 0 is the row's own node, so lane 0 holds the diagonal block and the
// node's current values.
struct RowOps {
    int ns, n;
    double b[9];
    double x0, x1, x2;
    double r0, r1, r2;
};

// The matrix is streamed once per sweep and is larger than L2: its loads
// are marked evict-first (ld.global.cs) so the solution vector, re-read by
// every colour phase, stays resident in L2.
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const float *p) { return (double)__ldcs(p); }

template <typename T>
__device__ __forceinline__ void load_row(const BlockDev &B, const T *__restrict__ blk, int p, int lane,
                                         const double *__restrict__ rhs, const double *sol, RowOps &o)
{
    o.ns = B.nslot[p];
    const bool on = lane < o.ns;
    const int m = on ? __ldcs(B.bcol + B.si(p, lane)) : 0;
    o.n = __shfl_sync(0xffffffffu, m, 0);
#pragma unroll
    for (int q = 0; q < 9; ++q) o.b[q] = on ? ld_stream(blk + B.bi(p, lane, q)) : 0.0;
    o.x0 = on ? sol[3 * m] : 0.0;
    o.x1 = on ? sol[3 * m + 1] : 0.0;
    o.x2 = on ? sol[3 * m + 2] : 0.0;
    if (lane == 0) {
        o.r0 = rhs[3 * m];
        o.r1 = rhs[3 * m + 1];
        o.r2 = rhs[3 * m + 2];
    }
}

// The point-SOR update of one row (FACSLS's inner loop, Stif_sol.f90:189-197,
// for the three DOFs of one node) by one warp: lanes 1..nslot-1 multiply
// their off-diagonal block by the solution at the column node, the warp sums
// the products, and lane 0 updates x, y, z in turn with the diagonal block.
// Adds to dv / vv (lane 0) the squared change and the squared new values;
// `base` (may be null) is added to the iterate for the latter.
__device__ __forceinline__ void sor_update(const RowOps &o, int lane, double *sol,
                                           const double *__restrict__ base, double &dv, double &vv)
{
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if (lane >= 1) {
        a0 = o.b[0] * o.x0 + o.b[1] * o.x1 + o.b[2] * o.x2;
        a1 = o.b[3] * o.x0 + o.b[4] * o.x1 + o.b[5] * o.x2;
        a2 = o.b[6] * o.x0 + o.b[7] * o.x1 + o.b[8] * o.x2;
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, k);
        a1 += __shfl_xor_sync(0xffffffffu, a1, k);
        a2 += __shfl_xor_sync(0xffffffffu, a2, k);
    }
    if (lane == 0) {
        const double *D = o.b;
        const int n = o.n;
        double x0 = o.x0, x1 = o.x1, x2 = o.x2;
        double t = (o.r0 - (a0 + D[1] * x1 + D[2] * x2)) / D[0];
        x0 = x0 + 1.2 * (t - x0);
        t = (o.r1 - (a1 + D[3] * x0 + D[5] * x2)) / D[4];
        x1 = x1 + 1.2 * (t - x1);
        t = (o.r2 - (a2 + D[6] * x0 + D[7] * x1)) / D[8];
        x2 = x2 + 1.2 * (t - x2);
        sol[3 * n] = x0;
        sol[3 * n + 1] = x1;
        sol[3 * n + 2] = x2;
        dv += (x0 - o.x0) * (x0 - o.x0) + (x1 - o.x1) * (x1 - o.x1) + (x2 - o.x2) * (x2 - o.x2);
        if (base) {
            x0 += base[3 * n];
            x1 += base[3 * n + 1];
            x2 += base[3 * n + 2];
        }
        vv += x0 * x0 + x1 * x1 + x2 * x2;
    }
}

// Rows p, p + stride, ... < p1 of one colour by one warp, with the next
// row's operands loaded while the current row is reduced and updated.
// Within a colour no row reads a value another row of the colour writes
// (same-colour nodes share no element), so the early loads see final values.
template <typename T>
__device__ __forceinline__ void sor_rows(const BlockDev &B, const T *__restrict__ blk, int p, int p1,
                                         int stride, int lane, const double *__restrict__ rhs,
                                         double *sol, const double *__restrict__ base, double &dv,
                                         double &vv)
{
    if (p >= p1) return;
    RowOps cur, nxt;
    load_row<T>(B, blk, p, lane, rhs, sol, cur);
    while (true) {
        const int pn = p + stride;
        const bool more = pn < p1;
        if (more) load_row<T>(B, blk, pn, lane, rhs, sol, nxt);
        sor_update(cur, lane, sol, base, dv, vv);
        if (!more) break;
        cur = nxt;
        p = pn;
    }
}

// The same warp-per-row update for rows of more than 32 slots: lane l holds
// slots l, l + 32, ... (K per lane); lane 0's first slot is the diagonal.
template <int K> struct RowOpsK {
    int ns, n;
    double b[K][9];
    double x0[K], x1[K], x2[K];
    double r0, r1, r2;
};

template <typename T, int K>
__device__ __forceinline__ void load_row_k(const BlockDev &B, const T *__restrict__ blk, int p, int lane,
                                           const double *__restrict__ rhs, const double *sol, RowOpsK<K> &o)
{
    o.ns = B.nslot[p];
    int m0 = 0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int sl = lane + 32 * k;
        const bool on = sl < o.ns;
        const int m = on ? __ldcs(B.bcol + B.si(p, sl)) : 0;
        if (k == 0) m0 = m;
#pragma unroll
        for (int q = 0; q < 9; ++q) o.b[k][q] = on ? ld_stream(blk + B.bi(p, sl, q)) : 0.0;
        o.x0[k] = on ? sol[3 * m] : 0.0;
        o.x1[k] = on ? sol[3 * m + 1] : 0.0;
        o.x2[k] = on ? sol[3 * m + 2] : 0.0;
    }
    o.n = __shfl_sync(0xffffffffu, m0, 0);
    if (lane == 0) {
        o.r0 = rhs[3 * m0];
        o.r1 = rhs[3 * m0 + 1];
        o.r2 = rhs[3 * m0 + 2];
    }
}

template <int K>
__device__ __forceinline__ void sor_update_k(const RowOpsK<K> &o, int lane, double *sol,
                                             const double *__restrict__ base, double &dv, double &vv)
{
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        if (lane + 32 * k >= 1) {
            a0 += o.b[k][0] * o.x0[k] + o.b[k][1] * o.x1[k] + o.b[k][2] * o.x2[k];
            a1 += o.b[k][3] * o.x0[k] + o.b[k][4] * o.x1[k] + o.b[k][5] * o.x2[k];
            a2 += o.b[k][6] * o.x0[k] + o.b[k][7] * o.x1[k] + o.b[k][8] * o.x2[k];
        }
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, k);
        a1 += __shfl_xor_sync(0xffffffffu, a1, k);
        a2 += __shfl_xor_sync(0xffffffffu, a2, k);
    }
    if (lane == 0) {
        const double *D = o.b[0];
        const int n = o.n;
        double x0 = o.x0[0], x1 = o.x1[0], x2 = o.x2[0];
        double t = (o.r0 - (a0 + D[1] * x1 + D[2] * x2)) / D[0];
        x0 = x0 + 1.2 * (t - x0);
        t = (o.r1 - (a1 + D[3] * x0 + D[5] * x2)) / D[4];
        x1 = x1 + 1.2 * (t - x1);
        t = (o.r2 - (a2 + D[6] * x0 + D[7] * x1)) / D[8];
        x2 = x2 + 1.2 * (t - x2);
        sol[3 * n] = x0;
        sol[3 * n + 1] = x1;
        sol[3 * n + 2] = x2;
        dv += (x0 - o.x0[0]) * (x0 - o.x0[0]) + (x1 - o.x1[0]) * (x1 - o.x1[0]) + (x2 - o.x2[0]) * (x2 - o.x2[0]);
        if (base) {
            x0 += base[3 * n];
            x1 += base[3 * n + 1];
            x2 += base[3 * n + 2];
        }
        vv += x0 * x0 + x1 * x1 + x2 * x2;
    }
}

template <typename T, int K>
__device__ __forceinline__ void sor_rows_k(const BlockDev &B, const T *__restrict__ blk, int p, int p1,
                                           int stride, int lane, const double *__restrict__ rhs,
                                           double *sol, const double *__restrict__ base, double &dv,
                                           double &vv)
{
    for (; p < p1; p += stride) {
        RowOpsK<K> o;
        load_row_k<T, K>(B, blk, p, lane, rhs, sol, o);
        sor_update_k<K>(o, lane, sol, base, dv, vv);
    }
}

// ---------------------------------------------------------------- bulk-copy SOR
// Shared-memory staging of block rows with the bulk-copy (TMA) engine:
// cp.async.bulk global -> shared, completion counted on an mbarrier.
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// L2 cache policies: the streamed matrix is evict-first, the solution
// vector gathered by every colour phase evict-last.
__device__ __forceinline__ uint64_t l2_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ double ld_keep(const double *ptr, uint64_t pol)
{
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar,
                                         uint64_t pol)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, "
        "[%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up (returns false) after 2^22 polls instead of
// spinning for ever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    for (int i = 0; i < (1 << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while the previous kernel of the stream drains.
// pdl_wait() returns once that kernel has completed and its writes are
// visible; before it, only data the previous kernel does not write may be
// touched.  Under an ordinary launch both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// End of one sweep, by one whole block: error = sum(dx^2) / sum(x^2) over
// the per-CTA partials of every colour (Stif_sol.f90:206-210).
__device__ __forceinline__ void sweep_test(const double *part, int nblk, SorCtl *ctl, double tolerl)
{
    double v[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        v[0] += part[i];
        v[1] += part[nblk + i];
    }
    __shared__ double red[2][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        double t = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) red[k][wid] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double a = 0.0, b = 0.0;
        for (int i = 0; i < nw; ++i) {
            a += red[0][i];
            b += red[1][i];
        }
        const double err = a / b;
        ctl->err = err;
        ctl->sweeps += 1;
        if (err < tolerl) ctl->conv = 1;
    }
}

// Launch shape of the colour kernel (compile-time; -D overrides for tuning).
#ifndef FAS_TMA_ROWS
#define FAS_TMA_ROWS 8
#endif
#ifndef FAS_TMA_LPR
#define FAS_TMA_LPR 4
#endif
#ifndef FAS_TMA_STAGES
#define FAS_TMA_STAGES 2
#endif
#ifndef FAS_TMA_PD
#define FAS_TMA_PD 1
#endif
constexpr int TMA_ROWS = FAS_TMA_ROWS;       // rows per chunk
constexpr int TMA_LPR = FAS_TMA_LPR;         // lanes per row of 27-slot rows (a power of two, at most 32)
#ifndef FAS_TMA_LPR81
#define FAS_TMA_LPR81 16
#endif
#ifndef FAS_TMA_ROWS81
#define FAS_TMA_ROWS81 4
#endif
constexpr int TMA_LPR81 = FAS_TMA_LPR81;     // lanes per row of 81-slot rows
constexpr int TMA_ROWS81 = FAS_TMA_ROWS81;   // rows per chunk of 81-slot rows
// The FP32-matrix sweeps of the tuned form have their own shape: their rings
// are half as large, so the same shared memory holds twice the rows in
// flight, and the shape that hides the consumer's latency differs.
#ifndef FAS_TMA_ROWS32
#define FAS_TMA_ROWS32 24
#endif
#ifndef FAS_TMA_LPR32
#define FAS_TMA_LPR32 4
#endif
#ifndef FAS_TMA_MINB32
#define FAS_TMA_MINB32 1
#endif
// 1: the FP32 colour kernel multiplies and sums a lane's blocks in FP32
// (the correction rounded to FP32 at the product, the lanes' sums and the
// point update in FP64): 103.7 against 110.1 us per 64^3 sweep, the same
// sweep counts, per-point stresses 1.5e-10 from the plain path at 16^3
#ifndef FAS_SOR32_ARITH
#define FAS_SOR32_ARITH 1
#endif
// and so have the FP32 sweeps of 81-slot rows
#ifndef FAS_TMA_ROWS81_32
#define FAS_TMA_ROWS81_32 16
#endif
#ifndef FAS_TMA_LPR81_32
#define FAS_TMA_LPR81_32 8
#endif
constexpr int TMA_ROWS81_32 = FAS_TMA_ROWS81_32;   // rows per chunk of FP32 81-slot rows
constexpr int TMA_LPR81_32 = FAS_TMA_LPR81_32;     // lanes per row of FP32 81-slot rows
// Symmetric FP32 rows (FAS_MODE_SOR_SYM) of 8-node meshes: the stiffness
// matrix is symmetric (K_mn = K_nm^T: symmetric element tangents, penalty
// terms on diagonal blocks only), so each off-diagonal block is stored once,
// in the row of one of its two nodes.  A row holds its diagonal block and at
// most SLOTS_SYM - 1 stored blocks (13 on the interior of a brick mesh):
// 608 bytes of FP32 values and column ids against 1,088 for full FP32 rows.
// 15 slots make a row 136 values long, 8 banks apart in shared memory, so
// the four rows a warp serves with 8 lanes each read without bank conflicts
// (14 slots, 128 values, put all four rows on the same banks).
constexpr int SLOTS_SYM = 15;
#ifndef FAS_TMA_ROWS_SYM
#define FAS_TMA_ROWS_SYM 16
#endif
#ifndef FAS_TMA_LPR_SYM
#define FAS_TMA_LPR_SYM 8   // us per 64^3 sweep: 16 x 8 121.6, 16 x 4 125.3, 32 x 8 125.9, 32 x 4 126.3
#endif
constexpr int TMA_ROWS_SYM = FAS_TMA_ROWS_SYM;   // rows per chunk of symmetric rows
constexpr int TMA_LPR_SYM = FAS_TMA_LPR_SYM;     // lanes per row of symmetric rows
static_assert(TMA_ROWS_SYM * TMA_LPR_SYM % 32 == 0 && (TMA_LPR_SYM & (TMA_LPR_SYM - 1)) == 0 &&
                  TMA_LPR_SYM <= 32,
              "whole warps per CTA");
constexpr int TMA_ROWS32 = FAS_TMA_ROWS32;   // rows per chunk of FP32 27-slot rows
constexpr int TMA_LPR32 = FAS_TMA_LPR32;     // lanes per row of FP32 27-slot rows
constexpr int TMA_MINB32 = FAS_TMA_MINB32;   // CTAs per SM the FP32 kernel's registers must allow
constexpr int TMA_STAGES = FAS_TMA_STAGES;   // chunks in flight per CTA
constexpr int TMA_PD = FAS_TMA_PD;           // chunks whose gathers run ahead of the computed one
static_assert(TMA_PD >= 1 && TMA_PD < TMA_STAGES, "gathers run ahead within the ring");
template <int LPR, int ROWS = TMA_ROWS> __host__ __device__ constexpr int tma_threads() { return ROWS * LPR; }
constexpr int TMA_THREADS = tma_threads<TMA_LPR>();
static_assert(TMA_LPR >= 1 && TMA_LPR <= 32 && (TMA_LPR & (TMA_LPR - 1)) == 0, "lanes per row");
static_assert(TMA_THREADS % 32 == 0 && tma_threads<TMA_LPR81, TMA_ROWS81>() % 32 == 0, "whole warps per CTA");

// rows per chunk of the S-slot layout in value type T
template <int S, typename T = double> __host__ __device__ constexpr int tma_rows()
{
    return S == SLOTS_SYM ? TMA_ROWS_SYM
           : S == SLOTS   ? (sizeof(T) == 4 ? TMA_ROWS32 : TMA_ROWS)
                          : (sizeof(T) == 4 ? TMA_ROWS81_32 : TMA_ROWS81);
}
// lanes per row of the S-slot layout in value type T
template <int S, typename T = double> __host__ __device__ constexpr int tma_lpr()
{
    return S == SLOTS_SYM ? TMA_LPR_SYM
           : S == SLOTS   ? (sizeof(T) == 4 ? TMA_LPR32 : TMA_LPR)
                          : (sizeof(T) == 4 ? TMA_LPR81_32 : TMA_LPR81);
}
static_assert(tma_threads<TMA_LPR81_32, TMA_ROWS81_32>() % 32 == 0 && (TMA_LPR81_32 & (TMA_LPR81_32 - 1)) == 0 &&
                  TMA_LPR81_32 <= 32,
              "whole warps per CTA");
// minimum CTAs per SM the kernel's register budget must allow (1: no bound)
template <int S, typename T> __host__ __device__ constexpr int tma_minb()
{
    return S == SLOTS && sizeof(T) == 4 ? TMA_MINB32 : 1;
}
static_assert(tma_threads<TMA_LPR32, TMA_ROWS32>() % 32 == 0 && (TMA_LPR32 & (TMA_LPR32 - 1)) == 0,
              "whole warps per CTA");
template <typename T, int S = SLOTS> __host__ __device__ constexpr int tma_stage_bytes()
{
    return tma_rows<S, T>() * brow_of(S) * (int)sizeof(T) + tma_rows<S, T>() * crow_of(S) * 4;
}
// the ring, its mbarriers and a 512-byte guard: lanes whose slots lie past
// the row (q + LPR j >= S) skip their reads, and the guard keeps even a
// speculated shared-memory read of the last row inside the allocation
template <typename T, int S = SLOTS> __host__ __device__ constexpr int tma_smem_bytes()
{
    return TMA_STAGES * tma_stage_bytes<T, S>() + TMA_STAGES * 8 + 512;
}
// CTAs of the FP64 kernel that fit on one SM (228 KB of shared memory,
// 1 KB of it reserved per CTA, at most 32 warps); the colour grid is sized
// to fill them.
template <int S, int LPR, typename T = double> __host__ __device__ constexpr int tma_ctas_per_sm()
{
    return (228 * 1024) / (tma_smem_bytes<T, S>() + 1024) < 32 / (tma_threads<LPR, tma_rows<S, T>()>() / 32)
               ? (228 * 1024) / (tma_smem_bytes<T, S>() + 1024)
               : 32 / (tma_threads<LPR, tma_rows<S, T>()>() / 32);
}
constexpr int TMA_CTAS_PER_SM = tma_ctas_per_sm<SLOTS, TMA_LPR>();
static_assert(TMA_CTAS_PER_SM >= 1 && tma_ctas_per_sm<SLOTS20, TMA_LPR81>() >= 1,
              "the ring must fit in shared memory");

// Operands of one chunk row for one lane, gathered before its point
// update: the solution at the lane's slots (x0, x1, x2) and, on the row's
// first lane, the right-hand side and reciprocal diagonal of the row's node (r).
template <int SPL, typename XT = double> struct SorOps {
    XT x0[SPL], x1[SPL], x2[SPL];
    double r[6];
};
// The FP32 sweeps' form: the slots' values from the FP32 mirror of the
// correction (exactly the values the FP32 products round them to), and the
// row node's own old values in FP64 for the point update.
// Symmetric rows add the row node's accumulated transposed products (acc).
template <int SPL> struct SorOps<SPL, float> {
    float x0[SPL], x1[SPL], x2[SPL];
    double r[6], own[3];
    float acc[3];
};

__device__ __forceinline__ float ld_keep_f32(const float *ptr, uint64_t pol)
{
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(ptr), "l"(pol));
    return v;
}
__device__ __forceinline__ float4 ld_keep_f32x4(const float *ptr, uint64_t pol)
{
    float4 v;
    asm volatile("ld.global.cg.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(ptr), "l"(pol));
    return v;
}

// Gather of lane q of chunk row `row` from a landed stage's column ids.
// r0 is the chunk's first row and nrow its row count.
// With SYM (symmetric rows) the row's first lane also reads the row node's
// accumulated transposed products acc[4 n .. 4 n + 2].
template <int S, int LPR, typename XT = double, bool SYM = false>
__device__ __forceinline__ void sor_gather(const int *stage_cols, int r0, int nrow, int row, int q,
                                           const double *sol, const double *__restrict__ rhs,
                                           const double *__restrict__ rdiag, uint64_t keep_pol,
                                           SorOps<(S + LPR - 1) / LPR, XT> &g, const float *sol32 = nullptr,
                                           const float *acc = nullptr)
{
    constexpr int SPL = (S + LPR - 1) / LPR, CR = crow_of(S);
    const bool live = row < nrow;
    const int *cols = stage_cols + (live ? row : 0) * CR;
    const int ns = live ? cols[S] : 0;
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
        const int sl = q + LPR * j;
        const bool on = sl < ns;
        const int m = on ? cols[sl] : 0;
        if constexpr (sizeof(XT) == 4) {
            g.x0[j] = on ? ld_keep_f32(sol32 + 3 * m, keep_pol) : 0.f;
            g.x1[j] = on ? ld_keep_f32(sol32 + 3 * m + 1, keep_pol) : 0.f;
            g.x2[j] = on ? ld_keep_f32(sol32 + 3 * m + 2, keep_pol) : 0.f;
        } else {
            g.x0[j] = on ? ld_keep(sol + 3 * m, keep_pol) : 0.0;
            g.x1[j] = on ? ld_keep(sol + 3 * m + 1, keep_pol) : 0.0;
            g.x2[j] = on ? ld_keep(sol + 3 * m + 2, keep_pol) : 0.0;
        }
    }
    const bool own = live && q == 0;
    const int n = cols[0];
    if constexpr (sizeof(XT) == 4) {
        g.own[0] = own ? ld_keep(sol + 3 * n, keep_pol) : 0.0;
        g.own[1] = own ? ld_keep(sol + 3 * n + 1, keep_pol) : 0.0;
        g.own[2] = own ? ld_keep(sol + 3 * n + 2, keep_pol) : 0.0;
        if constexpr (SYM) {
            const float4 a = own ? ld_keep_f32x4(acc + 4 * (size_t)n, keep_pol) : make_float4(0.f, 0.f, 0.f, 0.f);
            g.acc[0] = a.x;
            g.acc[1] = a.y;
            g.acc[2] = a.z;
        }
    } else {
        static_assert(!SYM, "symmetric rows are FP32 rows with FP32 gathers");
    }
    g.r[0] = own ? ld_keep(rhs + 3 * n, keep_pol) : 0.0;
    g.r[1] = own ? ld_keep(rhs + 3 * n + 1, keep_pol) : 0.0;
    g.r[2] = own ? ld_keep(rhs + 3 * n + 2, keep_pol) : 0.0;
    if (rdiag) {
        const double *rd = rdiag + 3 * (size_t)(own ? r0 + row : r0);
        g.r[3] = own ? rd[0] : 0.0;
        g.r[4] = own ? rd[1] : 0.0;
        g.r[5] = own ? rd[2] : 0.0;
    }
}

// Point update of chunk row `row` from a landed stage and its gathered
// operands: lane q multiplies the blocks of slots q, q+LPR, ... (slot 0,
// the diagonal, excluded), the LPR lanes of the row sum their products, and
// the first lane updates x, y and z in turn (omega = 1.2), stores them and
// adds |x_new - x_old|^2 to v0 and |x_new + base|^2 to v1.  With `rcp` the
// quotients come from the gathered reciprocal diagonal.
// With FP32 gathers (XT = float) the row's own old values come from g.own,
// and the new values also go, rounded, to the mirror sol32.
// With SYM (symmetric rows) the row's sum also takes the accumulated
// transposed products g.acc, and after the point update every lane pushes,
// for each stored block K_nm of its slots, K_nm^T (x32_new - x32_old) of
// the row node n into acc[4 m ..] of the column node m (one vector atomic
// add per block): acc[4 m ..] then always holds the products of the blocks
// stored in other rows with the current FP32 correction.
template <typename T, int S, int LPR, int ROWS, typename XT = double, bool SYM = false>
__device__ __forceinline__ void sor_update(const unsigned char *stage, int nrow, int row, int q,
                                           const SorOps<(S + LPR - 1) / LPR, XT> &g, bool rcp,
                                           const double *__restrict__ base, double *sol, double &v0,
                                           double &v1, float *sol32 = nullptr, float *acc = nullptr)
{
    static_assert(sizeof(XT) == 8 || (sizeof(T) == 4 && FAS_SOR32_ARITH), "FP32 gathers feed FP32 products only");
    constexpr int SPL = (S + LPR - 1) / LPR, BR = brow_of(S), CR = crow_of(S);
    constexpr int VB = ROWS * BR * (int)sizeof(T);
    const bool live = row < nrow;
    const T *vals = reinterpret_cast<const T *>(stage) + (live ? row : 0) * BR;
    const int *cols = reinterpret_cast<const int *>(stage + VB) + (live ? row : 0) * CR;
    const int ns = live ? cols[S] : 0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    // symmetric rows keep the lane's blocks in registers for the push
    float kb[SYM ? SPL : 1][9];
    if constexpr (sizeof(T) == 4 && FAS_SOR32_ARITH) {
        // FP32 products and lane sums of the FP32 blocks with the rounded
        // correction; the lanes' sums join in FP64
        float f0 = 0.f, f1 = 0.f, f2 = 0.f;
#pragma unroll
        for (int j = 0; j < SPL; ++j) {
            const int sl = q + LPR * j;
            if constexpr (SYM) {
#pragma unroll
                for (int qq = 0; qq < 9; ++qq) kb[j][qq] = (sl >= 1 && sl < ns) ? vals[sl + qq * S] : 0.f;
                const float y0 = g.x0[j], y1 = g.x1[j], y2 = g.x2[j];
                f0 += kb[j][0] * y0 + kb[j][1] * y1 + kb[j][2] * y2;
                f1 += kb[j][3] * y0 + kb[j][4] * y1 + kb[j][5] * y2;
                f2 += kb[j][6] * y0 + kb[j][7] * y1 + kb[j][8] * y2;
            } else if (sl >= 1 && sl < ns) {
                const T *b = vals + sl;
                const float y0 = (float)g.x0[j], y1 = (float)g.x1[j], y2 = (float)g.x2[j];
                f0 += b[0 * S] * y0 + b[1 * S] * y1 + b[2 * S] * y2;
                f1 += b[3 * S] * y0 + b[4 * S] * y1 + b[5 * S] * y2;
                f2 += b[6 * S] * y0 + b[7 * S] * y1 + b[8 * S] * y2;
            }
        }
        a0 = f0;
        a1 = f1;
        a2 = f2;
    } else {
#pragma unroll
        for (int j = 0; j < SPL; ++j) {
            const int sl = q + LPR * j;
            if (sl >= 1 && sl < ns) {
                const T *b = vals + sl;
                a0 += (double)b[0 * S] * g.x0[j] + (double)b[1 * S] * g.x1[j] + (double)b[2 * S] * g.x2[j];
                a1 += (double)b[3 * S] * g.x0[j] + (double)b[4 * S] * g.x1[j] + (double)b[5 * S] * g.x2[j];
                a2 += (double)b[6 * S] * g.x0[j] + (double)b[7 * S] * g.x1[j] + (double)b[8 * S] * g.x2[j];
            }
        }
    }
#pragma unroll
    for (int o = 1; o < LPR; o <<= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    float e0 = 0.f, e1 = 0.f, e2 = 0.f;   // the FP32 change of the row node (SYM)
    if (live && q == 0) {
        const int n = cols[0];
        if constexpr (SYM) {
            a0 += (double)g.acc[0];
            a1 += (double)g.acc[1];
            a2 += (double)g.acc[2];
        }
        double D[9];
#pragma unroll
        for (int qq = 0; qq < 9; ++qq) D[qq] = (double)vals[qq * S];
        double o0, o1, o2;
        if constexpr (sizeof(XT) == 4) {
            o0 = g.own[0];
            o1 = g.own[1];
            o2 = g.own[2];
        } else {
            o0 = g.x0[0];
            o1 = g.x1[0];
            o2 = g.x2[0];
        }
        double x0 = o0, x1 = o1, x2 = o2;
        double t;
        if (rcp) {
            // num / D from the correctly rounded reciprocal of D: with
            // q0 = num * (1/D) and the exact remainder e = num - q0 * D
            // (one FMA), q0 + e * (1/D) rounds to the correctly rounded
            // quotient (Markstein, IBM J. Res. Dev. 34 (1990) 111-119).
            const double i0 = g.r[3], i1 = g.r[4], i2 = g.r[5];
            double nm = g.r[0] - (a0 + D[1] * x1 + D[2] * x2);
            double q0 = nm * i0;
            t = fma(fma(-q0, D[0], nm), i0, q0);
            x0 = x0 + 1.2 * (t - x0);
            nm = g.r[1] - (a1 + D[3] * x0 + D[5] * x2);
            q0 = nm * i1;
            t = fma(fma(-q0, D[4], nm), i1, q0);
            x1 = x1 + 1.2 * (t - x1);
            nm = g.r[2] - (a2 + D[6] * x0 + D[7] * x1);
            q0 = nm * i2;
            t = fma(fma(-q0, D[8], nm), i2, q0);
            x2 = x2 + 1.2 * (t - x2);
        } else {
            t = (g.r[0] - (a0 + D[1] * x1 + D[2] * x2)) / D[0];
            x0 = x0 + 1.2 * (t - x0);
            t = (g.r[1] - (a1 + D[3] * x0 + D[5] * x2)) / D[4];
            x1 = x1 + 1.2 * (t - x1);
            t = (g.r[2] - (a2 + D[6] * x0 + D[7] * x1)) / D[8];
            x2 = x2 + 1.2 * (t - x2);
        }
        sol[3 * n] = x0;
        sol[3 * n + 1] = x1;
        sol[3 * n + 2] = x2;
        if constexpr (sizeof(XT) == 4) {
            sol32[3 * n] = (float)x0;
            sol32[3 * n + 1] = (float)x1;
            sol32[3 * n + 2] = (float)x2;
            if constexpr (SYM) {   // the mirror held (float) of the old value
                e0 = (float)x0 - (float)o0;
                e1 = (float)x1 - (float)o1;
                e2 = (float)x2 - (float)o2;
            }
        }
        v0 += (x0 - o0) * (x0 - o0) + (x1 - o1) * (x1 - o1) + (x2 - o2) * (x2 - o2);
        if (base) {
            x0 += base[3 * n];
            x1 += base[3 * n + 1];
            x2 += base[3 * n + 2];
        }
        v1 += x0 * x0 + x1 * x1 + x2 * x2;
    }
    if constexpr (SYM) {
        const int lead = (int)(threadIdx.x & 31u) & ~(LPR - 1);
        e0 = __shfl_sync(0xffffffffu, e0, lead);
        e1 = __shfl_sync(0xffffffffu, e1, lead);
        e2 = __shfl_sync(0xffffffffu, e2, lead);
        if (e0 != 0.f || e1 != 0.f || e2 != 0.f) {
#pragma unroll
            for (int j = 0; j < SPL; ++j) {
                const int sl = q + LPR * j;
                if (sl >= 1 && sl < ns) {
                    const float *b = kb[j];
                    const float t0 = b[0] * e0 + b[3] * e1 + b[6] * e2;
                    const float t1 = b[1] * e0 + b[4] * e1 + b[7] * e2;
                    const float t2 = b[2] * e0 + b[5] * e1 + b[8] * e2;
                    atomicAdd(reinterpret_cast<float4 *>(acc + 4 * (size_t)cols[sl]), make_float4(t0, t1, t2, 0.f));
                }
            }
        }
    }
}

// One colour phase of SOR with the colour's block rows streamed through a
// TMA_STAGES-deep shared-memory ring by the bulk-copy engine (evict-first in
// L2).  CTA b takes chunks b, b + grid, ... of TMA_ROWS consecutive rows;
// thread 0 issues the copies (values and column ids) and re-arms a stage
// once every row of it is done.  TMA_LPR lanes serve one row: lane q of the
// row's group multiplies the blocks of slots q, q+LPR, ... by the solution
// at their column nodes (gathered with evict-last so the vector stays in
// L2), the group sums its three partial products, and its first lane does the
// x, y, z point update with the diagonal block (slot 0).  Within a colour
// no row reads a value another row of the colour writes, so the gathers of
// chunk k+1 (and its right-hand side) are issued before chunk k is
// computed: one L2 round trip per chunk is hidden.  Every mbarrier
// wait is bounded; on a timeout the CTA waits (bounded) for its own copies
// still in flight, raises ctl->fault and leaves.
//
// With SYM the rows are symmetric FP32 rows (SLOTS_SYM slots: the diagonal
// and the blocks stored in this row) and acc holds, per node, the products
// of the blocks stored in other rows with the current FP32 correction
// (sor_update).  The rows of a colour push only into nodes of other
// colours, so no row of a phase reads an accumulator the phase writes.
template <typename T, int S, int LPR, bool SYM = false>
__global__ void __launch_bounds__(tma_rows<S, T>() * LPR, tma_minb<S, T>()) k_sor_colour_tma(const T *__restrict__ blk,
                                                                const int *__restrict__ bcol, int p0, int p1,
                                                                const double *__restrict__ rhs, double *sol,
                                                                const double *__restrict__ base,
                                                                const double *__restrict__ rdiag, SorCtl *ctl,
                                                                double *part, int boff, int nblk_tot,
                                                                float *sol32, float *acc)
{
    static_assert(!SYM || (S == SLOTS_SYM && sizeof(T) == 4 && FAS_SOR32_ARITH), "symmetric rows: FP32 products");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_pre, s_post;
    constexpr int BR = brow_of(S), CR = crow_of(S);
    // FP32 sweeps with FP32 products gather from the correction's FP32
    // mirror sol32 (kept equal to the correction rounded to FP32)
    using XT = std::conditional_t<sizeof(T) == 4 && FAS_SOR32_ARITH, float, double>;
    static_assert((BR * sizeof(T)) % 16 == 0 && (CR * 4) % 16 == 0, "bulk copies move 16-byte multiples");
    constexpr int SPL = (S + LPR - 1) / LPR;   // slots per lane
    constexpr int ROWS = tma_rows<S, T>();
    constexpr int VB = ROWS * BR * (int)sizeof(T);
    constexpr int SB = tma_stage_bytes<T, S>();
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + TMA_STAGES * SB);
    const int lane = threadIdx.x & 31;
    const int row = threadIdx.x / LPR;   // row of the chunk served by this group
    const int q = threadIdx.x % LPR;     // lane within the group
    const int nchunks = (p1 - p0 + ROWS - 1) / ROWS;
    const int myn = (int)blockIdx.x < nchunks ? (nchunks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const uint64_t stream_pol = l2_evict_first();
    const uint64_t keep_pol = l2_evict_last();
    auto issue = [&](int k) {
        const int c = blockIdx.x + k * gridDim.x;
        const int r0 = p0 + c * ROWS;
        const int nr = min(ROWS, p1 - r0);
        unsigned char *st = smem + (k % TMA_STAGES) * SB;
        const unsigned bv = (unsigned)(nr * BR * sizeof(T)), bc = (unsigned)(nr * CR * 4);
        mbar_expect_tx(&bars[k % TMA_STAGES], bv + bc);
        bulk_g2s(st, blk + (size_t)r0 * BR, bv, &bars[k % TMA_STAGES], stream_pol);
        bulk_g2s(st + VB, bcol + (size_t)r0 * CR, bc, &bars[k % TMA_STAGES], stream_pol);
    };
    // Prologue, overlapped with the previous kernel under a programmatic
    // launch.  The stopping flag only goes from 0 to 1 within a solve, so a
    // flag already set here is final and nothing is copied; the blocks and
    // column ids do not change during a solve, so their first copies may
    // start before the previous kernel has finished.
    if (threadIdx.x == 0) {
        for (int st = 0; st < TMA_STAGES; ++st) mbar_init(&bars[st], 1);
        mbar_fence_init();
        s_pre = ((volatile const SorCtl *)ctl)->conv;
        if (!s_pre)
            for (int k = 0; k < min(TMA_STAGES, myn); ++k) issue(k);
    }
    __syncthreads();
    pdl_launch_dependents();
    if (s_pre) return;
    pdl_wait();   // the previous colour's solution values and the flag are visible from here
    if (threadIdx.x == 0) s_post = ((volatile const SorCtl *)ctl)->conv;
    __syncthreads();
    if (s_post) {
        if (threadIdx.x == 0)   // the copies must land before the CTA's shared memory is released
            for (int k = 0; k < min(TMA_STAGES, myn); ++k) mbar_wait_bounded(&bars[k], 0u);
        return;
    }
    double v0 = 0.0, v1 = 0.0;
    // Gathered operands: set 0 belongs to the chunk being computed, set j
    // to chunk k + j.  No row of a colour reads a value written by another
    // row of the same colour, so the gathers of the next TMA_PD chunks are
    // in flight while chunk k is computed.
    SorOps<SPL, XT> g[TMA_PD + 1] = {};
    auto gather = [&](int kk, SorOps<SPL, XT> &o) {
        const int r0 = p0 + (blockIdx.x + kk * gridDim.x) * ROWS;
        sor_gather<S, LPR, XT, SYM>(reinterpret_cast<const int *>(smem + (kk % TMA_STAGES) * SB + VB), r0,
                                    min(ROWS, p1 - r0), row, q, sol, rhs, rdiag, keep_pol, o, sol32, acc);
    };
    // chunks [0, waited) have landed; chunks [0, min(myn, k + TMA_STAGES))
    // have been issued when iteration k starts
    int waited = 0, k = 0;
    bool fault = false;
#pragma unroll
    for (int i = 0; i < TMA_PD; ++i) {
        if (!fault && i < myn) {
            if (__syncthreads_and(mbar_wait_bounded(&bars[i], 0u) ? 1 : 0)) {
                waited = i + 1;
                gather(i, g[i]);
            } else {
                fault = true;
            }
        }
    }
    for (; !fault && k < myn; ++k) {
        if (k + TMA_PD < myn) {
            const int kk = k + TMA_PD;
            const unsigned par = (unsigned)((kk / TMA_STAGES) & 1);
            if (!__syncthreads_and(mbar_wait_bounded(&bars[kk % TMA_STAGES], par) ? 1 : 0)) {
                fault = true;
                break;
            }
            waited = kk + 1;
            gather(kk, g[TMA_PD]);
        }
        const int st = k % TMA_STAGES;
        const int nrow = min(ROWS, p1 - (p0 + (int)(blockIdx.x + k * gridDim.x) * ROWS));
        sor_update<T, S, LPR, ROWS, XT, SYM>(smem + st * SB, nrow, row, q, g[0], rdiag != nullptr, base, sol, v0,
                                             v1, sol32, acc);
        __syncthreads();   // every row of this stage is done
        if (threadIdx.x == 0 && k + TMA_STAGES < myn) {
            fence_proxy_async();
            issue(k + TMA_STAGES);
        }
#pragma unroll
        for (int i = 0; i < TMA_PD; ++i) g[i] = g[i + 1];
    }
    (void)lane;
    if (fault) {
        if (threadIdx.x == 0) {
            // copies issued and not yet seen to land may still write the ring
            for (int j = waited; j < min(myn, k + TMA_STAGES); ++j)
                mbar_wait_bounded(&bars[j % TMA_STAGES], (unsigned)((j / TMA_STAGES) & 1));
            atomicExch(&ctl->fault, 1);
        }
        return;
    }
    double v[2] = {v0, v1};
    block_sum_store<2>(v, part + boff, nblk_tot);
}

// Whole FACSLS solve in one CTA for small meshes: the same warp-per-row
// point update as k_sor_colour_tma, colours separated by __syncthreads, and the
// stopping test (Stif_sol.f90:206-210) evaluated in-block after every sweep.
// Bounded by maxitl sweeps.  cstart[c] .. cstart[c+1] are the colour ranges.
// K = slots per lane (1: rows of at most 32 slots, 3: up to 96), NT threads.
template <int K, int NT>
__global__ void __launch_bounds__(NT) k_sor_small(BlockDev B, const int *__restrict__ cstart,
                                                  int ncol, const double *__restrict__ rhs,
                                                  double *sol, SorCtl *ctl, double tolerl,
                                                  int maxitl)
{
    __shared__ double red[2][32];
    __shared__ int s_conv;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) s_conv = 0;
    __syncthreads();
    int sweeps = 0;
    double err = 0.0;
    while (!s_conv && sweeps < maxitl) {
        double v0 = 0.0, v1 = 0.0;
        for (int c = 0; c < ncol; ++c) {
            const int p1 = cstart[c + 1];
            if (K == 1)
                sor_rows<double>(B, B.blk, cstart[c] + wid, p1, nw, lane, rhs, sol, nullptr, v0, v1);
            else
                sor_rows_k<double, K>(B, B.blk, cstart[c] + wid, p1, nw, lane, rhs, sol, nullptr, v0, v1);
            __syncthreads();   // the next colour reads this colour's values
        }
        if (lane == 0) {
            red[0][wid] = v0;
            red[1][wid] = v1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0, b = 0.0;
            for (int i = 0; i < nw; ++i) {
                a += red[0][i];
                b += red[1][i];
            }
            err = a / b;
            if (err < tolerl) s_conv = 1;
            ctl->err = err;
        }
        ++sweeps;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ctl->sweeps = sweeps;
        ctl->conv = s_conv;
    }
}

// ---------------------------------------------------------------- FP32 SOR refinement
// FP64 residual of the assembled system, r = rhs - K x, one warp per row.
// Skipped once the solve has converged.
__global__ void __launch_bounds__(256) k_residual(BlockDev B, const double *__restrict__ rhs,
                                                  const double *__restrict__ x, double *r,
                                                  const SorCtl *ctl)
{
    if (((volatile const SorCtl *)ctl)->conv) return;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int p = blockIdx.x * wpb + (threadIdx.x >> 5); p < B.R; p += gridDim.x * wpb) {
        const int ns = B.nslot[p];
        const int S = B.slots;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int sl = lane; sl < ns; sl += 32) {
            const int m = B.bcol[B.si(p, sl)];
            const double *b = B.blk + B.bi(p, sl, 0);
            const double x0 = x[3 * m], x1 = x[3 * m + 1], x2 = x[3 * m + 2];
            a0 += b[0 * S] * x0 + b[1 * S] * x1 + b[2 * S] * x2;
            a1 += b[3 * S] * x0 + b[4 * S] * x1 + b[5 * S] * x2;
            a2 += b[6 * S] * x0 + b[7 * S] * x1 + b[8 * S] * x2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (lane == 0) {
            const int n = B.perm[p];
            r[3 * n] = rhs[3 * n] - a0;
            r[3 * n + 1] = rhs[3 * n + 1] - a1;
            r[3 * n + 2] = rhs[3 * n + 2] - a2;
        }
    }
}

// x += d, d = 0 and its FP32 mirror d32 = 0 (end of one refinement step);
// with symmetric rows also the nacc accumulator entries (the products of a
// zero correction).
__global__ void k_fold(int ndof, double *x, double *d, float *d32, float *acc = nullptr, int nacc = 0)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nacc) acc[i] = 0.f;
    if (i >= ndof) return;
    x[i] += d[i];
    d[i] = 0.0;
    if (d32) d32[i] = 0.f;
}

// Symmetric FP32 rows from the assembled FP64 rows (27-slot layout), one
// warp per row, lane s on slot s: the diagonal block and the slots whose bit
// is set in mask[row] (the blocks this row stores) are rounded to FP32 and
// packed, in slot order, into a SLOTS_SYM-slot row with its column ids and
// slot count.
__global__ void k_sym_pack(BlockDev B, const unsigned *__restrict__ mask, float *__restrict__ bs,
                           int *__restrict__ cs)
{
    constexpr int BRS = brow_of(SLOTS_SYM), CRS = crow_of(SLOTS_SYM);
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= B.R) return;
    const int r = (int)w;
    const int *cols = B.bcol + B.si(r, 0);
    const int ns = cols[SLOTS];
    const bool keep = lane < ns && (lane == 0 || ((mask[r] >> lane) & 1u));
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int pos = __popc(bal & ((1u << lane) - 1u));
    if (keep && pos < SLOTS_SYM) {
#pragma unroll
        for (int qq = 0; qq < 9; ++qq)
            bs[(size_t)r * BRS + qq * SLOTS_SYM + pos] = (float)B.blk[B.bi(r, lane, qq)];
        cs[(size_t)r * CRS + pos] = cols[lane];
    }
    if (lane == 0) cs[(size_t)r * CRS + SLOTS_SYM] = min(__popc(bal), SLOTS_SYM);
}

// End of one sweep: error = sum(dx^2) / sum(x^2) (Stif_sol.f90:206-210).
__global__ void __launch_bounds__(1024) k_sor_check(const double *part, int nblk, SorCtl *ctl,
                                                    double tolerl)
{
    pdl_launch_dependents();
    pdl_wait();   // every colour's partial sums are visible from here
    if (ctl->conv) return;
    sweep_test(part, nblk, ctl, tolerl);
}

// Correctly rounded reciprocals of the three diagonal entries of every row
// (row order), for the colour kernel's quotient.
__global__ void k_rdiag(BlockDev B, double *rdiag)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= B.R) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) rdiag[3 * (size_t)p + c] = 1.0 / B.blk[B.bi(p, 0, 4 * c)];
}

// 903 test (Stif_sol.f90:183-185): first DOF whose diagonal entry is zero.
__global__ void k_diag_check(BlockDev B, unsigned long long *firstbad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= B.R) return;
    const int n = B.perm[p];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if (B.blk[B.bi(p, 0, 4 * c)] == 0.0) atomicMin(firstbad, (unsigned long long)(3 * n + c));
}

// ---------------------------------------------------------------- updates
// NRITER's damped correction (Stif_sol.f90:70-74).
__global__ void k_nr_update(int ndof, double alp2, const double *ddx, double *x, double *dx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ndof) return;
    const double xc = alp2 * ddx[i];
    x[i] = x[i] - xc;
    dx[i] = dx[i] - xc;
}

// ---------------------------------------------------------------- graph-launched NRITER
// State of NRITER's loop when a whole increment runs as one CUDA graph
// (FAS_MODE_GRAPH): the loop and the SOR sweeps inside it are conditional
// while nodes whose conditions these kernels set on the device.
struct NrDev {
    int nit;        // Newton iterations done in this increment
    int status;     // 0, or the first error: a FAFERR code or FAS_E_* < 0
    double alp2;    // damping factor of the iteration just finished (0 after an error)
};

// Before the sweeps of a Newton iteration: sweep only when nothing has
// failed so far in it (an element's FAFERR code, a bad boundary code, a
// zero diagonal -- Stif_sol.f90:183-185 -- stop the reference before FACSLS).
// `hlast` (when `has_last`), the condition of the FP32 solve's shorter
// last cycle, starts cleared.
__global__ void k_graph_sor_begin(const unsigned long long *ekey, const int *flags,
                                  cudaGraphConditionalHandle hsor, cudaGraphConditionalHandle hlast,
                                  int has_last)
{
    if (threadIdx.x == 0) {
        cudaGraphSetConditional(hsor, (ekey[0] == ~0ull && ekey[1] == ~0ull && flags[0] == 0) ? 1u : 0u);
        if (has_last) cudaGraphSetConditional(hlast, 0u);
    }
}

// After a cycle of the FP32 solve (m sweeps, fold, FP64 residual): another
// full cycle while not converged, no wait gave up and fewer than `full`
// (the largest multiple of m within 1000) sweeps are done; the shorter
// last cycle of the remaining sweeps when exactly `full` are done and
// some remain.
__global__ void k_sor_cycle_cond(const SorCtl *ctl, int full, int rest, cudaGraphConditionalHandle hsor,
                                 cudaGraphConditionalHandle hlast)
{
    if (threadIdx.x != 0) return;
    const volatile SorCtl *c = ctl;
    const bool go = !c->conv && !c->fault;
    cudaGraphSetConditional(hsor, (go && c->sweeps < full) ? 1u : 0u);
    cudaGraphSetConditional(hlast, (go && c->sweeps == full && rest > 0) ? 1u : 0u);
}

// The stopping test of one sweep (k_sor_check) that also sets the sweep
// loop's condition: another four sweeps while not converged, below maxitl
// sweeps and no bounded wait gave up.
__global__ void __launch_bounds__(1024) k_sor_check_cond(const double *part, int nblk, SorCtl *ctl, double tolerl,
                                                         int maxitl, cudaGraphConditionalHandle hsor)
{
    pdl_launch_dependents();
    pdl_wait();
    if (!ctl->conv) sweep_test(part, nblk, ctl, tolerl);
    __syncthreads();
    if (threadIdx.x == 0) {
        const volatile SorCtl *c = ctl;
        cudaGraphSetConditional(hsor, (!c->conv && c->sweeps < maxitl && !c->fault) ? 1u : 0u);
    }
}

// The end of NRITER's loop body (Stif_sol.f90:46-75) on the device: the
// norms' sfc, errdx, erddx, sdx and the damping factor alp2, the report line
// of the iteration, the first error of the iteration (element key, boundary
// codes, zero diagonal, SOR fault or 904), and the loop's condition:
// another pass while sdx >= toler and nit < maxit and nothing failed.
__global__ void k_nr_decide(const double *sums, int ngps, const unsigned long long *ekey, const int *flags,
                            const SorCtl *ctl, double toler, double alpha, int maxit, double tolerl,
                            NrDev *nr, fas_iter_report *rep, int cap, cudaGraphConditionalHandle hnr)
{
    if (threadIdx.x != 0) return;
    const int nit = nr->nit + 1;
    int status = 0;
    if (ekey[0] != ~0ull)
        status = (int)(ekey[0] & 0xFFFFull);
    else if (flags[0])
        status = FAS_E_ARG;
    else if (ekey[1] != ~0ull)
        status = 903;
    else if (ctl->fault)
        status = FAS_E_TIMEOUT;
    else if (ctl->err > 10.0 * tolerl)
        status = 904;
    const double sfc = sqrt(sums[0]), errdx = sqrt(sums[1]), erddx = sqrt(sums[2]);
    const double sdx = errdx == 0.0 ? toler : erddx / errdx;
    // rounded like the host's 1 / (1 + alpha sdx): no fused multiply-add
    const double alp2 = 1.0 / __dadd_rn(1.0, __dmul_rn(alpha, sdx));
    if (nit <= cap && status == 0) {
        fas_iter_report &r = rep[nit - 1];
        r.nit = nit;
        r.sor_sweeps = ctl->sweeps;
        r.sdx = sdx;
        r.sfc = sfc;
        r.cp_err = sums[3] / (double)ngps;
        r.alp2 = alp2;
        r.sor_error = ctl->err;
    }
    nr->nit = nit;
    nr->status = status;
    nr->alp2 = status ? 0.0 : alp2;
    cudaGraphSetConditional(hnr, (status == 0 && sdx >= toler && nit < maxit) ? 1u : 0u);
}

// NRITER's correction x, dx -= alp2 ddx with the device's alp2 (none after
// an error: the reference stops before it).
__global__ void k_nr_update_dev(int ndof, const NrDev *nr, const double *ddx, double *x, double *dx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ndof || nr->status) return;
    const double xc = nr->alp2 * ddx[i];
    x[i] = x[i] - xc;
    dx[i] = dx[i] - xc;
}

// NRITER's cumslip tail, skipped after an error.
__global__ void k_cumslip_dev(DevGp G, int nsc, double tm, const NrDev *nr)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G.ngps || nr->status) return;
    for (int k = 0; k < nsc; ++k)
        G.cumslip[k * G.ngps + g] = G.cumslip[k * G.ngps + g] + (G.srate[k * G.ngps + g] * tm);
}

// UPDATE_NODE (src/fasolt/Fasolt3.f90:231-244)
__global__ void k_update_node(int ndof, double *x, const double *dx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ndof) x[i] = x[i] + dx[i];
}

// cumslip update after the Newton loop (src/fasolt/Stif_sol.f90:80-84)
__global__ void k_cumslip(DevGp G, int nsc, double tm)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G.ngps) return;
    for (int k = 0; k < nsc; ++k)
        G.cumslip[k * G.ngps + g] = G.cumslip[k * G.ngps + g] + (G.srate[k * G.ngps + g] * tm);
}

// UPDATE_GPTV (src/fasolt/Fasolt3.f90:254-284)
__global__ void k_update_gptv(DevGp G, int nsv)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G.ngps) return;
    const int ng = G.ngps;
    G.eps[g] = G.eps[g] + G.dep[g];
#pragma unroll
    for (int k = 0; k < 3; ++k) G.rt[k * ng + g] = G.rt[k * ng + g] + G.dr[k * ng + g];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        G.ep[k * ng + g] = G.ep[k * ng + g] + G.de[k * ng + g];
        G.st[k * ng + g] = G.st[k * ng + g] + G.ds[k * ng + g];
    }
    for (int k = 0; k < nsv; ++k) G.sv[k * ng + g] = G.sv[k * ng + g] + G.dsv[k * ng + g];
}

// DoReorient (src/fasolt/Fasolt3.f90:79-178): rotate a twinned GP by ssang
// about n x d of its twin system, using material 1's tables and
// pi = 3.14159 as the reference does.  Events are appended unordered; the
// host sorts them by GP.
struct TwinEv {
    int gp, sys;
    double eo[3], en[3];
};

__global__ void k_reorient(DevGp G, DevMat M, TwinEv *ev, int cap, int *nev)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= G.ngps) return;
    const int ts = G.twinsys[j];
    if (ts == 0) return;
    const int i = ts - 1;
    const int ng = G.ngps;
    const double e1 = G.sv[j], e2 = G.sv[ng + j], e3 = G.sv[2 * ng + j];
    const double ang = M.ssang[i] * 3.14159 / 180.0;
    double ss1, c1, s2, c2, s3, c3;
    sincos(e1, &ss1, &c1);
    sincos(e2, &s2, &c2);
    sincos(e3, &s3, &c3);
    double RM[3][3];
    RM[0][0] = c1 * c3 - c2 * ss1 * s3;
    RM[0][1] = -c1 * s3 - c2 * c3 * ss1;
    RM[0][2] = ss1 * s2;
    RM[1][0] = c3 * ss1 + c1 * c2 * s3;
    RM[1][1] = c1 * c2 * c3 - ss1 * s3;
    RM[1][2] = -c1 * s2;
    RM[2][0] = s2 * s3;
    RM[2][1] = c3 * s2;
    RM[2][2] = c2;
    double nv[3], dv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        nv[a] = RM[a][0] * M.an[3 * i] + RM[a][1] * M.an[3 * i + 1] + RM[a][2] * M.an[3 * i + 2];
        dv[a] = RM[a][0] * M.ab[3 * i] + RM[a][1] * M.ab[3 * i + 1] + RM[a][2] * M.ab[3 * i + 2];
    }
    const double u1 = nv[1] * dv[2] - nv[2] * dv[1];
    const double u2 = nv[2] * dv[0] - nv[0] * dv[2];
    const double u3 = nv[0] * dv[1] - nv[1] * dv[0];
    double s, c;
    sincos(ang, &s, &c);
    double E[3][3];
    E[0][0] = c + u1 * u1 * (1.0 - c);
    E[0][1] = u1 * u2 * (1.0 - c) - u3 * s;
    E[0][2] = u1 * u3 * (1.0 - c) + u2 * s;
    E[1][0] = u1 * u2 * (1.0 - c) + u3 * s;
    E[1][1] = c + u2 * u2 * (1.0 - c);
    E[1][2] = u2 * u3 * (1.0 - c) - u1 * s;
    E[2][0] = u1 * u3 * (1.0 - c) - u2 * s;
    E[2][1] = u2 * u3 * (1.0 - c) + u1 * s;
    E[2][2] = c + u3 * u3 * (1.0 - c);
    double F[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) F[a][b] = E[a][0] * RM[0][b] + E[a][1] * RM[1][b] + E[a][2] * RM[2][b];
    const double e1n = atan2(F[0][2], -F[1][2]);
    double f33 = F[2][2];
    if (fabs(f33) > 1.0) f33 = f33 / fabs(f33);
    const double e2n = acos(f33);
    const double e3n = atan2(F[2][0], F[2][1]);
    G.sv[j] = e1n;
    G.sv[ng + j] = e2n;
    G.sv[2 * ng + j] = e3n;
    const int slot = atomicAdd(nev, 1);
    if (slot < cap) {
        TwinEv &t = ev[slot];
        t.gp = j;
        t.sys = i;
        t.eo[0] = e1; t.eo[1] = e2; t.eo[2] = e3;
        t.en[0] = e1n; t.en[1] = e2n; t.en[2] = e3n;
    }
    G.twinsys[j] = 0;
    G.timestwinned[j] = G.timestwinned[j] + 1;
}

// ELASEPS (src/csvmkr/data_out.f90:263-361): elastic (lattice) strain of
// every GP, e = S(phi) sigma with the compliance of ELASTC at the committed
// Euler angles sv(1:3) and the GP's material; out[k * ngps + g].
__global__ void k_elaseps(DevMat M, DevGp G, const int *gp_iel, double *out)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G.ngps) return;
    const int ng = G.ngps;
    const int iel = gp_iel[g];
    const int mc = (iel < 0 ? -iel : iel) - 1;
    double S[6][6];
    elastc(M.e + 9 * mc, G.sv[g], G.sv[ng + g], G.sv[2 * ng + g], S);
    double st[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) st[k] = G.st[k * ng + g];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) acc = acc + S[i][c] * st[c];
        out[i * ng + g] = acc;
    }
}

// ---------------------------------------------------------------- exports
// SETPTA (src/fasolt/Stif_sol.f90:98-149) per DOF row: columns in the order
// of first touch over ascending elements and their local DOFs.  Writes the
// 1-based reference layout is[row * ld + k]; overflow raises 955.
__global__ void k_setpta(MeshDev Mh, int ld, int *is, int *overflow)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= 3 * Mh.nnod) return;
    const int n = row / 3;
    int *out = is + (size_t)row * ld;
    int cnt = 0;
    for (int k = 0; k < Mh.ne_cnt[n]; ++k) {
        const int e = Mh.ne_elem[k * Mh.nnod + n];
        for (int a = 0; a < Mh.nn; ++a) {
            const int m = Mh.ln[a * Mh.nlmnt + e];
            if (m < 0) break;   // a tie element's 2 nodes end its list
            for (int c = 0; c < 3; ++c) {
                const int col = 3 * m + c + 1;
                if (col == row + 1) continue;
                bool found = false;
                for (int q = 1; q <= cnt; ++q)
                    if (out[q] == col) { found = true; break; }
                if (!found) {
                    if (cnt + 1 >= ld) { *overflow = 1; return; }
                    out[++cnt] = col;
                }
            }
        }
    }
    out[0] = cnt;
    for (int q = cnt + 1; q < ld; ++q) out[q] = 0;
}

// Values of the block matrix in the reference layout ss(ld, ndof).
__global__ void k_to_ell(BlockDev B, const int *rowof, int nnod, int ld, const int *is, double *ss)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= 3 * nnod) return;
    const int n = row / 3, r = row % 3;
    const int p = rowof[n];
    const int *ir = is + (size_t)row * ld;
    double *out = ss + (size_t)row * ld;
    out[0] = B.blk[B.bi(p, 0, r * 3 + r)];
    for (int k = 1; k <= ir[0]; ++k) {
        const int col = ir[k] - 1;
        const int m = col / 3, c = col % 3;
        int slot = -1;
        for (int s = 0; s < B.nslot[p]; ++s)
            if (B.bcol[B.si(p, s)] == m) { slot = s; break; }
        out[k] = slot >= 0 ? B.blk[B.bi(p, slot, r * 3 + c)] : 0.0;
    }
    for (int k = ir[0] + 1; k < ld; ++k) out[k] = 0.0;
}

// ---------------------------------------------------------------- state I/O
// Gather a caller array laid out [g][k] (leading dimension ld, element size
// rb) into the structure-of-arrays [k][g] FP64 layout, and back.
__global__ void k_aos_to_soa(const void *src, int rb, int ld, int nk, int n, double *dst)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nk * n) return;
    const int k = (int)(t / n), g = (int)(t - (long long)k * n);
    const size_t si = (size_t)g * ld + k;
    dst[(size_t)k * n + g] = rb == 4 ? (double)((const float *)src)[si] : ((const double *)src)[si];
}

__global__ void k_soa_to_aos(const double *src, int nk, int n, void *dst, int rb, int ld)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)nk * n) return;
    const int g = (int)(t / nk), k = (int)(t - (long long)g * nk);
    const double v = src[(size_t)k * n + g];
    const size_t di = (size_t)g * ld + k;
    if (rb == 4) ((float *)dst)[di] = (float)v;
    else ((double *)dst)[di] = v;
}

}  // namespace fasdev
