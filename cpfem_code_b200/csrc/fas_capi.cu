// fas_capi.cu -- host side of libfasgpu.so: the handle, one-time set-up of
// the device layout, state transfer, the NRITER / FACSLS orchestration and
// the exported C ABI of include/fasolt_gpu.h.
//
// Everything runs on one CUDA stream per handle.  Host synchronisation
// happens once per global Newton iteration (to read the error key and the
// norms that decide the loop) and once per chunk of SOR sweeps (to read the
// convergence flag); nothing else waits for the device.  Chunks of sweeps
// are CUDA graphs whose colour and check kernels carry programmatic
// dependencies, so each colour's matrix stream starts while the previous
// colour drains.  A mesh is one brick family (8-node lt 12 or 20-node lt 22)
// plus optional tie elements (lt 1-6).

#include "../../include/fasolt_gpu.h"
#include "fas_kernels.cuh"
#include "fas_sor_tiles.cuh"
#include "fas_adjoint.cuh"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

using namespace fasdev;

// Quotients of the SOR point update from precomputed reciprocals (1) or by
// division (0); both give the correctly rounded quotient.
#ifndef FAS_SOR_RCP
#define FAS_SOR_RCP 1
#endif
// Constitutive passes pull their items from a device queue on a persistent
// grid (1), or launch one thread per item (0, the tuned choice).
#ifndef FAS_CP_QUEUE
#define FAS_CP_QUEUE 0
#endif
// Constitutive kernels launched in work-sorted order (1) or natural order (0).
#ifndef FAS_WORK_SORT
#define FAS_WORK_SORT 1
#endif

namespace {

template <class T> struct DVec {
    T *p = nullptr;
    size_t n = 0;
    DVec() = default;
    DVec(const DVec &) = delete;
    DVec &operator=(const DVec &) = delete;
    ~DVec() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t m)
    {
        release();
        n = m;
        if (!m) return cudaSuccess;
        cudaError_t e = cudaMalloc((void **)&p, m * sizeof(T));
        if (e != cudaSuccess) { p = nullptr; n = 0; }
        return e;
    }
    cudaError_t zero(cudaStream_t s) { return n ? cudaMemsetAsync(p, 0, n * sizeof(T), s) : cudaSuccess; }
    cudaError_t put(const T *h, size_t m, cudaStream_t s)
    {
        return m ? cudaMemcpyAsync(p, h, m * sizeof(T), cudaMemcpyHostToDevice, s) : cudaSuccess;
    }
};

inline double rdv(const void *p, int rb, size_t i)
{
    return rb == 4 ? (double)((const float *)p)[i] : ((const double *)p)[i];
}

inline unsigned nblocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

struct HostCtl {                 // pinned mirror of the small device results
    unsigned long long ekey[2];
    int flags[4];                // 0 bad_bc, 1 tflag, 2 overflow, 3 nev
    SorCtl sor;
    double sums[8];
    NrDev nr;                    // a graph-launched NRITER's outcome
};

}  // namespace

// Device buffers of the replay behind fas_gpu_adjoint_forward / _grad:
// the history and objective, checkpoints, per-GP records of the segment
// being swept back, the adjoints, and a private copy of the GP state that
// DSTRSS reads and writes (the handle's own state is left as it was).
struct ReplayBufs {
    DVec<double> de, dr, dt, w, y, chk, rec;
    DVec<double> sv, dsv, srate, erepmd, ops, jg, eq, gst, gsv, gp;
    DVec<int> twinsys, timestwinned, cp_iters, tflag;
};

struct fas_handle {
    int dev = 0, nsm = 148;
    cudaStream_t stream = nullptr;
    uint32_t mode = 0;
    int nlmnt = 0, nnod = 0, ngps = 0;
    int nn = 8, npg = 1;         // nodes and Gauss points per element (8, 1 or 20, 8)
    int slots = SLOTS;           // block slots per row (27 or 81)
    int maxns = 0, nsvld = 0, nsv = 0, ns_tmpl = 12;
    bool point_mode = false, have_state = false;
    int last_mat = 1;            // mat_code the last element leaves behind
    // host copies used by the set-up
    std::vector<int> h_ln, h_gpe, h_le, h_ib, h_gp_iel, h_colour;
    std::vector<int> ne_ptr, ne_list, ne_locl;   // node -> elements CSR
    std::vector<double> h_tiem;
    int ninc1 = 0, nxs = 0, nfs = 0;
    // device mesh
    DVec<int> ln, gpe, le, lt, ib, gp_iel, ne_elem, ne_loc, ne_cnt;
    // materials / control
    DVec<double> m_e, m_ssang, m_ab, m_an, m_ampar, m_sm;
    DevMat M{};
    DevCtrl C{};
    DVec<double> xspec, fspec;
    // nodal vectors
    DVec<double> x, dx, fc, ddx, rhs;
    // Gauss-point state (SoA)
    DVec<double> eps, dep, st, ep, ds, de, rt, dr, sv, dsv, srate, cumslip, erepmd, ops, chi_pts;
    DVec<int> timestwinned, twinsys, cp_iters;
    // element records
    DVec<double> rec;
    // block layout
    int ncol = 0;
    std::vector<int> col_start;
    std::vector<double> col_bytes, col_bytes32;   // algorithmic bytes per colour launch
    DVec<int> perm, rowof, nslot, bcol;
    DVec<unsigned long long> bloc;
    DVec<double> dnq;            // the quadratic element's local-derivative table (SHAPE_21/22/23)
    double wfac = 1.0;           // its GP weight factor
    int ltype = 12;              // element type of the mesh's elements
    int maxadj = 1;              // most elements on one node
    DVec<double> blk;
    DVec<float> blk32;           // FP32 copy for FAS_MODE_SOR_FP32
    DVec<double> sor_d, sor_r;   // correction and residual of the refinement
    DVec<float> sor_d32;         // the correction rounded to FP32 (the FP32 sweeps' gathers)
    // symmetric FP32 rows (FAS_MODE_SOR_SYM, 27-slot rows): the blocks each
    // row stores (bit s of sym_mask: slot s), the packed rows, and per node
    // the accumulated transposed products of the blocks stored elsewhere
    DVec<unsigned> sym_mask;
    DVec<float> blk_sym, sor_acc;
    DVec<int> bcol_sym;
    int sym_state = 0;           // 0 not set up, 1 usable, -1 the pattern does not fit SLOTS_SYM
    bool sym_on = false;         // the FP32 sweeps of this solve use the symmetric rows
    std::vector<int> sor_boff_sym, sor_nblk_sym;
    int sor_nblk_tot_sym = 0;
    DVec<double> rdiag;          // reciprocals of the diagonal entries, row order
    DVec<int> work_order, work_hist;   // work-sorted constitutive launch order
    DVec<int> cp_queue;          // head of the constitutive pass's device queue
    DVec<int> gp_item;           // GP of item e*npg + g (quadratic elements; -1 for ties)
    // tile layout of the persistent SOR solve (k_sor_tiles; 27-slot rows)
    int ntiles = 0;
    DVec<int> tseg, tadj_ptr, tadj, tsrc, tbcol, tprog;
    DVec<double> tblk64, trdiag, tpart, sol_scr;
    DVec<float> tblk32;
    DVec<TileSync> tsync;
    int tile_keep_rows = 0;      // rows per tile whose blocks stay in L2 across sweeps
    // NRITER of an increment as one CUDA graph (FAS_MODE_GRAPH): loop state,
    // report lines, the instantiated graph of each increment, and the two
    // side streams its nested loop bodies are captured on
    DVec<NrDev> nrdev;
    DVec<fas_iter_report> nrrep;
    std::map<int, cudaGraphExec_t> inc_graphs;
    cudaStream_t cap2 = nullptr, cap3 = nullptr;
    int64_t g_body_launches = 0, g_pass_launches = 0;   // per Newton iteration, per sweep pass
    int refine_every = 16;       // FP32 sweeps per FP64 residual
    cudaGraphExec_t sor_graph = nullptr;   // GRAPH_SWEEPS plain sweeps
    cudaGraphExec_t sor32_graph = nullptr; // one refinement cycle of the FP32 form
    bool sor32_graph_sym = false;          // ... on the symmetric rows
    bool blk32_fresh = false;    // the last assembly wrote blk32
    // reductions and control
    std::vector<int> sor_boff, sor_nblk;       // FP64 colour grids and their partial offsets
    std::vector<int> sor_boff32, sor_nblk32;   // FP32 colour grids (smaller rings, more CTAs)
    DVec<int> d_cstart;          // colour ranges for the one-CTA SOR
    bool sor_small = false;      // whole solve in one CTA (small meshes)
    int sor_nblk_tot = 0, sor_nblk_tot32 = 0, nr_nblk = 0;
    DVec<double> part_sor, part_nr, sums;
    bool mixed_phases = false;   // GPs of materials with different slip-system counts
    size_t stage_bytes = 0;      // shared memory of the constitutive kernels' table copy
    DVec<unsigned long long> ekey;
    DVec<int> flags;
    DVec<SorCtl> sorctl;
    HostCtl *hc = nullptr;
    // staging for state transfer
    DVec<unsigned char> stage;
    DVec<TwinEv> events;
    // profiling: 0 off, 1 counters + one event pair around the region,
    // 2 also an event pair around every phase kernel launch
    int prof = 0;
    fas_profile P{};
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<std::pair<cudaEvent_t, cudaEvent_t>, double *>> pending;
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;
    double asm_bytes = 0.0;      // algorithmic bytes of one assembly launch
    int64_t launches = 0;
    ReplayBufs rp;

    ~fas_handle()
    {
        if (sor_graph) cudaGraphExecDestroy(sor_graph);
        if (sor32_graph) cudaGraphExecDestroy(sor32_graph);
        for (auto &g : inc_graphs) cudaGraphExecDestroy(g.second);
        if (cap2) cudaStreamDestroy(cap2);
        if (cap3) cudaStreamDestroy(cap3);
        for (auto e : ev_pool) cudaEventDestroy(e);
        if (ev_t0) cudaEventDestroy(ev_t0);
        if (ev_t1) cudaEventDestroy(ev_t1);
        if (hc) cudaFreeHost(hc);
        if (stream) cudaStreamDestroy(stream);
    }
    DevGp gp()
    {
        DevGp G;
        G.ngps = ngps;
        G.ldsv = nsvld;
        G.ldsl = maxns;
        G.eps = eps.p; G.dep = dep.p; G.st = st.p; G.ep = ep.p; G.ds = ds.p; G.de = de.p;
        G.rt = rt.p; G.dr = dr.p; G.sv = sv.p; G.dsv = dsv.p; G.srate = srate.p;
        G.cumslip = cumslip.p; G.timestwinned = timestwinned.p; G.twinsys = twinsys.p;
        G.tflag = flags.p + 1; G.cp_iters = cp_iters.p; G.erepmd = erepmd.p; G.ops = ops.p;
        return G;
    }
    MeshDev mesh()
    {
        MeshDev m;
        m.nlmnt = nlmnt; m.nnod = nnod; m.nn = nn; m.npg = npg;
        m.ln = ln.p; m.gpe = gpe.p; m.le = le.p; m.lt = lt.p; m.ib = ib.p;
        m.ne_elem = ne_elem.p; m.ne_loc = ne_loc.p; m.ne_cnt = ne_cnt.p;
        return m;
    }
    BlockDev block()
    {
        BlockDev b;
        b.R = nnod; b.slots = slots; b.brow = brow_of(slots); b.crow = crow_of(slots);
        b.perm = perm.p; b.nslot = nslot.p; b.bcol = bcol.p; b.bloc = bloc.p; b.nbw = (maxadj + 7) / 8;
        b.blk = blk.p;
        b.blk32 = (mode & FAS_MODE_SOR_FP32) ? blk32.p : nullptr;
        return b;
    }
};

// meshes with at most this many nodes run each SOR solve in one CTA: 256
// for 27-slot rows (1024 threads, a slot per lane; measured us per sweep,
// one CTA against the colour kernels: 17 / 33 at 125 nodes, 74 / 27 at
// 729, 439 / 26 at 4,913); 512 for 81-slot rows, whose three slots per lane
// on 256 threads make a row about 12x slower than in the colour kernels,
// which cost about 64 us per sweep at that size
constexpr int SOR_SMALL_ROWS = 256;
constexpr int SOR_SMALL_ROWS81 = 512;

#define CK(expr)                                      \
    do {                                              \
        cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) {                      \
            std::fprintf(stderr, "fasgpu: %s: %s\n", #expr, cudaGetErrorString(e_)); \
            return FAS_E_CUDA;                        \
        }                                             \
    } while (0)
#define CKA(expr)                                     \
    do {                                              \
        cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return e_ == cudaErrorMemoryAllocation ? FAS_E_NOMEM : FAS_E_CUDA; \
    } while (0)
#define LAUNCHED(h)                                   \
    do {                                              \
        ++(h)->launches;                              \
        CK(cudaGetLastError());                       \
    } while (0)

namespace {

// ---------------------------------------------------------------- profiling
cudaEvent_t take_event(fas_handle *h)
{
    cudaEvent_t e;
    if (!h->ev_pool.empty()) {
        e = h->ev_pool.back();
        h->ev_pool.pop_back();
    } else {
        cudaEventCreate(&e);
    }
    return e;
}
struct Span {                    // event pair around one launch while profiling
    fas_handle *h;
    cudaEvent_t a = nullptr, b = nullptr;
    double *acc;
    explicit Span(fas_handle *hh, double *accum) : h(hh), acc(accum)
    {
        if (h->prof >= 2) {
            a = take_event(h);
            b = take_event(h);
            cudaEventRecord(a, h->stream);
        }
    }
    void end()
    {
        if (a) cudaEventRecord(b, h->stream);
    }
};
void keep(fas_handle *h, const Span &sp)
{
    if (sp.a) h->pending.push_back({{sp.a, sp.b}, sp.acc});
}
void settle_spans(fas_handle *h)
{
    for (auto &q : h->pending) {
        float ms = 0.f;
        cudaEventSynchronize(q.first.second);
        cudaEventElapsedTime(&ms, q.first.first, q.first.second);
        *q.second += ms;
        h->ev_pool.push_back(q.first.first);
        h->ev_pool.push_back(q.first.second);
    }
    h->pending.clear();
}

// ---------------------------------------------------------------- set-up
int greedy_colouring(fas_handle *h, const std::vector<double> &xyz)
{
    // Same rule as the checker: nodes visited in ascending (z, y, x, id)
    // order take the smallest colour unused by nodes sharing an element.
    const int nn = h->nnod;
    std::vector<int> order(nn);
    for (int i = 0; i < nn; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        for (int c = 2; c >= 0; --c) {
            const double xa = xyz[3 * (size_t)a + c], xb = xyz[3 * (size_t)b + c];
            if (xa != xb) return xa < xb;
        }
        return a < b;
    });
    h->h_colour.assign(nn, -1);
    int ncol = 0;
    std::vector<int> used(64, -1);
    for (int n : order) {
        for (int k = h->ne_ptr[n]; k < h->ne_ptr[n + 1]; ++k) {
            const int e = h->ne_list[k];
            for (int a = 0; a < h->nn; ++a) {
                const int m = h->h_ln[(size_t)e * h->nn + a];
                if (m < 0) break;   // end of a tie element's 2 nodes
                const int c = h->h_colour[m];
                if (c >= 0) {
                    if (c >= (int)used.size()) used.resize(c + 1, -1);
                    used[c] = n;
                }
            }
        }
        int c = 0;
        while (c < (int)used.size() && used[c] == n) ++c;
        h->h_colour[n] = c;
        ncol = std::max(ncol, c + 1);
    }
    h->ncol = ncol;
    return 0;
}

int build_tiles(fas_handle *h, const std::vector<double> &xyz, const std::vector<int> &bcol_host,
                const std::vector<int> &nslot_host, const std::vector<int> &rowof_host);

// Row permutation by colour, node block neighbourhoods and the per-slot
// element-local index words; allocates the block matrix.
int build_layout(fas_handle *h, const std::vector<double> &xyz)
{
    const int nn = h->nnod;
    greedy_colouring(h, xyz);
    std::vector<int> perm(nn), rowof(nn);
    for (int i = 0; i < nn; ++i) perm[i] = i;
    std::stable_sort(perm.begin(), perm.end(),
                     [&](int a, int b) { return h->h_colour[a] < h->h_colour[b]; });
    for (int p = 0; p < nn; ++p) rowof[perm[p]] = p;
    h->col_start.assign(h->ncol + 1, 0);
    for (int p = 0; p < nn; ++p) h->col_start[h->h_colour[perm[p]] + 1] = p + 1;
    for (int c = 1; c <= h->ncol; ++c) h->col_start[c] = std::max(h->col_start[c], h->col_start[c - 1]);

    // block neighbourhood of every row: the node itself, then the nodes it
    // shares an element with, ascending
    const int NN = h->nn;
    std::vector<std::vector<int>> nbs(nn);
    int maxs = 0;
    for (int p = 0; p < nn; ++p) {
        const int n = perm[p];
        std::vector<int> others;
        for (int k = h->ne_ptr[n]; k < h->ne_ptr[n + 1]; ++k) {
            const int e = h->ne_list[k];
            for (int a = 0; a < NN; ++a) {
                const int m = h->h_ln[(size_t)e * NN + a];
                if (m < 0) break;
                if (m != n && std::find(others.begin(), others.end(), m) == others.end()) others.push_back(m);
            }
        }
        std::sort(others.begin(), others.end());
        nbs[p].reserve(others.size() + 1);
        nbs[p].push_back(n);
        nbs[p].insert(nbs[p].end(), others.begin(), others.end());
        maxs = std::max(maxs, (int)nbs[p].size());
    }
    if (maxs > SLOTS20) return FAS_E_RANGE;
    h->slots = maxs <= SLOTS ? SLOTS : SLOTS20;
    const int crow = crow_of(h->slots), brow = brow_of(h->slots);
    std::vector<int> nslot(nn), bcol((size_t)crow * nn, 0);
    const int nbw = (h->maxadj + 7) / 8;   // local-index words per slot
    std::vector<unsigned long long> bloc((size_t)crow * nn * nbw, ~0ull);
    for (int p = 0; p < nn; ++p) {
        const int n = perm[p];
        const int cnt = (int)nbs[p].size();
        nslot[p] = cnt;
        bcol[(size_t)p * crow + h->slots] = cnt;   // the pad slot carries the slot count
        for (int s = 0; s < cnt; ++s) {
            bcol[(size_t)p * crow + s] = nbs[p][s];
            unsigned long long *words = &bloc[((size_t)p * crow + s) * nbw];
            int k = 0;
            for (int q = h->ne_ptr[n]; q < h->ne_ptr[n + 1]; ++q, ++k) {
                const int e = h->ne_list[q];
                unsigned long long b = 0xFF;
                for (int a = 0; a < NN; ++a)
                    if (h->h_ln[(size_t)e * NN + a] == nbs[p][s]) { b = (unsigned long long)a; break; }
                unsigned long long &word = words[k >> 3];
                word = (word & ~(0xFFull << (8 * (k & 7)))) | (b << (8 * (k & 7)));
            }
        }
    }
    // algorithmic bytes of one colour launch: blocks and column ids of the
    // row, perm + nslot, and rhs read + solution read/write of its node
    h->col_bytes.assign(h->ncol, 0.0);
    h->col_bytes32.assign(h->ncol, 0.0);
    for (int c = 0; c < h->ncol; ++c)
        for (int p = h->col_start[c]; p < h->col_start[c + 1]; ++p) {
            h->col_bytes[c] += nslot[p] * (72.0 + 4.0) + 8.0 + 72.0;
            h->col_bytes32[c] += nslot[p] * (36.0 + 4.0) + 8.0 + 72.0 + 24.0;
        }
    // algorithmic bytes of one assembly launch: each GP record read once
    // (3 nn + 28 used doubles), each block written once, the slot tables
    // and node adjacency read once, fc and ddx written
    double ab = (double)h->nlmnt * h->npg * (3.0 * NN + 28.0) * 8.0 + (double)nn * (48.0 + 8.0 + 12.0 * h->maxadj);
    for (int p = 0; p < nn; ++p) ab += nslot[p] * (72.0 + 4.0 + 8.0 * nbw);
    h->asm_bytes = ab;
    cudaStream_t s = h->stream;
    CKA(h->perm.alloc(nn));
    CKA(h->rowof.alloc(nn));
    CKA(h->nslot.alloc(nn));
    CKA(h->bcol.alloc((size_t)crow * nn));
    CKA(h->bloc.alloc(bloc.size()));
    CKA(h->blk.alloc((size_t)brow * nn));
    CK(h->perm.put(perm.data(), nn, s));
    CK(h->rowof.put(rowof.data(), nn, s));
    CK(h->nslot.put(nslot.data(), nn, s));
    CK(h->bcol.put(bcol.data(), bcol.size(), s));
    CK(h->bloc.put(bloc.data(), bloc.size(), s));
    CK(h->blk.zero(s));
    // SOR reduction partials
    h->sor_boff.assign(h->ncol, 0);
    h->sor_nblk.assign(h->ncol, 0);
    int tot = 0;
    for (int c = 0; c < h->ncol; ++c) {
        h->sor_boff[c] = tot;
        // chunks of TMA_ROWS rows; one wave of as many CTAs as the
        // shared-memory rings let reside per SM, which also keeps the
        // per-sweep partial sums few enough for a cheap deterministic check
        const int cps = h->slots == SLOTS ? TMA_CTAS_PER_SM : tma_ctas_per_sm<SLOTS20, TMA_LPR81>();
        const int rows = h->slots == SLOTS ? tma_rows<SLOTS>() : tma_rows<SLOTS20>();
        h->sor_nblk[c] = (int)std::min<long long>(nblocks(h->col_start[c + 1] - h->col_start[c], rows),
                                                   (long long)h->nsm * cps);
        tot += h->sor_nblk[c];
    }
    h->sor_nblk_tot = std::max(tot, 1);
    // the FP32 copies' rings are half as large, so twice as many CTAs reside
    h->sor_boff32.assign(h->ncol, 0);
    h->sor_nblk32.assign(h->ncol, 0);
    int tot32 = 0;
    for (int c = 0; c < h->ncol; ++c) {
        h->sor_boff32[c] = tot32;
        const int cps = h->slots == SLOTS ? tma_ctas_per_sm<SLOTS, TMA_LPR32, float>()
                                          : tma_ctas_per_sm<SLOTS20, TMA_LPR81_32, float>();
        const int rows = h->slots == SLOTS ? tma_rows<SLOTS, float>() : tma_rows<SLOTS20, float>();
        h->sor_nblk32[c] = (int)std::min<long long>(nblocks(h->col_start[c + 1] - h->col_start[c], rows),
                                                     (long long)h->nsm * cps);
        tot32 += h->sor_nblk32[c];
    }
    h->sor_nblk_tot32 = std::max(tot32, 1);
    // symmetric FP32 rows (27-slot meshes): rings of their own size; one
    // wave of the CTAs that reside per SM (their registers, not only the
    // rings, bound that)
    h->sor_boff_sym.assign(h->ncol, 0);
    h->sor_nblk_sym.assign(h->ncol, 0);
    int cps_sym = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &cps_sym, k_sor_colour_tma<float, SLOTS_SYM, TMA_LPR_SYM, true>, tma_threads<TMA_LPR_SYM, TMA_ROWS_SYM>(),
        tma_smem_bytes<float, SLOTS_SYM>()));
    cps_sym = std::max(1, std::min(cps_sym, tma_ctas_per_sm<SLOTS_SYM, TMA_LPR_SYM, float>()));
    int tots = 0;
    for (int c = 0; c < h->ncol; ++c) {
        h->sor_boff_sym[c] = tots;
        h->sor_nblk_sym[c] = (int)std::min<long long>(
            nblocks(h->col_start[c + 1] - h->col_start[c], tma_rows<SLOTS_SYM, float>()), (long long)h->nsm * cps_sym);
        tots += h->sor_nblk_sym[c];
    }
    h->sor_nblk_tot_sym = std::max(tots, 1);
    CKA(h->part_sor.alloc((size_t)2 *
                          std::max(std::max(h->sor_nblk_tot, h->sor_nblk_tot32), h->sor_nblk_tot_sym)));
    if (FAS_SOR_RCP) CKA(h->rdiag.alloc((size_t)3 * nn));
    CKA(h->d_cstart.alloc(h->ncol + 1));
    CK(h->d_cstart.put(h->col_start.data(), h->ncol + 1, s));
    h->sor_small = nn <= (h->slots == SLOTS ? SOR_SMALL_ROWS : SOR_SMALL_ROWS81);
    CK(cudaStreamSynchronize(s));
    return build_tiles(h, xyz, bcol, nslot, rowof);
}

// Recursive coordinate bisection of nodes[lo, hi) into nt tiles t0 ..
// t0 + nt - 1 of (nearly) equal node counts: cut across the longest extent
// of the bounding box, in proportion to the tiles on each side.
void rcb_tiles(std::vector<int> &nodes, int lo, int hi, int t0, int nt, const std::vector<double> &xyz,
               std::vector<int> &tile_of)
{
    if (nt <= 1 || hi - lo <= 1) {
        for (int k = lo; k < hi; ++k) tile_of[nodes[k]] = t0;
        return;
    }
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int k = lo; k < hi; ++k)
        for (int c = 0; c < 3; ++c) {
            mn[c] = std::min(mn[c], xyz[3 * (size_t)nodes[k] + c]);
            mx[c] = std::max(mx[c], xyz[3 * (size_t)nodes[k] + c]);
        }
    int ax = 0;
    for (int c = 1; c < 3; ++c)
        if (mx[c] - mn[c] > mx[ax] - mn[ax]) ax = c;
    const int ntl = nt / 2;
    const int cut = lo + (int)((long long)(hi - lo) * ntl / nt);
    std::nth_element(nodes.begin() + lo, nodes.begin() + cut, nodes.begin() + hi, [&](int a, int b) {
        const double xa = xyz[3 * (size_t)a + ax], xb = xyz[3 * (size_t)b + ax];
        return xa != xb ? xa < xb : a < b;
    });
    rcb_tiles(nodes, lo, cut, t0, ntl, xyz, tile_of);
    rcb_tiles(nodes, cut, hi, t0 + ntl, nt - ntl, xyz, tile_of);
}

// Tile layout of the persistent SOR solve (k_sor_tiles): one spatial tile
// of nodes per SM, rows ordered tile by tile and colour by colour inside a
// tile, the column ids marked by colour order, and the tiles each tile
// depends on.  27-slot rows only; other layouts keep the colour kernels.
int build_tiles(fas_handle *h, const std::vector<double> &xyz, const std::vector<int> &bcol_host,
                const std::vector<int> &nslot_host, const std::vector<int> &rowof_host)
{
    if (h->slots != SLOTS || h->ncol > TILE_MAXCOL) return 0;
    const int nn = h->nnod, ncol = h->ncol, crow = crow_of(SLOTS);
    int occ = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sor_tiles<double>, 32 * tile_warps<double>(),
                                                     tile_smem_bytes<double>()));
    int occ32 = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ32, k_sor_tiles<float>, 32 * tile_warps<float>(),
                                                     tile_smem_bytes<float>()));
    if (occ < 1 || occ32 < 1) return 0;   // the colour kernels serve this device
    const int nt = std::min(h->nsm, std::max(1, nn / 64));
    std::vector<int> nodes(nn), tile_of(nn, 0);
    for (int i = 0; i < nn; ++i) nodes[i] = i;
    rcb_tiles(nodes, 0, nn, 0, nt, xyz, tile_of);
    // rows: tile, then colour, then node id
    std::vector<int> order(nn);
    for (int i = 0; i < nn; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        if (tile_of[a] != tile_of[b]) return tile_of[a] < tile_of[b];
        if (h->h_colour[a] != h->h_colour[b]) return h->h_colour[a] < h->h_colour[b];
        return a < b;
    });
    std::vector<int> tseg((size_t)nt * (ncol + 1), 0), tsrc(nn), tbcol((size_t)crow * nn, 0);
    {
        std::vector<int> cnt((size_t)nt * ncol, 0);
        for (int n = 0; n < nn; ++n) ++cnt[(size_t)tile_of[n] * ncol + h->h_colour[n]];
        int r = 0;
        for (int t = 0; t < nt; ++t) {
            for (int c = 0; c < ncol; ++c) {
                tseg[(size_t)t * (ncol + 1) + c] = r;
                r += cnt[(size_t)t * ncol + c];
            }
            tseg[(size_t)t * (ncol + 1) + ncol] = r;
        }
    }
    std::vector<std::vector<int>> adj(nt);
    for (int r = 0; r < nn; ++r) {
        const int n = order[r], p = rowof_host[n], t = tile_of[n];
        tsrc[r] = p;
        const int ns = nslot_host[p];
        for (int sl = 0; sl < ns; ++sl) {
            const int m = bcol_host[(size_t)p * crow + sl];
            unsigned w = (unsigned)m;
            if (h->h_colour[m] < h->h_colour[n]) w |= TILE_LOWER;
            tbcol[(size_t)r * crow + sl] = (int)w;
            if (tile_of[m] != t) adj[t].push_back(tile_of[m]);
        }
        tbcol[(size_t)r * crow + SLOTS] = ns;
    }
    std::vector<int> aptr(nt + 1, 0), alist;
    for (int t = 0; t < nt; ++t) {
        std::sort(adj[t].begin(), adj[t].end());
        adj[t].erase(std::unique(adj[t].begin(), adj[t].end()), adj[t].end());
        if ((int)adj[t].size() > TILE_MAXADJ) return 0;   // the colour kernels serve this mesh
        aptr[t + 1] = aptr[t] + (int)adj[t].size();
        alist.insert(alist.end(), adj[t].begin(), adj[t].end());
    }
    cudaStream_t s = h->stream;
    h->ntiles = nt;
    CKA(h->tseg.alloc(tseg.size()));
    CKA(h->tadj_ptr.alloc(aptr.size()));
    CKA(h->tadj.alloc(std::max<size_t>(alist.size(), 1)));
    CKA(h->tsrc.alloc(nn));
    CKA(h->tbcol.alloc(tbcol.size()));
    CKA(h->tprog.alloc(nt));
    CKA(h->tpart.alloc((size_t)TILE_SLOTS_SYNC * nt * 2));
    CKA(h->tsync.alloc(1));
    CKA(h->trdiag.alloc((size_t)3 * nn));
    CKA(h->sol_scr.alloc((size_t)3 * nn));
    CK(h->tseg.put(tseg.data(), tseg.size(), s));
    CK(h->tadj_ptr.put(aptr.data(), aptr.size(), s));
    if (!alist.empty()) CK(h->tadj.put(alist.data(), alist.size(), s));
    CK(h->tsrc.put(tsrc.data(), nn, s));
    CK(h->tbcol.put(tbcol.data(), tbcol.size(), s));
    CK(cudaStreamSynchronize(s));
    return 0;
}

// SHAPE_22's local-derivative table (src/fasolt/Shapef.f90:259-316),
// t[(g*3 + j)*20 + i] = dndn(j+1, i+1, g+1): the serendipity functions of
// the 20-node brick at the GP coordinate 0.57735, rounded to 6 decimals as
// the reference tabulates them.  Node order is ADDEL_20NQ's; GPs 1-4 lie
// anticlockwise from node 1 at zeta < 0, 5-8 above them.
std::vector<double> shape22_table()
{
    static const int loc[20][3] = {{-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {1, 0, -1}, {1, 1, -1},
                                   {0, 1, -1},   {-1, 1, -1}, {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0},
                                   {1, 1, 0},    {-1, 1, 0},  {-1, -1, 1}, {0, -1, 1},  {1, -1, 1},
                                   {1, 0, 1},    {1, 1, 1},   {0, 1, 1},   {-1, 1, 1},  {-1, 0, 1}};
    static const int gsign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
    const double a = 0.57735;
    std::vector<double> t(480);
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
            } else {                       // mid-edge along its zero coordinate
                const int z = !c[0] ? 0 : (!c[1] ? 1 : 2);
                const int z1 = (z + 1) % 3, z2 = (z + 2) % 3;
                const double f1 = 1 + q[z1] * c[z1], f2 = 1 + q[z2] * c[z2], e = 1 - q[z] * q[z];
                d[z] = 0.25 * (-2 * q[z]) * f1 * f2;
                d[z1] = 0.25 * e * c[z1] * f2;
                d[z2] = 0.25 * e * f1 * c[z2];
            }
            for (int j = 0; j < 3; ++j) t[(g * 3 + j) * 20 + i] = std::round(d[j] * 1e6) / 1e6;
        }
    }
    return t;
}

// SHAPE_21's local-derivative table (src/fasolt/Shapef.f90:104-189):
// 10-node tetrahedron, corners 1, 3, 5, 10 with volume coordinates L1..L4,
// mid-edge nodes 2 (1,3), 4 (3,5), 6 (1,5), 7 (1,10), 8 (3,10), 9 (5,10); GP
// g at L_g = (5 + 3 sqrt5)/20, the others (5 - sqrt5)/20.  The reference's
// local directions are L4, L2, L1 with L3 dependent: t[(g*3 + j)*10 + i] =
// dN_i/dL_p(j) - dN_i/dL3, rounded to 6 decimals -- the reference's table.
std::vector<double> shape21_table()
{
    static const int corner[10] = {0, -1, 1, -1, 2, -1, -1, -1, -1, 3};
    static const int mid[10][2] = {{-1, -1}, {0, 1}, {-1, -1}, {1, 2}, {-1, -1},
                                   {0, 2},   {0, 3}, {1, 3},   {2, 3}, {-1, -1}};
    static const int dir[3] = {3, 1, 0};
    const double r5 = std::sqrt(5.0), a = (5.0 + 3.0 * r5) / 20.0, b = (5.0 - r5) / 20.0;
    std::vector<double> t(120);
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
                t[(g * 3 + j) * 10 + i] = std::round((dNdL(i, dir[j]) - dNdL(i, 2)) * 1e6) / 1e6;
    }
    return t;
}

// SHAPE_23's local-derivative table (src/fasolt/Shapef.f90:360-485):
// 15-node wedge, base corners 1, 3, 5 and top corners 10, 12, 14 with area
// coordinates L1..L3 at zeta -1 / +1, base mid-edges 2, 4, 6, top 11, 13,
// 15, vertical 7, 8, 9.  GPs 1-3 at L_(g) = 2/3 (others 1/6), zeta =
// -1/sqrt3, GPs 4-6 above them.  Local directions L1, L2 (L3 dependent)
// and zeta; the serendipity wedge functions' derivatives rounded to 6
// decimals (60 of the reference's 270 tabulated entries differ from these
// by one unit in the sixth decimal).  t[(g*3 + j)*15 + i].
std::vector<double> shape23_table()
{
    static const int kind[15] = {0, 1, 0, 1, 0, 1, 2, 2, 2, 0, 1, 0, 1, 0, 1};
    static const int la[15] = {0, 0, 1, 1, 2, 2, 0, 1, 2, 0, 0, 1, 1, 2, 2};
    static const int lb[15] = {-1, 1, -1, 2, -1, 0, -1, -1, -1, -1, 1, -1, 2, -1, 0};
    static const int side[15] = {-1, -1, -1, -1, -1, -1, 0, 0, 0, 1, 1, 1, 1, 1, 1};
    std::vector<double> t(270);
    for (int g = 0; g < 6; ++g) {
        double L[3] = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
        L[g % 3] = 2.0 / 3.0;
        const double z = (g < 3 ? -1.0 : 1.0) / std::sqrt(3.0);
        auto dNdL = [&](int i, int p) {
            const double sd = side[i];
            if (kind[i] == 0)
                return la[i] == p ? 0.5 * (4.0 * L[p] - 1.0) * (1.0 + sd * z) - 0.5 * (1.0 - z * z) : 0.0;
            if (kind[i] == 1) {
                const double f = 2.0 * (1.0 + sd * z);
                return p == la[i] ? f * L[lb[i]] : (p == lb[i] ? f * L[la[i]] : 0.0);
            }
            return la[i] == p ? 1.0 - z * z : 0.0;
        };
        auto dNdz = [&](int i) {
            const double sd = side[i], La = L[la[i]];
            if (kind[i] == 0) return 0.5 * La * (2.0 * La - 1.0) * sd + La * z;
            if (kind[i] == 1) return 2.0 * La * L[lb[i]] * sd;
            return -2.0 * z * La;
        };
        for (int i = 0; i < 15; ++i) {
            t[(g * 3 + 0) * 15 + i] = std::round((dNdL(i, 0) - dNdL(i, 2)) * 1e6) / 1e6;
            t[(g * 3 + 1) * 15 + i] = std::round((dNdL(i, 1) - dNdL(i, 2)) * 1e6) / 1e6;
            t[(g * 3 + 2) * 15 + i] = std::round(dNdz(i) * 1e6) / 1e6;
        }
    }
    return t;
}

int create_impl(fas_handle *h, const fas_mesh_desc *Md, const fas_matl_desc *T, const fas_ctrl_desc *Cd)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FAS_E_NODEVICE;
    CK(cudaGetDevice(&h->dev));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, h->dev));
    if (prop.major != 10) return FAS_E_NODEVICE;
    h->nsm = prop.multiProcessorCount;
    CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CK(cudaFuncSetAttribute(k_sor_colour_tma<double, SLOTS, TMA_LPR>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem_bytes<double, SLOTS>()));
    CK(cudaFuncSetAttribute(k_sor_colour_tma<float, SLOTS, TMA_LPR32>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem_bytes<float, SLOTS>()));
    CK(cudaFuncSetAttribute(k_sor_colour_tma<double, SLOTS20, TMA_LPR81>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem_bytes<double, SLOTS20>()));
    CK(cudaFuncSetAttribute(k_sor_colour_tma<float, SLOTS20, TMA_LPR81_32>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem_bytes<float, SLOTS20>()));
    CK(cudaFuncSetAttribute(k_sor_colour_tma<float, SLOTS_SYM, TMA_LPR_SYM, true>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem_bytes<float, SLOTS_SYM>()));
    CK(cudaFuncSetAttribute(k_sor_tiles<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            tile_smem_bytes<double>()));
    CK(cudaFuncSetAttribute(k_sor_tiles<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            tile_smem_bytes<float>()));
    CK(cudaMallocHost((void **)&h->hc, sizeof(HostCtl)));
    CK(cudaEventCreate(&h->ev_t0));
    CK(cudaEventCreate(&h->ev_t1));
    cudaStream_t s = h->stream;

    if (Md->nlmnt < 0 || Md->nnod < 0 || Md->ngps <= 0) return FAS_E_ARG;
    h->nlmnt = Md->nlmnt;
    h->nnod = Md->nnod;
    h->ngps = Md->ngps;
    h->point_mode = h->nlmnt == 0;
    h->h_gp_iel.assign(h->ngps, 1);
    if (!h->point_mode) {
        if (!Md->le || !Md->lt || !Md->nd || !Md->np || !Md->ln || !Md->lg || !Md->ib) return FAS_E_ARG;
        const int ne = h->nlmnt;
        // one element family per mesh -- 8-node one-GP bricks (lt 12),
        // 10-node four-GP tetrahedra (lt 21), 20-node eight-GP bricks (lt
        // 22) or 15-node six-GP wedges (lt 23) -- plus 2-node tie elements
        // (lt 1-6)
        int lt0 = 0;
        for (int e = 0; e < ne && !lt0; ++e)
            if (Md->lt[e] >= 9) lt0 = Md->lt[e];
        if (lt0 != 12 && lt0 != 21 && lt0 != 22 && lt0 != 23) return FAS_E_ELTYPE;
        h->ltype = lt0;
        h->nn = lt0 == 12 ? 8 : (lt0 == 21 ? 10 : (lt0 == 22 ? 20 : 15));
        h->npg = lt0 == 12 ? 1 : (lt0 == 21 ? 4 : (lt0 == 22 ? 8 : 6));
        const int NN = h->nn, NG = h->npg;
        if (Md->ld_ln < NN || Md->ld_lg < NG || h->nnod < 1) return FAS_E_ARG;
        h->h_ln.assign((size_t)ne * NN, -1);
        h->h_gpe.assign((size_t)ne * NG, -1);
        h->h_le.assign(Md->le, Md->le + ne);
        std::vector<int> h_lt(Md->lt, Md->lt + ne);
        std::vector<int> gp_seen(h->ngps, 0);
        for (int e = 0; e < ne; ++e) {
            if (Md->lt[e] >= 1 && Md->lt[e] <= 6) {   // tie element (Elvals.f90:62-77)
                if (Md->nd[e] != 2 || Md->np[e] != 0) return FAS_E_ARG;
                for (int a = 0; a < 2; ++a) {
                    const int id = Md->ln[(size_t)e * Md->ld_ln + a];
                    if (id < 1 || id > h->nnod) return FAS_E_ARG;
                    h->h_ln[(size_t)e * NN + a] = id - 1;
                }
                if (h->h_ln[(size_t)e * NN] == h->h_ln[(size_t)e * NN + 1]) return FAS_E_ARG;
                continue;
            }
            if (Md->lt[e] != lt0) return FAS_E_ELTYPE;
            if (Md->nd[e] != NN || Md->np[e] != NG) return FAS_E_ARG;
            for (int a = 0; a < NN; ++a) {
                const int id = Md->ln[(size_t)e * Md->ld_ln + a];
                if (id < 1 || id > h->nnod) return FAS_E_ARG;
                h->h_ln[(size_t)e * NN + a] = id - 1;
            }
            for (int q = 0; q < NG; ++q) {
                const int g = Md->lg[(size_t)e * Md->ld_lg + q];
                if (g < 1 || g > h->ngps || gp_seen[g - 1]) return FAS_E_ARG;
                gp_seen[g - 1] = 1;
                h->h_gpe[(size_t)e * NG + q] = g - 1;
                h->h_gp_iel[g - 1] = Md->le[e];
            }
        }
        // mat_code the last brick leaves behind (ties run no DSTRSS)
        for (int e = ne - 1; e >= 0; --e)
            if (Md->lt[e] >= 9) {
                if (std::abs(Md->le[e]) >= 1) h->last_mat = std::abs(Md->le[e]);
                break;
            }
        h->h_ib.assign(Md->ib, Md->ib + h->nnod);
        // node -> element CSR (ascending element ids)
        h->ne_ptr.assign(h->nnod + 1, 0);
        for (int e = 0; e < ne; ++e)
            for (int a = 0; a < NN && h->h_ln[(size_t)e * NN + a] >= 0; ++a) h->ne_ptr[h->h_ln[(size_t)e * NN + a] + 1]++;
        h->maxadj = 1;
        for (int n = 0; n < h->nnod; ++n) {
            if (h->ne_ptr[n + 1] > MAXADJ) return FAS_E_RANGE;
            h->maxadj = std::max(h->maxadj, h->ne_ptr[n + 1]);
            h->ne_ptr[n + 1] += h->ne_ptr[n];
        }
        const int maxadj = h->maxadj;
        h->ne_list.resize(h->ne_ptr[h->nnod]);
        h->ne_locl.resize(h->ne_ptr[h->nnod]);
        std::vector<int> fill(h->ne_ptr.begin(), h->ne_ptr.end() - 1);
        for (int e = 0; e < ne; ++e)
            for (int a = 0; a < NN && h->h_ln[(size_t)e * NN + a] >= 0; ++a) {
                const int n = h->h_ln[(size_t)e * NN + a];
                h->ne_list[fill[n]] = e;
                h->ne_locl[fill[n]] = a;
                fill[n]++;
            }
        std::vector<int> lnT((size_t)NN * ne), gpeT((size_t)NG * ne), nee((size_t)maxadj * h->nnod, -1),
            nel((size_t)maxadj * h->nnod, 0), nec(h->nnod);
        for (int e = 0; e < ne; ++e) {
            for (int a = 0; a < NN; ++a) lnT[(size_t)a * ne + e] = h->h_ln[(size_t)e * NN + a];
            for (int q = 0; q < NG; ++q) gpeT[(size_t)q * ne + e] = h->h_gpe[(size_t)e * NG + q];
        }
        for (int n = 0; n < h->nnod; ++n) {
            nec[n] = h->ne_ptr[n + 1] - h->ne_ptr[n];
            for (int k = 0; k < nec[n]; ++k) {
                nee[(size_t)k * h->nnod + n] = h->ne_list[h->ne_ptr[n] + k];
                nel[(size_t)k * h->nnod + n] = h->ne_locl[h->ne_ptr[n] + k];
            }
        }
        if (NN != 8) {
            const std::vector<double> t = NN == 20 ? shape22_table() : (NN == 10 ? shape21_table() : shape23_table());
            h->wfac = NN == 20 ? 1.0 : (NN == 10 ? -0.0416667 : 0.16666667);
            CKA(h->dnq.alloc(t.size()));
            CK(h->dnq.put(t.data(), t.size(), s));
            CKA(h->gp_item.alloc(h->h_gpe.size()));
            CK(h->gp_item.put(h->h_gpe.data(), h->h_gpe.size(), s));
        }
        CKA(h->ln.alloc(lnT.size()));
        CKA(h->gpe.alloc(gpeT.size()));
        CKA(h->le.alloc(ne));
        CKA(h->lt.alloc(ne));
        CKA(h->ib.alloc(h->nnod));
        CKA(h->ne_elem.alloc(nee.size()));
        CKA(h->ne_loc.alloc(nel.size()));
        CKA(h->ne_cnt.alloc(nec.size()));
        CK(h->ln.put(lnT.data(), lnT.size(), s));
        CK(h->gpe.put(gpeT.data(), gpeT.size(), s));
        CK(h->le.put(h->h_le.data(), ne, s));
        CK(h->lt.put(h_lt.data(), ne, s));
        CK(h->ib.put(h->h_ib.data(), h->nnod, s));
        CK(h->ne_elem.put(nee.data(), nee.size(), s));
        CK(h->ne_loc.put(nel.data(), nel.size(), s));
        CK(h->ne_cnt.put(nec.data(), nec.size(), s));
        CK(cudaStreamSynchronize(s));
    } else {
        if (!Md->le) return FAS_E_ARG;
        for (int g = 0; g < h->ngps; ++g) h->h_gp_iel[g] = Md->le[g];
    }
    // ---- materials
    if (!T || (T->real_bytes != 4 && T->real_bytes != 8)) return FAS_E_ARG;
    const int rb = T->real_bytes, L = T->ld_ss, nm = T->nmatl;
    if (nm < 1 || nm > 12 || L < 1 || L > MAXSS) return FAS_E_ARG;
    std::vector<double> e(9 * nm, 0.0), ssang((size_t)nm * MAXSS, 0.0), ab((size_t)nm * MAXSS * 3, 0.0),
        an((size_t)nm * MAXSS * 3, 0.0), ampar((size_t)nm * MAXSS * 6, 0.0),
        sm((size_t)nm * MAXSS * MAXSS, 0.0);
    h->M = DevMat{};
    h->M.nmatl = nm;
    h->M.tld = MAXSS;
    h->M.sld = MAXSS * MAXSS;
    for (int m = 0; m < nm; ++m) {
        const int ns = T->nss[m];
        if (ns < 1 || ns > L) return FAS_E_ARG;
        h->M.ns[m] = ns;
        h->maxns = std::max(h->maxns, ns);
        for (int k = 0; k < 9; ++k) e[9 * m + k] = rdv(T->e, rb, (size_t)9 * m + k);
        double amx = -1e300;
        for (int i = 0; i < ns; ++i) {
            ssang[(size_t)m * MAXSS + i] = rdv(T->ssang, rb, (size_t)m * L + i);
            for (int k = 0; k < 3; ++k) {
                ab[((size_t)m * MAXSS + i) * 3 + k] = rdv(T->ab, rb, ((size_t)m * L + i) * 3 + k);
                an[((size_t)m * MAXSS + i) * 3 + k] = rdv(T->an, rb, ((size_t)m * L + i) * 3 + k);
            }
            for (int k = 0; k < 6; ++k)
                ampar[((size_t)m * MAXSS + i) * 6 + k] =
                    k < T->nmpar ? rdv(T->ampar, rb, ((size_t)m * L + i) * 10 + k) : 0.0;
            amx = std::max(amx, ampar[((size_t)m * MAXSS + i) * 6]);
            for (int j = 0; j < ns; ++j)
                sm[(size_t)m * MAXSS * MAXSS + (size_t)i * ns + j] =
                    rdv(T->smatrx, rb, (size_t)m * L * L + (size_t)j * L + i);
        }
        h->M.amax[m] = amx;
    }
    int ns_used = 0;   // the slip-system count shared by every GP's material, or -1
    for (int g = 0; g < h->ngps; ++g) {
        const int mc = std::abs(h->h_gp_iel[g]);
        if (mc < 1 || mc > nm) return FAS_E_ARG;
        const int ns = h->M.ns[mc - 1];
        ns_used = ns_used == 0 ? ns : (ns_used == ns ? ns : -1);
    }
    h->mixed_phases = ns_used < 0;
    h->ns_tmpl = h->maxns <= 12 ? 12 : (h->maxns <= 32 ? 32 : 60);
    // tables in shared memory (FAS_SMEM_TABLES builds) when they fit the
    // default 48 KB of a launch
    if (FAS_SMEM_TABLES && staged_doubles(nm, h->maxns) * 8 <= 48 * 1024) {
        h->M.stage_t = h->maxns;
        h->stage_bytes = (size_t)staged_doubles(nm, h->maxns) * 8;
    }
    h->nsvld = 3 + h->maxns;
    CKA(h->m_e.alloc(e.size()));
    CKA(h->m_ssang.alloc(ssang.size()));
    CKA(h->m_ab.alloc(ab.size()));
    CKA(h->m_an.alloc(an.size()));
    CKA(h->m_ampar.alloc(ampar.size()));
    CKA(h->m_sm.alloc(sm.size()));
    CK(h->m_e.put(e.data(), e.size(), s));
    CK(h->m_ssang.put(ssang.data(), ssang.size(), s));
    CK(h->m_ab.put(ab.data(), ab.size(), s));
    CK(h->m_an.put(an.data(), an.size(), s));
    CK(h->m_ampar.put(ampar.data(), ampar.size(), s));
    CK(h->m_sm.put(sm.data(), sm.size(), s));
    h->M.e = h->m_e.p; h->M.ssang = h->m_ssang.p; h->M.ab = h->m_ab.p; h->M.an = h->m_an.p;
    h->M.ampar = h->m_ampar.p; h->M.sm = h->m_sm.p;
    h->M.twinlim = T->twinlim;
    h->M.twinprob = T->twinprob;
    // ---- control
    if (!Cd || (Cd->real_bytes != 4 && Cd->real_bytes != 8) || Cd->ninc1 < 1 || !Cd->tiem) return FAS_E_ARG;
    const int cb = Cd->real_bytes;
    h->C.toler = Cd->toler; h->C.alpha = Cd->alpha; h->C.afactor = Cd->afactor; h->C.efix = Cd->efix;
    h->C.smale = Cd->smale; h->C.smalr = Cd->smalr; h->C.maxit = Cd->maxit; h->C.seed = Cd->twin_seed;
    h->C.tangent = (h->mode & FAS_MODE_TANGENT_CONSISTENT) ? 1 : 0;
    h->ninc1 = Cd->ninc1; h->nxs = Cd->nxs; h->nfs = Cd->nfs;
    if (h->nxs < 0 || h->nfs < 0 || (h->nxs > 0 && (!Cd->x_spec || Cd->ld_xs < h->nxs)) ||
        (h->nfs > 0 && (!Cd->f_spec || Cd->ld_xs < h->nfs)))
        return FAS_E_ARG;
    h->h_tiem.resize(h->ninc1);
    for (int i = 0; i < h->ninc1; ++i) h->h_tiem[i] = rdv(Cd->tiem, cb, i);
    std::vector<double> xs((size_t)h->ninc1 * std::max(h->nxs, 1) * 15, 0.0),
        fs((size_t)h->ninc1 * std::max(h->nfs, 1) * 3, 0.0);
    for (int i = 0; i < h->ninc1; ++i) {
        for (int j = 0; j < h->nxs; ++j)
            for (int k = 0; k < 15; ++k)
                xs[((size_t)i * h->nxs + j) * 15 + k] = rdv(Cd->x_spec, cb, ((size_t)i * Cd->ld_xs + j) * 15 + k);
        for (int j = 0; j < h->nfs; ++j)
            for (int k = 0; k < 3; ++k)
                fs[((size_t)i * h->nfs + j) * 3 + k] = rdv(Cd->f_spec, cb, ((size_t)i * Cd->ld_xs + j) * 3 + k);
    }
    CKA(h->xspec.alloc(xs.size()));
    CKA(h->fspec.alloc(fs.size()));
    CK(h->xspec.put(xs.data(), xs.size(), s));
    CK(h->fspec.put(fs.data(), fs.size(), s));
    // ---- state
    const size_t nd3 = 3 * (size_t)h->nnod, ng = h->ngps;
    CKA(h->x.alloc(nd3)); CKA(h->dx.alloc(nd3)); CKA(h->fc.alloc(nd3));
    CKA(h->ddx.alloc(nd3)); CKA(h->rhs.alloc(nd3));
    CKA(h->eps.alloc(ng)); CKA(h->dep.alloc(ng));
    CKA(h->st.alloc(6 * ng)); CKA(h->ep.alloc(6 * ng)); CKA(h->ds.alloc(6 * ng)); CKA(h->de.alloc(6 * ng));
    CKA(h->rt.alloc(3 * ng)); CKA(h->dr.alloc(3 * ng));
    CKA(h->sv.alloc((size_t)h->nsvld * ng)); CKA(h->dsv.alloc((size_t)h->nsvld * ng));
    CKA(h->srate.alloc((size_t)h->maxns * ng)); CKA(h->cumslip.alloc((size_t)h->maxns * ng));
    CKA(h->erepmd.alloc(ng)); CKA(h->ops.alloc(ng));
    CKA(h->timestwinned.alloc(ng)); CKA(h->twinsys.alloc(ng)); CKA(h->cp_iters.alloc(ng));
    CKA(h->gp_iel.alloc(ng));
    CK(h->gp_iel.put(h->h_gp_iel.data(), ng, s));
    for (DVec<double> *v : {&h->x, &h->dx, &h->fc, &h->ddx, &h->rhs, &h->eps, &h->dep, &h->st, &h->ep,
                            &h->ds, &h->de, &h->rt, &h->dr, &h->sv, &h->dsv, &h->srate, &h->cumslip,
                            &h->erepmd, &h->ops})
        CK(v->zero(s));
    CK(h->timestwinned.zero(s));
    CK(h->twinsys.zero(s));
    CK(h->cp_iters.zero(s));
    if (h->point_mode) {
        CKA(h->chi_pts.alloc(36 * ng));
        CK(h->chi_pts.zero(s));
    } else {
        CKA(h->rec.alloc((size_t)(3 * h->nn + 32) * h->nlmnt * h->npg));
        CK(h->rec.zero(s));
    }
    h->nr_nblk = (int)std::min<long long>(nblocks(std::max<long long>(h->nnod, h->ngps), 256), 1184);
    h->nr_nblk = std::max(h->nr_nblk, 1);
    CKA(h->part_nr.alloc((size_t)4 * h->nr_nblk));
    CKA(h->sums.alloc(8));
    CKA(h->ekey.alloc(2));
    CKA(h->flags.alloc(4));
    CKA(h->sorctl.alloc(1));
    CK(h->flags.zero(s));
    CK(cudaStreamSynchronize(s));
    return 0;
}

// ---------------------------------------------------------------- state I/O
int ensure_stage(fas_handle *h, size_t bytes)
{
    if (h->stage.n >= bytes) return 0;
    CKA(h->stage.alloc(bytes));
    return 0;
}

// caller array [n][ld] (element size rb): its first nk columns -> device
// SoA [nk][n] in FP64.  A pitched copy moves only the nk used columns.
int up_field(fas_handle *h, const void *src, int rb, int ld, int nk, int n, double *dst)
{
    if (!src || nk <= 0 || n <= 0) return 0;
    const size_t bytes = (size_t)n * nk * rb;
    int rc = ensure_stage(h, bytes);
    if (rc) return rc;
    if (ld == nk) CK(cudaMemcpyAsync(h->stage.p, src, bytes, cudaMemcpyHostToDevice, h->stream));
    else CK(cudaMemcpy2DAsync(h->stage.p, (size_t)nk * rb, src, (size_t)ld * rb, (size_t)nk * rb, n,
                              cudaMemcpyHostToDevice, h->stream));
    k_aos_to_soa<<<nblocks((long long)nk * n, 256), 256, 0, h->stream>>>(h->stage.p, rb, nk, nk, n, dst);
    LAUNCHED(h);
    return 0;
}

// device SoA [nk][n] -> the first nk columns of the caller's [n][ld] array;
// columns beyond nk are left untouched.
int down_field(fas_handle *h, void *dst, int rb, int ld, int nk, int n, const double *src)
{
    if (!dst || nk <= 0 || n <= 0) return 0;
    const size_t bytes = (size_t)n * nk * rb;
    int rc = ensure_stage(h, bytes);
    if (rc) return rc;
    k_soa_to_aos<<<nblocks((long long)nk * n, 256), 256, 0, h->stream>>>(src, nk, n, h->stage.p, rb, nk);
    LAUNCHED(h);
    if (ld == nk) CK(cudaMemcpyAsync(dst, h->stage.p, bytes, cudaMemcpyDeviceToHost, h->stream));
    else CK(cudaMemcpy2DAsync(dst, (size_t)ld * rb, h->stage.p, (size_t)nk * rb, (size_t)nk * rb, n,
                              cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int upload_impl(fas_handle *h, const fas_state_desc *S)
{
    if (!S || (S->real_bytes != 4 && S->real_bytes != 8)) return FAS_E_ARG;
    if (S->nsv < 0 || S->nsv > S->ld_sv) return FAS_E_ARG;
    const int rb = S->real_bytes, nd3 = 3 * h->nnod, ng = h->ngps;
    if (S->nsv > 0) h->nsv = std::min(S->nsv, h->nsvld);
    int rc;
#define UP(ptr, ld, nk, n, dst) if ((rc = up_field(h, ptr, rb, ld, nk, n, dst))) return rc
    UP(S->x, 1, 1, nd3, h->x.p);
    UP(S->dx, 1, 1, nd3, h->dx.p);
    UP(S->fc, 1, 1, nd3, h->fc.p);
    UP(S->ddx, 1, 1, nd3, h->ddx.p);
    UP(S->eps, 1, 1, ng, h->eps.p);
    UP(S->dep, 1, 1, ng, h->dep.p);
    UP(S->st, 6, 6, ng, h->st.p);
    UP(S->ep, 6, 6, ng, h->ep.p);
    UP(S->ds, 6, 6, ng, h->ds.p);
    UP(S->de, 6, 6, ng, h->de.p);
    UP(S->rt, 3, 3, ng, h->rt.p);
    UP(S->dr, 3, 3, ng, h->dr.p);
    const int nsvk = std::min(S->ld_sv, h->nsvld);
    UP(S->sv, S->ld_sv, nsvk, ng, h->sv.p);
    UP(S->dsv, S->ld_sv, nsvk, ng, h->dsv.p);
    if (S->srate || S->cumslip) {
        if (S->ld_slip < 1) return FAS_E_ARG;
        const int nsl = std::min(S->ld_slip, h->maxns);
        UP(S->srate, S->ld_slip, nsl, ng, h->srate.p);
        UP(S->cumslip, S->ld_slip, nsl, ng, h->cumslip.p);
    }
#undef UP
    if (S->timestwinned)
        CK(cudaMemcpyAsync(h->timestwinned.p, S->timestwinned, ng * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    if (S->twinsys)
        CK(cudaMemcpyAsync(h->twinsys.p, S->twinsys, ng * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    if (!h->have_state && !h->point_mode) {
        if (!S->x) return FAS_E_STATE;
        std::vector<double> xyz(nd3);
        for (int i = 0; i < nd3; ++i) xyz[i] = rdv(S->x, rb, i);
        rc = build_layout(h, xyz);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(h->stream));
    h->have_state = true;
    return 0;
}

int download_impl(fas_handle *h, const fas_state_desc *S)
{
    if (!S || (S->real_bytes != 4 && S->real_bytes != 8)) return FAS_E_ARG;
    const int rb = S->real_bytes, nd3 = 3 * h->nnod, ng = h->ngps;
    int rc;
#define DN(ptr, ld, nk, n, src) if ((rc = down_field(h, ptr, rb, ld, nk, n, src))) return rc
    DN(S->x, 1, 1, nd3, h->x.p);
    DN(S->dx, 1, 1, nd3, h->dx.p);
    DN(S->fc, 1, 1, nd3, h->fc.p);
    DN(S->ddx, 1, 1, nd3, h->ddx.p);
    DN(S->eps, 1, 1, ng, h->eps.p);
    DN(S->dep, 1, 1, ng, h->dep.p);
    DN(S->st, 6, 6, ng, h->st.p);
    DN(S->ep, 6, 6, ng, h->ep.p);
    DN(S->ds, 6, 6, ng, h->ds.p);
    DN(S->de, 6, 6, ng, h->de.p);
    DN(S->rt, 3, 3, ng, h->rt.p);
    DN(S->dr, 3, 3, ng, h->dr.p);
    const int nsvk = std::min(S->ld_sv, h->nsvld);
    DN(S->sv, S->ld_sv, nsvk, ng, h->sv.p);
    DN(S->dsv, S->ld_sv, nsvk, ng, h->dsv.p);
    if (S->srate || S->cumslip) {
        const int nsl = std::min(S->ld_slip, h->maxns);
        DN(S->srate, S->ld_slip, nsl, ng, h->srate.p);
        DN(S->cumslip, S->ld_slip, nsl, ng, h->cumslip.p);
    }
#undef DN
    if (S->timestwinned)
        CK(cudaMemcpyAsync(S->timestwinned, h->timestwinned.p, ng * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (S->twinsys)
        CK(cudaMemcpyAsync(S->twinsys, h->twinsys.p, ng * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

// ---------------------------------------------------------------- phases
// The work-sorted order of n items (elements whose GP is gp_of[i], or points
// when gp_of is null), from the operation counts of their last update; null
// when sorting is off.
const int *work_order(fas_handle *h, int n, const int *gp_of)
{
    if (!FAS_WORK_SORT || n <= 0) return nullptr;
    if ((int)h->work_order.n < n) {
        if (h->work_order.alloc(n) != cudaSuccess) return nullptr;
    }
    if (!h->work_hist.p && h->work_hist.alloc(WORK_BINS) != cudaSuccess) return nullptr;
    cudaStream_t s = h->stream;
    if (cudaMemsetAsync(h->work_hist.p, 0, WORK_BINS * sizeof(int), s) != cudaSuccess) return nullptr;
    k_work_hist<<<nblocks(n, 256), 256, 0, s>>>(n, gp_of, h->ops.p, h->work_hist.p);
    k_work_scan<<<1, WORK_BINS, 0, s>>>(h->work_hist.p);
    k_work_scatter<<<nblocks(n, 256), 256, 0, s>>>(n, gp_of, h->ops.p, h->work_hist.p, h->work_order.p);
    h->launches += 3;
    return h->work_order.p;
}

// Grid of a constitutive pass over n items (for_each_item).  With the
// queue (FAS_MODE_CP_QUEUE, meshes whose GPs' materials differ in their
// slip-system counts, or built in with FAS_CP_QUEUE=1): as many
// 128-thread CTAs as reside at once, at most one item per thread, and the
// queue head zeroed; otherwise one thread per item.
// CTA size of a constitutive pass over n items: 128 threads, halved (down
// to one warp) while that leaves fewer than two CTAs per SM, so that a
// small mesh spreads its long serial threads over every SM.  Items are
// independent, so the size changes no result.
int cp_block(const fas_handle *h, long long n)
{
    int bs = 128;
    while (bs > 32 && n < 2LL * h->nsm * bs) bs >>= 1;
    return bs;
}

template <typename K> unsigned cp_grid(fas_handle *h, K kern, long long n, int **queue, int *bs)
{
    *queue = nullptr;
    *bs = cp_block(h, n);
    const unsigned full = nblocks(n, *bs);
    if (!FAS_CP_QUEUE && !(h->mode & FAS_MODE_CP_QUEUE) && !h->mixed_phases) return full;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, *bs, h->stage_bytes) != cudaSuccess || occ < 1)
        return full;
    if (!h->cp_queue.p && h->cp_queue.alloc(1) != cudaSuccess) return full;
    if (cudaMemsetAsync(h->cp_queue.p, 0, sizeof(int), h->stream) != cudaSuccess) return full;
    *queue = h->cp_queue.p;
    return std::min<unsigned>(full, (unsigned)occ * (unsigned)h->nsm);
}

template <int NS> int launch_elem(fas_handle *h, int inc, int nit)
{
    Span sp(h, &h->P.ms_constitutive);
    if (h->nn != 8) {   // quadratic elements: one thread per (element, GP)
        auto go = [&](auto kern) {
            const long long nit_items = (long long)h->npg * h->nlmnt;
            const int *order = work_order(h, (int)nit_items, h->gp_item.p);
            int *queue = nullptr, bs = 128;
            const unsigned grid = cp_grid(h, kern, nit_items, &queue, &bs);
            kern<<<grid, bs, h->stage_bytes, h->stream>>>(h->mesh(), h->M, h->C, h->gp(), h->dnq.p, h->wfac, h->x.p, h->dx.p,
                                              h->rec.p, h->h_tiem[inc - 1], inc, nit, h->ekey.p, order, queue);
        };
        if (h->nn == 20)
            go(k_elemq<NS, 20, 8>);
        else if (h->nn == 10)
            go(k_elemq<NS, 10, 4>);
        else
            go(k_elemq<NS, 15, 6>);
    }
    else if (!(h->mode & FAS_MODE_CP_WARP)) {
        const int *order = work_order(h, h->nlmnt, h->gpe.p);
        int *queue = nullptr, bs = 128;
        const unsigned grid = cp_grid(h, k_elem<NS>, h->nlmnt, &queue, &bs);
        k_elem<NS><<<grid, bs, h->stage_bytes, h->stream>>>(
            h->mesh(), h->M, h->C, h->gp(), h->x.p, h->dx.p, h->rec.p, h->h_tiem[inc - 1], inc, nit, h->ekey.p,
            order, queue);
    }
    else
        k_elem_wc<(NS > 12 ? 32 : 12)><<<nblocks(32LL * h->nlmnt, 128), 128, 0, h->stream>>>(
            h->mesh(), h->M, h->C, h->gp(), h->x.p, h->dx.p, h->rec.p, h->h_tiem[inc - 1], inc, nit, h->ekey.p);
    sp.end();
    keep(h, sp);
    LAUNCHED(h);
    h->P.n_constitutive++;
    h->P.gp_updates += h->ngps;
    return 0;
}

// ELVALS (+ SUVALS when bc): element pass then row-gather assembly.
// Returns the first element's FAFERR code in element order, if any.
int ensure_fp32(fas_handle *h)
{
    if (!(h->mode & FAS_MODE_SOR_FP32) || h->blk32.p || h->point_mode) return 0;
    const size_t nd3 = 3 * (size_t)h->nnod;
    CKA(h->blk32.alloc((size_t)brow_of(h->slots) * h->nnod));
    CKA(h->sor_d.alloc(nd3));
    CKA(h->sor_d32.alloc(nd3));
    CKA(h->sor_r.alloc(nd3));
    CK(h->blk32.zero(h->stream));
    return 0;
}

// Symmetric FP32 rows (FAS_MODE_SOR_SYM with FAS_MODE_SOR_FP32, 27-slot
// rows), set up once per handle since the pattern is fixed: every
// off-diagonal block pair of the pattern is given to one of its two rows,
// in ascending node order, to the row that stores fewer blocks so far (13
// per row on the interior of a brick mesh).  A pattern that needs more than
// SLOTS_SYM - 1 stored blocks in some row, or is not symmetric, leaves the
// FP32 sweeps on the full FP32 rows (sym_state -1).
int ensure_sym(fas_handle *h)
{
    if (h->sym_state || !(h->mode & FAS_MODE_SOR_SYM) || !(h->mode & FAS_MODE_SOR_FP32) || h->slots != SLOTS ||
        h->point_mode)
        return 0;
    cudaStream_t s = h->stream;
    const int R = h->nnod;
    std::vector<int> bc((size_t)CROW * R), rowof(R);
    CK(cudaMemcpyAsync(bc.data(), h->bcol.p, bc.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(rowof.data(), h->rowof.p, (size_t)R * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<int> cnt(R, 0);
    std::vector<unsigned> mask(R, 0u);
    bool ok = true;
    for (int a = 0; a < R && ok; ++a) {
        const int r = rowof[a];
        const int *ca = &bc[(size_t)r * CROW];
        for (int sl = 1; sl < ca[SLOTS] && ok; ++sl) {
            const int m = ca[sl];
            if (m <= a) continue;
            if (cnt[m] < cnt[a]) {
                const int *cm = &bc[(size_t)rowof[m] * CROW];
                int s2 = -1;
                for (int t = 1; t < cm[SLOTS]; ++t)
                    if (cm[t] == a) s2 = t;
                if (s2 < 0) ok = false;
                else {
                    mask[rowof[m]] |= 1u << s2;
                    ++cnt[m];
                }
            } else {
                mask[r] |= 1u << sl;
                ++cnt[a];
            }
        }
    }
    for (int a = 0; a < R && ok; ++a) ok = cnt[a] <= SLOTS_SYM - 1;
    if (!ok) {
        h->sym_state = -1;
        return 0;
    }
    CKA(h->sym_mask.alloc(R));
    CKA(h->blk_sym.alloc((size_t)brow_of(SLOTS_SYM) * R));
    CKA(h->bcol_sym.alloc((size_t)crow_of(SLOTS_SYM) * R));
    CKA(h->sor_acc.alloc((size_t)4 * R));
    CK(h->sym_mask.put(mask.data(), R, s));
    CK(h->blk_sym.zero(s));
    CK(h->bcol_sym.zero(s));
    CK(h->sor_acc.zero(s));
    CK(cudaStreamSynchronize(s));
    h->sym_state = 1;
    return 0;
}

int elvals_impl(fas_handle *h, int inc, int nit, bool bc)
{
    cudaStream_t s = h->stream;
    if (int rc = ensure_fp32(h)) return rc;
    if (int rc = ensure_sym(h)) return rc;
    CK(cudaMemsetAsync(h->ekey.p, 0xFF, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(h->flags.p, 0, sizeof(int), s));
    int rc;
    switch (h->ns_tmpl) {
    case 12: rc = launch_elem<12>(h, inc, nit); break;
    case 32: rc = launch_elem<32>(h, inc, nit); break;
    default: {   // more than 32 systems: one thread per GP only
        const uint32_t m = h->mode;
        h->mode &= ~FAS_MODE_CP_WARP;
        rc = launch_elem<60>(h, inc, nit);
        h->mode = m;
    } break;
    }
    if (rc) return rc;
    {
        Span sp(h, &h->P.ms_assembly);
        const long long nthr = (long long)h->slots * h->nnod;   // thread (row, slot), row-major
        auto kern = h->nn == 20   ? k_assemble<20, 8>
                    : h->nn == 10 ? k_assemble<10, 4>
                    : h->nn == 15 ? k_assemble<15, 6>
                                  : k_assemble<8, 1>;
        kern<<<nblocks(nthr, 256), 256, 0, s>>>(
            h->mesh(), h->block(), h->rec.p, h->x.p, h->dx.p, h->fc.p, h->ddx.p,
            h->xspec.p + (size_t)(inc - 1) * std::max(h->nxs, 1) * 15,
            h->fspec.p + (size_t)(inc - 1) * std::max(h->nfs, 1) * 3, h->nxs, h->nfs, h->C.efix,
            bc ? 1 : 0, h->flags.p);
        sp.end();
        keep(h, sp);
        LAUNCHED(h);
        h->P.n_assembly++;
        h->blk32_fresh = h->block().blk32 != nullptr;
        h->P.assembly_bytes += h->asm_bytes;
    }
    CK(cudaMemcpyAsync(h->hc->ekey, h->ekey.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(h->hc->flags, h->flags.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    settle_spans(h);
    if (h->hc->ekey[0] != ~0ull) return (int)(h->hc->ekey[0] & 0xFFFFull);
    if (h->hc->flags[0]) return FAS_E_ARG;
    return 0;
}

int suvals_impl(fas_handle *h, int inc)
{
    cudaStream_t s = h->stream;
    CK(cudaMemsetAsync(h->flags.p, 0, sizeof(int), s));
    k_suvals<<<nblocks(h->nnod, 256), 256, 0, s>>>(
        h->mesh(), h->block(), h->rowof.p, h->x.p, h->dx.p, h->fc.p, h->ddx.p,
        h->xspec.p + (size_t)(inc - 1) * std::max(h->nxs, 1) * 15,
        h->fspec.p + (size_t)(inc - 1) * std::max(h->nfs, 1) * 3, h->nxs, h->nfs, h->C.efix, h->flags.p);
    LAUNCHED(h);
    CK(cudaMemcpyAsync(h->hc->flags, h->flags.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return h->hc->flags[0] ? FAS_E_ARG : 0;
}

// GRAPH_SWEEPS plain sweeps (ncol colour launches + the check, each)
// captured once into a CUDA graph: one graph launch replaces
// GRAPH_SWEEPS * (ncol + 1) kernel launches.
constexpr int GRAPH_SWEEPS = 4;

// Launch with programmatic stream serialisation: the kernel may start while
// the previous kernel of the stream drains and waits for it with
// pdl_wait() (the SOR colour and check kernels do).
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                Args... args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

// One colour-kernel launch of the row layout's instantiation (27 or 81
// slots), with programmatic serialisation when `pdl` is set.
template <typename T>
void launch_colour_kernel(fas_handle *h, int c, bool pdl, const T *blk, const double *rhs, double *sol,
                          const double *base, const double *rdiag, SorCtl *ctl, double *part,
                          float *sol32 = nullptr)
{
    const int p0 = h->col_start[c], p1 = h->col_start[c + 1];
    if (p1 <= p0) return;
    const bool f32 = sizeof(T) == 4;
    const int nblk = f32 ? h->sor_nblk32[c] : h->sor_nblk[c];
    const int boff = f32 ? h->sor_boff32[c] : h->sor_boff[c];
    const int ntot = f32 ? h->sor_nblk_tot32 : h->sor_nblk_tot;
    if (h->slots == SLOTS) {
        constexpr int LPR = sizeof(T) == 4 ? TMA_LPR32 : TMA_LPR;
        auto k = k_sor_colour_tma<T, SLOTS, LPR>;
        const unsigned nt = tma_threads<LPR, tma_rows<SLOTS, T>()>();
        if (pdl)
            launch_pdl(k, nblk, nt, tma_smem_bytes<T, SLOTS>(), h->stream, blk, h->bcol.p, p0,
                       p1, rhs, sol, base, rdiag, ctl, part, boff, ntot, sol32, (float *)nullptr);
        else
            k<<<nblk, nt, tma_smem_bytes<T, SLOTS>(), h->stream>>>(
                blk, h->bcol.p, p0, p1, rhs, sol, base, rdiag, ctl, part, boff, ntot, sol32, nullptr);
    } else {
        constexpr int LPR = tma_lpr<SLOTS20, T>();
        auto k = k_sor_colour_tma<T, SLOTS20, LPR>;
        const unsigned nt = tma_threads<LPR, tma_rows<SLOTS20, T>()>();
        if (pdl)
            launch_pdl(k, nblk, nt, tma_smem_bytes<T, SLOTS20>(), h->stream, blk, h->bcol.p, p0, p1,
                       rhs, sol, base, rdiag, ctl, part, boff, ntot, sol32, (float *)nullptr);
        else
            k<<<nblk, nt, tma_smem_bytes<T, SLOTS20>(), h->stream>>>(
                blk, h->bcol.p, p0, p1, rhs, sol, base, rdiag, ctl, part, boff, ntot, sol32, nullptr);
    }
}

// The whole solve in one CTA (meshes of at most SOR_SMALL_ROWS nodes).
void launch_sor_small(fas_handle *h, const BlockDev &B, SorCtl *ctl, double tolerl)
{
    if (h->slots == SLOTS)
        k_sor_small<1, 1024><<<1, 1024, 0, h->stream>>>(B, h->d_cstart.p, h->ncol, h->rhs.p, h->ddx.p, ctl,
                                                         tolerl, 1000);
    else
        k_sor_small<3, 256><<<1, 256, 0, h->stream>>>(B, h->d_cstart.p, h->ncol, h->rhs.p, h->ddx.p, ctl,
                                                       tolerl, 1000);
}

// One colour phase of the symmetric FP32 rows on the refinement's
// (residual, correction), with the iterate as base.
void launch_sym_colour(fas_handle *h, int c)
{
    const int p0 = h->col_start[c], p1 = h->col_start[c + 1];
    if (p1 <= p0) return;
    auto k = k_sor_colour_tma<float, SLOTS_SYM, TMA_LPR_SYM, true>;
    launch_pdl(k, h->sor_nblk_sym[c], tma_threads<TMA_LPR_SYM, TMA_ROWS_SYM>(), tma_smem_bytes<float, SLOTS_SYM>(),
               h->stream, (const float *)h->blk_sym.p, (const int *)h->bcol_sym.p, p0, p1, (const double *)h->sor_r.p,
               h->sor_d.p, (const double *)h->ddx.p, (const double *)nullptr, h->sorctl.p, h->part_sor.p,
               h->sor_boff_sym[c], h->sor_nblk_tot_sym, h->sor_d32.p, h->sor_acc.p);
}

// One colour phase: FP64 blocks on (rhs, sol), or the FP32 copy on the
// refinement's (residual, correction) with the iterate as base.
void launch_colour(fas_handle *h, int c, bool fp32)
{
    if (fp32 && h->sym_on)
        launch_sym_colour(h, c);
    else if (fp32)
        launch_colour_kernel<float>(h, c, true, h->blk32.p, h->sor_r.p, h->sor_d.p, h->ddx.p, nullptr,
                                    h->sorctl.p, h->part_sor.p, h->sor_d32.p);
    else
        launch_colour_kernel<double>(h, c, true, h->blk.p, h->rhs.p, h->ddx.p, nullptr,
                                     FAS_SOR_RCP ? h->rdiag.p : nullptr, h->sorctl.p, h->part_sor.p);
}

void launch_check(fas_handle *h, double tolerl, bool fp32 = false)
{
    launch_pdl(k_sor_check, 1, 1024, 0, h->stream, h->part_sor.p,
               fp32 ? (h->sym_on ? h->sor_nblk_tot_sym : h->sor_nblk_tot32) : h->sor_nblk_tot, h->sorctl.p, tolerl);
}

// End of one refinement cycle of the FP32 form: x += d, d = 0, the FP32
// mirror and (symmetric rows) the accumulators cleared.
void launch_fold(fas_handle *h)
{
    const long long nd3 = 3LL * h->nnod, nacc = h->sym_on ? 4LL * h->nnod : 0;
    k_fold<<<nblocks(std::max(nd3, nacc), 256), 256, 0, h->stream>>>((int)nd3, h->ddx.p, h->sor_d.p, h->sor_d32.p,
                                                                      h->sor_acc.p, (int)nacc);
}

// Start of an FP32 solve: whether its sweeps take the symmetric rows, and
// if so their packing from the assembled FP64 rows and zero accumulators
// (the correction starts at zero).
void sym_begin(fas_handle *h, const BlockDev &B)
{
    h->sym_on = h->sym_state == 1 && (h->mode & FAS_MODE_SOR_SYM) && (h->mode & FAS_MODE_SOR_FP32);
    if (!h->sym_on) return;
    k_sym_pack<<<nblocks(32LL * h->nnod, 256), 256, 0, h->stream>>>(B, h->sym_mask.p, h->blk_sym.p, h->bcol_sym.p);
    cudaMemsetAsync(h->sor_acc.p, 0, (size_t)4 * h->nnod * sizeof(float), h->stream);
}

void launch_plain_sweep(fas_handle *h, const BlockDev &B, double tolerl)
{
    (void)B;
    for (int c = 0; c < h->ncol; ++c) launch_colour(h, c, false);
    launch_check(h, tolerl);
}

int ensure_sor_graph(fas_handle *h, const BlockDev &B, double tolerl)
{
    if (h->sor_graph) return 0;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < GRAPH_SWEEPS; ++it) launch_plain_sweep(h, B, tolerl);
    CK(cudaStreamEndCapture(h->stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&h->sor_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->sor_graph = nullptr;
        return FAS_E_CUDA;
    }
    return 0;
}

// One refinement cycle of the FP32 form: refine_every FP32 sweeps on the
// correction, the fold into the iterate and the FP64 residual.
void launch_fp32_cycle(fas_handle *h, const BlockDev &B, double tolerl, int sweeps)
{
    const size_t nd3 = 3 * (size_t)h->nnod;
    const unsigned rblk = (unsigned)std::min<long long>(nblocks(h->nnod, 8), (long long)h->nsm * 8);
    for (int it = 0; it < sweeps; ++it) {
        for (int c = 0; c < h->ncol; ++c) launch_colour(h, c, true);
        launch_check(h, tolerl, true);
    }
    launch_fold(h);
    k_residual<<<rblk, 256, 0, h->stream>>>(B, h->rhs.p, h->ddx.p, h->sor_r.p, h->sorctl.p);
}

int ensure_fp32_graph(fas_handle *h, const BlockDev &B, double tolerl)
{
    if (h->sor32_graph && h->sor32_graph_sym == h->sym_on) return 0;
    if (h->sor32_graph) cudaGraphExecDestroy(h->sor32_graph);
    h->sor32_graph = nullptr;
    h->sor32_graph_sym = h->sym_on;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    launch_fp32_cycle(h, B, tolerl, h->refine_every);
    CK(cudaStreamEndCapture(h->stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&h->sor32_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->sor32_graph = nullptr;
        return FAS_E_CUDA;
    }
    return 0;
}

// One cooperative launch of the persistent tile solve: at most maxsw
// sweeps from sol0, sweep counts reported from sweep_base on.
template <typename T>
int launch_tiles(fas_handle *h, const T *blk, const double *rhs, const double *base, const double *rdiag,
                 double *sol0, int maxsw, int sweep_base, double tolerl)
{
    cudaStream_t s = h->stream;
    CK(h->tprog.zero(s));
    CK(h->tsync.zero(s));
    TileArgs<T> a;
    a.blk = blk;
    a.bcol = h->tbcol.p;
    a.tseg = h->tseg.p;
    a.tadj_ptr = h->tadj_ptr.p;
    a.tadj = h->tadj.p;
    a.rhs = rhs;
    a.base = base;
    a.rdiag = rdiag;
    a.sol0 = sol0;
    a.sol1 = h->sol_scr.p;
    a.progress = h->tprog.p;
    a.part = h->tpart.p;
    a.sync = h->tsync.p;
    a.ctl = h->sorctl.p;
    a.ntiles = h->ntiles;
    a.ncol = h->ncol;
    a.maxsw = maxsw;
    a.sweep_base = sweep_base;
    a.tolerl = tolerl;
    a.keep_rows = h->tile_keep_rows;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(h->ntiles);
    cfg.blockDim = dim3(32 * tile_warps<T>());
    cfg.dynamicSmemBytes = tile_smem_bytes<T>();
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k_sor_tiles<T>, a));
    LAUNCHED(h);
    return 0;
}

// FACSLS by the persistent tile kernel: the assembled rows are copied into
// the tile layout, then one launch runs the FP64 solve to convergence; the
// FP32 form runs refinement cycles of refine_every sweeps (one launch, the
// fold and the FP64 residual each).  Leaves the verdict in h->hc->sor.
int facsls_tiles(fas_handle *h, const BlockDev &B, double tolerl, bool fp32)
{
    cudaStream_t s = h->stream;
    const int rows = h->nnod;
    const size_t nd3 = 3 * (size_t)rows;
    const unsigned pblk = (unsigned)std::min<long long>(nblocks(rows, 8), (long long)h->nsm * 8);
    if (!fp32) {
        if (!h->tblk64.p) CKA(h->tblk64.alloc((size_t)BROW * rows));
        k_tile_pack<double><<<pblk, 256, 0, s>>>(B, h->tsrc.p, rows, h->tblk64.p, h->trdiag.p);
        LAUNCHED(h);
        Span sp(h, &h->P.ms_sor_colour);
        const int rc = launch_tiles<double>(h, h->tblk64.p, h->rhs.p, nullptr, FAS_SOR_RCP ? h->trdiag.p : nullptr,
                                            h->ddx.p, 1000, 0, tolerl);
        sp.end();
        keep(h, sp);
        if (rc) return rc;
        CK(cudaMemcpyAsync(&h->hc->sor, h->sorctl.p, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        return 0;
    }
    if (!h->tblk32.p) CKA(h->tblk32.alloc((size_t)BROW * rows));
    k_tile_pack<float><<<pblk, 256, 0, s>>>(B, h->tsrc.p, rows, h->tblk32.p, nullptr);
    LAUNCHED(h);
    // x (= ddx) starts at 0, so the first residual is rhs itself
    CK(cudaMemcpyAsync(h->sor_r.p, h->rhs.p, nd3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(h->sor_d.p, 0, nd3 * sizeof(double), s));
        CK(cudaMemsetAsync(h->sor_d32.p, 0, nd3 * sizeof(float), s));
    const int m = h->refine_every;
    const unsigned rblk = (unsigned)std::min<long long>(nblocks(rows, 8), (long long)h->nsm * 8);
    int done = 0, outer_per_chunk = 1;
    while (done < 1000) {
        for (int o = 0; o < outer_per_chunk && done < 1000; ++o) {
            const int k = std::min(m, 1000 - done);
            Span sp(h, &h->P.ms_sor_colour);
            const int rc = launch_tiles<float>(h, h->tblk32.p, h->sor_r.p, h->ddx.p, nullptr, h->sor_d.p, k, done,
                                               tolerl);
            sp.end();
            keep(h, sp);
            if (rc) return rc;
            k_fold<<<nblocks((long long)nd3, 256), 256, 0, s>>>((int)nd3, h->ddx.p, h->sor_d.p, h->sor_d32.p);
            LAUNCHED(h);
            k_residual<<<rblk, 256, 0, s>>>(B, h->rhs.p, h->ddx.p, h->sor_r.p, h->sorctl.p);
            LAUNCHED(h);
            done += k;
        }
        CK(cudaMemcpyAsync(&h->hc->sor, h->sorctl.p, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (h->hc->sor.conv || h->hc->sor.fault) break;
        outer_per_chunk = std::min(outer_per_chunk * 2, 4);
    }
    return 0;
}

// FACSLS: rhs <- ddx, ddx <- 0, multicolour SOR sweeps until the relative
// change drops below toler^2 or 1000 sweeps (Stif_sol.f90:173-213).
int facsls_impl(fas_handle *h, int *sweeps, double *error)
{
    cudaStream_t s = h->stream;
    const size_t nd3 = 3 * (size_t)h->nnod;
    CK(cudaMemcpyAsync(h->rhs.p, h->ddx.p, nd3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(h->ddx.p, 0, nd3 * sizeof(double), s));
    CK(cudaMemsetAsync(h->ekey.p + 1, 0xFF, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(h->sorctl.p, 0, sizeof(SorCtl), s));
    BlockDev B = h->block();
    k_diag_check<<<nblocks(h->nnod, 256), 256, 0, s>>>(B, h->ekey.p + 1);
    LAUNCHED(h);
    CK(cudaMemcpyAsync(&h->hc->ekey[1], h->ekey.p + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h->hc->ekey[1] != ~0ull) return 903;
    const double tolerl = h->C.toler * h->C.toler;
    const bool small = h->sor_small && !(h->mode & FAS_MODE_SOR_GRID);
    const bool tiles = !small && h->ntiles > 0 && (h->mode & FAS_MODE_SOR_TILES);
    if (!small && !tiles && FAS_SOR_RCP) {
        k_rdiag<<<nblocks(h->nnod, 256), 256, 0, s>>>(B, h->rdiag.p);
        LAUNCHED(h);
    }
    if (small) {
        Span sp(h, &h->P.ms_sor_colour);
        launch_sor_small(h, B, h->sorctl.p, tolerl);
        sp.end();
        keep(h, sp);
        LAUNCHED(h);
        CK(cudaMemcpyAsync(&h->hc->sor, h->sorctl.p, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    int done = small ? 1000 : 0, chunk = 4;
    const bool fp32 = !small && (h->mode & FAS_MODE_SOR_FP32) && h->blk32.p && h->blk32_fresh;
    if (tiles) {
        const int rc = facsls_tiles(h, B, tolerl, fp32);
        if (rc) return rc;
        done = 1000;
    }
    h->sym_on = false;
    if (fp32 && !tiles) {
        // x (= ddx) starts at 0, so the first residual is rhs itself
        CK(cudaMemcpyAsync(h->sor_r.p, h->rhs.p, nd3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemsetAsync(h->sor_d.p, 0, nd3 * sizeof(double), s));
        CK(cudaMemsetAsync(h->sor_d32.p, 0, nd3 * sizeof(float), s));
        sym_begin(h, B);
        CK(cudaGetLastError());
        const int m = h->refine_every;
        const unsigned rblk = (unsigned)std::min<long long>(nblocks(h->nnod, 8), (long long)h->nsm * 8);
        const bool graph32 = h->prof < 2 && ensure_fp32_graph(h, B, tolerl) == 0;
        int outer_per_chunk = 1;
        while (done < 1000) {
            for (int o = 0; o < outer_per_chunk && done < 1000; ++o) {
                const int k = std::min(m, 1000 - done);
                if (graph32 && k == m) {
                    CK(cudaGraphLaunch(h->sor32_graph, s));
                    h->launches += (int64_t)k * (h->ncol + 1) + 2;
                    done += k;
                    continue;
                }
                for (int it = 0; it < k; ++it) {
                    for (int c = 0; c < h->ncol; ++c) {
                        if (h->col_start[c + 1] <= h->col_start[c]) continue;
                        Span sp(h, &h->P.ms_sor_colour);
                        launch_colour(h, c, true);
                        sp.end();
                        keep(h, sp);
                        LAUNCHED(h);
                    }
                    launch_check(h, tolerl, true);
                    LAUNCHED(h);
                }
                done += k;
                launch_fold(h);
                LAUNCHED(h);
                k_residual<<<rblk, 256, 0, s>>>(B, h->rhs.p, h->ddx.p, h->sor_r.p, h->sorctl.p);
                LAUNCHED(h);
            }
            CK(cudaMemcpyAsync(&h->hc->sor, h->sorctl.p, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (h->hc->sor.conv) break;
            outer_per_chunk = std::min(outer_per_chunk * 2, 4);
        }
        done = 1000;
    }
    const bool graph = h->prof < 2 && done < 1000 && ensure_sor_graph(h, B, tolerl) == 0;
    while (done < 1000) {
        const int k = std::min(chunk, 1000 - done);
        if (graph && k % GRAPH_SWEEPS == 0) {
            for (int it = 0; it < k; it += GRAPH_SWEEPS) CK(cudaGraphLaunch(h->sor_graph, s));
            h->launches += (int64_t)k * (h->ncol + 1);
        } else for (int it = 0; it < k; ++it) {
            for (int c = 0; c < h->ncol; ++c) {
                if (h->col_start[c + 1] <= h->col_start[c]) continue;
                Span sp(h, &h->P.ms_sor_colour);
                launch_colour(h, c, false);
                sp.end();
                keep(h, sp);
                LAUNCHED(h);
            }
            launch_check(h, tolerl);
            LAUNCHED(h);
        }
        done += k;
        CK(cudaMemcpyAsync(&h->hc->sor, h->sorctl.p, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (h->hc->sor.conv) break;
        chunk = std::min(chunk * 2, 64);
    }
    settle_spans(h);
    const int nsw = h->hc->sor.sweeps;
    h->P.sor_sweeps += nsw;
    h->P.n_sor_colour += small ? 1 : (int64_t)nsw * h->ncol;
    double bytes = 0.0;
    for (double b : h->col_bytes) bytes += b;
    if (fp32) {   // FP32 blocks: 36 + 4 bytes per slot, plus the xs read
        bytes = 0.0;
        for (double b : h->col_bytes32) bytes += b;
    }
    if (fp32 && h->sym_on)   // symmetric rows as streamed: values and column ids
        bytes = (double)h->nnod * (brow_of(SLOTS_SYM) + crow_of(SLOTS_SYM)) * 4.0;
    h->P.sor_bytes += bytes * nsw;
    if (sweeps) *sweeps = nsw;
    if (error) *error = h->hc->sor.err;
    if (h->hc->sor.fault) return FAS_E_TIMEOUT;
    if (h->hc->sor.err > 10.0 * tolerl) return 904;
    return 0;
}

// One pass of NRITER's loop body (Stif_sol.f90:32-77): ELVALS + SUVALS,
// the residual norm, FACSLS, the damping factor and the correction of x and
// dx.  *more = the reference's loop condition for another pass.
int nr_step_impl(fas_handle *h, int inc, int nit, fas_iter_report *r, bool *more)
{
    cudaStream_t s = h->stream;
    const int ndof = 3 * h->nnod;
    int rc = elvals_impl(h, inc, nit, true);
    if (rc) return rc;
    int sweeps = 0;
    double serr = 0.0;
    rc = facsls_impl(h, &sweeps, &serr);
    if (rc) return rc;
    k_nr_norms<<<h->nr_nblk, 256, 0, s>>>(h->nnod, h->ngps, h->ib.p, h->rhs.p, h->dx.p, h->ddx.p,
                                          h->erepmd.p, h->part_nr.p, h->nr_nblk);
    LAUNCHED(h);
    k_final_sum<4><<<1, 1024, 0, s>>>(h->part_nr.p, h->nr_nblk, h->sums.p);
    LAUNCHED(h);
    CK(cudaMemcpyAsync(h->hc->sums, h->sums.p, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const double sfc = std::sqrt(h->hc->sums[0]);
    const double errdx = std::sqrt(h->hc->sums[1]);
    const double erddx = std::sqrt(h->hc->sums[2]);
    const double sdx = errdx == 0.0 ? h->C.toler : erddx / errdx;
    const double alp2 = 1.0 / (1.0 + h->C.alpha * sdx);
    if (r) {
        r->nit = nit;
        r->sor_sweeps = sweeps;
        r->sdx = sdx;
        r->sfc = sfc;
        r->cp_err = h->hc->sums[3] / (double)h->ngps;
        r->alp2 = alp2;
        r->sor_error = serr;
    }
    k_nr_update<<<nblocks(ndof, 256), 256, 0, s>>>(ndof, alp2, h->ddx.p, h->x.p, h->dx.p);
    LAUNCHED(h);
    if (more) *more = (sdx >= h->C.toler) && (nit < h->C.maxit);
    return 0;
}

// NRITER's tail after the loop (Stif_sol.f90:80-84): cumslip += srate *
// tiem(inc) over nss(mat_code) of the last element evaluated.
int nr_finish_impl(fas_handle *h, int inc)
{
    const int nsc = h->M.ns[h->last_mat - 1];
    k_cumslip<<<nblocks(h->ngps, 256), 256, 0, h->stream>>>(h->gp(), nsc, h->h_tiem[inc - 1]);
    LAUNCHED(h);
    CK(cudaStreamSynchronize(h->stream));
    return 0;
}

// ---------------------------------------------------------------- graphed NRITER
// Creates a condition in the graph that the stream `s` is capturing into.
int make_condition(cudaStream_t s, unsigned default_value, bool assign_default, cudaGraphConditionalHandle *hc)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr));
    if (st != cudaStreamCaptureStatusActive || !g) return FAS_E_STATE;
    CK(cudaGraphConditionalHandleCreate(hc, g, default_value, assign_default ? cudaGraphCondAssignDefault : 0));
    return 0;
}

// Adds a conditional node (a while loop or an if) on condition `hc` at the
// current end of the capture on `s`, and returns its body graph.
int add_conditional(cudaStream_t s, cudaGraphConditionalHandle hc, cudaGraphConditionalNodeType type,
                    cudaGraph_t *body)
{
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps));
    if (st != cudaStreamCaptureStatusActive || !g) return FAS_E_STATE;
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.handle = hc;
    prm.conditional.type = type;
    prm.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, ndeps, &prm));
    CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    *body = prm.conditional.phGraph_out[0];
    return 0;
}

// Captures what `issue` launches on h->stream into `body`, on the side
// stream `side` (h->stream points at it meanwhile).
template <typename F> int capture_into(fas_handle *h, cudaStream_t &side, cudaGraph_t body, F issue)
{
    std::swap(h->stream, side);
    int rc = 0;
    cudaError_t e = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = issue();
        cudaGraph_t done = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(h->stream, &done);
        if (e2 != cudaSuccess) e = e2;
    }
    std::swap(h->stream, side);
    if (rc) return rc;
    return e == cudaSuccess ? 0 : FAS_E_CUDA;
}

// One Newton iteration (nr_step_impl) with no host read: ELVALS + SUVALS,
// FACSLS's prologue, the sweeps in a conditional node that runs only when
// nothing failed so far (a while loop of GRAPH_SWEEPS sweeps per pass, or
// the one-CTA solve under an if), the norms, the decision and the
// correction.  Issued on h->stream while it captures the body of the
// increment graph's Newton loop `hnr`.
int capture_nr_body(fas_handle *h, int inc, cudaGraphConditionalHandle hnr)
{
    const size_t nd3 = 3 * (size_t)h->nnod;
    const int ndof = (int)nd3;
    const int64_t l0 = h->launches;
    CK(cudaMemsetAsync(h->ekey.p, 0xFF, sizeof(unsigned long long), h->stream));
    CK(cudaMemsetAsync(h->flags.p, 0, sizeof(int), h->stream));
    int rc;
    switch (h->ns_tmpl) {
    case 12: rc = launch_elem<12>(h, inc, 0); break;
    case 32: rc = launch_elem<32>(h, inc, 0); break;
    default: {
        const uint32_t m = h->mode;
        h->mode &= ~FAS_MODE_CP_WARP;
        rc = launch_elem<60>(h, inc, 0);
        h->mode = m;
    } break;
    }
    if (rc) return rc;
    cudaStream_t s = h->stream;
    {
        const long long nthr = (long long)h->slots * h->nnod;
        auto kern = h->nn == 20   ? k_assemble<20, 8>
                    : h->nn == 10 ? k_assemble<10, 4>
                    : h->nn == 15 ? k_assemble<15, 6>
                                  : k_assemble<8, 1>;
        kern<<<nblocks(nthr, 256), 256, 0, s>>>(
            h->mesh(), h->block(), h->rec.p, h->x.p, h->dx.p, h->fc.p, h->ddx.p,
            h->xspec.p + (size_t)(inc - 1) * std::max(h->nxs, 1) * 15,
            h->fspec.p + (size_t)(inc - 1) * std::max(h->nfs, 1) * 3, h->nxs, h->nfs, h->C.efix, 1, h->flags.p);
        LAUNCHED(h);
    }
    CK(cudaMemcpyAsync(h->rhs.p, h->ddx.p, nd3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(h->ddx.p, 0, nd3 * sizeof(double), s));
    CK(cudaMemsetAsync(h->ekey.p + 1, 0xFF, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(h->sorctl.p, 0, sizeof(SorCtl), s));
    const BlockDev B = h->block();
    k_diag_check<<<nblocks(h->nnod, 256), 256, 0, s>>>(B, h->ekey.p + 1);
    LAUNCHED(h);
    const double tolerl = h->C.toler * h->C.toler;
    const bool small = h->sor_small && !(h->mode & FAS_MODE_SOR_GRID);
    if (!small && FAS_SOR_RCP) {
        k_rdiag<<<nblocks(h->nnod, 256), 256, 0, s>>>(B, h->rdiag.p);
        LAUNCHED(h);
    }
    // the FP32 solve (facsls_impl): cycles of refine_every sweeps on the
    // FP32 copy, each closed by the fold and the FP64 residual
    const bool fp32 = !small && (h->mode & FAS_MODE_SOR_FP32) && h->blk32.p;
    const int m = h->refine_every, full = (1000 / m) * m, rest = 1000 - full;
    h->sym_on = false;
    if (fp32) {
        CK(cudaMemcpyAsync(h->sor_r.p, h->rhs.p, nd3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        CK(cudaMemsetAsync(h->sor_d.p, 0, nd3 * sizeof(double), s));
        CK(cudaMemsetAsync(h->sor_d32.p, 0, nd3 * sizeof(float), s));
        sym_begin(h, B);
        CK(cudaGetLastError());
    }
    cudaGraphConditionalHandle hsor, hlast = 0;
    if (int r = make_condition(s, 0, false, &hsor)) return r;
    if (fp32)
        if (int r = make_condition(s, 0, false, &hlast)) return r;
    k_graph_sor_begin<<<1, 32, 0, s>>>(h->ekey.p, h->flags.p, hsor, hlast, fp32 ? 1 : 0);
    LAUNCHED(h);
    int ncolours = 0;
    for (int c = 0; c < h->ncol; ++c) ncolours += h->col_start[c + 1] > h->col_start[c];
    cudaGraph_t sbody = nullptr;
    if (int r = add_conditional(s, hsor, small ? cudaGraphCondTypeIf : cudaGraphCondTypeWhile, &sbody)) return r;
    rc = capture_into(h, h->cap3, sbody, [&]() -> int {
        if (small) {
            launch_sor_small(h, B, h->sorctl.p, tolerl);
            LAUNCHED(h);
            return 0;
        }
        if (fp32) {
            launch_fp32_cycle(h, B, tolerl, m);
            k_sor_cycle_cond<<<1, 32, 0, h->stream>>>(h->sorctl.p, full, rest, hsor, hlast);
            h->g_pass_launches = (int64_t)m * (ncolours + 1) + 3;
        } else {
            for (int it = 0; it < GRAPH_SWEEPS; ++it) {
                for (int c = 0; c < h->ncol; ++c) launch_colour(h, c, false);
                launch_pdl(k_sor_check_cond, 1, 1024, 0, h->stream, h->part_sor.p, h->sor_nblk_tot,
                           h->sorctl.p, tolerl, 1000, hsor);
            }
            h->g_pass_launches = (int64_t)GRAPH_SWEEPS * (ncolours + 1);
        }
        CK(cudaGetLastError());
        return 0;
    });
    if (rc) return rc;
    if (fp32 && rest > 0) {   // the shorter last cycle
        cudaGraph_t lbody = nullptr;
        if (int r = add_conditional(s, hlast, cudaGraphCondTypeIf, &lbody)) return r;
        rc = capture_into(h, h->cap3, lbody, [&]() -> int {
            launch_fp32_cycle(h, B, tolerl, rest);
            CK(cudaGetLastError());
            return 0;
        });
        if (rc) return rc;
    }
    k_nr_norms<<<h->nr_nblk, 256, 0, s>>>(h->nnod, h->ngps, h->ib.p, h->rhs.p, h->dx.p, h->ddx.p, h->erepmd.p,
                                          h->part_nr.p, h->nr_nblk);
    LAUNCHED(h);
    k_final_sum<4><<<1, 1024, 0, s>>>(h->part_nr.p, h->nr_nblk, h->sums.p);
    LAUNCHED(h);
    k_nr_decide<<<1, 32, 0, s>>>(h->sums.p, h->ngps, h->ekey.p, h->flags.p, h->sorctl.p, h->C.toler, h->C.alpha,
                                 h->C.maxit, tolerl, h->nrdev.p, h->nrrep.p, (int)h->nrrep.n, hnr);
    LAUNCHED(h);
    k_nr_update_dev<<<nblocks(ndof, 256), 256, 0, s>>>(ndof, h->nrdev.p, h->ddx.p, h->x.p, h->dx.p);
    LAUNCHED(h);
    h->g_body_launches = h->launches - l0;
    return 0;
}

// The graph of NRITER for increment `inc`, built on first use and kept:
// the loop state zeroed, a while node whose body is one Newton iteration,
// and the cumslip tail.
int ensure_inc_graph(fas_handle *h, int inc, cudaGraphExec_t *out)
{
    auto it = h->inc_graphs.find(inc);
    if (it != h->inc_graphs.end()) {
        *out = it->second;
        return 0;
    }
    if (!h->cap2) CK(cudaStreamCreateWithFlags(&h->cap2, cudaStreamNonBlocking));
    if (!h->cap3) CK(cudaStreamCreateWithFlags(&h->cap3, cudaStreamNonBlocking));
    if (!h->nrdev.p) CKA(h->nrdev.alloc(1));
    if (!h->nrrep.p) CKA(h->nrrep.alloc((size_t)std::max(h->C.maxit, 1)));
    if (!h->cp_queue.p) CKA(h->cp_queue.alloc(1));
    if (int rc = ensure_fp32(h)) return rc;
    // the work-order buffers are sized outside the capture
    if (h->nn != 8)
        work_order(h, h->npg * h->nlmnt, h->gp_item.p);
    else if (!(h->mode & FAS_MODE_CP_WARP))
        work_order(h, h->nlmnt, h->gpe.p);
    CK(cudaStreamSynchronize(h->stream));
    const fas_profile P0 = h->P;
    const int64_t L0 = h->launches;
    const DevCtrl C0 = h->C;
    h->C.nit_dev = &h->nrdev.p->nit;
    cudaStream_t s = h->stream;
    cudaGraph_t g = nullptr;
    int rc = 0;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    if (cudaMemsetAsync(h->nrdev.p, 0, sizeof(NrDev), s) != cudaSuccess) rc = FAS_E_CUDA;
    cudaGraphConditionalHandle hnr;
    cudaGraph_t body = nullptr;
    if (!rc) rc = make_condition(s, 1, true, &hnr);
    if (!rc) rc = add_conditional(s, hnr, cudaGraphCondTypeWhile, &body);
    if (!rc) rc = capture_into(h, h->cap2, body, [&]() { return capture_nr_body(h, inc, hnr); });
    if (!rc) {
        const int nsc = h->M.ns[h->last_mat - 1];
        k_cumslip_dev<<<nblocks(h->ngps, 256), 256, 0, s>>>(h->gp(), nsc, h->h_tiem[inc - 1], h->nrdev.p);
    }
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    h->C = C0;
    h->P = P0;
    h->launches = L0;
    if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc ? rc : FAS_E_CUDA;
    }
    cudaGraphExec_t ge = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
    h->inc_graphs[inc] = ge;
    *out = ge;
    return 0;
}

// NRITER of increment `inc` as one graph launch and one host read: the
// report lines, the iteration count and the first error come back together.
int nriter_graph_impl(fas_handle *h, int inc, fas_iter_report *rep, int cap, int *n_rep)
{
    cudaGraphExec_t ge;
    if (int rc = ensure_inc_graph(h, inc, &ge)) return rc;
    cudaStream_t s = h->stream;
    CK(cudaGraphLaunch(ge, s));
    CK(cudaMemcpyAsync(&h->hc->nr, h->nrdev.p, sizeof(NrDev), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const NrDev nr = h->hc->nr;
    const int n = std::min(nr.nit - (nr.status ? 1 : 0), (int)h->nrrep.n);
    std::vector<fas_iter_report> r(std::max(n, 1));
    if (n > 0) CK(cudaMemcpy(r.data(), h->nrrep.p, n * sizeof(fas_iter_report), cudaMemcpyDeviceToHost));
    if (n_rep) *n_rep = nr.nit;
    if (rep)
        for (int k = 0; k < std::min(n, cap); ++k) rep[k] = r[k];
    // the counters of the iterations the graph ran
    const bool small = h->sor_small && !(h->mode & FAS_MODE_SOR_GRID);
    const bool fp32 = !small && (h->mode & FAS_MODE_SOR_FP32) && h->blk32.p;
    const int per_pass = fp32 ? h->refine_every : GRAPH_SWEEPS;
    double bytes = 0.0;
    for (double b : fp32 ? h->col_bytes32 : h->col_bytes) bytes += b;
    h->launches += 1 + (int64_t)nr.nit * h->g_body_launches;   // cumslip, and every iteration's body
    for (int k = 0; k < n; ++k) {
        const int sw = r[k].sor_sweeps;
        h->P.n_constitutive++;
        h->P.gp_updates += h->ngps;
        h->P.n_assembly++;
        h->P.assembly_bytes += h->asm_bytes;
        h->P.sor_sweeps += sw;
        h->P.sor_bytes += bytes * sw;
        h->P.n_sor_colour += small ? 1 : (int64_t)sw * h->ncol;
        if (!small) h->launches += (int64_t)((sw + per_pass - 1) / per_pass) * h->g_pass_launches;
    }
    return nr.status;
}

int nriter_impl(fas_handle *h, int inc, fas_iter_report *rep, int cap, int *n_rep)
{
    if ((h->mode & FAS_MODE_GRAPH) && !(h->mode & FAS_MODE_SOR_TILES) && h->prof < 2)
        return nriter_graph_impl(h, inc, rep, cap, n_rep);
    int nit = 0;
    bool l_conv = true;
    while (l_conv) {
        ++nit;
        if (n_rep) *n_rep = nit;
        const int rc = nr_step_impl(h, inc, nit, rep && nit <= cap ? &rep[nit - 1] : nullptr, &l_conv);
        if (rc) return rc;
    }
    return nr_finish_impl(h, inc);
}

int reorient_impl(fas_handle *h, int inc, fas_twin_event *ev, int cap, int *n_ev)
{
    cudaStream_t s = h->stream;
    if (!h->events.p) CKA(h->events.alloc(std::max(h->ngps, 1)));
    CK(cudaMemsetAsync(h->flags.p + 3, 0, sizeof(int), s));
    k_reorient<<<nblocks(h->ngps, 256), 256, 0, s>>>(h->gp(), h->M, h->events.p, h->ngps, h->flags.p + 3);
    LAUNCHED(h);
    CK(cudaMemsetAsync(h->flags.p + 1, 0, sizeof(int), s));   // tflag = 0
    CK(cudaMemcpyAsync(&h->hc->flags[3], h->flags.p + 3, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const int n = h->hc->flags[3];
    if (n_ev) *n_ev = n;
    if (ev && n > 0 && cap > 0) {
        std::vector<TwinEv> tv(n);
        CK(cudaMemcpy(tv.data(), h->events.p, n * sizeof(TwinEv), cudaMemcpyDeviceToHost));
        std::sort(tv.begin(), tv.end(), [](const TwinEv &a, const TwinEv &b) { return a.gp < b.gp; });
        for (int i = 0; i < std::min(n, cap); ++i) {
            ev[i].inc = inc;
            ev[i].gp = tv[i].gp + 1;
            ev[i].sys = tv[i].sys + 1;
            ev[i].pad = 0;
            for (int k = 0; k < 3; ++k) {
                ev[i].euler_old[k] = tv[i].eo[k];
                ev[i].euler_new[k] = tv[i].en[k];
            }
        }
    }
    return 0;
}

int pattern_device(fas_handle *h, int ld, DVec<int> &isd)
{
    const size_t ndof = 3 * (size_t)h->nnod;
    CKA(isd.alloc(ndof * ld));
    CK(cudaMemsetAsync(h->flags.p + 2, 0, sizeof(int), h->stream));
    k_setpta<<<nblocks((long long)ndof, 128), 128, 0, h->stream>>>(h->mesh(), ld, isd.p, h->flags.p + 2);
    LAUNCHED(h);
    CK(cudaMemcpyAsync(&h->hc->flags[2], h->flags.p + 2, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return h->hc->flags[2] ? 955 : 0;
}

// ------------------------------------------------------------------ adjoint
// Grow-only allocation of a replay buffer.
template <class T> cudaError_t ensure(DVec<T> &v, size_t n)
{
    return v.n >= n && v.p ? cudaSuccess : v.alloc(std::max<size_t>(n, 1));
}

// Uploads a replay's history, copies the GP state the replay works on and
// sizes its buffers; fills the kernels' descriptors.
int replay_prepare(fas_handle *h, const fas_replay_desc *d, bool grad, ReplayDev &H, DevGp &G, int &rs)
{
    if (!h || !d || !d->de || !d->dr || !d->dt || !d->w || !d->y) return FAS_E_ARG;
    if (!h->have_state) return FAS_E_STATE;
    if (d->ninc < 1 || d->chk_every < 1) return FAS_E_ARG;
    if (h->ns_tmpl > 32) return FAS_E_RANGE;
    const double qn = std::sqrt(d->q[0] * d->q[0] + d->q[1] * d->q[1] + d->q[2] * d->q[2]);
    if (!(qn > 0.0) || !std::isfinite(qn)) return FAS_E_ARG;
    ReplayBufs &B = h->rp;
    cudaStream_t s = h->stream;
    const size_t ng = h->ngps, ninc = d->ninc;
    const int chk = std::min(d->chk_every, d->ninc);
    const int nseg = (d->ninc + chk - 1) / chk;
    const int zs = 9 + h->maxns;
    rs = zs + 7 + h->ns_tmpl;
    CKA(ensure(B.de, 6 * ng * ninc));
    CKA(ensure(B.dr, 3 * ng * ninc));
    CKA(ensure(B.dt, ninc));
    CKA(ensure(B.w, ng));
    CKA(ensure(B.y, ng));
    CKA(ensure(B.chk, (size_t)nseg * zs * ng));
    if (grad) {
        CKA(ensure(B.rec, (size_t)chk * rs * ng));
        CKA(ensure(B.gst, 6 * ng));
        CKA(ensure(B.gsv, (size_t)(zs - 6) * ng));
        CKA(ensure(B.gp, (size_t)ADJ_NP * ng));
    }
    CKA(ensure(B.sv, (size_t)h->nsvld * ng));
    CKA(ensure(B.dsv, (size_t)h->nsvld * ng));
    CKA(ensure(B.srate, (size_t)h->maxns * ng));
    CKA(ensure(B.erepmd, ng));
    CKA(ensure(B.ops, ng));
    CKA(ensure(B.jg, ng));
    CKA(ensure(B.eq, ng));
    CKA(ensure(B.twinsys, ng));
    CKA(ensure(B.timestwinned, ng));
    CKA(ensure(B.cp_iters, ng));
    CKA(ensure(B.tflag, 1));
    CK(cudaMemcpyAsync(B.de.p, d->de, 6 * ng * ninc * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.dr.p, d->dr, 3 * ng * ninc * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.dt.p, d->dt, ninc * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.w.p, d->w, ng * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.y.p, d->y, ng * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(B.sv.p, h->sv.p, (size_t)h->nsvld * ng * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(B.twinsys.p, h->twinsys.p, ng * sizeof(int), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(B.timestwinned.p, h->timestwinned.p, ng * sizeof(int), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(B.tflag.p, 0, sizeof(int), s));
    CK(cudaMemsetAsync(h->ekey.p, 0xFF, sizeof(unsigned long long), s));
    H.de = B.de.p;
    H.dr = B.dr.p;
    H.dt = B.dt.p;
    H.w = B.w.p;
    H.y = B.y.p;
    for (int k = 0; k < 3; ++k) H.q[k] = d->q[k] / qn;
    H.ninc = d->ninc;
    H.chk = chk;
    H.zs = zs;
    G = DevGp{};
    G.ngps = h->ngps;
    G.ldsv = h->nsvld;
    G.ldsl = h->maxns;
    G.sv = B.sv.p;
    G.dsv = B.dsv.p;
    G.srate = B.srate.p;
    G.erepmd = B.erepmd.p;
    G.ops = B.ops.p;
    G.cp_iters = B.cp_iters.p;
    G.twinsys = B.twinsys.p;
    G.timestwinned = B.timestwinned.p;
    G.tflag = B.tflag.p;
    return 0;
}

// CTA size of the replay kernels: 128 threads, halved (down to one warp)
// while that leaves fewer than two CTAs per SM, so that a small GP count
// still spreads its long serial threads over every SM.  Each GP is
// independent, so the size changes no result.
int replay_block(const fas_handle *h)
{
    int bs = 128;
    while (bs > 32 && (long long)h->ngps < 2LL * h->nsm * bs) bs >>= 1;
    return bs;
}

// The forward sweep; with rs > 0 it also records the last segment for
// the reverse sweep.
template <int NS>
void launch_replay_fwd(fas_handle *h, const ReplayDev &H, const DevGp &G, int rs)
{
    const int bs = replay_block(h);
    k_replay_fwd<NS><<<nblocks(h->ngps, bs), bs, 0, h->stream>>>(h->M, h->C, G, h->gp_iel.p, h->st.p, H,
                                                                  h->rp.chk.p, rs > 0 ? h->rp.rec.p : nullptr,
                                                                  rs, h->rp.jg.p, h->rp.eq.p, h->ekey.p);
}

template <int NS>
void launch_replay_adj(fas_handle *h, const ReplayDev &H, const DevGp &G, int rs)
{
    const int bs = replay_block(h);
    k_replay_adj<NS><<<nblocks(h->ngps, bs), bs, 0, h->stream>>>(h->M, h->C, G, h->gp_iel.p, H, h->rp.chk.p,
                                                                  h->rp.rec.p, rs, h->rp.jg.p, h->rp.gst.p,
                                                                  h->rp.gsv.p, h->rp.gp.p, h->ekey.p);
}

// Waits for the replay kernels; the objective summed over the GPs in GP order.
int replay_finish(fas_handle *h, double *J)
{
    std::vector<double> jg(h->ngps);
    CK(cudaMemcpyAsync(h->hc->ekey, h->ekey.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(jg.data(), h->rp.jg.p, jg.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->hc->ekey[0] != ~0ull) return (int)(h->hc->ekey[0] & 0xFFFFull);
    double acc = 0.0;
    for (double v : jg) acc += v;
    if (J) *J = acc;
    return 0;
}

}  // namespace

// ================================================================ C ABI
extern "C" {

int32_t fas_gpu_create(const fas_mesh_desc *mesh, const fas_matl_desc *matl, const fas_ctrl_desc *ctrl,
                       uint32_t mode, fas_handle **out)
{
    if (!out || !mesh || !matl || !ctrl) return FAS_E_ARG;
    *out = nullptr;
    fas_handle *h = new (std::nothrow) fas_handle;
    if (!h) return FAS_E_NOMEM;
    h->mode = mode;
    const int rc = create_impl(h, mesh, matl, ctrl);
    if (rc) {
        delete h;
        return rc;
    }
    *out = h;
    return 0;
}

void fas_gpu_destroy(fas_handle *h) { delete h; }

int32_t fas_gpu_set_mode(fas_handle *h, uint32_t mode)
{
    if (!h) return FAS_E_ARG;
    h->mode = mode;
    h->C.tangent = (mode & FAS_MODE_TANGENT_CONSISTENT) ? 1 : 0;
    // increment graphs hold the launches of the old mode
    for (auto &g : h->inc_graphs) cudaGraphExecDestroy(g.second);
    h->inc_graphs.clear();
    // and so does the FP32 cycle's graph (full or symmetric rows)
    if (h->sor32_graph) cudaGraphExecDestroy(h->sor32_graph);
    h->sor32_graph = nullptr;
    return 0;
}

int32_t fas_gpu_upload_state(fas_handle *h, const fas_state_desc *s)
{
    if (!h) return FAS_E_ARG;
    return upload_impl(h, s);
}

int32_t fas_gpu_download_state(fas_handle *h, const fas_state_desc *s)
{
    if (!h) return FAS_E_ARG;
    return download_impl(h, s);
}

int32_t fas_gpu_update_node(fas_handle *h)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state) return FAS_E_STATE;
    const int nd3 = 3 * h->nnod;
    if (nd3 > 0) {
        k_update_node<<<nblocks(nd3, 256), 256, 0, h->stream>>>(nd3, h->x.p, h->dx.p);
        LAUNCHED(h);
    }
    return 0;
}

int32_t fas_gpu_elvals(fas_handle *h, int32_t inc, int32_t nit)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    if (inc < 1 || inc > h->ninc1) return FAS_E_ARG;
    return elvals_impl(h, inc, nit, false);
}

int32_t fas_gpu_suvals(fas_handle *h, int32_t inc)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    if (inc < 1 || inc > h->ninc1) return FAS_E_ARG;
    return suvals_impl(h, inc);
}

int32_t fas_gpu_facsls(fas_handle *h, int32_t *sweeps, double *error)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    return facsls_impl(h, sweeps, error);
}

int32_t fas_gpu_nriter(fas_handle *h, int32_t inc, fas_iter_report *rep, int32_t cap, int32_t *n_rep)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    if (inc < 1 || inc > h->ninc1) return FAS_E_ARG;
    int n = 0;
    const int rc = nriter_impl(h, inc, rep, cap, &n);
    if (n_rep) *n_rep = n;
    return rc;
}

int32_t fas_gpu_nr_step(fas_handle *h, int32_t inc, int32_t nit, fas_iter_report *rep, int32_t *more)
{
    if (!h || nit < 1) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    if (inc < 1 || inc > h->ninc1) return FAS_E_ARG;
    bool m = false;
    const int rc = nr_step_impl(h, inc, nit, rep, &m);
    if (more) *more = m ? 1 : 0;
    return rc;
}

int32_t fas_gpu_nr_finish(fas_handle *h, int32_t inc)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    if (inc < 1 || inc > h->ninc1) return FAS_E_ARG;
    return nr_finish_impl(h, inc);
}

int32_t fas_gpu_update_gptv(fas_handle *h)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state) return FAS_E_STATE;
    k_update_gptv<<<nblocks(h->ngps, 256), 256, 0, h->stream>>>(h->gp(), h->nsv);
    LAUNCHED(h);
    return 0;
}

int32_t fas_gpu_reorient(fas_handle *h, int32_t inc, fas_twin_event *ev, int32_t cap, int32_t *n_ev)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state) return FAS_E_STATE;
    return reorient_impl(h, inc, ev, cap, n_ev);
}

int32_t fas_gpu_increment(fas_handle *h, int32_t inc, fas_iter_report *rep, int32_t cap, int32_t *n_rep,
                          fas_twin_event *ev, int32_t ev_cap, int32_t *n_ev)
{
    int32_t rc = fas_gpu_update_node(h);
    if (rc) return rc;
    rc = fas_gpu_nriter(h, inc, rep, cap, n_rep);
    if (rc) return rc;
    rc = fas_gpu_update_gptv(h);
    if (rc) return rc;
    if (n_ev) *n_ev = 0;
    CK(cudaMemcpyAsync(&h->hc->flags[1], h->flags.p + 1, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->hc->flags[1]) rc = reorient_impl(h, inc, ev, ev_cap, n_ev);
    return rc;
}

int32_t fas_gpu_get_pattern(fas_handle *h, int32_t *is, int32_t ld_is)
{
    if (!h || !is || ld_is < 2) return FAS_E_ARG;
    if (h->point_mode) return FAS_E_STATE;
    DVec<int> isd;
    int rc = pattern_device(h, ld_is, isd);
    if (rc) return rc;
    CK(cudaMemcpy(is, isd.p, isd.n * sizeof(int), cudaMemcpyDeviceToHost));
    return 0;
}

int32_t fas_gpu_get_stiffness(fas_handle *h, void *ss, int32_t ld_ss, int32_t real_bytes)
{
    if (!h || !ss || ld_ss < 2 || (real_bytes != 4 && real_bytes != 8)) return FAS_E_ARG;
    if (h->point_mode || !h->have_state) return FAS_E_STATE;
    DVec<int> isd;
    int rc = pattern_device(h, ld_ss, isd);
    if (rc) return rc;
    const size_t n = 3 * (size_t)h->nnod * ld_ss;
    DVec<double> ssd;
    CKA(ssd.alloc(n));
    k_to_ell<<<nblocks(3LL * h->nnod, 128), 128, 0, h->stream>>>(h->block(), h->rowof.p, h->nnod, ld_ss,
                                                                 isd.p, ssd.p);
    LAUNCHED(h);
    std::vector<double> tmp(n);
    CK(cudaMemcpyAsync(tmp.data(), ssd.p, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (size_t i = 0; i < n; ++i) {
        if (real_bytes == 4) ((float *)ss)[i] = (float)tmp[i];
        else ((double *)ss)[i] = tmp[i];
    }
    return 0;
}

int32_t fas_gpu_get_colouring(fas_handle *h, int32_t *colour, int32_t *ncol)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    if (colour) std::copy(h->h_colour.begin(), h->h_colour.end(), colour);
    if (ncol) *ncol = h->ncol;
    return 0;
}

int32_t fas_gpu_constitutive(fas_handle *h, int32_t inc, int32_t nit)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state) return FAS_E_STATE;
    if (inc < 1 || inc > h->ninc1) return FAS_E_ARG;
    if (!h->chi_pts.p) {
        CKA(h->chi_pts.alloc(36 * (size_t)h->ngps));
        CK(h->chi_pts.zero(h->stream));
    }
    cudaStream_t s = h->stream;
    CK(cudaMemsetAsync(h->ekey.p, 0xFF, sizeof(unsigned long long), s));
    Span sp(h, &h->P.ms_constitutive);
    const double dt = h->h_tiem[inc - 1];
    const unsigned nbw = nblocks(32LL * h->ngps, 128);
    const bool thr = !(h->mode & FAS_MODE_CP_WARP) || h->maxns > 32;
    const int *order = thr ? work_order(h, h->ngps, nullptr) : nullptr;
    switch (h->ns_tmpl) {
    case 12:
        if (thr) {
            int *queue = nullptr;
            int bs = 128;
            const unsigned grid = cp_grid(h, k_points<12>, h->ngps, &queue, &bs);
            k_points<12><<<grid, bs, h->stage_bytes, s>>>(h->M, h->C, h->gp(), h->gp_iel.p, h->chi_pts.p, dt, inc, nit, h->ekey.p, order, queue);
        }
        else k_points_wc<12><<<nbw, 128, 0, s>>>(h->M, h->C, h->gp(), h->gp_iel.p, h->chi_pts.p, dt, inc, nit, h->ekey.p);
        break;
    case 32:
        if (thr) {
            int *queue = nullptr;
            int bs = 128;
            const unsigned grid = cp_grid(h, k_points<32>, h->ngps, &queue, &bs);
            k_points<32><<<grid, bs, h->stage_bytes, s>>>(h->M, h->C, h->gp(), h->gp_iel.p, h->chi_pts.p, dt, inc, nit, h->ekey.p, order, queue);
        }
        else k_points_wc<32><<<nbw, 128, 0, s>>>(h->M, h->C, h->gp(), h->gp_iel.p, h->chi_pts.p, dt, inc, nit, h->ekey.p);
        break;
    default: {
        int *queue = nullptr;
        int bs = 128;
        const unsigned grid = cp_grid(h, k_points<60>, h->ngps, &queue, &bs);
        k_points<60><<<grid, bs, h->stage_bytes, s>>>(h->M, h->C, h->gp(), h->gp_iel.p, h->chi_pts.p, dt, inc, nit, h->ekey.p, order, queue);
        break;
    }
    }
    sp.end();
    keep(h, sp);
    LAUNCHED(h);
    h->P.n_constitutive++;
    h->P.gp_updates += h->ngps;
    CK(cudaMemcpyAsync(h->hc->ekey, h->ekey.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    settle_spans(h);
    if (h->hc->ekey[0] != ~0ull) return (int)(h->hc->ekey[0] & 0xFFFFull);
    return 0;
}

int32_t fas_gpu_get_tangent(fas_handle *h, void *chi, int32_t real_bytes)
{
    if (!h || !chi || (real_bytes != 4 && real_bytes != 8)) return FAS_E_ARG;
    const size_t ng = h->ngps;
    std::vector<double> out(36 * ng, 0.0);
    if (h->point_mode || !h->rec.p) {
        if (!h->chi_pts.p) return FAS_E_STATE;
        std::vector<double> t(36 * ng);
        CK(cudaMemcpy(t.data(), h->chi_pts.p, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (size_t g = 0; g < ng; ++g)
            for (int q = 0; q < 36; ++q) out[g * 36 + q] = t[(size_t)q * ng + g];
    } else {
        std::vector<double> r((size_t)REC * h->nlmnt);
        CK(cudaMemcpy(r.data(), h->rec.p, r.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int e = 0; e < h->nlmnt; ++e) {
            const size_t g = h->h_gpe[e];
            for (int i = 0; i < 6; ++i)
                for (int j = i; j < 6; ++j) {
                    const double v = r[(size_t)e * REC + REC_D + utri(i, j)];
                    out[g * 36 + i + 6 * j] = v;
                    out[g * 36 + j + 6 * i] = v;
                }
        }
    }
    for (size_t i = 0; i < out.size(); ++i) {
        if (real_bytes == 4) ((float *)chi)[i] = (float)out[i];
        else ((double *)chi)[i] = out[i];
    }
    return 0;
}

int32_t fas_gpu_get_cp_stats(fas_handle *h, int32_t *iters, double *erepmd)
{
    if (!h) return FAS_E_ARG;
    if (iters) CK(cudaMemcpy(iters, h->cp_iters.p, h->ngps * sizeof(int), cudaMemcpyDeviceToHost));
    if (erepmd) CK(cudaMemcpy(erepmd, h->erepmd.p, h->ngps * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int32_t fas_gpu_lattice_strain(fas_handle *h, void *strain, int32_t real_bytes)
{
    if (!h || !strain || (real_bytes != 4 && real_bytes != 8)) return FAS_E_ARG;
    if (!h->have_state) return FAS_E_STATE;
    DVec<double> d;
    CKA(d.alloc(6 * (size_t)h->ngps));
    k_elaseps<<<nblocks(h->ngps, 128), 128, 0, h->stream>>>(h->M, h->gp(), h->gp_iel.p, d.p);
    LAUNCHED(h);
    return down_field(h, strain, real_bytes, 6, 6, h->ngps, d.p);
}

int32_t fas_gpu_adjoint_forward(fas_handle *h, const fas_replay_desc *d, double *J, double *eq)
{
    ReplayDev H;
    DevGp G;
    int rs = 0;
    int rc = replay_prepare(h, d, false, H, G, rs);
    if (rc) return rc;
    if (h->ns_tmpl == 12) launch_replay_fwd<12>(h, H, G, 0);
    else launch_replay_fwd<32>(h, H, G, 0);
    LAUNCHED(h);
    rc = replay_finish(h, J);
    if (rc) return rc;
    if (eq) CK(cudaMemcpy(eq, h->rp.eq.p, h->ngps * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int32_t fas_gpu_adjoint_grad(fas_handle *h, const fas_replay_desc *d, double *J, double *g_st, double *g_sv,
                             double *g_ampar)
{
    ReplayDev H;
    DevGp G;
    int rs = 0;
    int rc = replay_prepare(h, d, true, H, G, rs);
    if (rc) return rc;
    const size_t ng = h->ngps;
    if (h->ns_tmpl == 12) launch_replay_fwd<12>(h, H, G, rs);
    else launch_replay_fwd<32>(h, H, G, rs);
    LAUNCHED(h);
    // the reverse sweep starts from the same twin state as the forward one
    CK(cudaMemcpyAsync(h->rp.twinsys.p, h->twinsys.p, ng * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
    if (h->ns_tmpl == 12) launch_replay_adj<12>(h, H, G, rs);
    else launch_replay_adj<32>(h, H, G, rs);
    LAUNCHED(h);
    rc = replay_finish(h, J);
    if (rc) return rc;
    const int nsv = 3 + h->maxns;
    if (g_st) {
        std::vector<double> t(6 * ng);
        CK(cudaMemcpy(t.data(), h->rp.gst.p, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (size_t g = 0; g < ng; ++g)
            for (int k = 0; k < 6; ++k) g_st[g * 6 + k] = t[(size_t)k * ng + g];
    }
    if (g_sv) {
        std::vector<double> t((size_t)nsv * ng);
        CK(cudaMemcpy(t.data(), h->rp.gsv.p, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (size_t g = 0; g < ng; ++g) {
            const int ns = h->M.ns[std::abs(h->h_gp_iel[g]) - 1];
            for (int k = 0; k < FAS_MAXSVS; ++k) g_sv[g * FAS_MAXSVS + k] = k < 3 + ns ? t[(size_t)k * ng + g] : 0.0;
        }
    }
    if (g_ampar) {
        std::vector<double> t((size_t)ADJ_NP * ng);
        CK(cudaMemcpy(t.data(), h->rp.gp.p, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int m = 0; m < h->M.nmatl; ++m)
            for (int k = 0; k < 10; ++k) g_ampar[m * 10 + k] = 0.0;
        for (size_t g = 0; g < ng; ++g) {
            const int m = std::abs(h->h_gp_iel[g]) - 1;
            for (int j = 0; j < ADJ_NP; ++j) g_ampar[m * 10 + adj_ampar_index(j)] += t[(size_t)j * ng + g];
        }
    }
    return 0;
}

int32_t fas_gpu_get_cp_ops(fas_handle *h, double *ops)
{
    if (!h || !ops) return FAS_E_ARG;
    CK(cudaMemcpy(ops, h->ops.p, h->ngps * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int32_t fas_gpu_profile(fas_handle *h, int32_t enable, fas_profile *out)
{
    if (!h) return FAS_E_ARG;
    if (h->prof) {
        CK(cudaEventRecord(h->ev_t1, h->stream));
        CK(cudaEventSynchronize(h->ev_t1));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, h->ev_t0, h->ev_t1));
        h->P.ms_total = ms;
        settle_spans(h);
    }
    h->P.n_launches = h->launches;
    if (out) *out = h->P;
    if (enable) {
        h->P = fas_profile{};
        h->launches = 0;
        h->prof = enable >= 2 ? 2 : 1;
        CK(cudaEventRecord(h->ev_t0, h->stream));
    } else {
        h->prof = 0;
    }
    return 0;
}

}  // extern "C"

// ================================================================ FACSLS
// without device allocation.  No counterpart in the reference: it exists
// for callers that must not allocate device memory once set-up is over
// (fas_gpu_facsls_noalloc in fasolt_gpu.h says who and why).
//
// The SOR kernels' scratch -- the control words of the stopping test
// (SorCtl) and the per-CTA reduction partials -- lives in this file-scope
// array instead of in buffers of the handle: a 256-byte block for the
// control words, then FAS_NOALLOC_PARTIALS pairs of doubles (the sums of
// |dx|^2 and |x|^2 of every colour CTA).  262,400 bytes per device.
static __device__ __align__(256) unsigned char fas_noalloc_scratch[256 + 2 * sizeof(double) * FAS_NOALLOC_PARTIALS];

namespace {

constexpr size_t NOALLOC_CTL_BYTES = 256;
constexpr int NOALLOC_MAXDEV = 64;
static_assert(sizeof(SorCtl) <= NOALLOC_CTL_BYTES, "control words exceed their block");

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[NOALLOC_MAXDEV] = {};

// The device address of fas_noalloc_scratch on device `dev`, looked up
// once per device (with that device current) and cached.
int noalloc_scratch(int dev, unsigned char **out)
{
    if (dev < 0 || dev >= NOALLOC_MAXDEV) return FAS_E_RANGE;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        int cur = -1;
        CK(cudaGetDevice(&cur));
        if (cur != dev) CK(cudaSetDevice(dev));
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, fas_noalloc_scratch);
        if (cur != dev) CK(cudaSetDevice(cur));
        if (e != cudaSuccess || !p) return FAS_E_CUDA;
        g_noalloc_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_addr[dev];
    return 0;
}

// The FP64 FACSLS of facsls_impl (same colour kernels, colour order,
// reciprocal-diagonal quotients, sweep chunks and stopping test) on the
// static scratch; no CUDA graph, no FP32-matrix sweeps, no profiling
// spans.  The reciprocal diagonal goes to the handle's own buffer, which
// set-up allocated.
int facsls_noalloc_impl(fas_handle *h, int *sweeps, double *error)
{
    if (h->sor_nblk_tot > FAS_NOALLOC_PARTIALS) return FAS_E_RANGE;
    unsigned char *scr = nullptr;
    const int rc = noalloc_scratch(h->dev, &scr);
    if (rc) return rc;
    SorCtl *ctl = reinterpret_cast<SorCtl *>(scr);
    double *part = reinterpret_cast<double *>(scr + NOALLOC_CTL_BYTES);
    cudaStream_t s = h->stream;
    const size_t nd3 = 3 * (size_t)h->nnod;
    CK(cudaMemcpyAsync(h->rhs.p, h->ddx.p, nd3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemsetAsync(h->ddx.p, 0, nd3 * sizeof(double), s));
    CK(cudaMemsetAsync(h->ekey.p + 1, 0xFF, sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(ctl, 0, sizeof(SorCtl), s));   // the control words start every solve at zero
    BlockDev B = h->block();
    k_diag_check<<<nblocks(h->nnod, 256), 256, 0, s>>>(B, h->ekey.p + 1);
    LAUNCHED(h);
    CK(cudaMemcpyAsync(&h->hc->ekey[1], h->ekey.p + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h->hc->ekey[1] != ~0ull) return 903;
    const double tolerl = h->C.toler * h->C.toler;
    if (h->sor_small && !(h->mode & FAS_MODE_SOR_GRID)) {
        launch_sor_small(h, B, ctl, tolerl);
        LAUNCHED(h);
    } else {
        const double *rdiag = FAS_SOR_RCP ? h->rdiag.p : nullptr;
        if (rdiag) {
            k_rdiag<<<nblocks(h->nnod, 256), 256, 0, s>>>(B, h->rdiag.p);
            LAUNCHED(h);
        }
        int done = 0, chunk = 4;
        while (done < 1000) {
            const int k = std::min(chunk, 1000 - done);
            for (int it = 0; it < k; ++it) {
                for (int c = 0; c < h->ncol; ++c) {
                    if (h->col_start[c + 1] <= h->col_start[c]) continue;
                    launch_colour_kernel<double>(h, c, false, h->blk.p, h->rhs.p, h->ddx.p, nullptr, rdiag, ctl,
                                                 part);
                    LAUNCHED(h);
                }
                k_sor_check<<<1, 1024, 0, s>>>(part, h->sor_nblk_tot, ctl, tolerl);
                LAUNCHED(h);
            }
            done += k;
            CK(cudaMemcpyAsync(&h->hc->sor, ctl, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (h->hc->sor.conv || h->hc->sor.fault) break;
            chunk = std::min(chunk * 2, 64);
        }
    }
    CK(cudaMemcpyAsync(&h->hc->sor, ctl, sizeof(SorCtl), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (sweeps) *sweeps = h->hc->sor.sweeps;
    if (error) *error = h->hc->sor.err;
    if (h->hc->sor.fault) return FAS_E_TIMEOUT;
    if (h->hc->sor.err > 10.0 * tolerl) return 904;
    return 0;
}

}  // namespace

extern "C" int32_t fas_gpu_facsls_noalloc(fas_handle *h, int32_t *sweeps, double *error)
{
    if (!h) return FAS_E_ARG;
    if (!h->have_state || h->point_mode) return FAS_E_STATE;
    return facsls_noalloc_impl(h, sweeps, error);
}
