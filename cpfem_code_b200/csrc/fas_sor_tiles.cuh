// fas_sor_tiles.cuh -- FACSLS (src/fasolt/Stif_sol.f90:161-215) as one
// persistent kernel per solve: multicolour point SOR over spatial tiles
// with tile-to-tile dataflow instead of one launch per colour.
//
// Why.  The colour kernels (k_sor_colour_tma) end every colour phase at a
// kernel boundary: nine launch ramps per sweep (eight colours and the
// stopping test) and a pipeline that refills from empty every phase.  The
// dependence that forces the boundary is local: a row of colour c reads
// only the nodes it shares an element with.  So the rows are split into
// spatial tiles (one per CTA, all CTAs resident), and a tile starts colour
// c of sweep j as soon as every tile adjacent to it has finished colour
// c - 1 of sweep j (colour ncol - 1 of sweep j - 1 for c = 0).  Each row
// then sees exactly the values it sees in the global colour order -- a
// neighbour of lower colour already updated in this sweep, one of higher
// colour still holding the previous sweep's value (that neighbour cannot
// pass colour c before this tile has finished c) -- and the iterates equal
// the colour kernels' to the bit.  The block rows stream through each
// warp's bulk-copy ring without pause across phases and sweeps: the matrix
// is constant during a solve, so a ring runs ahead into the next phase
// while the tile waits for its neighbours.
//
// Rows are ordered tile by tile, and inside a tile colour by colour:
// tseg[t * (ncol + 1) + c] is the first row of colour c of tile t (the
// entry c = ncol the end of the tile).  The rows of one colour of one tile
// are cut into chunks of TILE_ROWS; warp w of the CTA serves chunks w, w +
// nwarps, ... of every phase.
//
// Stopping test without a global barrier.  Sweep j writes its iterate into
// sol[j & 1] (sol0 = the caller's vector, sol1 = scratch; slot bit 31 of a
// column id says whether the column node has a lower colour than the row,
// i.e. whether its value for this sweep is in sol[j & 1] or still in
// sol[(j - 1) & 1]).  Every tile adds its share of |x_j - x_{j-1}|^2 and
// |x_j|^2 to a per-sweep slot; the last tile to arrive sums the tiles'
// shares in tile order and publishes err and the verdict for sweep j.
// Sweep j overwrites the iterate of sweep j - 2, so a tile waits for sweep
// j - 2's verdict only before it starts sweep j: the verdict of sweep j - 1
// is never waited for while the tiles move on.  When sweep j* converges
// (err < toler^2) every tile has computed at most one further sweep into
// the other buffer; each tile then copies its rows of sweep j* into sol0
// if j* is odd.  The returned sweep count and error are sweep j*'s, as
// FACSLS reports them.
//
// Every wait (neighbour progress, verdicts, bulk copies) is bounded; on a
// timeout the kernel raises ctl->fault, every tile leaves at its next wait,
// and each CTA first waits (bounded) for its own copies still in flight.
#pragma once

#include "fas_kernels.cuh"

namespace fasdev {

#ifndef FAS_TILE_WARPS64
#define FAS_TILE_WARPS64 6
#endif
#ifndef FAS_TILE_WARPS32
#define FAS_TILE_WARPS32 12
#endif
// warps (each with its own 2-stage ring of 8-row chunks) per tile CTA
template <typename T> __host__ __device__ constexpr int tile_warps()
{
    return sizeof(T) == 8 ? FAS_TILE_WARPS64 : FAS_TILE_WARPS32;
}
// chunk shape and ring depth of the tile kernel (fixed, independent of
// the colour kernels' tuned shapes): 8 rows x 4 lanes = one warp per chunk
constexpr int TILE_ROWS = 8, TILE_LPR = 4, TILE_STAGES = 2;
// a ring stage: TILE_ROWS rows of 27 slots (values and column ids)
template <typename T> __host__ __device__ constexpr int tile_stage_bytes()
{
    return TILE_ROWS * brow_of(SLOTS) * (int)sizeof(T) + TILE_ROWS * crow_of(SLOTS) * 4;
}
template <typename T> __host__ __device__ constexpr int tile_smem_bytes()
{
    return tile_warps<T>() * (TILE_STAGES * tile_stage_bytes<T>() + TILE_STAGES * 8) + 512;
}
static_assert(tile_smem_bytes<double>() <= 227 * 1024 && tile_smem_bytes<float>() <= 227 * 1024,
              "the tile CTA's rings must fit in shared memory");

constexpr unsigned TILE_LOWER = 0x80000000u;   // column-id bit: lower colour than the row
constexpr int TILE_SLOTS_SYNC = 4;             // per-sweep slots of the stopping test
// a tile's colour bounds and neighbour list live in shared memory (global
// reads of them after every acquire would cost an L2 round trip each)
constexpr int TILE_MAXCOL = 64;
constexpr int TILE_MAXADJ = 128;

// Per-sweep stopping-test state, zeroed before every launch.
struct TileSync {
    int cnt[TILE_SLOTS_SYNC];      // tiles that have added their share of sweep j
    int dsw[TILE_SLOTS_SYNC];      // sweep whose verdict the slot holds (0: none yet)
    int dconv[TILE_SLOTS_SYNC];
    int fault;
    double derr[TILE_SLOTS_SYNC];
};

template <typename T> struct TileArgs {
    const T *blk;                  // [rows][brow] tile-layout block rows
    const int *bcol;               // [rows][crow] column nodes (| TILE_LOWER), [S] = slot count
    const int *tseg;               // [ntiles][ncol + 1] first row of each colour of each tile
    const int *tadj_ptr, *tadj;    // tiles adjacent to each tile (CSR)
    const double *rhs, *base, *rdiag;   // rdiag: reciprocal diagonal, tile-row order
    double *sol0, *sol1;
    int *progress;                 // [ntiles] phases finished (sweep-major), zeroed per launch
    double *part;                  // [TILE_SLOTS_SYNC][ntiles][2] per-tile sweep shares
    TileSync *sync;
    SorCtl *ctl;
    int ntiles, ncol, maxsw, sweep_base;
    double tolerl;
    int keep_rows;                 // rows at the start of each tile whose blocks stay in L2
};

__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bound of the polls of one wait: far above any legitimate wait (a
// sweep takes well under a millisecond), short enough that a lost peer
// ends the kernel in well under a minute.
constexpr int TILE_POLLS = 1 << 21;

// Waits until every tile of adj[0, nadj) has finished `target` phases.
// One warp polls up to 32 neighbours at a time.  Returns false on a
// timeout or when another tile raised the fault.
__device__ __forceinline__ bool tile_wait_neighbours(const int *adj, int nadj, const int *progress, int target,
                                                     TileSync *sync)
{
    const int lane = threadIdx.x & 31;
    for (int b = 0; b < nadj; b += 32) {
        const int k = b + lane;
        const int nb = k < nadj ? adj[k] : -1;
        int it = 0;
        while (true) {
            const bool ok = nb < 0 || ld_acquire(progress + nb) >= target;
            if (__all_sync(0xffffffffu, ok)) break;
            if (++it > TILE_POLLS || ld_acquire(&sync->fault)) return false;
            __nanosleep(64);
        }
    }
    return true;
}

// Waits for the verdict of sweep j; false on a timeout or fault.
__device__ __forceinline__ bool tile_wait_verdict(TileSync *sync, int j)
{
    const int s = j & (TILE_SLOTS_SYNC - 1);
    for (int it = 0; it <= TILE_POLLS; ++it) {
        if (ld_acquire(&sync->dsw[s]) == j) return true;
        if (ld_acquire(&sync->fault)) return false;
        __nanosleep(64);
    }
    return false;
}

// Gather of lane q of chunk row `row` for the tile kernel: as sor_gather,
// with each column's value taken from the new-sweep buffer when the column
// node has a lower colour than the row and from the previous sweep's
// buffer otherwise (the row's own old value included).
template <int S, int LPR>
__device__ __forceinline__ void tile_gather(const int *stage_cols, int r0, int nrow, int row, int q,
                                            const double *sol_new, const double *sol_old,
                                            const double *__restrict__ rhs, const double *__restrict__ rdiag,
                                            uint64_t keep_pol, SorOps<(S + LPR - 1) / LPR> &g)
{
    constexpr int SPL = (S + LPR - 1) / LPR, CR = crow_of(S);
    const bool live = row < nrow;
    const int *cols = stage_cols + (live ? row : 0) * CR;
    const int ns = live ? cols[S] : 0;
#pragma unroll
    for (int j = 0; j < SPL; ++j) {
        const int sl = q + LPR * j;
        const bool on = sl < ns;
        const unsigned w = on ? (unsigned)cols[sl] : 0u;
        const int m = (int)(w & ~TILE_LOWER);
        const double *src = (w & TILE_LOWER) ? sol_new : sol_old;
        g.x0[j] = on ? ld_keep(src + 3 * m, keep_pol) : 0.0;
        g.x1[j] = on ? ld_keep(src + 3 * m + 1, keep_pol) : 0.0;
        g.x2[j] = on ? ld_keep(src + 3 * m + 2, keep_pol) : 0.0;
    }
    const bool own = live && q == 0;
    const int n = cols[0] & (int)~TILE_LOWER;
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

// The chunk sequence of one warp: for every sweep j = 1..maxsw and colour
// c, the chunks w, w + nw, ... of (tile, c).  k counts the chunks taken.
struct TileCursor {
    int j, c, i;
};

template <typename T>
__global__ void __launch_bounds__(32 * tile_warps<T>(), 1) k_sor_tiles(TileArgs<T> a)
{
    constexpr int S = SLOTS, LPR = TILE_LPR, ROWS = TILE_ROWS;
    constexpr int BR = brow_of(S), CR = crow_of(S);
    constexpr int SPL = (S + LPR - 1) / LPR;
    constexpr int VB = ROWS * BR * (int)sizeof(T);
    constexpr int SB = tile_stage_bytes<T>();
    constexpr int NW = tile_warps<T>();
    static_assert(ROWS * LPR == 32, "one warp serves one chunk");
    static_assert((BR * sizeof(T)) % 16 == 0 && (CR * 4) % 16 == 0, "bulk copies move 16-byte multiples");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_flag[2];
    __shared__ double s_red[2][NW];
    __shared__ int seg[TILE_MAXCOL + 1];   // first row of each colour of this tile
    __shared__ int s_adj[TILE_MAXADJ];      // the tiles this tile waits for

    // a launch queued behind the one that converged does nothing
    if (((volatile const SorCtl *)a.ctl)->conv) return;
    const int t = blockIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int row = lane / LPR, q = lane % LPR;
    const int ncol = a.ncol;
    const int a0 = a.tadj_ptr[t], nadj = a.tadj_ptr[t + 1] - a0;   // at most TILE_MAXADJ (set-up checks)
    for (int k = threadIdx.x; k <= ncol; k += blockDim.x) seg[k] = a.tseg[(size_t)t * (ncol + 1) + k];
    for (int k = threadIdx.x; k < nadj; k += blockDim.x) s_adj[k] = a.tadj[a0 + k];
    __syncthreads();
    unsigned char *ring = smem + (size_t)w * TILE_STAGES * SB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + (size_t)NW * TILE_STAGES * SB) + w * TILE_STAGES;
    const uint64_t stream_pol = l2_evict_first();
    const uint64_t keep_pol = l2_evict_last();
    const int tile_row0 = seg[0];

    auto nch = [&](int c) { return (seg[c + 1] - seg[c] + ROWS - 1) / ROWS; };
    // first chunk of this warp at or after (j, c, i0)
    auto settle = [&](TileCursor &u) {
        while (u.j <= a.maxsw) {
            if (u.i < nch(u.c)) return;
            u.i = w;
            if (++u.c == ncol) {
                u.c = 0;
                ++u.j;
            }
        }
    };
    auto advance = [&](TileCursor &u) {
        u.i += NW;
        settle(u);
    };
    auto issue = [&](const TileCursor &u, int k) {
        const int r0 = seg[u.c] + u.i * ROWS;
        const int nr = min(ROWS, seg[u.c + 1] - r0);
        unsigned char *st = ring + (k % TILE_STAGES) * SB;
        const unsigned bv = (unsigned)(nr * BR * sizeof(T)), bc = (unsigned)(nr * CR * 4);
        const uint64_t pol = r0 - tile_row0 < a.keep_rows ? keep_pol : stream_pol;
        mbar_expect_tx(&bars[k % TILE_STAGES], bv + bc);
        bulk_g2s(st, a.blk + (size_t)r0 * BR, bv, &bars[k % TILE_STAGES], pol);
        bulk_g2s(st + VB, a.bcol + (size_t)r0 * CR, bc, &bars[k % TILE_STAGES], pol);
    };

    TileCursor ic{1, 0, w};   // next chunk to issue (every lane keeps the same cursor)
    settle(ic);
    int issued = 0, taken = 0;
    if (lane == 0) {
        for (int st = 0; st < TILE_STAGES; ++st) mbar_init(&bars[st], 1);
        mbar_fence_init();
    }
    __syncwarp();
    for (int st = 0; st < TILE_STAGES && ic.j <= a.maxsw; ++st) {
        if (lane == 0) issue(ic, issued);
        ++issued;
        advance(ic);
    }
    __syncthreads();

    bool fault = false;
    int jf = 0;   // converged sweep, 0 while none is known
    int j = 1;
    for (; j <= a.maxsw && !fault; ++j) {
        // sweep j overwrites sweep j - 2's iterate: its verdict first
        if (j >= 3) {
            if (threadIdx.x == 0) {
                const bool ok = tile_wait_verdict(a.sync, j - 2);
                s_flag[0] = ok ? a.sync->dconv[(j - 2) & (TILE_SLOTS_SYNC - 1)] : -1;
            }
            __syncthreads();
            if (s_flag[0] < 0) {
                fault = true;
                break;
            }
            if (s_flag[0]) {
                jf = j - 2;
                break;
            }
        }
        double *sol_new = (j & 1) ? a.sol1 : a.sol0;
        const double *sol_old = (j & 1) ? a.sol0 : a.sol1;
        double v0 = 0.0, v1 = 0.0;
        for (int c = 0; c < ncol && !fault; ++c) {
            if (w == 0) {
                const bool ok = tile_wait_neighbours(s_adj, nadj, a.progress, (j - 1) * ncol + c, a.sync);
                __threadfence();
                if (lane == 0) s_flag[1] = ok ? 1 : 0;
            }
            __syncthreads();
            if (!s_flag[1]) {
                fault = true;
                break;
            }
            const int nc = nch(c);
            SorOps<SPL> gcur = {}, gnxt = {};
            bool have = false;
            for (int i = w; i < nc; i += NW) {
                // the chunk of this phase taken now (taken-th of the warp's
                // sequence): wait for its copy, gather, then compute
                if (!have) {
                    const unsigned par = (unsigned)((taken / TILE_STAGES) & 1);
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[taken % TILE_STAGES], par))) {
                        fault = true;
                        break;
                    }
                    const int r0 = seg[c] + i * ROWS;
                    tile_gather<S, LPR>(reinterpret_cast<const int *>(ring + (taken % TILE_STAGES) * SB + VB), r0,
                                        min(ROWS, seg[c + 1] - r0), row, q, sol_new, sol_old, a.rhs, a.rdiag,
                                        keep_pol, gcur);
                }
                // gathers of the warp's next chunk of this phase run ahead
                const int i2 = i + NW;
                have = false;
                if (i2 < nc && TILE_STAGES > 1) {
                    const int k2 = taken + 1;
                    const unsigned par = (unsigned)((k2 / TILE_STAGES) & 1);
                    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&bars[k2 % TILE_STAGES], par))) {
                        fault = true;
                        break;
                    }
                    const int r2 = seg[c] + i2 * ROWS;
                    tile_gather<S, LPR>(reinterpret_cast<const int *>(ring + (k2 % TILE_STAGES) * SB + VB), r2,
                                        min(ROWS, seg[c + 1] - r2), row, q, sol_new, sol_old, a.rhs, a.rdiag,
                                        keep_pol, gnxt);
                    have = true;
                }
                const int r0 = seg[c] + i * ROWS;
                sor_update<T, S, LPR, ROWS>(ring + (taken % TILE_STAGES) * SB, min(ROWS, seg[c + 1] - r0), row, q, gcur,
                                      a.rdiag != nullptr, a.base, sol_new, v0, v1);
                __syncwarp();
                // the stage is free: refill it with the warp's next chunk
                if (lane == 0 && ic.j <= a.maxsw) {
                    fence_proxy_async();
                    issue(ic, issued);
                }
                if (ic.j <= a.maxsw) {
                    ++issued;
                    advance(ic);
                }
                ++taken;
                gcur = gnxt;
            }
            if (__syncthreads_or(fault ? 1 : 0)) {
                fault = true;
                break;
            }
            if (threadIdx.x == 0) {
                __threadfence();
                st_release(a.progress + t, (j - 1) * ncol + c + 1);
            }
        }
        if (fault) break;
        // this tile's share of the sweep's stopping test, then the verdict
        // by the last tile to arrive
        double r0v = v0, r1v = v1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r0v += __shfl_down_sync(0xffffffffu, r0v, o);
            r1v += __shfl_down_sync(0xffffffffu, r1v, o);
        }
        if (lane == 0) {
            s_red[0][w] = r0v;
            s_red[1][w] = r1v;
        }
        __syncthreads();
        const int slot = j & (TILE_SLOTS_SYNC - 1);
        if (threadIdx.x == 0) {
            double s0 = 0.0, s1 = 0.0;
            for (int k = 0; k < NW; ++k) {
                s0 += s_red[0][k];
                s1 += s_red[1][k];
            }
            double *pp = a.part + ((size_t)slot * a.ntiles + t) * 2;
            pp[0] = s0;
            pp[1] = s1;
            __threadfence();
            s_flag[0] = atomicAdd(&a.sync->cnt[slot], 1) == a.ntiles - 1;
        }
        __syncthreads();
        if (s_flag[0] && w == 0) {
            __threadfence();
            const volatile double *pp = a.part + (size_t)slot * a.ntiles * 2;
            double s0 = 0.0, s1 = 0.0;
            for (int k = lane; k < a.ntiles; k += 32) {
                s0 += pp[2 * k];
                s1 += pp[2 * k + 1];
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s0 += __shfl_xor_sync(0xffffffffu, s0, o);
                s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            }
            if (lane == 0) {
                const double err = s0 / s1;
                a.sync->derr[slot] = err;
                a.sync->dconv[slot] = err < a.tolerl ? 1 : 0;
                a.sync->cnt[slot] = 0;
                __threadfence();
                st_release(&a.sync->dsw[slot], j);
            }
        }
        __syncthreads();
    }
    const int last = min(j, a.maxsw + 1) - 1;   // last sweep this tile computed
    // the final sweep: a converged one among the last two unknown verdicts,
    // else the last computed
    if (!fault && jf == 0) {
        if (threadIdx.x == 0) {
            int f = last, bad = 0;
            for (int jj = max(1, last - 1); jj <= last; ++jj) {
                if (!tile_wait_verdict(a.sync, jj)) {
                    bad = 1;
                    break;
                }
                if (a.sync->dconv[jj & (TILE_SLOTS_SYNC - 1)]) {
                    f = jj;
                    break;
                }
            }
            s_flag[0] = bad ? -1 : f;
        }
        __syncthreads();
        if (s_flag[0] < 0)
            fault = true;
        else
            jf = s_flag[0];
    }
    // copies issued and not taken may still write the ring
    if (lane == 0)
        for (int k = taken; k < issued; ++k)
            mbar_wait_bounded(&bars[k % TILE_STAGES], (unsigned)((k / TILE_STAGES) & 1));
    if (fault) {
        if (threadIdx.x == 0) {
            atomicExch(&a.sync->fault, 1);
            atomicExch(&a.ctl->fault, 1);
        }
        return;
    }
    // sweep jf's iterate into sol0: odd sweeps wrote sol1
    if (jf & 1) {
        const int r1 = seg[ncol];
        for (int r = tile_row0 + threadIdx.x; r < r1; r += blockDim.x) {
            const int n = a.bcol[(size_t)r * CR] & (int)~TILE_LOWER;
            a.sol0[3 * n] = a.sol1[3 * n];
            a.sol0[3 * n + 1] = a.sol1[3 * n + 1];
            a.sol0[3 * n + 2] = a.sol1[3 * n + 2];
        }
    }
    if (t == 0 && threadIdx.x == 0 && jf > 0) {
        const int s = jf & (TILE_SLOTS_SYNC - 1);
        a.ctl->err = a.sync->derr[s];
        a.ctl->conv = a.sync->dconv[s];
        a.ctl->sweeps = a.sweep_base + jf;
    }
}

// Tile-layout copy of the assembled rows: block values (FP64 or rounded to
// FP32) and the reciprocal diagonal, one warp per tile row.  src_row[r] is
// the colour-layout row of tile row r.
template <typename T>
__global__ void __launch_bounds__(256) k_tile_pack(BlockDev B, const int *__restrict__ src_row, int rows,
                                                   T *__restrict__ dst, double *__restrict__ rdiag)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int brow = B.brow;
    for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < rows; r += gridDim.x * wpb) {
        const int p = src_row[r];
        const double *s = B.blk + (size_t)p * brow;
        T *d = dst + (size_t)r * brow;
        for (int k = lane; k < brow; k += 32) d[k] = (T)s[k];
        if (lane < 3 && rdiag) rdiag[3 * (size_t)r + lane] = 1.0 / s[(size_t)(4 * lane) * B.slots];
    }
}

}  // namespace fasdev
