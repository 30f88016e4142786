/*
 * fasolt_gpu.h -- C ABI of the B200 (sm_100a) implementation of FASOLT3's
 * per-increment hot path: the crystal-plasticity Gauss-point update, element
 * assembly, penalty boundary conditions, SOR solve and the increment commit.
 *
 * The Fortran driver (src/fasolt/Fasolt3.f90) keeps its module arrays
 * (FAS_COM / FAS_CPL in src/fasolt/fas-com-mod.f90:9-43,54-80) and reaches
 * this library through ISO_C_BINDING.  Every pointer below may point straight
 * at a Fortran module array: arrays are column-major with explicit leading
 * dimensions, index arrays are 1-based, and reals are REAL(4) or REAL(8) as
 * the caller says in `real_bytes`.  Nothing crosses this boundary as a C++ or
 * torch type.
 *
 * Return codes of every `int32_t` entry point:
 *    0                 success
 *  > 0                 the reference's own FAFERR code, raised at the point
 *                      where the reference would raise it (first failing
 *                      element / DOF in the reference's loop order):
 *                      903 zero SOR diagonal, 904 SOR not converged,
 *                      905 rotation increment too large, 906 strain increment
 *                      too large, 910 singular local Jacobian, 920 element
 *                      weight too small, 987 slip Newton failed (tauerr>0.5)
 *  < 0                 FAS_E_* errors of this ABI (bad argument, no sm_100
 *                      device, CUDA failure, unsupported element type).
 * There is no CPU fallback: without an sm_100 device fas_gpu_create returns
 * FAS_E_NODEVICE.
 */
#ifndef FASOLT_GPU_H
#define FASOLT_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define FAS_API __attribute__((visibility("default")))
#else
#define FAS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes of the ABI itself (reference FAFERR codes are > 0) ---- */
#define FAS_OK              0
#define FAS_E_ARG          (-1)  /* null / inconsistent argument            */
#define FAS_E_NODEVICE     (-2)  /* no sm_100 (B200) device visible          */
#define FAS_E_CUDA         (-3)  /* a CUDA runtime call failed               */
#define FAS_E_ELTYPE       (-4)  /* element type not implemented: lt other than 12, 21, 22 or 23 (ties 1-6 aside), or two of them in one mesh */
#define FAS_E_NOMEM        (-5)  /* device allocation failed                 */
#define FAS_E_RANGE        (-6)  /* size beyond a documented maximum         */
#define FAS_E_STATE        (-7)  /* call out of order (e.g. no state yet)    */
#define FAS_E_TIMEOUT      (-8)  /* a device-side bounded wait gave up       */

#define FAS_MAXSS  60            /* maxss, src/fasolt/fas-com-mod.f90:57     */
#define FAS_MAXSVS 63            /* maxsvs, src/fasolt/fas-com-mod.f90:14    */

/* ---- mode flags for fas_gpu_create / fas_gpu_set_mode ------------------ */
#define FAS_MODE_PLAIN        0u  /* FP64 everywhere, reference tangent      */
#define FAS_MODE_SOR_FP32     1u  /* SOR sweeps on an FP32 copy of the
                                     matrix (FP32 products, FP64 point
                                     update and stopping test) with an FP64
                                     residual every 16 sweeps               */
#define FAS_MODE_SOR_NATURAL  2u  /* (oracle only) natural-order SOR        */
#define FAS_MODE_CP_WARP      8u  /* Gauss-point update with one warp per GP
                                     (lanes = slip systems) instead of one
                                     thread per GP; at most 32 systems      */
#define FAS_MODE_SOR_GRID     4u  /* always use the grid-wide SOR launches,
                                     also for meshes small enough for the
                                     one-CTA solve                          */
#define FAS_MODE_TANGENT_CONSISTENT 32u  /* element tangent (B X^-1 B^T + S)^-1
                                     of the local system re-evaluated at
                                     the converged stress (the implicit-
                                     function derivative of the converged
                                     CPSTRS update, no counterpart in the
                                     reference) instead of CPSTRS's chi of
                                     the last iterate (Cpstrs.f90:154-162);
                                     symmetrised like chi                  */
#define FAS_MODE_CP_QUEUE    64u  /* constitutive passes on a persistent grid
                                     whose warps take the next 32 GPs of the
                                     work-sorted (heaviest first) order from
                                     a device queue, instead of one thread
                                     per GP in that order.  Meshes whose GPs'
                                     materials differ in their slip-system
                                     counts (mixed FCC/HCP) take the queue
                                     without the flag                       */
#define FAS_MODE_SOR_TILES   16u  /* grid-wide SOR as one persistent launch
                                     per solve: spatial tiles of rows, one
                                     per SM, that start each colour once
                                     their neighbour tiles have finished the
                                     previous one (8-node bricks; other
                                     meshes keep one launch per colour)     */
#define FAS_MODE_GRAPH      128u  /* fas_gpu_nriter as one CUDA graph per
                                     increment: the Newton loop and the SOR
                                     loop are conditional while nodes whose
                                     conditions the device sets (sdx >=
                                     toler and nit < maxit; not converged
                                     and below 1000 sweeps), so the
                                     increment runs with one launch and one
                                     host read.  Same arithmetic and launch
                                     shapes as the host-driven loop, so the
                                     same results to the bit; combines with
                                     FAS_MODE_SOR_FP32 (cycles of sweeps,
                                     fold and residual as the loop body).
                                     With FAS_MODE_SOR_TILES, and while
                                     profiling with prof >= 2, the host loop
                                     runs.  The graph of an increment is
                                     built on its first call and kept until
                                     the mode changes                       */
#define FAS_MODE_SOR_SYM    256u  /* with FAS_MODE_SOR_FP32 on 8-node meshes:
                                     the FP32 sweeps stream each off-diagonal
                                     block once (K_mn = K_nm^T), from the
                                     row of one of its two nodes, and push
                                     its transposed product with each change
                                     of that node into a per-node FP32
                                     accumulator of the other (vector atomic
                                     adds): 608 instead of 1,088 bytes per
                                     row.  The same iteration as
                                     FAS_MODE_SOR_FP32 to FP32 rounding, but
                                     the order of the atomic adds varies, so
                                     results are not bit-reproducible from
                                     run to run.  No effect on 20-node or
                                     quadratic meshes, nor on a pattern
                                     whose rows would store more than 14
                                     blocks                                 */

/*
 * Mesh: the FAS_COM element and node tables.
 * Replaces the element/node arrays read by RDDATA
 * (src/fasolt/Faslt_io_nowin.f90:36-53).  ln(1:ld_ln,1:nlmnt) and
 * lg(1:ld_lg,1:nlmnt) are Fortran column-major with 1-based ids.
 * nlmnt == 0 makes a mesh-free "point batch" of ngps independent Gauss
 * points; `le` then holds one material code per point (length ngps).
 */
typedef struct fas_mesh_desc {
    int32_t nlmnt, nnod, ngps;
    const int32_t *le, *lt, *nd, *np;    /* [nlmnt]                        */
    const int32_t *ln;  int32_t ld_ln;   /* node ids, ln(ld_ln, nlmnt)     */
    const int32_t *lg;  int32_t ld_lg;   /* GP ids,   lg(ld_lg, nlmnt)     */
    const int32_t *ib;                   /* [nnod] boundary codes ccbbaa   */
} fas_mesh_desc;

/*
 * Materials: the FAS_CPL tables (src/fasolt/fas-com-mod.f90:59-78), as read
 * by RDDATA (src/fasolt/Faslt_io_nowin.f90:66-116).
 */
typedef struct fas_matl_desc {
    int32_t real_bytes;                  /* 4 (REAL(4)) or 8 (REAL(8))     */
    int32_t nmatl, nmpar;
    int32_t ld_ss;                       /* leading dim of the ss tables
                                            (maxss = 60 in the reference)  */
    const int32_t *nss;                  /* [nmatl]                        */
    const void *e;                       /* e(9, nmatl) compliances 1/MPa  */
    const void *ssang;                   /* ssang(ld_ss, nmatl) degrees    */
    const void *ab, *an;                 /* (3, ld_ss, nmatl)              */
    const void *ampar;                   /* ampar(10, ld_ss, nmatl)        */
    const void *smatrx;                  /* smatrx(ld_ss, ld_ss, nmatl)    */
    int32_t twinlim;
    double  twinprob;
} fas_matl_desc;

/*
 * Control: fafcdf.dat scalars read by FSINIT (src/fasolt/Fasolt3.f90:216-218)
 * and the per-increment loading read by RDDATA
 * (src/fasolt/Faslt_io_nowin.f90:123-138).
 */
typedef struct fas_ctrl_desc {
    int32_t real_bytes;                  /* element size of tiem/x/f_spec  */
    int32_t maxit;
    double  toler, alpha, afactor, efix, smale, smalr;
    int32_t ninc1, nxs, nfs;
    int32_t ld_xs;                       /* 2nd dim of x_spec/f_spec (99)  */
    const void *tiem;                    /* [ninc1]                        */
    const void *x_spec;                  /* x_spec(15, ld_xs, ninc1)       */
    const void *f_spec;                  /* f_spec(3,  ld_xs, ninc1) or 0  */
    uint64_t twin_seed;                  /* key of the counter-based twin
                                            RNG (stands in for RANDOM_NUMBER,
                                            src/fasolt/crys-cons.f90:169)  */
} fas_ctrl_desc;

/*
 * Nodal and Gauss-point state (FAS_COM / FAS_CPL arrays).  Used for upload
 * (read) and download (written).  Any pointer may be null to skip it.
 */
typedef struct fas_state_desc {
    int32_t real_bytes;
    int32_t nsv;                         /* state variables per GP used    */
    int32_t ld_sv;                       /* leading dim of sv/dsv (63)     */
    int32_t ld_slip;                     /* leading dim of srate/cumslip   */
    void *x, *dx, *fc, *ddx;             /* [3*nnod]                       */
    void *eps, *dep;                     /* [ngps]                         */
    void *st, *ep, *ds, *de;             /* (6, ngps)                      */
    void *rt, *dr;                       /* (3, ngps)                      */
    void *sv, *dsv;                      /* (ld_sv, ngps)                  */
    int32_t *timestwinned, *twinsys;     /* [ngps]                         */
    void *srate, *cumslip;               /* (ld_slip, ngps)                */
} fas_state_desc;

/* One line of the NRITER progress report (ITEREP,
 * src/fasolt/Faslt_io_nowin.f90:309-344), plus the SOR statistics. */
typedef struct fas_iter_report {
    int32_t nit;
    int32_t sor_sweeps;
    double  sdx, sfc, cp_err, alp2;
    double  sor_error;
} fas_iter_report;

/* One twin reorientation (the unit-55 "twins" record written by DoReorient,
 * src/fasolt/Fasolt3.f90:164).  gp and sys are 1-based. */
typedef struct fas_twin_event {
    int32_t inc, gp, sys, pad;
    double  euler_old[3], euler_new[3];
} fas_twin_event;

typedef struct fas_handle fas_handle;

/* Creates a device problem: uploads mesh, materials and loading, builds the
 * node adjacency, the node colouring for SOR and the block-ELL stiffness
 * layout.  Replaces the set-up half of SETPTA (src/fasolt/Stif_sol.f90:98-149)
 * and the table reads of RDDATA.  `mode` is a FAS_MODE_* mask. */
FAS_API int32_t fas_gpu_create(const fas_mesh_desc *mesh, const fas_matl_desc *matl,
                       const fas_ctrl_desc *ctrl, uint32_t mode,
                       fas_handle **out);
FAS_API void    fas_gpu_destroy(fas_handle *h);
FAS_API int32_t fas_gpu_set_mode(fas_handle *h, uint32_t mode);

/* Copies Fortran-side state to the device (promoted to FP64) / back. */
FAS_API int32_t fas_gpu_upload_state(fas_handle *h, const fas_state_desc *s);
FAS_API int32_t fas_gpu_download_state(fas_handle *h, const fas_state_desc *s);

/* UPDATE_NODE, src/fasolt/Fasolt3.f90:231-244:  x += dx. */
FAS_API int32_t fas_gpu_update_node(fas_handle *h);

/* ELVALS, src/fasolt/Elvals.f90:11-275 (with fc zeroed first, as
 * NRITER does at src/fasolt/Stif_sol.f90:38-39).  `nit` is the global
 * Newton iteration number (keys the twin RNG). */
FAS_API int32_t fas_gpu_elvals(fas_handle *h, int32_t inc, int32_t nit);

/* SUVALS, src/fasolt/Bconds.f90:19-113. */
FAS_API int32_t fas_gpu_suvals(fas_handle *h, int32_t inc);

/* FACSLS, src/fasolt/Stif_sol.f90:161-215: SOR on the assembled system,
 * right-hand side taken from ddx, solution left in ddx.  Multicolour node
 * order (see fas_gpu_get_colouring). */
FAS_API int32_t fas_gpu_facsls(fas_handle *h, int32_t *sweeps, double *error);

/* NRITER, src/fasolt/Stif_sol.f90:10-88: the damped global Newton loop of
 * increment `inc` including the cumslip update.  Up to `cap` report lines
 * are written to `rep` (may be null); *n_rep receives the iteration count. */
FAS_API int32_t fas_gpu_nriter(fas_handle *h, int32_t inc, fas_iter_report *rep,
                       int32_t cap, int32_t *n_rep);

/* One pass of NRITER's loop body, src/fasolt/Stif_sol.f90:32-77: ELVALS,
 * SUVALS, the residual norm, FACSLS, the damping factor and the correction
 * of x and dx, for a driver that keeps its own Newton loop (ITEREP after
 * every pass).  `nit` is the 1-based iteration number; *more receives the
 * reference's loop condition (sdx >= toler and nit < maxit).  After the last
 * pass call fas_gpu_nr_finish.  fas_gpu_nriter is this loop. */
FAS_API int32_t fas_gpu_nr_step(fas_handle *h, int32_t inc, int32_t nit, fas_iter_report *rep,
                        int32_t *more);

/* NRITER's tail after its loop, src/fasolt/Stif_sol.f90:80-84: cumslip +=
 * srate * tiem(inc) over nss(mat_code) of the last element evaluated. */
FAS_API int32_t fas_gpu_nr_finish(fas_handle *h, int32_t inc);

/* UPDATE_GPTV, src/fasolt/Fasolt3.f90:254-284. */
FAS_API int32_t fas_gpu_update_gptv(fas_handle *h);

/* DoReorient, src/fasolt/Fasolt3.f90:79-178.  Events are returned in
 * ascending GP order; *n_ev may exceed cap (then only cap are written). */
FAS_API int32_t fas_gpu_reorient(fas_handle *h, int32_t inc, fas_twin_event *ev,
                         int32_t cap, int32_t *n_ev);

/* One whole increment of the driver loop (src/fasolt/Fasolt3.f90:38-46):
 * UPDATE_NODE, NRITER, UPDATE_GPTV and, when a twin fired, DoReorient. */
FAS_API int32_t fas_gpu_increment(fas_handle *h, int32_t inc, fas_iter_report *rep,
                          int32_t cap, int32_t *n_rep, fas_twin_event *ev,
                          int32_t ev_cap, int32_t *n_ev);

/* The compact stiffness pattern of SETPTA (src/fasolt/Stif_sol.f90:98-149),
 * rebuilt on the device: is(1,row) = off-diagonal count, is(2..,row) = 1-based
 * columns in first-touch order.  `is` is (ld_is, 3*nnod), column-major. */
FAS_API int32_t fas_gpu_get_pattern(fas_handle *h, int32_t *is, int32_t ld_is);

/* The assembled stiffness (after ELVALS [+ SUVALS]) in the reference layout
 * ss(ld_ss, 3*nnod): ss(1,row) = diagonal, ss(k,row) = value of column
 * is(k,row).  Replaces reading the module array ss. */
FAS_API int32_t fas_gpu_get_stiffness(fas_handle *h, void *ss, int32_t ld_ss,
                              int32_t real_bytes);

/* Node colour of every node (0-based colours, [nnod]) and the colour count:
 * the SOR visits colours in ascending order, nodes of one colour in any
 * order, and the three DOFs of a node in x, y, z order. */
FAS_API int32_t fas_gpu_get_colouring(fas_handle *h, int32_t *colour, int32_t *ncol);

/* DSTRSS, src/fasolt/Sig_eps.f90:84-151, for every GP of the handle, taking
 * the strain increment de(:,j) and spin dr(:,j) from the uploaded state
 * (the constitutive micro-benchmark).  Updates ds, dsv, dep, srate and the
 * twin flags on the device; the 6x6 tangent is kept for fas_gpu_get_tangent. */
FAS_API int32_t fas_gpu_constitutive(fas_handle *h, int32_t inc, int32_t nit);

/* The symmetrised tangent chi(6,6,ngps) of the last constitutive pass
 * (upper triangle mirrored), column-major. */
FAS_API int32_t fas_gpu_get_tangent(fas_handle *h, void *chi, int32_t real_bytes);

/* Per-GP diagnostics of the last constitutive pass: outer (CPSTRS) iteration
 * count and final erepmd.  Either pointer may be null. */
FAS_API int32_t fas_gpu_get_cp_stats(fas_handle *h, int32_t *iters, double *erepmd);

/* ELASEPS (src/csvmkr/data_out.f90:263-361): the elastic lattice strain
 * e = S(sv(1:3)) st of every GP, engineering shears, into strain(6, ngps)
 * (column-major, element size real_bytes).  The forward map of csvmkr's
 * el_eps columns. */
FAS_API int32_t fas_gpu_lattice_strain(fas_handle *h, void *strain, int32_t real_bytes);

/* Adjoint of the constitutive update (no counterpart in the reference).
 *
 * A replay drives every GP through a recorded history of ninc increments:
 * DSTRSS from the uploaded stress st and state sv with the increment's
 * strain increment, spin and time step, then UPDATE_GPTV's commit.  Each
 * increment starts from its own orientation and slip resistances and from
 * the elastic predictor as the stress guess, as an increment's first
 * Newton iteration does.  Twins are flagged but not reoriented.  The
 * handle's own state is not changed.
 *
 * The objective is J = sum_g w(g) (q^T e_g q - y(g))^2 / 2, where e_g is the
 * lattice strain S(sv(1:3)) st of GP g after the last increment (as
 * fas_gpu_lattice_strain gives it) and q the scattering direction.  The
 * weights select and scale GPs, e.g. 1/count for the GPs of one orientation
 * bin and 0 elsewhere.
 *
 * Gradients come from the implicit function theorem at each increment's
 * converged CPSTRS system, swept backwards over the increments from
 * checkpoints taken every chk_every increments (the forward sweep keeps
 * the last segment; each earlier one is recomputed from its checkpoint
 * before it is swept).  They are exact for the replay
 * as converged: a tight toler makes them agree with finite differences of
 * fas_gpu_adjoint_forward.  Materials of at most 32 slip systems. */
typedef struct fas_replay_desc {
    int32_t ninc;          /* increments in the history (>= 1)                 */
    int32_t chk_every;     /* checkpoint interval of the reverse sweep (>= 1)  */
    const double *de;      /* de(6, ngps, ninc): strain increments, eng. shears */
    const double *dr;      /* dr(3, ngps, ninc): spins, as DSTRNS returns them  */
    const double *dt;      /* dt(ninc): time increments (tiem)                 */
    const double *w;       /* w(ngps): objective weight of each GP             */
    const double *y;       /* y(ngps): target lattice strain of each GP        */
    double q[3];           /* scattering direction (normalised by the call)    */
} fas_replay_desc;

/* The replay and its objective: J, and when eq is non-null the final
 * lattice strain q^T e_g q of every GP into eq(ngps).  Returns 0, a FAFERR
 * code of DSTRSS, or an ABI error (FAS_E_RANGE for more than 32 systems). */
FAS_API int32_t fas_gpu_adjoint_forward(fas_handle *h, const fas_replay_desc *d, double *J, double *eq);

/* J and its gradients with respect to the replay's starting stress
 * g_st(6, ngps), starting state g_sv(FAS_MAXSVS, ngps) (Euler angles in rows 1-3,
 * slip resistances in rows 4..3+ns, zero elsewhere) and hardening
 * parameters g_ampar(10, nmatl): entry k of material m is dJ/dc for
 * ampar(k, i, m) + c on every slip system i, filled for k = 1 (rate
 * exponent), 2, 3 and 5 (saturation stress), zero for the others.  Column-
 * major; any of the three may be null. */
FAS_API int32_t fas_gpu_adjoint_grad(fas_handle *h, const fas_replay_desc *d, double *J, double *g_st,
                                     double *g_sv, double *g_ampar);

/* Per-GP algorithmic operation count of the last constitutive pass (the
 * formulas of fas_flops.h summed over the iterations each GP took). */
FAS_API int32_t fas_gpu_get_cp_ops(fas_handle *h, double *ops);

/* Device time per phase, measured with CUDA events on the handle's stream
 * while profiling is on, plus launch counts and algorithmic work. */
typedef struct fas_profile {
    double  ms_constitutive;   /* element kernel (kinematics + DSTRSS)      */
    double  ms_assembly;       /* row-gather assembly (+ fused SUVALS)      */
    double  ms_sor_colour;     /* multicolour SOR colour-phase kernels      */
    double  ms_total;          /* everything on the stream while profiling  */
    int64_t n_constitutive, n_assembly, n_sor_colour;
    int64_t n_launches;        /* all kernels this library launched         */
    int64_t gp_updates;        /* DSTRSS evaluations                        */
    int64_t sor_sweeps;
    double  sor_bytes;         /* algorithmic bytes of the colour kernels   */
    double  assembly_bytes;    /* algorithmic bytes of the assembly kernel  */
} fas_profile;

/* enable = 1 starts (and zeroes) profiling with counters and one event
 * pair around the whole region (ms_total); enable = 2 also brackets every
 * phase kernel launch with an event pair (the per-phase ms_*, at some
 * launch-rate cost); 0 stops.  When `out` is non-null the counters so far
 * are written to it first. */
FAS_API int32_t fas_gpu_profile(fas_handle *h, int32_t enable, fas_profile *out);

/* FACSLS that allocates no device memory in the call.  No counterpart in
 * the reference.
 *
 * Who needs it: a driver that must not allocate device memory once set-up
 * is over -- one that hands all memory left after fas_gpu_create to
 * another allocator (a coupled solver's pool, a caching allocator) or runs
 * under a fixed device-memory cap.  fas_gpu_facsls allocates on first use
 * (it instantiates a CUDA graph of its sweeps), which can then fail in
 * the middle of a run; this entry point never does.
 *
 * What it does: the same solve as fas_gpu_facsls -- the same iterates
 * (one launch per colour, the colour order, the reciprocal-diagonal
 * quotients), sweep count and stopping test, same return codes (903, 904,
 * FAS_E_TIMEOUT) -- on the FP64 blocks, with the kernels' scratch (the
 * stopping-test control words and one pair of partial sums per colour
 * CTA) in a static device array of this library instead of buffers of the
 * handle.  It ignores FAS_MODE_SOR_FP32 and FAS_MODE_SOR_TILES and is not
 * timed by fas_gpu_profile.  It reads the stopping flag between chunks of
 * sweeps, so it synchronises the handle's stream before it returns.
 *
 * Limits and rules:
 *  - the array holds FAS_NOALLOC_PARTIALS partial pairs (262,400 bytes per
 *    device, held by every GPU that loads the library until the process
 *    exits); a handle whose layout needs more (colours x colour-kernel CTAs
 *    per colour) gets FAS_E_RANGE.  On a 148-SM B200 the 64^3 8-node cube
 *    needs 8 x 888 = 7,104 pairs and the 32^3 20-node brick mesh about
 *    15 x 592 = 8,880; meshes of 27-slot rows with more than 18 colours,
 *    or of 81-slot rows with more than 27, can exceed the array;
 *  - the first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress, with the handle's device made current for the
 *    look-up); make that first call before any stream capture begins;
 *  - the control words must be zero when a solve starts: every call zeroes
 *    them itself on the handle's stream before its first sweep; the
 *    partial sums need no initial value (each is written before it is
 *    read);
 *  - there is one array per device and process, so calls that overlap in
 *    time on the same device (two host threads, two handles) race on it:
 *    the caller must serialise them. */
#define FAS_NOALLOC_PARTIALS 16384
FAS_API int32_t fas_gpu_facsls_noalloc(fas_handle *h, int32_t *sweeps, double *error);

#ifdef __cplusplus
}
#endif
#endif /* FASOLT_GPU_H */
