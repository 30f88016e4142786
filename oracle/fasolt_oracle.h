/*
 * fasolt_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of FASOLT3's per-increment hot path (gabortimar/CPFEM_code,
 * src/fasolt/, all .f90 files), used by the tests, the smoke check and the CPU-baseline
 * leg of the benchmark as the checker.  The product path never links or calls
 * it.  Parity status: unpinned by the reference -- the reference ships no
 * tests, golden outputs or fixtures with expected results, and no Fortran
 * compiler exists here to run it; the restatement is pinned instead by
 * physics known-answer tests (tests/test_oracle_kat.py).
 *
 * The entry points mirror include/fasolt_gpu.h one for one (ora_* for
 * fas_gpu_*), take the same descriptors, and return the same codes.
 * ora_create's `real_bytes` picks the arithmetic: 8 = the reference promoted
 * to double (-freal-4-real-8), 4 = the FP32-faithful restatement.
 */
#ifndef FASOLT_ORACLE_H
#define FASOLT_ORACLE_H

#include "../include/fasolt_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_problem ora_problem;

int32_t ora_create(const fas_mesh_desc *mesh, const fas_matl_desc *matl,
                   const fas_ctrl_desc *ctrl, int32_t real_bytes,
                   uint32_t mode, ora_problem **out);
void    ora_destroy(ora_problem *p);
int32_t ora_set_mode(ora_problem *p, uint32_t mode);
int32_t ora_set_threads(ora_problem *p, int32_t nthreads);
int32_t ora_upload_state(ora_problem *p, const fas_state_desc *s);
int32_t ora_download_state(ora_problem *p, const fas_state_desc *s);
int32_t ora_update_node(ora_problem *p);
int32_t ora_elvals(ora_problem *p, int32_t inc, int32_t nit);
int32_t ora_suvals(ora_problem *p, int32_t inc);
int32_t ora_facsls(ora_problem *p, int32_t *sweeps, double *error);
int32_t ora_facsls_limited(ora_problem *p, int32_t max_sweeps, int32_t *sweeps,
                           double *error);
int32_t ora_nriter(ora_problem *p, int32_t inc, fas_iter_report *rep,
                   int32_t cap, int32_t *n_rep);
/* One pass of NRITER's loop body; *more = 1 when NRITER would go on. */
int32_t ora_nr_step(ora_problem *p, int32_t inc, int32_t nit, fas_iter_report *rep,
                    int32_t *more);
/* NRITER's cumslip update after its loop. */
int32_t ora_nr_finish(ora_problem *p, int32_t inc);
int32_t ora_update_gptv(ora_problem *p);
int32_t ora_reorient(ora_problem *p, int32_t inc, fas_twin_event *ev,
                     int32_t cap, int32_t *n_ev);
int32_t ora_increment(ora_problem *p, int32_t inc, fas_iter_report *rep,
                      int32_t cap, int32_t *n_rep, fas_twin_event *ev,
                      int32_t ev_cap, int32_t *n_ev);
int32_t ora_get_pattern(ora_problem *p, int32_t *is, int32_t ld_is);
int32_t ora_get_stiffness(ora_problem *p, void *ss, int32_t ld_ss,
                          int32_t real_bytes);
int32_t ora_get_colouring(ora_problem *p, int32_t *colour, int32_t *ncol);
int32_t ora_constitutive(ora_problem *p, int32_t inc, int32_t nit);
int32_t ora_get_tangent(ora_problem *p, void *chi, int32_t real_bytes);
int32_t ora_get_cp_stats(ora_problem *p, int32_t *iters, double *erepmd);
/* Per-GP algorithmic operation counts of the last constitutive pass. */
int32_t ora_get_cp_ops(ora_problem *p, double *ops);

/* ELASEPS (src/csvmkr/data_out.f90:263-361): out[g*6 + k]. */
int32_t ora_lattice_strain(ora_problem *p, double *out);

/* The replay of fas_gpu_adjoint_forward (its checker): DSTRSS per
 * increment from the elastic predictor, then UPDATE_GPTV's commit. */
int32_t ora_adjoint_forward(ora_problem *p, const fas_replay_desc *d, double *J, double *eq);

/* Low-level single-routine checks for the known-answer tests (double). */
double  ora_spower(double a, double b);
double  ora_fj2vom(int32_t stress, const double *x6);
int32_t ora_factor_solve(int32_t n, const double *a_colmajor, double *x);
void    ora_ctmatrx(double ph1, double phi, double ph2, double *a9_colmajor,
                    double *aug3);
void    ora_elastc(const double *e9, const double *euler3, double *s36_colmajor);
void    ora_tens_rot(const double *r3, const double *a6, double *b6);
double  ora_shape12(const double *xnode_3x8_colmajor, double *dndx_3x8_colmajor);
/* SHAPE_22 at Gauss point g (0-based) and its local-derivative table
 * dn[(g*3 + j)*20 + i] = dndn(j+1, i+1, g+1). */
double  ora_shape22(int g, const double *xnode_3x20_colmajor, double *dndx_3x20_colmajor);
void    ora_shape22_table(double *dn_8x3x20);

/* SHAPE_21/22/23 of type lt at GP g (tests) and the SHAPE_21/23 tables. */
double ora_shape_elem(int lt, int g, const double *x, double *d);
void ora_shape21_table(double *dn);
void ora_shape23_table(double *dn);
#ifdef __cplusplus
}
#endif
#endif /* FASOLT_ORACLE_H */
