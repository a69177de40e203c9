/*
 * CPU oracle for the fdfault time-stepping path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-process restatement of the reference solver's per-stage
 * update (domain::do_rk_stage, src/domain.cpp:228-305 of edaub/fdfault) and of
 * the set-up it depends on (input parsing, transfinite grid, SBP metrics,
 * boundary/interface normals, friction parameters, time step).  Every
 * function in fdf_oracle.c cites the reference file:line it restates and keeps
 * the reference's floating-point operation order, so on the same input it
 * produces bit-identical doubles to the reference built without FMA
 * contraction (checked against oracle/_ref by tests/test_oracle_ref.py).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product path never calls
 * it.
 */
#ifndef FDF_ORACLE_H
#define FDF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

/* field selectors for orc_field() */
enum { ORC_F = 0, ORC_DF = 1, ORC_X = 2, ORC_METRIC = 3, ORC_JAC = 4, ORC_S = 5 };
/* fault array selectors for orc_fault() */
enum {
    ORC_U = 0, ORC_DU = 1, ORC_V = 2, ORC_SS = 3, ORC_SN = 4, ORC_UX = 5, ORC_DUX = 6,
    ORC_VX = 7, ORC_SX = 8, ORC_STATE = 9, ORC_DSTATE = 10, ORC_DSTATEDT = 11, ORC_TFRONT = 12
};

orc_problem *orc_load(const char *infile, char *err, int errlen);
void orc_free(orc_problem *p);

/* ints[0..]: ndim, mode, nx, ny, nz, nfields, nfieldsp, nifaces, nstages, nt, sbporder,
 *            nblocks0, nblocks1, nblocks2, is_plastic, rkorder
 * dbls[0..]: dt, ttot, cfl */
void orc_info(const orc_problem *p, int *ints, double *dbls);
double *orc_field(orc_problem *p, int which);
/* n[0], n[1]: fault plane size; returns 0 if the interface has no such array */
double *orc_fault(orc_problem *p, int iface, int which, int *n0, int *n1);
int orc_iface_info(const orc_problem *p, int iface, int *ints);

/* one Runge-Kutta stage / one step / nsteps steps; return 0 or an error code */
int orc_do_rk_stage(orc_problem *p, double dt, int stage, double t);
int orc_step(orc_problem *p, int step_index);
int orc_run(orc_problem *p, int first_step, int nsteps);

/* absolute/relative stress conversions of the whole field array */
void orc_set_stress(orc_problem *p);
void orc_remove_stress(orc_problem *p);
void orc_abs_field(const orc_problem *p, int c, double *out);

const char *orc_last_error(const orc_problem *p);

#ifdef __cplusplus
}
#endif

#endif
