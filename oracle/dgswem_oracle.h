/*
 * dgswem_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C API of the CPU FP64 restatement of the DG-SWEM explicit hydro time step
 * (reference: src/DG_hydro_timestep.F and the routines it calls).  The oracle
 * is the checker for the CUDA library: only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may load it.  No product code path calls it.
 *
 * State exchange layout is the reference's Fortran layout of one stage slice:
 * ZE(DOFH, NE) column-major, i.e. ze[k + dofh*e] with 0-based k and e.
 */
#ifndef DGSWEM_ORACLE_H
#define DGSWEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;

/* Read fort.14/15/dg (+fort.13) from `dir`, run PREP_DG.  NULL on error,
 * message copied into err. */
orc_model* orc_open(const char* dir, char* err, int errlen);
void orc_close(orc_model* m);
/* Number of OpenMP threads the oracle uses (1 = scalar). */
void orc_set_threads(int n);

/* ints: ne, np, dofh, nrk, nt, nedges, nieds, nleds, needs, nfeds, nreds,
 *       nebseg, nibseg, nspoolge, nolifa, slopeflag, ics, nws, rainfall */
int orc_info_int(const orc_model* m, const char* key);
double orc_info_real(const orc_model* m, const char* key);

/* One call of DG_HYDRO_TIMESTEP(IT). */
int orc_step(orc_model* m, int it);
/* Run steps it0..it1 inclusive. */
int orc_run(orc_model* m, int it0, int it1);

/* Stage-1 state in Fortran layout (dofh*ne), wdflg (ne). */
void orc_get_state(const orc_model* m, double* ze, double* qx, double* qy, int* wdflg);
void orc_set_state(orc_model* m, const double* ze, const double* qx, const double* qy, const int* wdflg);
void orc_get_hb(const orc_model* m, double* hb);
void orc_get_nodecode(const orc_model* m, int* nodecode);

/* modal2nodal (reference write_results.F:14-170) on the stage-1 state. */
void orc_modal2nodal(const orc_model* m, double* eta2, double* uu2, double* vv2);

/* Uniform-in-time nodal met forcing for NWS=1 (kinematic stress, pressure
 * head); each stage applies RAMPDG * value, as MET_FORCING does. */
void orc_set_met(orc_model* m, const double* wsx, const double* wsy, const double* pr);

/* Integer edge tables, 1-based as in the reference (for bit-exact checks).
 * which: "NEDNO" (2*nedges), "NEDEL" (2*nedges), "NELED" (3*ne),
 * "NEDSD" (2*nedges), "NIEDN","NLEDN","NEEDN","NFEDN","NREDN","NEBSEGN",
 * "NIBSEGN" (2*nibseg), "ELEM_EDGE" (3*ne).  Returns the element count. */
int orc_get_int_table(const orc_model* m, const char* which, int* out, int cap);
/* Real tables: "XLEN","COSNX","SINNX" (nedges), "AREAS" (ne), "DP" (np),
 * "X","Y" (np), "HB" (dofh*ne); basis and area rule: "PHI_AREA"
 * (dofh*NAGP, [k*NAGP + i]), "XAGP","YAGP","WAGP" (NAGP, reference
 * triangle (-1,-1),(1,-1),(-1,1), weights summing to 2), "M_INV" (dofh). */
int orc_get_real_table(const orc_model* m, const char* which, double* out, int cap);

/* The Manning depth factor DEPTH**(1.D0/3.D0) as the oracle evaluates it
 * (correctly rounded), over xs[0..n) into out. */
void orc_pow_third(const double* xs, long n, double* out);

/* Full reference-style run writing fort.63 (elevation) to out_path. */
int orc_run_case(const char* dir, const char* out_path, char* err, int errlen);

#ifdef __cplusplus
}
#endif
#endif
