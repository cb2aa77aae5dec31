/*
 * jk_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of the J-Kogbetliantz hyperbolic SVD step loop of
 * venovako/JKogb (real `djk` and complex `zjk`), written from the reference's
 * Fortran sources and cited function by function in jk_oracle.c / jk_oracle_z.c.
 * It is the checker for the CUDA product and the CPU baseline of the benchmark;
 * nothing in the product links, loads or calls it.
 *
 * Arithmetic contract (shared, operation for operation, with the CUDA kernels):
 *   - every FMAD(a,b,c) of the reference is a fused fma(a,b,c); the file is
 *     compiled with -ffp-contract=off so no other operation is fused;
 *   - division and sqrt are IEEE-754 round-to-nearest;
 *   - HYPOT / complex ABS use jo_hypot(), a project-own hypot (one Newton
 *     correction with an error-free residual), not libm;
 *   - EXPONENT / SCALE are exact integer restatements (frexp exponent,
 *     correctly rounded x*2^e);
 *   - MIN/MAX that must ignore NaN are fmin/fmax.
 *
 * Index convention: matrices are column-major with leading dimension ld;
 * pivot indices p, q in traces and records are 1-based, as in the reference.
 */
#ifndef JK_ORACLE_H
#define JK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } jo_z;

/* The reference's AW record (src/shared/atypes.F90:18-24). */
typedef struct { double w; int p, q, b, i; } jo_aw;

/* Optional per-step trace of a solve. */
typedef struct {
  int max_steps;       /* capacity of the per-step arrays (may be 0) */
  int *sl;             /* SL after the build (selected pivots), per step */
  int *nl;             /* NL returned by the transform (effective pivots), per step; -1 if not run */
  int *trig;           /* trigonometric / hyperbolic effective pivots per step */
  int *hyp;
  double *tw;          /* NORMF2D column: sum of weights of effective pivots, per step */
  long long max_piv;   /* capacity of piv (pairs) */
  int *piv;            /* 2 ints per selected pivot (p,q), 1-based, in STEP order, all steps */
  long long n_piv;     /* out: number of pivots written */
  int n_steps;         /* out: number of EXEC calls recorded */
} jo_trace;

/* ---- scalar helpers (src/shared/params.F90, src/shared/utils.F90) ---- */
double jo_quiet_nan(int64_t payload);
int    jo_exponent(double x);
double jo_scale(double x, int e);
double jo_hypot(double x, double y);
/* the multiplication-scaled form of jo_hypot that the GPU's complex column scan uses, and
 * the count of seeded operand pairs on which the two differ (jk_hypot_check.c) */
double jo_hypot_mulscaled(double x, double y);
long long jo_hypot_identity_check(long long n, unsigned long long seed);
double jo_dasum2(double x1, double x2);
double jo_dasum4(double x1, double x2, double x3, double x4);

/* ---- 2x2 kernels (src/D/dtransf.F90, src/Z/ztransf.F90, src/shared/ktransf.F90) ---- */
void jo_dhsvd2(double A[4], const int J[2], double U[4], double Z[4], double th1, int *info);
void jo_zhsvd2(jo_z A[4], const int J[2], jo_z U[4], jo_z Z[4], double th1, int *info);
void jo_dba(const double B[4], int n, double *x, double *y, int lda);
void jo_dab(const double B[4], int m, double *x, double *y);
double jo_abodndf2(const double B[4], int m, const double *x, const double *y, double aqp, double apq, int p, int q);
void jo_zba(const jo_z B[4], int n, jo_z *x, jo_z *y, int lda);
void jo_zab(const jo_z B[4], int m, jo_z *x, jo_z *y);
double jo_abodnzf2(const jo_z B[4], int m, const jo_z *x, const jo_z *y, jo_z aqp, jo_z apq, int p, int q);
/* 1: reproduce the complex BA branch of src/Z/ztransf.F90:325 (R1 used where the
 * real code uses R2); 0: use R2 as src/D/dtransf.F90:155 does. Default 1. */
void jo_set_zba_quirk(int on);

/* ---- pair weights (src/D/dstep.F90:12-72, src/Z/zstep.F90:12-74) ---- */
double jo_dmagf2t(int n, int p, int q, const double *A, int lda, const int *J);
double jo_dmagf2h(int n, int p, int q, const double *A, int lda, const int *J);
double jo_zmagf2t(int n, int p, int q, const jo_z *A, int lda, const int *J);
double jo_zmagf2h(int n, int p, int q, const jo_z *A, int lda, const int *J);

/* ---- pivot strategy (src/shared/jstep.F90, src/shared/atypes.F90) ---- */
int  jo_jstep_len(int n, int n_2);
int  jo_tru1(int n, const int *J, int nn, int *P, int *Q, int pn[2]);
int  jo_tru2(int n, const int *J, int nn, int *P, int *Q, int pn[2]);
int  jo_aw_cmp(const jo_aw *a, const jo_aw *b);
int  jo_aw_srt1(int nn, int nm, jo_aw *dz, int nt);
int  jo_aw_srt2(int nn, int nm, jo_aw *dz);
int  jo_aw_ncp1(int n, int nn, int nm, jo_aw *dz, int n_2, int *sl, int *step, int nt);
int  jo_aw_ncp2(int n, int nn, int nm, jo_aw *dz, int n_2, int *sl, int *step);
int  jo_aw_ncp3(int n, int nn, int nm, jo_aw *dz, int n_2, int *sl, int *step, int nt);

/* ---- the step loop (src/D/dstep.F90:472-604, src/Z/zstep.F90:482-615) ----
 * Returns INFO: >= 0 the number of steps, < 0 an error, as DSTEP_LOOP does.
 * nt = number of OpenMP threads (>1 selects AW_SRT1/AW_NCP1 as the reference's
 * DPROC_INIT does; 1 selects AW_SRT2/AW_NCP2). id_ncp/id_tru as on the djk
 * command line (0 = default). tr may be NULL. */
int jo_dstep_loop(int n, double *U, int ldu, double *A, int lda, double *Z, int ldz,
                  const int *J, double *sigma, int n_2, int id_ncp, int id_tru, int nt,
                  jo_trace *tr);
int jo_zstep_loop(int n, jo_z *U, int ldu, jo_z *A, int lda, jo_z *Z, int ldz,
                  const int *J, double *sigma, int n_2, int id_ncp, int id_tru, int nt,
                  jo_trace *tr);

/* Stop every later loop after m steps (0: run to convergence); test helper. */
void jo_set_max_steps(int m);

/* One build phase alone: weights of all pairs in the reference's record order
 * (TRU1/TRU2), NaN where the reference stores a NaN. w must hold NN doubles.
 * Returns TT (number of trigonometric pairs) or < 0. */
int jo_dweights(int n, const double *A, int lda, const int *J, int id_tru, int nt, double *w, int *P, int *Q);
int jo_zweights(int n, const jo_z *A, int lda, const int *J, int id_tru, int nt, double *w, int *P, int *Q);

/* Sort + greedy selection of one step from given weights of the NN pairs (P,Q
 * 1-based); -inf weights of hyperbolic pairs must already be NaN. Writes SL
 * pivots (1-based p,q) in selection order. Returns SL or < 0. */
int jo_select(int n, int nn, const double *w, const int *P, const int *Q, int n_2, int id_ncp, int nt, int *piv);

#ifdef __cplusplus
}
#endif
#endif /* !JK_ORACLE_H */
