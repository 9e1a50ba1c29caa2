/*
 * CPU oracle for the doubly periodic contour-advection (CLAM / "caps") time
 * step.  TEST INFRASTRUCTURE ONLY: this library is the checker that the CUDA
 * path is compared against, and the timed CPU baseline.  Nothing in the
 * product (hydra_b200/) links, loads or calls it.
 *
 * It restates, in plain C with Fortran semantics kept exact (1-based
 * indices, int() truncation toward zero, nint() rounding half away from zero,
 * SIGN(), MOD(), left-to-right evaluation, no FMA contraction), the
 * reference's Fortran 90 sources of ca/plane/qg/caps:
 *   contours.f90  init_contours, velint, con2grid, surgery, renode
 *   evolution.f90 advect, init, prepare, advance, source, inversion, adapt,
 *                 energy
 *   spectral.f90  init_spectral, main_invert, gradient, spec1d
 *   congen.f90    recontour, ugrid2con, con2ugrid   (beta = 0 build)
 *   caps.f90      initialise (loopinit = 0 path), recont
 *   generic.f90   contint, l2norm
 * and lib/stafft (sta2dfft.f90 ptospc/spctop/xderiv/yderiv, stafft.f90
 * forfft/revfft): the FFT is restated as the transform it computes (the
 * "Hermitian" real layout and its normalisation), not as stafft's radix
 * loops, so FFT-derived values agree with the Fortran to rounding only.
 *
 * PARITY UNPINNED: the reference ships no tests, fixtures or golden vectors,
 * and no Fortran compiler exists on the build or GPU machines, so the oracle
 * cannot be checked against outputs of the reference itself.  It is checked
 * against hand-derived known answers read off the reference sources, numpy,
 * and analytic solutions instead.
 */
#ifndef CASL_ORACLE_H
#define CASL_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct o_state o_state;

/* Physical and numerical parameters (parameters.f90 / constants.f90). */
typedef struct {
  int nx, ny;          /* inversion grid (N_X, N_Y) */
  int ncontq;          /* number of PV jumps (N_CONTQ) */
  double ellx, elly;   /* domain lengths (L_X, L_Y) */
  double kd, beta;     /* deformation wavenumber, planetary PV gradient */
  double rtherm, rekman;
  double cdamp, nnu;   /* hyperdiffusion coefficient and power */
  long npm;            /* node capacity (reference: 500*nx*ny) */
  long nm;             /* contour capacity (reference: npm/20+npm/200) */
  int nlevm;           /* max contour levels (reference: 2000) */
  /* Run-control overrides used by the synthetic workloads.  The reference's
   * own behaviour is fixed_dt <= 0 (adaptive dt) and force_surgery = 0
   * (surgery when twist > 2.5). */
  double fixed_dt;
  double dtmax;        /* adapt's cap, 0.2*min(tgsave,tcsave) in the reference */
  int force_surgery;
  int nregmax;         /* regularisations between recontourings (20) */
  double twistmax;     /* 2.5 */
} o_params;

o_state *o_create(const o_params *p);
void o_destroy(o_state *s);

/* --- FFT (sta2dfft.f90 / stafft.f90), arrays in Fortran order ----------- */
void o_forfft(int m, int n, double *x);          /* x(m,n), m transforms of length n */
void o_revfft(int m, int n, double *x);
void o_ptospc(o_state *s, double *rvar, double *svar); /* rvar(ny,nx) destroyed */
void o_spctop(o_state *s, double *svar, double *rvar); /* svar(nx,ny) destroyed */

/* --- spectral tables (spectral.f90:42-158) ------------------------------ */
/* which: 0 green,1 flo,2 fhi,3 qdiss,4 rksq,5 rk  -> (nx,ny)
 *        6 rkx(nx), 7 hrkx(nx), 8 rky(ny), 9 hrky(ny), 10 bety(ny) */
const double *o_table(o_state *s, int which);

/* --- contours ------------------------------------------------------------ */
/* Index arrays are 1-based as in the reference (nextq values 1..nptq). */
int o_set_contours(o_state *s, int nq, int nptq, double qjump,
                   const double *xq, const double *yq, const int *nextq,
                   const int *indq, const int *npq, const int *i1q, const int *i2q);
void o_get_counts(o_state *s, int *nq, int *nptq, double *qjump);
void o_get_contours(o_state *s, double *xq, double *yq, int *nextq,
                    int *indq, int *npq, int *i1q, int *i2q);

/* --- module procedures ---------------------------------------------------- */
/* con2grid (contours.f90:173-346).  qc(ny,nx).  If levels != NULL it receives
 * the fine-grid PV level index field L(iy,ix), iy=1..nyf, ix=1..nxf (Fortran
 * order, nyf*nxf ints) that the fine-grid q values are qjump multiples of. */
void o_con2grid(o_state *s, double *qc, int *levels);
void o_velint(o_state *s, const double *uu, const double *vv, double *uq, double *vq);
int o_surgery(o_state *s);   /* nonzero: capacity exceeded */
/* renode (contours.f90:687-933): xd,yd 1..npd in, xr,yr 1..npr out (0-based
 * C arrays holding elements 1..n at [0..n-1]). Returns npr. */
int o_renode(o_state *s, const double *xd, const double *yd, int npd, double *xr, double *yr);
void o_main_invert(o_state *s, const double *qq, double *uu, double *vv, double *pp);
void o_gradient(o_state *s, const double *ff, double *ffx, double *ffy);
void o_inversion(o_state *s);
void o_advance(o_state *s);
int  o_recontour(o_state *s, double *qq);

/* --- driver (caps.f90 / evolution.f90:advect) ---------------------------- */
/* initialise (caps.f90:106-361, loopinit=0) from q(ny,nx) at t=0, then
 * recont (caps.f90:380-395) and the evolution init (evolution.f90:96-131). */
int o_initialise(o_state *s, const double *qq_init);
/* One pass of the advect loop body (evolution.f90:55-79): regularise
 * (surgery, or prepare + recontour + init every nregmax) then advance. */
int o_step(o_state *s);

/* --- field access ---------------------------------------------------------- */
/* which: 0 qs,1 qd,2 qc,3 qq,4 pp,5 qspre,6 emq,7 epq (spectral, nx*ny)
 *        8 uu, 9 vv, 10 qr (physical, ny*nx) */
double *o_field(o_state *s, int which);
/* scalars: 0 t,1 dt,2 twist,3 ireg,4 zzrms,5 zzmax,6 uumax */
double o_scalar(o_state *s, int which);
void o_set_scalar(o_state *s, int which, double v);

/* diagnostics: ekin, epot (evolution.f90:612-644), enstrophy-like l2 norm of
 * q - beta*y (generic.f90:48-62), circulation sum over contours */
void o_diagnostics(o_state *s, double *out4);
/* 1-D spectrum of a spectral field (spectral.f90:370-424) and its tables
 * (spectral.f90:109-134); arrays of max(nx,ny)+1 entries. */
void o_spec1d(o_state *s, double *ss, double *spec, int iopt);
void o_spec_tables(o_state *s, int *kmax, int *kmaxred, double *spmf, double *alk);
/* genfg's ultra-fine PV (post/genfg.f90:79-113): float32 (nyu, nxu). */
void o_genfg(o_state *s, const double *qq, float *out);

/* Forcing (evolution.f90:330-428, spectral.f90:160-285) with the uniform
 * random numbers supplied by the caller, in the reference's draw order. */
void o_pvforce(o_state *s, int ivor, double vorvor, int nvor, const double *rnd);
int o_nb_forcing_init(o_state *s, double kfmid, double fwid, double famp);
void o_nb_forcing(o_state *s, double dt, const double *rnd);

#ifdef __cplusplus
}
#endif
#endif
