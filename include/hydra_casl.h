/*
 * hydra_casl.h -- C ABI of the B200 contour-advection (CLAM / "caps") time
 * step for the doubly periodic plane.
 *
 * Drop-in boundary for the module procedures of Hydra's
 * basic_hydra/ca/plane/qg/caps Fortran program.  Each entry point below
 * names the reference procedure (file:line) whose body it replaces.  The
 * reference keeps its state in module globals (contours.f90:12-15,
 * evolution.f90:10-16, common.f90:12-16); here that state lives on one GPU
 * behind an opaque handle, and the Fortran host passes its arrays by pointer
 * (iso_c_binding) when it needs to move them in or out.
 *
 * Conventions
 *   - Plain C types only; every pointer argument is HOST memory unless the
 *     name says "_dev".
 *   - Physical fields are Fortran (ny,nx) column-major double arrays
 *     (iy fastest); spectral fields are Fortran (nx,ny) (kx fastest), in
 *     stafft's "Hermitian" layout (lib/stafft/stafft.f90:55-58).
 *   - Contour index arrays are 1-based exactly as in the reference:
 *     nextq(i) in 1..nptq, i1q/i2q in 1..nptq.
 *   - Every function returns 0 on success or a CASL_E* code; nothing aborts
 *     the host process, and no device wait is unbounded.
 *   - One handle is used by one host thread at a time; all work is ordered
 *     on the handle's own CUDA stream.
 */
#ifndef HYDRA_CASL_H
#define HYDRA_CASL_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define CASL_OK 0
#define CASL_EINVAL 1      /* bad argument (size, null pointer, parameter) */
#define CASL_ECAPACITY 2   /* node / contour / crossing capacity exceeded */
#define CASL_ECUDA 3       /* CUDA runtime error (see casl_last_cuda_error) */
#define CASL_ENOMEM 4      /* device allocation failed */
#define CASL_EDOMAIN 5     /* a node left the domain or became non-finite */
#define CASL_ETIMEOUT 6    /* a bounded device-side wait gave up */
#define CASL_EUNSUPPORTED 7
#define CASL_EIO 8         /* a file could not be opened, read or written */

/* ---- parameters (parameters.f90 / constants.f90 of QG caps) ------------- */
typedef struct casl_params {
  int nx, ny;            /* inversion grid; nx == ny, a power of two 32..2048 */
  int ncontq;            /* number of PV jumps used to set qjump (N_CONTQ) */
  double ellx, elly;     /* domain lengths (L_X, L_Y), domain centred on 0 */
  double kd, beta;       /* deformation wavenumber (K_D), PV gradient (PV_GRAD) */
  double rtherm, rekman; /* thermal / Ekman damping rates */
  double cdamp, nnu;     /* hyperdiffusion coefficient (C_DAMP) and power */
  long long npm;         /* node capacity (reference: 500*nx*ny) */
  long long nm;          /* contour capacity (reference: npm/20+npm/200) */
  int nlevm;             /* level offset used by recontouring (2000) */
  double fixed_dt;       /* > 0: use this dt instead of adapt's choice */
  double dtmax;          /* adapt's cap on dt (0.2*min(tgsave,tcsave)) */
  int force_surgery;     /* 1: regularise every step (else when twist > twistmax) */
  int nregmax;           /* regularisations between recontourings (20) */
  double twistmax;       /* 2.5 */
} casl_params;

typedef struct casl_handle casl_handle;

/* Field selectors for casl_get_field / casl_set_field. */
#define CASL_QS 0   /* spectral (nx,ny): q_s, evolved PV anomaly   (common.f90:15) */
#define CASL_QD 1   /* spectral: q_d, residual PV                  (evolution.f90:14) */
#define CASL_QC 2   /* spectral: contour PV                         (evolution.f90:14) */
#define CASL_QQ 3   /* spectral: full PV anomaly                    (evolution.f90:14) */
#define CASL_PP 4   /* spectral: streamfunction                     (evolution.f90:14) */
#define CASL_QSPRE 5
#define CASL_EMQ 6
#define CASL_EPQ 7
#define CASL_UU 8   /* physical (ny,nx): velocity u                 (evolution.f90:11) */
#define CASL_VV 9   /* physical: velocity v */
#define CASL_QR 10  /* physical: residual PV for recontouring       (common.f90:12) */

/* Scalar selectors for casl_get_scalar / casl_set_scalar. */
#define CASL_T 0
#define CASL_DT 1
#define CASL_TWIST 2
#define CASL_IREG 3
#define CASL_ZZRMS 4
#define CASL_ZZMAX 5
#define CASL_UUMAX 6
#define CASL_QJUMP 7
#define CASL_NODESTEPS 8  /* sum over casl_step passes of the node count advanced */

/* ---- lifetime ------------------------------------------------------------ */
/* init_spectral + init_contours (spectral.f90:42-158, contours.f90:48-132):
 * builds wavenumber, filter and Green-function tables and allocates the
 * device state for the given capacities. */
int casl_create(const casl_params *p, int device, casl_handle **out);
void casl_destroy(casl_handle *h);
const char *casl_error_string(int code);
int casl_last_cuda_error(casl_handle *h);   /* cudaError_t of the last failure */
int casl_synchronize(casl_handle *h);

/* ---- state transfer (host <-> device) ------------------------------------ */
/* Replaces the module state xq,yq,nextq,indq,npq,i1q,i2q,nq,nptq,qjump
 * (contours.f90:12-15).  Arrays are 1-based in content (nextq values).
 * The uploaded state is checked on the device before it is accepted: a
 * non-finite node or one outside [-ellx/2,ellx/2) x [-elly/2,elly/2) returns
 * CASL_EDOMAIN, a successor or contour range outside 1..nptq (or npq !=
 * i2q-i1q+1) CASL_EINVAL, more nodes or contours than the capacities
 * CASL_ECAPACITY; a rejected state leaves the handle with no contours. */
int casl_set_contours(casl_handle *h, int nq, int nptq, double qjump,
                      const double *xq, const double *yq, const int *nextq,
                      const int *indq, const int *npq, const int *i1q, const int *i2q);
int casl_get_counts(casl_handle *h, int *nq, int *nptq, double *qjump);
int casl_get_contours(casl_handle *h, double *xq, double *yq, int *nextq,
                      int *indq, int *npq, int *i1q, int *i2q);
int casl_set_field(casl_handle *h, int which, const double *host);
int casl_get_field(casl_handle *h, int which, double *host);
int casl_get_scalar(casl_handle *h, int which, double *value);
int casl_set_scalar(casl_handle *h, int which, double value);

/* ---- module procedures ---------------------------------------------------- */
/* ptospc / spctop (lib/stafft/sta2dfft.f90:103-165): rvar(ny,nx) <-> svar(nx,ny).
 * Unlike the reference the input is not destroyed. */
int casl_ptospc(casl_handle *h, const double *rvar, double *svar);
int casl_spctop(casl_handle *h, const double *svar, double *rvar);

/* con2grid (contours.f90:173-346) on the current contours.  qc(ny,nx) may be
 * NULL.  levels (optional, (4ny,4nx) ints, iy fastest) receives the fine-grid
 * PV level index whose qjump multiples the reference's fine grid holds. */
int casl_con2grid(casl_handle *h, double *qc, int *levels);

/* velint (contours.f90:136-169): bilinear interpolation of uu,vv (ny,nx) to
 * the current nodes; uq, vq have nptq entries. */
int casl_velint(casl_handle *h, const double *uu, const double *vv, double *uq, double *vq);

/* main_invert (spectral.f90:304-342): qq (nx,ny) spectral -> uu,vv (ny,nx)
 * physical, pp (nx,ny) spectral.  Any output may be NULL. */
int casl_main_invert(casl_handle *h, const double *qq, double *uu, double *vv, double *pp);

/* gradient (spectral.f90:345-366): ff spectral -> ffx, ffy physical. */
int casl_gradient(casl_handle *h, const double *ff, double *ffx, double *ffy);

/* inversion (evolution.f90:494-520) on the device state. */
int casl_inversion(casl_handle *h);

/* advance (evolution.f90:166-326): one RK4 step of nodes, qs and qd. */
int casl_advance(casl_handle *h);

/* surgery (contours.f90:350-683), including renode of every contour. */
int casl_surgery(casl_handle *h);

/* renode (contours.f90:687-933) of one closed contour given on the host;
 * xr, yr must hold cap entries; *npr receives the new node count (0 = the
 * contour is too small and is dropped). */
int casl_renode(casl_handle *h, const double *xd, const double *yd, int npd,
                double *xr, double *yr, int cap, int *npr);

/* recontour (congen.f90:24-128): new contours from the current contours plus
 * the residual qq (ny,nx); with no contours, qq is the full field. */
int casl_recontour(casl_handle *h, const double *qq);

/* ---- driver (caps.f90 / evolution.f90:advect) ------------------------------ */
/* initialise (caps.f90:106-361, loopinit = 0) from the initial PV q(ny,nx),
 * then recont (caps.f90:380-395) and the evolution init
 * (evolution.f90:96-131). */
int casl_initialise(casl_handle *h, const double *qq_init);

/* nsteps passes of the advect loop body (evolution.f90:55-79): regularise
 * (surgery; or prepare + recontour + init every nregmax) then advance. */
int casl_step(casl_handle *h, int nsteps);

/* ---- forcing of the residual PV (row f3) ---------------------------------- */
/* The reference adds these to qd at the end of advance (evolution.f90:316-
 * 323); a host that runs them calls them after casl_advance.  The reference
 * draws its random numbers from GNU rand() inside the procedures; here the
 * caller passes them in, in the reference's draw order.
 * pvforce (evolution.f90:330-428): nvor point vortices of alternating sign
 * +-vorvor (ivor = 1; rnd holds x, y in [0,1) per vortex, in grid units of
 * nx, ny) or dipoles of strength vorvor (ivor != 1; theta, x, y in [0,1)),
 * spread over their grid box by inverse bilinear interpolation, transformed
 * and added to qd.  The caller computes nvor as the reference does,
 * 2*nint((dnvor*t - totnvor)/2) or nint(dnvor*t - totnvor). */
int casl_pvforce(casl_handle *h, int ivor, double vorvor, int nvor, const double *rnd);
/* init_forcing (spectral.f90:160-229): the band |k - kfmid| <= fwid of the
 * narrow-band forcing with amplitude famp = fbase*2^nfamp; *nrand receives
 * the number of random values each casl_nb_forcing call consumes.  A band
 * reaching wavenumber 0 or the Nyquist wavenumber (where the reference
 * stops) returns CASL_EINVAL. */
int casl_nb_forcing_init(casl_handle *h, double kfmid, double fwid, double famp, int *nrand);
/* nb_forcing (spectral.f90:232-285) then qd = qd + dqdt: rnd holds nrand
 * values of myrand (2*rand()-1) in the reference's order. */
int casl_nb_forcing(casl_handle *h, double dt, const double *rnd);

/* ---- batched ensembles (no counterpart in the reference) ------------------ */
/* M independent simulations of one grid size and parameter set in one
 * handle, stepped together by casl_step: every stage of the RK4 advance, the
 * surgery and the renode run as single launches over all members (each
 * member keeps its own dt, qjump and scalars, as M separate runs of the
 * reference would); recontouring runs member by member.  force_surgery is
 * set (every member regularises every step, so all members recontour at the
 * same step).  Members' contours are stored one member after another with
 * member m's levels offset by m*2^20 (casl_get_contours returns that raw
 * form; casl_ensemble_member_contours one member in its own numbering).
 * The closure and the FP32-inversion mode serve single simulations only. */
int casl_ensemble_create(const casl_params *p, int members, int device, casl_handle **out);
int casl_ensemble_members(casl_handle *h, int *members);
/* initialise (caps.f90:106-361) of every member: q_all holds the M initial
 * fields (ny,nx) one after another; ncontq (nullable) each member's number
 * of PV jumps. */
int casl_ensemble_initialise(casl_handle *h, const double *q_all, const int *ncontq);
int casl_ensemble_member_counts(casl_handle *h, int m, int *nq, int *nptq, double *qjump);
int casl_ensemble_member_contours(casl_handle *h, int m, double *xq, double *yq, int *nextq,
                                  int *indq, int *npq, int *i1q, int *i2q);
/* which: CASL_T, CASL_DT, CASL_TWIST, CASL_ZZRMS, CASL_ZZMAX, CASL_UUMAX, CASL_QJUMP */
int casl_ensemble_member_scalar(casl_handle *h, int m, int which, double *value);

/* Precision of the inversion inside casl_advance / casl_step.
 * CASL_PREC_FP64 (default): everything FP64, the parity mode.
 * CASL_PREC_FP32_INVERSION: the inverse transform pair of every RK4 stage
 * (velocities from green*qq and the x/y derivatives of qd and qs,
 * spectral.f90:304-366) stores its intermediate and its physical outputs in
 * FP32 (arithmetic stays FP64 in registers); velint and the advection
 * products read those FP32 fields; the state (qs, qd, nodes), the forward
 * transforms, adapt's reductions and every contour operation stay FP64.
 * casl_get_field(CASL_UU / CASL_VV) then returns the last stage's FP32
 * velocity widened to FP64; casl_diagnostics recomputes the FP64 velocity
 * from qq first. */
#define CASL_PREC_FP64 0
#define CASL_PREC_FP32_INVERSION 1
int casl_set_precision(casl_handle *h, int mode);
int casl_get_precision(casl_handle *h, int *mode);

/* Diagnostics: out[0] kinetic energy, out[1] potential energy
 * (evolution.f90:612-644), out[2] integral of (q - beta y)^2 (generic.f90:48),
 * out[3] contour circulation qjump * sum of signed contour areas. */
int casl_diagnostics(casl_handle *h, double out[4]);

/* spec1d (spectral.f90:370-424): 1-D spectrum of the spectral field
 * ss(nx,ny) (host array); spec receives max(nx,ny)+1 shell sums, zero above
 * kmax.  iopt = 1 multiplies ss by the filtered K^2 first and returns it so
 * modified, as the reference does; iopt = 0 leaves ss untouched. */
int casl_spec1d(casl_handle *h, double *ss, double *spec, int iopt);

/* The spectrum tables of init_spectral (spectral.f90:109-134): kmax, kmaxred
 * and, when non-NULL, spmf and alk (max(nx,ny)+1 entries each) as savegrid
 * (evolution.f90:683-719) uses them. */
int casl_spec_tables(casl_handle *h, int *kmax, int *kmaxred, double *spmf, double *alk);

/* ---- output files and restart (row f1) ----------------------------------- */
/* The caps output files, byte-compatible with the reference's gfortran I/O
 * (evolution.f90:582-583, 648-774; caps.f90:233-248; common.f90:30-100).
 * Paths are files; `dir` arguments are the run directory holding cont/.
 * ASCII writers append one formatted line (spectrum: header + kmaxred lines)
 * with the reference's edit descriptors; sequential records carry 4-byte
 * length markers; r4 files are direct access with recl = 4*(nx*ny+1). */
int casl_io_append_synopsis(const char *path, int nq, int nptq, double t, double qjump);
int casl_io_append_ene(const char *path, double tgrid, double ekin, double epot);
int casl_io_append_norms(const char *path, double tgrid, double qql2);
int casl_io_append_spectrum(const char *path, double tgrid, double sumqspec, double qql2,
                            int kmaxred, const double *alk, const double *qspec);
int casl_io_append_monitor(const char *path, double t, double cfl, double zzrms, double zzmax,
                           double uumax, double twist);
int casl_io_append_complexity(const char *path, double t, int nq, int nptq);
int casl_io_write_index(const char *path, int nq, const int *npq, const int *i1q, const int *indq);
int casl_io_read_index(const char *path, int nq, int *npq, int *i1q, int *indq);
int casl_io_write_nodes(const char *path, int nptq, const double *xq, const double *yq);
int casl_io_read_nodes(const char *path, int nptq, double *xq, double *yq);
int casl_io_write_r4(const char *path, int irec, int nx, int ny, float t, const float *a);
int casl_io_read_r4(const char *path, int irec, int nx, int ny, float *t, float *a);
int casl_io_read_synopsis(const char *path, int iind, int *nq, int *nptq, double *t,
                          double *qjump);

/* savecont (evolution.f90:731-774) of the current state into dir/cont/
 * (record icrec, 1..999).  The device work and copies are enqueued on the
 * handle's stream and a host thread writes the files; the call returns
 * without waiting for them.  casl_io_wait joins the writer and returns its
 * status; the next save, readcont and casl_destroy join it too. */
int casl_savecont(casl_handle *h, const char *dir, int icrec);
/* savegrid (evolution.f90:648-727) at the current time (no interpolation
 * between steps): ene.asc, norms.asc, spectra.asc and record irec of qq.r4,
 * written by the same host thread. */
int casl_savegrid(casl_handle *h, const char *dir, int irec);
/* The save schedule of the time loop (evolution.f90:586-600, 200-204):
 * casl_step writes savegrid output every tgsave and savecont output every
 * tcsave time units from tinit into dir (a value <= 0 turns that kind off;
 * dir NULL turns the schedule off).  The step whose t + dt reaches a grid
 * save time keeps its PV and energies; the next step writes qq.r4 record
 * igrec+1, ene.asc, norms.asc and spectra.asc at the save time, interpolated
 * linearly between the two steps (evolution.f90:665-677), then (for a
 * contour save time) savecont record icrec at its own time.  igrec and
 * icrec are the reference's counters (a fresh run: 0 and 1; caps.f90:
 * 227-230); each save advances its own.  The flagging step's PV is kept in
 * CASL_QSPRE, the reference's qspre.  Every init (casl_initialise,
 * casl_readcont, a recontouring) drops pending flags, as the reference's
 * init does.  Replaces the save logic of advect/adapt; one simulation
 * (M = 1) only. */
int casl_set_saves(casl_handle *h, const char *dir, double tinit, double tgsave, double tcsave,
                   int igrec, int icrec);
int casl_get_saves(casl_handle *h, int *igrec, int *icrec);
int casl_io_wait(casl_handle *h);
/* readcont (common.f90:30-100) followed by init (evolution.f90:96-131):
 * contours, residual and time of save iind; qs = ptospc(con2grid + qr). */
int casl_readcont(casl_handle *h, const char *dir, int iind);

/* genfg (post/genfg.f90:79-194): the PV on the ultra-fine (16n)^2 grid,
 * con2ugrid of the current contours plus the bilinear interpolation of the
 * residual field qr (CASL_QR, e.g. as casl_readcont leaves it), as float32.
 * out is (nyv, nxv) column-major with out(iy, ix) = qa(iy1v + (iy-1)*stride,
 * ix1v + (ix-1)*stride), 1-based and periodic: stride 1 over the whole grid
 * is genfg's option 1, stride n its option 2, a wrapped window option 3. */
int casl_genfg(casl_handle *h, int ix1v, int nxv, int iy1v, int nyv, int stride, float *out);

/* ---- con2grid without device allocation ---------------------------------- */
/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * -- their GPU memory is handed out by their own pool or another framework,
 * they must not hit cudaMalloc's implicit device synchronisation inside a
 * time-critical loop, or they hold no casl handle -- this runs con2grid
 * (contours.f90:173-346, beta = 0) on device arrays the caller owns:
 * xq_dev, yq_dev (nptq doubles), nextq_dev (nptq ints, 1-based successors as
 * in the reference) and qc_dev (n*n doubles, Fortran (ny,nx) order).  It
 * allocates nothing: its scratch is one fixed file-scope device array of
 * 4.3 MB, so n is limited to 32..256 (a power of two; larger n returns
 * CASL_EINVAL), and every GPU on which the library's device code is loaded
 * holds that array until the process exits.  The first call on a device
 * looks the array's address up (cudaGetSymbolAddress); under CUDA's default
 * lazy module loading that first call is also what loads the library's
 * device code and the array onto the device, so it may allocate and
 * synchronise: make it once as a warm-up, outside any time-critical loop and
 * before any stream capture.  The address is kept per device for the
 * device's primary context (the runtime API's), so the entry point serves
 * that context only, and not across a cudaDeviceReset.  An error the caller
 * left pending in the runtime (cudaPeekAtLastError) makes the call return
 * CASL_ECUDA at once and is left in place for the caller.
 * All calls on a device share the array and it keeps the last call's
 * contents (the call clears what must start at zero), so calls that overlap
 * on the GPU (e.g. on two streams at once) race.  `stream` is a cudaStream_t
 * (NULL = default stream); the call synchronises it before returning. */
int casl_con2grid_noalloc(int n, double ellx, double elly, int nptq, double qjump,
                          const double *xq_dev, const double *yq_dev, const int *nextq_dev,
                          double *qc_dev, void *stream);

/* ---- learned velocity closure (no counterpart in the reference) ----------- */
/* The reference interpolates the coarse inversion's velocity bilinearly to
 * the nodes (velint, contours.f90:136-169).  The closure adds to the gridded
 * velocity that velint reads a correction predicted by a small CNN from the
 * coarse grid's PV and velocity: four periodic 5x5 convolutions 3 -> 32 ->
 * 32 -> 32 -> 2 channels with GELU after the first three, BF16 weights and
 * activations, FP32 accumulation, forward and backward on the tensor cores.
 * Parameters are float32 in the order W1[co][ci][ky][kx], b1, ..., W4, b4
 * (casl_net_param_count of them).  Host arrays are channel-major
 * (C, nx, ny) float32 with ny fastest, like the physical fields.  n is a
 * multiple of 128, 128..2048. */
typedef struct casl_net casl_net;
int casl_net_param_count(void);
int casl_net_create(int n, int device, casl_net **out);
void casl_net_destroy(casl_net *net);
/* qscale, uscale: the PV and velocity scales the network's inputs are
 * divided by and its output multiplied by when it runs inside a step. */
int casl_net_set_params(casl_net *net, const float *params, float qscale, float uscale);
int casl_net_get_params(casl_net *net, float *params, float *qscale, float *uscale);
/* x: (CASL_NET_IN, n, n) network input (already scaled: the coarse contour
 * PV, u and v, then qjump (L - C/256) for the fine contour levels L at the
 * 3 x 3 points (4ix + 2a - 2, 4iy + 2b - 2) of each coarse cell, channel
 * 3 + 3a + b, C the cell's con2grid sum); y: (CASL_NET_OUT, n, n)
 * output, the velocity correction on a grid twice as fine as n: channel
 * comp*4 + a*2 + b holds component comp (0: u, 1: v) at the fine point
 * (2 ix + a, 2 iy + b).  Keeps what casl_net_backward needs. */
#define CASL_NET_IN 12
#define CASL_NET_OUT 8
int casl_net_forward(casl_net *net, const float *x, float *y);
/* Gradient of sum(dy * y) for the last casl_net_forward with respect to the
 * parameters (grad: casl_net_param_count floats, may be NULL); also keeps it
 * for casl_net_adam. */
int casl_net_backward(casl_net *net, const float *dy, float *grad);
/* One Adam step (b1 = 0.9, b2 = 0.999, eps = 1e-8) with the last gradient. */
int casl_net_adam(casl_net *net, float lr);

/* The fine-grid judge of node velocities.  `judge` is a handle of the same
 * domain with 2, 4 or 8 times h's grid (the reference's main_invert,
 * spectral.f90:304-342, at that resolution): it inverts h's contours on its
 * own grid plus the spectrum of h's non-contour PV (qq - qc of an inversion
 * of h, carried over unchanged) and interpolates its velocity bilinearly to
 * the nodes.  uJ, vJ (and uP, vP, the plain velint of h's own inversion,
 * nullable) are host arrays of nptq doubles. */
int casl_closure_judge(casl_handle *h, casl_handle *judge, double *uJ, double *vJ, double *uP,
                       double *vP);
/* Attach a network to h: from now on every RK4 stage of casl_advance /
 * casl_step runs it on the stage's coarse PV and velocity, and each node's
 * velocity is velint's plus uscale times the bilinear interpolation of the
 * network's output on the grid twice as fine (see casl_net_forward).  With a judge and check_every > 0, every
 * check_every-th casl_step first compares the node velocities of both forms
 * with the judge's: the correction stays on while its relative error
 * (sqrt(sum |u - uJ|^2 / sum |uJ|^2) over the nodes) is at most `budget` and
 * at most the plain form's, and falls back to plain velint otherwise, until a
 * later check passes.  net = NULL detaches.  The network and judge are not
 * owned by h. */
int casl_closure_attach(casl_handle *h, casl_net *net, casl_handle *judge, int check_every,
                        double budget);
int casl_closure_status(casl_handle *h, int *active, double *err_plain, double *err_net,
                        long long *checks, long long *fallbacks);
/* One check now (needs an attached network and judge). */
int casl_closure_check(casl_handle *h, double *err_plain, double *err_net);
/* One training sample at h's current state: judge, network forward, the node
 * loss sum |corrected - judge|^2 / (nptq uscale^2), backward and one Adam
 * step.  out: plain relative error, corrected relative error (before the
 * step), loss.  casl_closure_evaluate does the same without training. */
int casl_closure_train(casl_handle *h, casl_net *net, casl_handle *judge, float lr,
                       double out[3]);
int casl_closure_evaluate(casl_handle *h, casl_net *net, casl_handle *judge, double out[3]);
/* The network input of an inversion of h's current state (run by the call),
 * (CASL_NET_IN, n, n) float32, already divided by the network's scales. */
int casl_closure_features(casl_handle *h, casl_net *net, float *x);
/* The network's correction at h's nodes (du, dv: host arrays of nptq
 * doubles) from an inversion of h's current state, as the node update inside
 * a step adds it. */
int casl_closure_correction(casl_handle *h, casl_net *net, double *du, double *dv);

/* ---- benchmarking hooks (no counterpart in the reference) ---------------- */
/* The cudaStream_t (as void*) on which all of the handle's work is ordered,
 * so a caller can bracket work with its own CUDA events. */
int casl_get_stream(casl_handle *h, void **stream);
/* Kernel launches issued by this library in this process so far. */
int casl_launch_count(long long *count);
/* Kernel-class timing: while a class is selected, each launch of that class
 * is bracketed by CUDA events on the handle's stream; casl_profile_read
 * returns the summed device time, the number of launches and their
 * algorithmic bytes (a 2-D transform reads each field once and writes it
 * once, 16 B per FP64 element; each of its two passes counts half), then
 * resets the tally.  Classes: */
#define CASL_PROF_OFF 0
#define CASL_PROF_FFT 1   /* the batched real-FFT passes (ptospc/spctop halves) */
int casl_profile(casl_handle *h, int kernel_class);
int casl_profile_read(casl_handle *h, double *total_ms, long long *launches, double *bytes);
/* Per-launch timing of every kernel of this library (process-wide):
 * mode 1 switches it on (each launch bracketed by two CUDA events on its
 * stream, up to 65536 launches), 0 switches it off, 2 writes a report into
 * buf (one line per kernel: launches, total ms, mean us; by total) and
 * starts a new tally.  A diagnostic, not a part of the reference interface. */
int casl_kernel_times(int mode, char *buf, long long cap);

#ifdef __cplusplus
}
#endif
#endif
