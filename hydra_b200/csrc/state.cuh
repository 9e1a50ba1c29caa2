// Device state of one simulation handle and internal entry points shared
// between the translation units of the library.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/hydra_casl.h"
#include "common.cuh"

namespace casl {
struct ClosureState;  // the learned velocity closure attached to a handle (closure.cu)
struct ForcingState;  // narrow-band spectral forcing tables (forcing.cu)
}

struct casl_handle {
  casl_params p;
  casl::Consts c;
  int device;
  cudaStream_t stream;
  double *gtmp;                  // 6 fields of scratch for the batched inversion + gradients
  int last_cuda;
  int n;                 // nx == ny
  long long npm, nm;     // capacities
  double qjump;          // host copy
  int nq, nptq;          // host copies of the counts
  int ireg;              // regularisations since the last recontouring
  int contex;
  double node_steps;     // sum of nptq over advanced steps (casl_step)

  // nodes (structure of arrays; nextq 0-based internally)
  double *xq, *yq;
  int *nextq;
  double *xqi, *yqi, *xqf, *yqf, *uq, *vq;
  // contours (0-based i1q, i2q internally)
  int *i1q, *i2q, *npq, *indq;

  // fields, n*n doubles each
  double *qr, *qs, *qd, *qc, *qq, *pp, *uu, *vv, *emq, *epq, *qspre;
  double *sqs, *sqd, *qsi, *qsf, *qdi, *qdf;
  double *w[6];          // work fields
  // tables
  double *green, *flo, *fhi, *qdiss, *hrkx, *hrky, *bety, *betac;
  double2 *tw;           // exp(-2 pi i k / n), k < n
  // 1-D spectrum (spectral.f90:109-134): spectral indices grouped by shell
  int *shell_off, *shell_idx;  // kmax+2 offsets; n*n indices kx + nx*ky
  double *rkxf, *rkyf;         // filtered wavenumbers for K^2 (spec1d iopt = 1)
  int kmax, kmaxred;
  double *spmf_h, *alk_h;      // host, n+1 entries each
  void *io;                    // output writer (thread + pinned staging), see io.cu

  // con2grid scratch
  int *fineJ;            // (nyf, nxf): row 0 = bottom level, rows 1.. = jump counts
  int *ljx;              // (nxf)
  int *coarseC;          // (n*n) coarse integer cells
  // reductions
  double *part;          // per-block partials
  casl::Scalars *scal;   // device scalars
  casl::Scalars *hscal;  // pinned host mirror

  // surgery / renode / recontour scratch (allocated on first use)
  void *sx;
  size_t sx_bytes;
  void *sx2;             // second arena (recontouring's per-crossing data)
  size_t sx2_bytes;
  void *sxe;             // beta != 0 recontouring: the extension rows' level codes
  size_t sxe_bytes;

  // kernel-class timing for benchmarks (events on the handle's stream)
  int prof_class;
  int prof_n;
  double prof_bytes;
  cudaEvent_t *prof_ev;  // 2 * CASL_PROF_MAX events, created on first use

  casl::ClosureState *closure;  // learned velocity closure (nullable)
  int *c2g_feat;                // its sub-cell input, written by con2grid when set (9 n^2)

  // FP32-inversion mode (casl_set_precision): the velocity and gradient
  // fields of each stage in FP32, u, v, dqd/dx, dqd/dy, dqs/dx, dqs/dy
  int prec;
  float *f32;            // 6 * n*n floats, allocated when the mode is first selected
  int uv_fp32;           // the latest stage velocity exists only in f32 (uu, vv stale)

  casl::ForcingState *forcing;  // nb_forcing tables (nullable)

  // Ensemble of M independent members (casl_ensemble_create; M = 1 for one
  // simulation).  Members share the grid size and parameters; their fields
  // are stacked (member m's field at offset m*n*n), their contours
  // concatenated member after member with member m's levels offset by
  // m*CASL_LSTRIDE, and scal holds one Scalars per member (member 0's also
  // carries the total counts and the error word).
  int M;
  int *mnode;            // device, M+1: first node of each member (mnode[M] = nptq)
  int *mcont;            // device, M+1: first contour of each member
  int *hmnode, *hmcont;  // pinned host copies
  double *mqjump;        // host, M: each member's qjump
  casl_handle *view;     // one-member view used to recontour each member in turn
};
#define CASL_LSTRIDE (1 << 20)   // level offset between ensemble members
#define CASL_LBIAS (1 << 19)     // |level| < CASL_LBIAS within a member

#define CASL_PROF_MAX 8192

namespace casl {

int set_cuda_error(casl_handle *h, cudaError_t e);
int check_launch(casl_handle *h);

// Spectral transforms on device buffers (in/out may alias only where noted).
// ptospc: phys (n*n, [ix][iy]) -> spec ([ky][kx]); spec must not alias phys.
int ptospc_dev(casl_handle *h, const double *phys, double *spec, int batch = 1);
// spctop: spec -> phys using tmp (n*n); spec is preserved.
int spctop_dev(casl_handle *h, const double *spec, double *phys, double *tmp, int batch = 1);

int con2grid_dev(casl_handle *h, bool want_levels);  // -> coarseC, scal->csum
int con2grid_to_spec(casl_handle *h, double *spec); // con2grid + ptospc fused load
int con2grid_to_phys(casl_handle *h, double *phys, bool want_levels);  // -> qc(ny,nx)

int surgery_dev(casl_handle *h);
int recontour_dev(casl_handle *h, const double *qq_dev);
int renode_host(casl_handle *h, const double *xd, const double *yd, int npd, double *xr,
                double *yr, int cap, int *npr);

int sync_counts(casl_handle *h);    // device counts -> host copies
int debug_check(casl_handle *h, const char *phase);  // CASL_CHECK=1: node sanity after a phase
int get_scalars(casl_handle *h);    // device scalars -> hscal
int put_scalars(casl_handle *h);    // hscal -> device scalars
int inversion_dev(casl_handle *h, bool reset);  // evolution.f90:494-520
int evo_init(casl_handle *h);       // evolution.f90:96-131 (qc, qd, qspre)
int spec1d_dev(casl_handle *h, const double *ss, double *dspec);
void io_release(casl_handle *h);    // joins the output writer, frees its staging
// Save schedule of casl_step (casl_set_saves; no-ops without one): the saves
// flagged by the previous step and this step's copies before the advance,
// adapt's flags after it; evo_init (initialise, restart, recontouring)
// clears the flags.
int saves_before_advance(casl_handle *h);
int saves_after_advance(casl_handle *h);
void saves_clear_flags(casl_handle *h);

// Opt-in phase trace (environment variable CASL_TRACE=1): records CUDA
// events at named points on the handle's stream and prints the device time
// between consecutive points to stderr when flushed.  CASL_TRACE=2 instead
// synchronises the stream at every point and prints the point's name and
// the host time since the previous point at once, so that a phase which
// never ends is named by the last line printed.
struct Trace {
  bool on = false;
  bool eager = false;
  double t_last = 0.0;
  int n = 0;
  cudaEvent_t ev[64];
  const char *name[64];
  cudaStream_t st;
  void begin(cudaStream_t s, const char *what);
  void point(const char *what);
  void flush(const char *title);
};
int ensure_scratch(casl_handle *h, size_t bytes);
int ensure_scratch2(casl_handle *h, size_t bytes);

// The fine-grid judge of node velocities: hf (nf = 2, 4 or 8 times h's n)
// inverts h's contours at its own resolution plus the spectrum of h's
// non-contour PV (qq - qc, after an inversion of h) and interpolates the
// result bilinearly to the nodes.  uJ, vJ, uP, vP: device arrays of nptq
// doubles (uP, vP = plain velint of h's inversion; nullable).  On h's stream.
int judge_velocity(casl_handle *h, casl_handle *hf, double *uJ, double *vJ, double *uP,
                   double *vP);
// Learned velocity closure hooks (closure.cu).  closure_stage runs after a
// stage's inversion; while the closure is active it sets du, dv to the
// correction at every node (added to velint's velocity in the node update),
// else leaves them null.
int closure_stage(casl_handle *h, const double **du, const double **dv);
int closure_stage32(casl_handle *h, const float *u, const float *v, const double **du,
                    const double **dv);  // FP32-inversion mode
// Before each advance of casl_step: the periodic fine-grid check.
int closure_step_check(casl_handle *h);
void closure_release(casl_handle *h);
void forcing_release(casl_handle *h);  // forcing.cu
// Ensembles (ensemble.cu): handle creation with M members, each member's
// node and contour ranges (mnode, mcont) from the level offsets, the
// member-by-member recontouring, and the view's release.
int create_handle_members(const casl_params *p, int device, int M, casl_handle **out);
int member_ranges(casl_handle *h);
int ensemble_recontour(casl_handle *h);
void ensemble_release(casl_handle *h);

}  // namespace casl
