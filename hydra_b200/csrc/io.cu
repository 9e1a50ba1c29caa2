// The caps output files and the restart reader, byte-compatible with the
// reference's Fortran I/O (gfortran conventions):
//
//   cont/qqsynopsis.asc  (i9,1x,i10,1x,f12.5,1x,f16.12) nq,nptq,t,qjump
//                        (evolution.f90:746)
//   cont/qqindexNNN      one unformatted sequential record: npq(1:nq),
//                        i1q(1:nq), indq(1:nq) as int32 (evolution.f90:760-762)
//   cont/qqnodesNNN      one record: xq(1:nptq), yq(1:nptq) as float64
//                        (evolution.f90:764-766)
//   cont/qqresi.r4       direct access, recl = 4*(nx*ny+1): t, qd(ny,nx) as
//                        float32 (evolution.f90:749-752, caps.f90:247)
//   qq.r4                the same record layout for the full PV
//                        (evolution.f90:696-703, caps.f90:242)
//   ene.asc              (f9.2,3(1x,f17.11))  (evolution.f90:682)
//   norms.asc            (f9.2,1x,f16.9)      (evolution.f90:707)
//   spectra.asc          (f9.2,2(1x,f16.9),1x,i5) then kmaxred lines of
//                        (2(1x,f12.8))        (evolution.f90:714-719)
//   monitor.asc          (1x,f12.5,1x,f6.4,4(1x,f12.6),1x,f5.3)
//                        (evolution.f90:582-583)
//   complexity.asc       (1x,f12.5,1x,i9,1x,i10) (evolution.f90:73)
//
// An unformatted sequential record is a 4-byte little-endian length, the
// payload, and the length again; payloads of 2^31 bytes or more (which
// gfortran splits into subrecords) are rejected with CASL_EUNSUPPORTED.
// Direct-access record r (1-based) starts at byte (r-1)*recl.
//
// The device-state entry points (casl_savecont, casl_savegrid) enqueue the
// device work and the device-to-host copies into pinned staging on the
// handle's stream and hand the file writing to a host thread, so the GPU
// keeps stepping while the files are written; casl_io_wait joins it.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "state.cuh"

namespace casl {

// ---------------------------------------------------------------------------
// Fortran edit descriptors
// ---------------------------------------------------------------------------
// Fw.d: d decimals, right-justified in w columns; the optional leading zero
// of |x| < 1 is dropped when it does not fit; w asterisks when the value
// does not fit at all.  Exact decimal ties round as C's printf does.
// Infinities print as Infinity (Inf in narrow fields), NaN as NaN.
static void put_f(std::string &out, double x, int w, int d) {
  char buf[512];
  std::string v;
  if (isnan(x)) {
    v = "NaN";
  } else if (isinf(x)) {
    // gfortran spells infinities out where the field allows
    const bool neg = x < 0;
    v = (w - (neg ? 1 : 0) >= 8) ? "Infinity" : "Inf";
    if (neg) v = "-" + v;
  } else {
    snprintf(buf, sizeof buf, "%.*f", d, x);
    v = buf;
  }
  if ((int)v.size() > w) {
    size_t z = v[0] == '-' ? 1 : 0;
    if (v.size() > z + 1 && v[z] == '0' && v[z + 1] == '.') v.erase(z, 1);
  }
  if ((int)v.size() > w)
    out.append((size_t)w, '*');
  else
    out.append((size_t)(w - (int)v.size()), ' ').append(v);
}

static void put_i(std::string &out, long long x, int w) {
  char buf[64];
  snprintf(buf, sizeof buf, "%lld", x);
  std::string v(buf);
  if ((int)v.size() > w)
    out.append((size_t)w, '*');
  else
    out.append((size_t)(w - (int)v.size()), ' ').append(v);
}

static int append_line(const char *path, const std::string &line) {
  FILE *f = fopen(path, "ab");
  if (!f) return CASL_EIO;
  bool ok = fwrite(line.data(), 1, line.size(), f) == line.size() && fputc('\n', f) != EOF;
  ok = (fclose(f) == 0) && ok;
  return ok ? CASL_OK : CASL_EIO;
}

// ---------------------------------------------------------------------------
// Records
// ---------------------------------------------------------------------------
static int write_seq_record(const char *path, const void *const *parts, const size_t *bytes,
                            int nparts) {
  size_t total = 0;
  for (int i = 0; i < nparts; i++) total += bytes[i];
  if (total >= ((size_t)1 << 31)) return CASL_EUNSUPPORTED;
  FILE *f = fopen(path, "wb");
  if (!f) return CASL_EIO;
  int32_t m = (int32_t)total;
  bool ok = fwrite(&m, 4, 1, f) == 1;
  for (int i = 0; i < nparts && ok; i++)
    ok = bytes[i] == 0 || fwrite(parts[i], 1, bytes[i], f) == bytes[i];
  ok = ok && fwrite(&m, 4, 1, f) == 1;
  ok = (fclose(f) == 0) && ok;
  return ok ? CASL_OK : CASL_EIO;
}

static int read_seq_record(const char *path, void *const *parts, const size_t *bytes, int nparts) {
  size_t total = 0;
  for (int i = 0; i < nparts; i++) total += bytes[i];
  FILE *f = fopen(path, "rb");
  if (!f) return CASL_EIO;
  int32_t m0 = 0, m1 = 0;
  bool ok = fread(&m0, 4, 1, f) == 1 && m0 >= 0 && (size_t)m0 == total;
  for (int i = 0; i < nparts && ok; i++)
    ok = bytes[i] == 0 || fread(parts[i], 1, bytes[i], f) == bytes[i];
  ok = ok && fread(&m1, 4, 1, f) == 1 && m1 == m0;
  fclose(f);
  return ok ? CASL_OK : CASL_EIO;
}

static int write_r4_record(const char *path, int irec, int nx, int ny, float t, const float *a) {
  if (irec < 1 || nx < 1 || ny < 1 || !a) return CASL_EINVAL;
  FILE *f = fopen(path, "r+b");
  if (!f) f = fopen(path, "w+b");
  if (!f) return CASL_EIO;
  const long long recl = 4LL * ((long long)nx * ny + 1);
  bool ok = fseeko(f, (off_t)((irec - 1) * recl), SEEK_SET) == 0;
  ok = ok && fwrite(&t, 4, 1, f) == 1;
  ok = ok && fwrite(a, 4, (size_t)nx * ny, f) == (size_t)nx * ny;
  ok = (fclose(f) == 0) && ok;
  return ok ? CASL_OK : CASL_EIO;
}

static int read_r4_record(const char *path, int irec, int nx, int ny, float *t, float *a) {
  if (irec < 1 || nx < 1 || ny < 1 || !a || !t) return CASL_EINVAL;
  FILE *f = fopen(path, "rb");
  if (!f) return CASL_EIO;
  const long long recl = 4LL * ((long long)nx * ny + 1);
  bool ok = fseeko(f, (off_t)((irec - 1) * recl), SEEK_SET) == 0;
  ok = ok && fread(t, 4, 1, f) == 1;
  ok = ok && fread(a, 4, (size_t)nx * ny, f) == (size_t)nx * ny;
  fclose(f);
  return ok ? CASL_OK : CASL_EIO;
}

static std::string cont_file(const char *dir, const char *name, int rec) {
  char b[16];
  snprintf(b, sizeof b, "%03d", rec);  // write(pind,'(i3.3)')
  return std::string(dir) + "/cont/" + name + b;
}

static void ensure_cont_dir(const char *dir) {
  mkdir(dir, 0777);
  mkdir((std::string(dir) + "/cont").c_str(), 0777);
}

// ---------------------------------------------------------------------------
// Asynchronous writer state kept on the handle
// ---------------------------------------------------------------------------
// Save schedule of the time loop (evolution.f90:586-600, 200-204): gridded
// data every tgsave and contours every tcsave time units from tinit.  adapt
// of step k flags a save when t_k + dt_k reaches the next save time (and
// keeps its PV in the handle's qspre); step k+1 writes it after its
// inversion (and surgery), the gridded data interpolated between the two
// steps.
struct SaveSchedule {
  bool on = false;
  std::string dir;
  double tinit = 0.0, tgsave = 0.0, tcsave = 0.0;
  int igrec = 0, icrec = 1;       // the reference's record counters
  double tgrid = 0.0, tcont = 0.0;
  double tstep = 0.0;             // t at the start of the current step
  bool snap = false;              // qspre and the energies hold this step's values
  bool gpend = false, cpend = false;  // gsave / csave set by the previous step
  double ekinpre = 0.0, epotpre = 0.0;  // the flagging step's PV is the handle's qspre
  double *qqs = nullptr;          // the interpolated PV (n^2, device)
};

struct IoJob {
  std::thread th;
  int status = CASL_OK;
  bool active = false;
  // pinned staging
  void *pin = nullptr;
  size_t pin_bytes = 0;
  SaveSchedule sv;
};

static IoJob *job_of(casl_handle *h) {
  if (!h->io) h->io = new IoJob();
  return (IoJob *)h->io;
}

static int io_join(casl_handle *h) {
  if (!h->io) return CASL_OK;
  IoJob *j = (IoJob *)h->io;
  if (j->active) {
    j->th.join();
    j->active = false;
  }
  int st = j->status;
  j->status = CASL_OK;
  return st;
}

static int io_stage(casl_handle *h, size_t bytes, void **p) {
  IoJob *j = job_of(h);
  if (j->pin_bytes < bytes) {
    if (j->pin) cudaFreeHost(j->pin);
    j->pin = nullptr;
    j->pin_bytes = 0;
    if (cudaMallocHost(&j->pin, bytes) != cudaSuccess) return CASL_ENOMEM;
    j->pin_bytes = bytes;
  }
  *p = j->pin;
  return CASL_OK;
}

void io_release(casl_handle *h) {
  if (!h->io) return;
  io_join(h);
  IoJob *j = (IoJob *)h->io;
  if (j->pin) cudaFreeHost(j->pin);
  cudaFree(j->sv.qqs);
  delete j;
  h->io = nullptr;
}

__global__ void k_io_sub(const double *__restrict__ a, const double *__restrict__ b,
                         double *__restrict__ c, long long nn) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x)
    c[k] = a[k] - b[k];
}

// real(a(iy,ix) + bety(iy)) as float32 (bety may be null)
__global__ void k_io_add(const double *__restrict__ a, const double *__restrict__ b,
                         double *__restrict__ c, long long nn) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x)
    c[k] = a[k] + b[k];
}

__global__ void k_io_f32(const double *__restrict__ a, const double *__restrict__ bety,
                         float *__restrict__ out, int n, long long nn) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)(bety ? a[k] + bety[k % n] : a[k]);
}

// qqs = pt*qspre + ptc*qq (evolution.f90:669), each product rounded
__global__ void k_io_interp(const double *__restrict__ qspre, const double *__restrict__ qq,
                            double pt, double ptc, double *__restrict__ out, long long nn) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x)
    out[k] = __dadd_rn(__dmul_rn(pt, qspre[k]), __dmul_rn(ptc, qq[k]));
}

// sum of a^2 over nn values, one block (the sum of l2norm, generic.f90:198-212)
__global__ void __launch_bounds__(1024) k_io_sumsq(const double *__restrict__ a, long long nn,
                                                    double *__restrict__ out) {
  CASL_PDL_ENTRY();
  __shared__ double sh[1024];
  double v = 0.0;
  for (long long k = threadIdx.x; k < nn; k += blockDim.x) v += a[k] * a[k];
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_io_i1q(const int *__restrict__ i1q, int *__restrict__ out, int nq) {
  CASL_PDL_ENTRY();
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x)
    out[j] = i1q[j] + 1;
}

}  // namespace casl

using namespace casl;

extern "C" {

// ---- pure host: formats and records ---------------------------------------

int casl_io_append_synopsis(const char *path, int nq, int nptq, double t, double qjump) {
  if (!path) return CASL_EINVAL;
  std::string s;
  put_i(s, nq, 9); s += ' ';
  put_i(s, nptq, 10); s += ' ';
  put_f(s, t, 12, 5); s += ' ';
  put_f(s, qjump, 16, 12);
  return append_line(path, s);
}

int casl_io_append_ene(const char *path, double tgrid, double ekin, double epot) {
  if (!path) return CASL_EINVAL;
  std::string s;
  put_f(s, tgrid, 9, 2);
  s += ' '; put_f(s, ekin, 17, 11);
  s += ' '; put_f(s, epot, 17, 11);
  s += ' '; put_f(s, ekin + epot, 17, 11);
  return append_line(path, s);
}

int casl_io_append_norms(const char *path, double tgrid, double qql2) {
  if (!path) return CASL_EINVAL;
  std::string s;
  put_f(s, tgrid, 9, 2);
  s += ' '; put_f(s, qql2, 16, 9);
  return append_line(path, s);
}

int casl_io_append_spectrum(const char *path, double tgrid, double sumqspec, double qql2,
                            int kmaxred, const double *alk, const double *qspec) {
  if (!path || kmaxred < 0 || (kmaxred > 0 && (!alk || !qspec))) return CASL_EINVAL;
  std::string s;
  put_f(s, tgrid, 9, 2);
  s += ' '; put_f(s, sumqspec, 16, 9);
  s += ' '; put_f(s, qql2, 16, 9);
  s += ' '; put_i(s, kmaxred, 5);
  for (int k = 1; k <= kmaxred; k++) {
    s += "\n ";
    put_f(s, alk[k], 12, 8);
    s += ' ';
    put_f(s, log10(qspec[k]), 12, 8);
  }
  return append_line(path, s);
}

int casl_io_append_monitor(const char *path, double t, double cfl, double zzrms, double zzmax,
                           double uumax, double twist) {
  if (!path) return CASL_EINVAL;
  std::string s = " ";
  put_f(s, t, 12, 5);
  s += ' '; put_f(s, cfl, 6, 4);
  s += ' '; put_f(s, 0.5 * (zzrms * zzrms), 12, 6);
  s += ' '; put_f(s, zzrms, 12, 6);
  s += ' '; put_f(s, zzmax, 12, 6);
  s += ' '; put_f(s, uumax, 12, 6);
  s += ' '; put_f(s, twist, 5, 3);
  return append_line(path, s);
}

int casl_io_append_complexity(const char *path, double t, int nq, int nptq) {
  if (!path) return CASL_EINVAL;
  std::string s = " ";
  put_f(s, t, 12, 5);
  s += ' '; put_i(s, nq, 9);
  s += ' '; put_i(s, nptq, 10);
  return append_line(path, s);
}

int casl_io_write_index(const char *path, int nq, const int *npq, const int *i1q, const int *indq) {
  if (!path || nq < 0 || (nq > 0 && (!npq || !i1q || !indq))) return CASL_EINVAL;
  const void *parts[3] = {npq, i1q, indq};
  size_t b = (size_t)nq * 4;
  size_t bytes[3] = {b, b, b};
  return write_seq_record(path, parts, bytes, 3);
}

int casl_io_read_index(const char *path, int nq, int *npq, int *i1q, int *indq) {
  if (!path || nq < 0 || (nq > 0 && (!npq || !i1q || !indq))) return CASL_EINVAL;
  void *parts[3] = {npq, i1q, indq};
  size_t b = (size_t)nq * 4;
  size_t bytes[3] = {b, b, b};
  return read_seq_record(path, parts, bytes, 3);
}

int casl_io_write_nodes(const char *path, int nptq, const double *xq, const double *yq) {
  if (!path || nptq < 0 || (nptq > 0 && (!xq || !yq))) return CASL_EINVAL;
  const void *parts[2] = {xq, yq};
  size_t b = (size_t)nptq * 8;
  size_t bytes[2] = {b, b};
  return write_seq_record(path, parts, bytes, 2);
}

int casl_io_read_nodes(const char *path, int nptq, double *xq, double *yq) {
  if (!path || nptq < 0 || (nptq > 0 && (!xq || !yq))) return CASL_EINVAL;
  void *parts[2] = {xq, yq};
  size_t b = (size_t)nptq * 8;
  size_t bytes[2] = {b, b};
  return read_seq_record(path, parts, bytes, 2);
}

int casl_io_write_r4(const char *path, int irec, int nx, int ny, float t, const float *a) {
  if (!path) return CASL_EINVAL;
  return write_r4_record(path, irec, nx, ny, t, a);
}

int casl_io_read_r4(const char *path, int irec, int nx, int ny, float *t, float *a) {
  if (!path) return CASL_EINVAL;
  return read_r4_record(path, irec, nx, ny, t, a);
}

// readcont's list-directed read of line iind of qqsynopsis.asc (common.f90:50-53)
int casl_io_read_synopsis(const char *path, int iind, int *nq, int *nptq, double *t,
                          double *qjump) {
  if (!path || iind < 1 || !nq || !nptq || !t || !qjump) return CASL_EINVAL;
  FILE *f = fopen(path, "rb");
  if (!f) return CASL_EIO;
  char line[1024];
  int rc = CASL_EIO;
  for (int i = 1; i <= iind; i++) {
    if (!fgets(line, sizeof line, f)) break;
    if (i < iind) continue;
    for (char *c = line; *c; c++)
      if (*c == 'd' || *c == 'D') *c = 'e';  // Fortran exponent letter
    char *e1, *e2, *e3, *e4;
    long a = strtol(line, &e1, 10);
    long b = strtol(e1, &e2, 10);
    double c = strtod(e2, &e3);
    double d = strtod(e3, &e4);
    if (e1 != line && e2 != e1 && e3 != e2 && e4 != e3) {
      *nq = (int)a;
      *nptq = (int)b;
      *t = c;
      *qjump = d;
      rc = CASL_OK;
    }
  }
  fclose(f);
  return rc;
}

// ---- device state -----------------------------------------------------------

// savecont (evolution.f90:731-774): PV contours and residual qq - qc at the
// current time.  Enqueues the inversion, the residual transform and the
// copies; the files are written by a host thread (casl_io_wait joins it).
int casl_savecont(casl_handle *h, const char *dir, int icrec) {
  if (!h || !dir || icrec < 1 || icrec > 999) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // the files of one simulation
  int rc = io_join(h);
  if (rc) return rc;
  rc = sync_counts(h);
  if (rc) return rc;
  rc = get_scalars(h);
  if (rc) return rc;
  const int n = h->n, nq = h->nq, npt = h->nptq;
  const long long nn = (long long)n * n;
  const double t = h->hscal->t, qjump = h->hscal->qjump;
  cudaStream_t st = h->stream;
  // residual qq - qc after an inversion (evolution.f90:87, 749-751)
  rc = inversion_dev(h, false);
  if (rc) return rc;
  CASL_K(k_io_sub, 1184, 256, 0, st)(h->qq, h->qc, h->w[4], nn);
  rc = spctop_dev(h, h->w[4], h->w[5], h->w[0]);
  if (rc) return rc;
  float *resid_d = (float *)h->w[4];
  CASL_K(k_io_f32, 1184, 256, 0, st)(h->w[5], nullptr, resid_d, n, nn);
  int *i1q1 = (int *)h->w[3];
  if (nq > 0) CASL_K(k_io_i1q, (nq + 255) / 256, 256, 0, st)(h->i1q, i1q1, nq);
  rc = check_launch(h);
  if (rc) return rc;
  size_t bytes = (size_t)nn * 4 + (size_t)npt * 16 + (size_t)nq * 12;
  void *pin;
  rc = io_stage(h, bytes, &pin);
  if (rc) return rc;
  float *resid = (float *)pin;
  double *xq = (double *)(resid + nn), *yq = xq + npt;
  int *npq = (int *)(yq + npt), *i1q = npq + nq, *indq = i1q + nq;
  CASL_CUDA_TRY(cudaMemcpyAsync(resid, resid_d, nn * 4, cudaMemcpyDeviceToHost, st));
  if (npt > 0) {
    CASL_CUDA_TRY(cudaMemcpyAsync(xq, h->xq, (size_t)npt * 8, cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(yq, h->yq, (size_t)npt * 8, cudaMemcpyDeviceToHost, st));
  }
  if (nq > 0) {
    CASL_CUDA_TRY(cudaMemcpyAsync(npq, h->npq, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(i1q, i1q1, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaMemcpyAsync(indq, h->indq, (size_t)nq * 4, cudaMemcpyDeviceToHost, st));
  }
  cudaEvent_t ev;
  CASL_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CASL_CUDA_TRY(cudaEventRecord(ev, st));
  IoJob *j = job_of(h);
  std::string d(dir);
  j->active = true;
  j->th = std::thread([=]() {
    int s = cudaEventSynchronize(ev) == cudaSuccess ? CASL_OK : CASL_ECUDA;
    cudaEventDestroy(ev);
    if (!s) {
      ensure_cont_dir(d.c_str());
      s = casl_io_append_synopsis((d + "/cont/qqsynopsis.asc").c_str(), nq, npt, t, qjump);
    }
    if (!s) s = write_r4_record((d + "/cont/qqresi.r4").c_str(), icrec, n, n, (float)t, resid);
    if (!s && npt > 0) {
      s = casl_io_write_index(cont_file(d.c_str(), "qqindex", icrec).c_str(), nq, npq, i1q, indq);
      if (!s) s = casl_io_write_nodes(cont_file(d.c_str(), "qqnodes", icrec).c_str(), npt, xq, yq);
    }
    j->status = s;
  });
  return CASL_OK;
}

// savegrid's output (evolution.f90:648-727) for the spectral PV anomaly qsrc
// (device, not one of the work fields) at time tsave with the energies
// given: ene.asc, spectra.asc (spec1d), norms.asc (l2norm of spctop(qsrc))
// and record irec of qq.r4 (spctop(qsrc) + beta*y as float32).  The device
// work and copies are enqueued; a host thread writes the files.  The caller
// has joined the previous writer.
static int savegrid_write(casl_handle *h, const char *dir, int irec, double tsave,
                          const double *qsrc, double ekin, double epot) {
  const int n = h->n, kmax = h->kmax, kred = h->kmaxred;
  const long long nn = (long long)n * n;
  cudaStream_t st = h->stream;
  double *dspec = h->w[3];
  double *dl2 = h->w[3] + n + 8;
  int rc = spec1d_dev(h, qsrc, dspec);
  if (rc) return rc;
  rc = spctop_dev(h, qsrc, h->w[5], h->w[0]);
  if (rc) return rc;
  CASL_K(k_io_sumsq, 1, 1024, 0, st)(h->w[5], nn, dl2);
  float *q4_d = (float *)h->w[4];
  CASL_K(k_io_f32, 1184, 256, 0, st)(h->w[5], h->c.beffect ? h->bety : nullptr, q4_d, n, nn);
  rc = check_launch(h);
  if (rc) return rc;
  void *pin;
  rc = io_stage(h, (size_t)nn * 4 + (size_t)(n + 2) * 8, &pin);
  if (rc) return rc;
  float *q4 = (float *)pin;
  double *spec = (double *)(q4 + nn), *l2 = spec + n + 1;
  CASL_CUDA_TRY(cudaMemcpyAsync(q4, q4_d, nn * 4, cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(spec, dspec, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(l2, dl2, sizeof(double), cudaMemcpyDeviceToHost, st));
  cudaEvent_t ev;
  CASL_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CASL_CUDA_TRY(cudaEventRecord(ev, st));
  const double dsumi = h->c.dsumi, garea = h->c.garea;
  std::vector<double> spmf(h->spmf_h, h->spmf_h + n + 1), alk(h->alk_h, h->alk_h + n + 1);
  IoJob *j = job_of(h);
  std::string d(dir);
  j->active = true;
  j->th = std::thread([=]() mutable {
    int s = cudaEventSynchronize(ev) == cudaSuccess ? CASL_OK : CASL_ECUDA;
    cudaEventDestroy(ev);
    if (!s) {
      mkdir(d.c_str(), 0777);
      s = casl_io_append_ene((d + "/ene.asc").c_str(), tsave, ekin, epot);
    }
    if (!s) {
      // evolution.f90:685-692
      double sum = 0.0;
      std::vector<double> q(spec, spec + n + 1);
      for (int k = 1; k <= kmax; k++) {
        sum = sum + q[k];
        q[k] = spmf[k] * q[k];
      }
      sum = 8.0 * sum * dsumi;
      const double qql2 = garea * l2[0];
      s = write_r4_record((d + "/qq.r4").c_str(), irec, n, n, (float)tsave, q4);
      if (!s) s = casl_io_append_norms((d + "/norms.asc").c_str(), tsave, qql2);
      if (!s)
        s = casl_io_append_spectrum((d + "/spectra.asc").c_str(), tsave, sum, qql2, kred,
                                    alk.data(), q.data());
    }
    j->status = s;
  });
  return CASL_OK;
}

// savegrid (evolution.f90:648-727) at the current time: the inversion, the
// energies (evolution.f90:612-644) and savegrid_write of qq.  The schedule
// of casl_set_saves writes the same files interpolated to each save time.
int casl_savegrid(casl_handle *h, const char *dir, int irec) {
  if (!h || !dir || irec < 1) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;
  int rc = io_join(h);
  if (rc) return rc;
  rc = get_scalars(h);
  if (rc) return rc;
  const double t = h->hscal->t;
  rc = inversion_dev(h, false);
  if (rc) return rc;
  double diag[4];
  rc = casl_diagnostics(h, diag);  // energy (evolution.f90:612-644)
  if (rc) return rc;
  return savegrid_write(h, dir, irec, t, h->qq, diag[0], diag[1]);
}

int casl_set_saves(casl_handle *h, const char *dir, double tinit, double tgsave, double tcsave,
                   int igrec, int icrec) {
  if (!h) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // the files of one simulation
  IoJob *j = job_of(h);
  SaveSchedule &s = j->sv;
  if (!dir) {
    s.on = false;
    return CASL_OK;
  }
  if (!(tgsave > 0.0 || tcsave > 0.0) || igrec < 0 || icrec < 1) return CASL_EINVAL;
  if (!std::isfinite(tinit) || !std::isfinite(tgsave) || !std::isfinite(tcsave)) return CASL_EINVAL;
  const size_t bytes = (size_t)h->n * h->n * sizeof(double);
  if (!s.qqs) CASL_CUDA_TRY(cudaMalloc(&s.qqs, bytes));
  s.dir = dir;
  s.tinit = tinit;
  s.tgsave = tgsave;
  s.tcsave = tcsave;
  s.igrec = igrec;
  s.icrec = icrec;
  s.snap = s.gpend = s.cpend = false;
  s.on = true;
  return CASL_OK;
}

int casl_get_saves(casl_handle *h, int *igrec, int *icrec) {
  if (!h || !igrec || !icrec) return CASL_EINVAL;
  const IoJob *j = (const IoJob *)h->io;
  *igrec = j ? j->sv.igrec : 0;
  *icrec = j ? j->sv.icrec : 1;
  return CASL_OK;
}

int casl_io_wait(casl_handle *h) {
  if (!h) return CASL_EINVAL;
  return io_join(h);
}

// readcont (common.f90:30-100): contours, residual and time of save iind;
// qs = ptospc(con2grid + qr) on the device, qd = 0.
int casl_readcont(casl_handle *h, const char *dir, int iind) {
  if (!h || !dir || iind < 1 || iind > 999) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;
  int rc = io_join(h);
  if (rc) return rc;
  std::string d(dir);
  int nq = 0, npt = 0;
  double t = 0.0, qjump = 0.0;
  rc = casl_io_read_synopsis((d + "/cont/qqsynopsis.asc").c_str(), iind, &nq, &npt, &t, &qjump);
  if (rc) return rc;
  if (nq < 0 || npt < 0 || npt > h->npm || nq > h->nm) return CASL_ECAPACITY;
  std::vector<int> npq(nq), i1q(nq), indq(nq), i2q(nq), nextq(npt);
  std::vector<double> xq(npt), yq(npt);
  if (npt > 0) {
    rc = casl_io_read_index(cont_file(dir, "qqindex", iind).c_str(), nq, npq.data(), i1q.data(),
                            indq.data());
    if (rc) return rc;
    rc = casl_io_read_nodes(cont_file(dir, "qqnodes", iind).c_str(), npt, xq.data(), yq.data());
    if (rc) return rc;
  }
  const int n = h->n;
  std::vector<float> r4((size_t)n * n);
  float tr4;
  rc = read_r4_record((d + "/cont/qqresi.r4").c_str(), iind, n, n, &tr4, r4.data());
  if (rc) return rc;
  // i2q and nextq from npq / i1q (common.f90:75-85)
  for (int c = 0; c < nq; c++) {
    int ibeg = i1q[c], iend = ibeg + npq[c] - 1;
    if (ibeg < 1 || iend > npt || npq[c] < 1) return CASL_EINVAL;
    i2q[c] = iend;
    for (int i = ibeg; i < iend; i++) nextq[i - 1] = i + 1;
    nextq[iend - 1] = ibeg;
  }
  rc = casl_set_contours(h, nq, npt, qjump, xq.data(), yq.data(), nextq.data(), indq.data(),
                         npq.data(), i1q.data(), i2q.data());
  if (rc) return rc;
  std::vector<double> qr((size_t)n * n);
  for (size_t k = 0; k < qr.size(); k++) qr[k] = (double)r4[k];
  rc = casl_set_field(h, CASL_QR, qr.data());
  if (rc) return rc;
  // qs = ptospc(con2grid + qr); time = t of the save (common.f90:89-99)
  const long long nn = (long long)n * n;
  cudaStream_t st = h->stream;
  rc = con2grid_to_phys(h, h->w[5], false);
  if (rc) return rc;
  CASL_K(k_io_add, 1184, 256, 0, st)(h->w[5], h->qr, h->w[4], nn);
  rc = ptospc_dev(h, h->w[4], h->qs);
  if (rc) return rc;
  rc = get_scalars(h);
  if (rc) return rc;
  h->hscal->t = t;
  h->hscal->dt = 0.0;
  h->hscal->twist = 0.0;
  rc = put_scalars(h);
  if (rc) return rc;
  // then init (evolution.f90:96-131) as the restarted advect does
  rc = evo_init(h);
  if (rc) return rc;
  h->ireg = 0;
  return sync_counts(h);
}

}  // extern "C"

namespace casl {
static SaveSchedule *schedule_of(casl_handle *h) {
  if (!h->io) return nullptr;
  SaveSchedule *s = &((IoJob *)h->io)->sv;
  return s->on ? s : nullptr;
}

// Start of a step, after its surgery or recontouring: the saves flagged by
// the previous step (advance at evolution.f90:200-204: savegrid, then
// savecont), then this step's save times and, when this step's adapt can
// reach the next grid save time (t + dtmax >= tgrid, dt <= dtmax), the
// copies that the interpolation needs (evolution.f90:587-595).
int saves_before_advance(casl_handle *h) {
  SaveSchedule *s = schedule_of(h);
  if (!s) return CASL_OK;
  int rc = sync_counts(h);
  if (rc) return rc;
  if ((rc = get_scalars(h))) return rc;
  const double t = h->hscal->t, dtprev = h->hscal->dt, dtmax = h->hscal->dtmax;
  const long long nn = (long long)h->n * h->n;
  double diag[4];
  bool have = false;  // an inversion of this state and its energies in diag
  if (s->gpend) {
    if ((rc = io_join(h))) return rc;
    if ((rc = inversion_dev(h, false))) return rc;
    if ((rc = casl_diagnostics(h, diag))) return rc;
    have = true;
    // weights for time interpolation (evolution.f90:665-677)
    const double pt = (t - s->tgrid) / dtprev, ptc = 1.0 - pt;
    CASL_K(k_io_interp, 1184, 256, 0, h->stream)(h->qspre, h->qq, pt, ptc, s->qqs, nn);
    const double ekin = pt * s->ekinpre + ptc * diag[0];
    const double epot = pt * s->epotpre + ptc * diag[1];
    if ((rc = savegrid_write(h, s->dir.c_str(), s->igrec + 1, s->tgrid, s->qqs, ekin, epot)))
      return rc;
    s->igrec++;
    s->gpend = false;
  }
  if (s->cpend) {
    if ((rc = casl_savecont(h, s->dir.c_str(), s->icrec))) return rc;
    s->icrec++;
    s->cpend = false;
  }
  s->tgrid = s->tinit + s->tgsave * (double)s->igrec;
  s->tcont = s->tinit + s->tcsave * (double)s->icrec;
  s->tstep = t;
  s->snap = s->tgsave > 0.0 && t + dtmax >= s->tgrid;
  if (s->snap) {
    if (!have) {
      if ((rc = inversion_dev(h, false))) return rc;
      if ((rc = casl_diagnostics(h, diag))) return rc;
    }
    // qspre = qs after the reset, the same values as qq (evolution.f90:592)
    CASL_CUDA_TRY(cudaMemcpyAsync(h->qspre, h->qq, nn * sizeof(double), cudaMemcpyDeviceToDevice,
                                  h->stream));
    s->ekinpre = diag[0];
    s->epotpre = diag[1];
  }
  return CASL_OK;
}

// End of a step: adapt's flags, t + dt >= tgrid and t + dt >= tcont with the
// step's own t and dt (evolution.f90:589, 599).
int saves_after_advance(casl_handle *h) {
  SaveSchedule *s = schedule_of(h);
  if (!s) return CASL_OK;
  int rc = get_scalars(h);
  if (rc) return rc;
  const double tnext = s->tstep + h->hscal->dt;
  if (s->snap && tnext >= s->tgrid) s->gpend = true;
  if (s->tcsave > 0.0 && tnext >= s->tcont) s->cpend = true;
  return CASL_OK;
}

// init clears both flags (evolution.f90:113-116): after a recontouring, a
// save flagged by the step before is taken up again by the next adapt.
void saves_clear_flags(casl_handle *h) {
  SaveSchedule *s = schedule_of(h);
  if (s) s->gpend = s->cpend = false;
}
}  // namespace casl
