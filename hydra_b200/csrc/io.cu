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
struct IoJob {
  std::thread th;
  int status = CASL_OK;
  bool active = false;
  // pinned staging
  void *pin = nullptr;
  size_t pin_bytes = 0;
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

// savegrid (evolution.f90:648-727) at the current time: ene.asc, spectra.asc,
// norms.asc and record irec of qq.r4.  The reference interpolates to the
// save time between two steps (pt); here the state is written at t itself.
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
  rc = casl_diagnostics(h, diag);  // energy (evolution.f90:612-644) and l2norm of spctop(qq)
  if (rc) return rc;
  const int n = h->n, kmax = h->kmax, kred = h->kmaxred;
  const long long nn = (long long)n * n;
  cudaStream_t st = h->stream;
  double *dspec = h->w[3];
  rc = spec1d_dev(h, h->qq, dspec);
  if (rc) return rc;
  rc = spctop_dev(h, h->qq, h->w[5], h->w[0]);
  if (rc) return rc;
  float *q4_d = (float *)h->w[4];
  CASL_K(k_io_f32, 1184, 256, 0, st)(h->w[5], h->c.beffect ? h->bety : nullptr, q4_d, n, nn);
  rc = check_launch(h);
  if (rc) return rc;
  void *pin;
  rc = io_stage(h, (size_t)nn * 4 + (size_t)(n + 1) * 8, &pin);
  if (rc) return rc;
  float *q4 = (float *)pin;
  double *spec = (double *)(q4 + nn);
  CASL_CUDA_TRY(cudaMemcpyAsync(q4, q4_d, nn * 4, cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(spec, dspec, (n + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
  cudaEvent_t ev;
  CASL_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CASL_CUDA_TRY(cudaEventRecord(ev, st));
  const double ekin = diag[0], epot = diag[1], qql2 = diag[2], dsumi = h->c.dsumi;
  std::vector<double> spmf(h->spmf_h, h->spmf_h + n + 1), alk(h->alk_h, h->alk_h + n + 1);
  IoJob *j = job_of(h);
  std::string d(dir);
  j->active = true;
  j->th = std::thread([=]() mutable {
    int s = cudaEventSynchronize(ev) == cudaSuccess ? CASL_OK : CASL_ECUDA;
    cudaEventDestroy(ev);
    if (!s) {
      mkdir(d.c_str(), 0777);
      s = casl_io_append_ene((d + "/ene.asc").c_str(), t, ekin, epot);
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
      s = write_r4_record((d + "/qq.r4").c_str(), irec, n, n, (float)t, q4);
      if (!s) s = casl_io_append_norms((d + "/norms.asc").c_str(), t, qql2);
      if (!s)
        s = casl_io_append_spectrum((d + "/spectra.asc").c_str(), t, sum, qql2, kred, alk.data(),
                                    q.data());
    }
    j->status = s;
  });
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
