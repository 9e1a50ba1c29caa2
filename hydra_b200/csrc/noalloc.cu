// con2grid without device allocation: casl_con2grid_noalloc.
//
// Some callers cannot call cudaMalloc: applications whose GPU memory is all
// handed out by their own pool or by another framework, codes that must not
// hit cudaMalloc's implicit device-wide synchronisation inside a
// time-critical loop, and callers that hold no casl handle (the handle is
// where this library keeps its allocations).  For them this entry point runs
// con2grid (contours.f90:173-346) on device arrays the caller already owns,
// with its scratch -- the 4n x 4n fine grid of jump counts and PV levels,
// the bottom-row jumps, the coarse integer cells and two counters -- in one
// file-scope __device__ array of fixed size.  Limits and sharing rules are
// stated in include/hydra_casl.h beside the declaration.
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "../../include/hydra_casl.h"
#include "common.cuh"

namespace casl {
// kernels of the handle-based con2grid (casl.cu), reused unchanged
__global__ void k_c2g_lbot(const int *__restrict__ ljx, int *__restrict__ J, int nxf, int nyf);
__global__ void k_c2g_colscan(int *__restrict__ J, int nxf, int nyf);
__global__ void k_c2g_coarsen(const int *__restrict__ L, int *__restrict__ C,
                              unsigned long long *__restrict__ csum, int n, int nf);
}  // namespace casl

namespace {

constexpr int NA_MAX_N = 256;                         // largest grid served
constexpr long long NA_FINE = 16LL * NA_MAX_N * NA_MAX_N;  // (4n)^2 fine cells
constexpr long long NA_LJX = 4LL * NA_MAX_N;
constexpr long long NA_COARSE = 1LL * NA_MAX_N * NA_MAX_N;
constexpr long long NA_MISC = 64;                     // csum (8 B) + error flag + spare
constexpr long long NA_INTS = NA_FINE + NA_LJX + NA_COARSE + NA_MISC;
// Offsets (in ints) of the per-call counters inside the misc region; the
// whole region is cleared at the start of every call.
constexpr long long NA_MISC_OFF = NA_FINE + NA_LJX + NA_COARSE;
constexpr long long NA_CSUM_OFF = NA_MISC_OFF;        // unsigned long long, 2 ints
constexpr long long NA_ERR_OFF = NA_MISC_OFF + 2;     // int
static_assert(NA_MISC_OFF % 2 == 0, "csum must be 8-byte aligned");
static_assert(NA_CSUM_OFF + 2 <= NA_MISC_OFF + NA_MISC && NA_ERR_OFF + 1 <= NA_MISC_OFF + NA_MISC,
              "the per-call counters must lie inside the cleared misc region");

// The scratch.  Every GPU that loads the library holds it (4.3 MB) until the
// process exits; all calls on a device share it.
static __device__ __align__(256) int g_na_scratch[NA_INTS];

struct NaConsts {
  int nxf, nyf;
  double ellx, elly, hlx, hly, hlxi, hlyi, xmin, xmax, ymin, ymax, glxf, glxfi, glyfi, small;
};

// Segment crossings of fine x grid lines and of y = ymin, as +-1 PV jumps
// (contours.f90:206-269); nextq holds 1-based successors as in the reference.
__global__ void k_na_scatter(const double *__restrict__ xq, const double *__restrict__ yq,
                             const int *__restrict__ nextq1, int npt, int *__restrict__ J,
                             int *__restrict__ ljx, NaConsts c, int *__restrict__ err) {
  CASL_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int ia = nextq1[i] - 1;
    if (ia < 0 || ia >= npt) { atomicExch(err, CASL_EINVAL); continue; }
    double xi = xq[i], yi = yq[i], xa = xq[ia], ya = yq[ia];
    if (!(xi >= c.xmin && xi < c.xmax && yi >= c.ymin && yi < c.ymax)) {
      atomicExch(err, CASL_EDOMAIN);
      continue;
    }
    int ixci = 1 + casl::f_int(c.glxfi * (xi - c.xmin));
    int ixca = 1 + casl::f_int(c.glxfi * (xa - c.xmin));
    double xx = xa - xi;
    double dx = xx - c.ellx * casl::f_dint(xx * c.hlxi);
    double yy = ya - yi;
    double dy = yy - c.elly * casl::f_dint(yy * c.hlyi);
    int ixdif = ixca - ixci;
    int nxc = ixdif - c.nxf * ((2 * ixdif) / c.nxf);
    if (fabs(yy) > c.hly) {
      double cc = casl::f_sign1(dy);
      double p = -(yi - c.hly * cc) / (dy + c.small);
      int ix = 1 + casl::f_int(c.glxfi * fmod(c.ellx + c.hlx + xi + p * dx, c.ellx));
      ix = ix < 1 ? 1 : (ix > c.nxf ? c.nxf : ix);
      atomicAdd(&ljx[ix - 1], -(int)cc);
    }
    if (nxc != 0 && nxc >= -c.nxf && nxc <= c.nxf) {
      int jump = casl::f_isign1(nxc);
      int ixbeg = ixci + (jump - 1) / 2 + c.nxf;
      int sgn = (int)casl::f_sign1(dx);
      for (int ncr = 0; ncr != nxc; ncr += jump) {
        int m = (ixbeg + ncr) % c.nxf;
        if (m < 0) m += c.nxf;
        int ix = 1 + m;
        double xgf = c.xmin + c.glxf * (double)(ix - 1);
        double x2 = xgf - xi;
        double px0 = (x2 - c.ellx * casl::f_dint(x2 * c.hlxi)) / dx;
        double y2 = yi + px0 * dy;
        int iy = 2 + casl::f_int(c.glyfi * (y2 - c.elly * casl::f_dint(y2 * c.hlyi) - c.ymin));
        if (iy >= 2 && iy <= c.nyf) atomicAdd(&J[(long long)(ix - 1) * c.nyf + (iy - 1)], sgn);
      }
    }
  }
}

// qc = qjump*(C*n^2 - S)/(256 n^2): the exact integer coarse cells with the
// mean removed, as the handle-based con2grid computes them.
__global__ void k_na_final(const int *__restrict__ C, const unsigned long long *__restrict__ csum,
                           double qjump, double *__restrict__ qc, int n) {
  CASL_PDL_ENTRY();
  const long long nn = (long long)n * n;
  const double inv = 1.0 / (256.0 * (double)n * (double)n);
  const long long S = (long long)*csum;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x) {
    long long num = (long long)C[t] * nn - S;
    qc[t] = qjump * ((double)num * inv);
  }
}

// Device address of g_na_scratch per device, looked up once per device in the
// device's primary context (the runtime API's context).  The lookup is also
// where CUDA's lazy module loading brings the library's device code, and with
// it the array, onto the device.
std::mutex g_na_mutex;
int *g_na_ptr[64] = {nullptr};

int scratch_for_current_device(int **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CASL_ECUDA;
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    int *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_na_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return CASL_ECUDA;
    }
    g_na_ptr[dev] = p;
  }
  *out = g_na_ptr[dev];
  return CASL_OK;
}

}  // namespace

extern "C" int casl_con2grid_noalloc(int n, double ellx, double elly, int nptq, double qjump,
                                     const double *xq_dev, const double *yq_dev,
                                     const int *nextq_dev, double *qc_dev, void *stream) {
  if (n < 32 || n > NA_MAX_N || (n & (n - 1)) || !(ellx > 0.0) || !(elly > 0.0) || nptq < 0 ||
      !qc_dev)
    return CASL_EINVAL;
  if (nptq > 0 && (!xq_dev || !yq_dev || !nextq_dev)) return CASL_EINVAL;
  // An error the caller left pending is the caller's: report it without
  // consuming it, so that the error checks after the launches below see only
  // this call's own errors.
  if (cudaPeekAtLastError() != cudaSuccess) return CASL_ECUDA;
  cudaStream_t st = (cudaStream_t)stream;
  const long long nn = (long long)n * n;
  if (nptq == 0) {
    if (cudaMemsetAsync(qc_dev, 0, nn * sizeof(double), st) != cudaSuccess) return CASL_ECUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? CASL_OK : CASL_ECUDA;
  }
  int *base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  const int nf = 4 * n;
  int *J = base;                                   // (nf, nf) jump counts -> levels
  int *ljx = base + NA_FINE;                       // (nf) bottom-row jumps
  int *C = base + NA_FINE + NA_LJX;                // (n, n) coarse integer cells
  unsigned long long *csum = (unsigned long long *)(base + NA_CSUM_OFF);
  int *err = base + NA_ERR_OFF;

  // constants as constants.f90 / contours.f90 define them
  NaConsts c;
  c.nxf = nf;
  c.nyf = nf;
  c.ellx = ellx;
  c.elly = elly;
  c.hlx = 0.5 * ellx;
  c.hly = 0.5 * elly;
  c.hlxi = 1.0 / c.hlx;
  c.hlyi = 1.0 / c.hly;
  c.xmin = -c.hlx;
  c.xmax = c.hlx;
  c.ymin = -c.hly;
  c.ymax = c.hly;
  c.glxf = ellx / (double)nf;
  c.glxfi = (double)nf / ellx;
  c.glyfi = (double)nf / elly;
  c.small = 1.0e-12;

  // The array keeps the previous call's contents: clear what accumulates.
  if (cudaMemsetAsync(J, 0, (size_t)nf * nf * sizeof(int), st) != cudaSuccess) return CASL_ECUDA;
  if (cudaMemsetAsync(ljx, 0, (size_t)nf * sizeof(int), st) != cudaSuccess) return CASL_ECUDA;
  if (cudaMemsetAsync(base + NA_MISC_OFF, 0, NA_MISC * sizeof(int), st) != cudaSuccess)
    return CASL_ECUDA;
  int g = (nptq + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  CASL_K(k_na_scatter, g, 256, 0, st)(xq_dev, yq_dev, nextq_dev, nptq, J, ljx, c, err);
  CASL_K(casl::k_c2g_lbot, 1, 1024, 0, st)(ljx, J, nf, nf);
  CASL_K(casl::k_c2g_colscan, (nf * 32 + 255) / 256, 256, 0, st)(J, nf, nf);
  int gc = (int)((nn + 255) / 256);
  if (gc > 148 * 16) gc = 148 * 16;
  CASL_K(casl::k_c2g_coarsen, gc, 256, 0, st)(J, C, csum, n, nf);
  CASL_K(k_na_final, gc, 256, 0, st)(C, csum, qjump, qc_dev, n);
  if (cudaGetLastError() != cudaSuccess) return CASL_ECUDA;
  int herr = 0;
  if (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return CASL_ECUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CASL_ECUDA;
  return herr ? herr : CASL_OK;
}
