// B200 contour-advection time step: handle, tables, transforms, con2grid,
// node advection, spectral source terms, adapt and the RK4 advance.
//
// Reference: basic_hydra/ca/plane/qg/caps (Fortran 90).  File:line citations
// name the reference procedure each piece restates.
#include <cxxabi.h>
#include <string>
#include <typeinfo>
#include <chrono>
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "common.cuh"
#include "fft.cuh"
#include "scan.cuh"
#include "state.cuh"

using namespace casl;

namespace casl {

unsigned long long g_launches = 0;

// ---- per-launch timing ------------------------------------------------------
namespace {
constexpr int KT_MAX = 1 << 16;  // launches recorded between two reports
struct KTime {
  bool on = false;
  cudaEvent_t *ev = nullptr;  // 2 * KT_MAX, created when switched on
  const char **name = nullptr;
  int n = 0, open = -1;
  cudaStream_t st = 0;
};
KTime g_kt;
}  // namespace

bool kt_begin(const char *name, dim3, dim3, size_t, cudaStream_t st) {
  ++g_launches;
  if (g_kt.on && g_kt.n < KT_MAX) {
    g_kt.open = g_kt.n;
    g_kt.st = st;
    g_kt.name[g_kt.n] = name;
    cudaEventRecord(g_kt.ev[2 * g_kt.n], st);
  }
  return true;
}
bool kt_end() {
  if (g_kt.open >= 0) {
    cudaEventRecord(g_kt.ev[2 * g_kt.open + 1], g_kt.st);
    g_kt.n = g_kt.open + 1;
    g_kt.open = -1;
  }
  return false;
}

struct FillJobs {
  unsigned int *p[6];
  long long n[6];
  unsigned int v[6];
  int nj;
};
__global__ void k_fill(FillJobs J) {
  CASL_PDL_ENTRY();
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
#pragma unroll
  for (int j = 0; j < 6; j++) {
    if (j >= J.nj) break;
    unsigned int *p = J.p[j];
    const long long n = J.n[j];
    const unsigned int v = J.v[j];
    long long head = 0;
    if (((uintptr_t)p & 15) == 0) {
      uint4 *q = reinterpret_cast<uint4 *>(p);
      const uint4 w = make_uint4(v, v, v, v);
      for (long long i = tid; i < n / 4; i += stride) q[i] = w;
      head = (n / 4) * 4;
    }
    for (long long i = head + tid; i < n; i += stride) p[i] = v;
  }
}

int fill_words(cudaStream_t st, const FillJob *jobs, int njobs) {
  if (njobs < 1 || njobs > 6) return CASL_EINVAL;
  FillJobs J{};
  long long most = 0;
  for (int j = 0; j < njobs; j++) {
    J.p[j] = static_cast<unsigned int *>(jobs[j].p);
    J.n[j] = jobs[j].words;
    J.v[j] = jobs[j].value;
    most = std::max(most, jobs[j].words);
  }
  J.nj = njobs;
  long long g = (most / 4 + 255) / 256;
  g = std::max(1LL, std::min(g, 148LL * 16));
  CASL_K(k_fill, (int)g, 256, 0, st)(J);
  return check_launch(nullptr);
}

int set_cuda_error(casl_handle *h, cudaError_t e) {
  if (h) h->last_cuda = (int)e;
  cudaGetLastError();  // clear sticky non-fatal error state
  if (e == cudaErrorMemoryAllocation) return CASL_ENOMEM;
  return CASL_ECUDA;
}

int check_launch(casl_handle *h) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(h, e);
  return CASL_OK;
}


// ---------------------------------------------------------------------------
// Transform launches
// ---------------------------------------------------------------------------
// A functor type's name without its namespace, for launch names.
static std::string short_type_name(const std::type_info &t) {
  int status = 0;
  char *d = abi::__cxa_demangle(t.name(), nullptr, nullptr, &status);
  std::string r = (status == 0 && d) ? d : t.name();
  free(d);
  for (size_t at; (at = r.find("casl::")) != std::string::npos;) r.erase(at, 6);
  return r;
}

// One batched transform pass (all vectors of `batch` fields along one axis).
template <int LOGH, bool FWD, bool LVF, bool SVF, class LD, class ST>
static int launch_rfft(casl_handle *h, LD ld, ST st, int batch) {
  using Sh = RfftShape<LOGH, LVF || SVF>;
  dim3 grid(Sh::N / Sh::V, batch);
  const bool prof = h->prof_class == CASL_PROF_FFT && h->prof_ev && h->prof_n < CASL_PROF_MAX;
  if (prof) cudaEventRecord(h->prof_ev[2 * h->prof_n], h->stream);
  auto kern = k_rfft_r<LOGH, FWD, LVF, SVF, LD, ST>;
  const size_t sm = rfft_smem<LOGH, FWD, LVF, SVF, staged_rows<LD, LVF>()>();
  static bool configured = false;  // one per template instance
  if (!configured) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    configured = true;
  }
  // named by size, direction and functors for the per-launch timing report
  static char name[160];
  if (!name[0])
    snprintf(name, sizeof name, "k_rfft_r<%d %s, %s, %s>", Sh::N, FWD ? "fwd" : "inv",
             short_type_name(typeid(LD)).c_str(), short_type_name(typeid(ST)).c_str());
  for (bool once = kt_begin(name, grid, Sh::NT, sm, h->stream); once; once = kt_end())
    launch_of(kern, grid, Sh::NT, sm, h->stream)(ld, st, h->tw);
  if (prof) {
    cudaEventRecord(h->prof_ev[2 * h->prof_n + 1], h->stream);
    h->prof_n++;
    // algorithmic bytes of a 2-D transform: each field read once and written
    // once (16 B per FP64 element); each of its two passes accounts for half
    h->prof_bytes += (double)batch * (double)Sh::N * (double)Sh::N * 8.0;
  }
  return check_launch(h);
}

template <bool FWD, bool LVF, bool SVF, class LD, class ST>
static int rfft_dispatch(casl_handle *h, LD ld, ST st, int batch) {
  switch (h->n) {
    case 32: return launch_rfft<4, FWD, LVF, SVF>(h, ld, st, batch);
    case 64: return launch_rfft<5, FWD, LVF, SVF>(h, ld, st, batch);
    case 128: return launch_rfft<6, FWD, LVF, SVF>(h, ld, st, batch);
    case 256: return launch_rfft<7, FWD, LVF, SVF>(h, ld, st, batch);
    case 512: return launch_rfft<8, FWD, LVF, SVF>(h, ld, st, batch);
    case 1024: return launch_rfft<9, FWD, LVF, SVF>(h, ld, st, batch);
    case 2048: return launch_rfft<10, FWD, LVF, SVF>(h, ld, st, batch);
    default: return CASL_EINVAL;
  }
}
#define RFFT_DISPATCH(FWD, LVF, SVF, ld, st, batch) rfft_dispatch<FWD, LVF, SVF>(h, ld, st, batch)

// A 2-D transform is separable, so each one takes the axis whose vectors are
// contiguous first: forward transforms run along iy (phys columns, vector v =
// ix) and then along ix (rows of the intermediate, v = ky); inverse ones run
// along kx (spectral rows, v = ky) and then along ky (v = ix).  Only one of
// the four global sides is vector-fastest.  The intermediate of both is
// T[ky*n + ix].  The order of the axes changes results by rounding only.
int ptospc_dev(casl_handle *h, const double *phys, double *spec, int batch) {
  long long n = h->n, nn = n * n;
  // along iy for each ix: phys[ix*n+iy] -> spec[ky*n+ix] (spec != phys)
  int rc = RFFT_DISPATCH(true, false, true, (LoadRow{phys, nn, n, (int)n, &h->scal->error}),
                         (StoreStrided{spec, nn, 1, n}), batch);
  if (rc) return rc;
  // along ix for each ky, in place by rows: spec[ky*n + kx]
  return RFFT_DISPATCH(true, false, false, (LoadRow{spec, nn, n, (int)n, &h->scal->error}),
                       (StoreStrided{spec, nn, n, 1}), batch);
}

int spctop_dev(casl_handle *h, const double *spec, double *phys, double *tmp, int batch) {
  long long n = h->n, nn = n * n;
  // along kx for each ky: spec[ky*n+kx] -> tmp[ky*n+ix]
  int rc = RFFT_DISPATCH(false, false, false, (LoadRow{spec, nn, n, (int)n, &h->scal->error}),
                         (StoreStrided{tmp, nn, n, 1}), batch);
  if (rc) return rc;
  // along ky for each ix: tmp[ky*n+ix] -> phys[ix*n+iy]
  return RFFT_DISPATCH(false, true, false, (LoadStrided{tmp, nn, 1, n}),
                       (StoreStrided{phys, nn, n, 1}), batch);
}

// ---------------------------------------------------------------------------
// Fused load / store functors
// ---------------------------------------------------------------------------

// Element (v = kx-1, j = ky-1) of xderiv / yderiv (sta2dfft.f90:169-245) of
// a spectral field, optionally of green*field (main_invert, spectral.f90:321).
// Batch index b selects field and direction.
// MB: an ensemble transform (batch entry b is entry b % nb of member b / nb,
// whose fields lie ms elements after the previous member's).  A single
// simulation instantiates MB = false, whose index arithmetic has no integer
// division: with it the derivative load, at its 80-register budget, spilled.
template <bool MB>
struct LoadDerivT {
  static constexpr bool wide = MB;  // the ensemble's index arithmetic needs 80 registers
  // bytes per element, averaged over the batch's entries
  __host__ double bytes() const {
    int nb = 0, ng = 0;
    for (int b = 0; b < 6; b++)
      if (f[b]) {
        nb++;
        ng += wg[b];
      }
    return nb ? 8.0 + 8.0 * ng / nb : 8.0;
  }
  const double *f[6];
  int dir[6];  // 0: d/dx, 1: d/dy
  int wg[6];   // 1: entry multiplied by the Green function
  const double *green;
  const double *hrkx, *hrky;
  int n;
  int nb = 6;
  long long ms = 0;
  __device__ __forceinline__ int ent(int b) const { return MB ? b % nb : b; }
  __device__ __forceinline__ long long mof(int b) const { return MB ? (long long)(b / nb) * ms : 0; }
  __device__ __forceinline__ double base(int b, int kx0, int ky0) const {
    long long k = (long long)ky0 * n + kx0;
    const int e = ent(b);
    double v = pick(f, e)[mof(b) + k];
    return pick(wg, e) ? green[k] * v : v;
  }
  // first pass of an inverse transform: vector v = ky, element j = kx.
  // Branch-free, so that a thread's loads are issued together: the factor
  // is 0 at k = 0 and k = n/2, -hrk(2k-1) below n/2 and +hrk(2(n-k)-1) above,
  // and the reflected index (n-k) mod n is always a valid element.
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    const int nw = n >> 1, kx = j, ky = v;
    const bool dx = pick(dir, ent(b)) == 0;
    const int k = dx ? kx : ky;
    const int kr = (n - k) & (n - 1);
    const int hi = k < nw ? 2 * k - 1 : 2 * (n - k) - 1;
    const double *hrk = dx ? hrkx : hrky;
    const double h = hrk[hi < 0 ? 0 : hi];
    const double fac = (k == 0 || k == nw) ? 0.0 : (k < nw ? -h : h);
    return fac * (dx ? base(b, kr, ky) : base(b, kx, kr));
  }
  // elements j, j+1 (j even).  For d/dy the factor is the vector's and the
  // two values are adjacent: one 16-byte load each from f and green.  For
  // d/dx the reflected indices n-j, n-j-1 run backwards from an odd start,
  // so they stay two loads.
  __device__ __forceinline__ double2 pair(int b, int v, int j) const {
    const int e = ent(b);
    if (pick(dir, e) == 0) return make_double2((*this)(b, v, j), (*this)(b, v, j + 1));
    const int nw = n >> 1, k = v;
    const int kr = (n - k) & (n - 1);
    const int hi = k < nw ? 2 * k - 1 : 2 * (n - k) - 1;
    const double h = hrky[hi < 0 ? 0 : hi];
    const double fac = (k == 0 || k == nw) ? 0.0 : (k < nw ? -h : h);
    const long long o = (long long)kr * n + j;
    double2 q = *reinterpret_cast<const double2 *>(pick(f, e) + mof(b) + o);
    if (pick(wg, e)) {
      const double2 g = *reinterpret_cast<const double2 *>(green + o);
      q = make_double2(g.x * q.x, g.y * q.y);
    }
    return make_double2(fac * q.x, fac * q.y);
  }
  // Bulk staging (the pass is along kx, one row per vector): vector v of
  // entry b reads row v of f (d/dx, reflected within the row) or row
  // (n - v) mod n (d/dy), and the same row of the Green function.
  static constexpr int NROWS = 2;
  int *err = nullptr;
  __device__ __forceinline__ uint32_t stage_bytes(int b, int) const {
    return (uint32_t)n * 8u * (pick(wg, ent(b)) ? 2u : 1u);
  }
  __device__ __forceinline__ void stage(int b, int v, double *dst, uint64_t *bar) const {
    const int e = ent(b);
    const long long r = (long long)(pick(dir, e) == 0 ? v : (n - v) & (n - 1)) * n;
    tc::bulk_g2s(dst, pick(f, e) + mof(b) + r, (uint32_t)n * 8u, bar);
    if (pick(wg, e)) tc::bulk_g2s(dst + n, green + r, (uint32_t)n * 8u, bar);
  }
  __device__ __forceinline__ void fail() const {
    if (err) atomicExch(err, CASL_ETIMEOUT);
  }
  // operator() on the staged rows R (f, then the Green function)
  __device__ __forceinline__ double staged(int b, int v, int j, const double *R) const {
    const int e = ent(b);
    const bool dx = pick(dir, e) == 0;
    const int nw = n >> 1;
    const int k = dx ? j : v;
    const int idx = dx ? (n - j) & (n - 1) : j;
    const int hi = k < nw ? 2 * k - 1 : 2 * (n - k) - 1;
    const double h = (dx ? hrkx : hrky)[hi < 0 ? 0 : hi];
    const double fac = (k == 0 || k == nw) ? 0.0 : (k < nw ? -h : h);
    const double val = R[idx];
    return fac * (pick(wg, e) ? R[n + idx] * val : val);
  }
};
using LoadDeriv = LoadDerivT<false>;

// qa(iy,ix) of con2grid from the exact integer coarse cells:
// qc = qjump*(C*n^2 - S)/(256 n^2) (+ beta field), phys layout [ix][iy].
struct LoadQC {
  __host__ double bytes() const { return 4.0; }
  const int *C;
  const Scalars *s;
  const double *betac;  // nullable
  long long nn;
  double inv;           // 1/(256 n^2)
  int n;
  // batch entry b = ensemble member b (its cells and scalars)
  __device__ __forceinline__ double operator()(int b, int v /*ix*/, int j /*iy*/) const {
    long long k = (long long)b * nn + (long long)v * n + j;
    long long num = (long long)C[k] * nn - s[b].csum;
    double q = s[b].qjump * ((double)num * inv);
    if (betac) q = q + betac[j];
    return q;
  }
  __device__ __forceinline__ double2 pair(int b, int v, int j) const {
    long long k = (long long)b * nn + (long long)v * n + j;
    const int2 c = *reinterpret_cast<const int2 *>(C + k);
    const long long S = s[b].csum;
    const double qj = s[b].qjump;
    double q0 = qj * ((double)((long long)c.x * nn - S) * inv);
    double q1 = qj * ((double)((long long)c.y * nn - S) * inv);
    if (betac) {
      q0 = q0 + betac[j];
      q1 = q1 + betac[j + 1];
    }
    return make_double2(q0, q1);
  }
};

// Advection product -u*fx - v*(fy [+ beta]) of evolution.f90:449,456-461,
// read from physical arrays ([ix][iy]); b = 0 for qd, 1 for qs.
// Two adjacent elements of an FP64 or FP32 field, as FP64.
__device__ __forceinline__ double2 ld2(const double *p) { return *reinterpret_cast<const double2 *>(p); }
__device__ __forceinline__ double2 ld2(const float *p) {
  const float2 f = *reinterpret_cast<const float2 *>(p);
  return make_double2((double)f.x, (double)f.y);
}
template <class T>
struct LoadAdvectT {
  __host__ double bytes() const { return 4.0 * sizeof(T); }
  const T *uu, *vv;
  const T *fx[2], *fy[2];
  double betab[2];  // beta added to fy for the qs term when beffect
  int n;
  long long ms = 0;  // ensemble: entry b is term b % 2 of member b / 2, fields ms apart
  __device__ __forceinline__ double operator()(int b, int v /*ix*/, int j /*iy*/) const {
    const int e = b & 1;
    long long k = (long long)(b >> 1) * ms + (long long)v * n + j;
    const double bb = pick(betab, e);
    double gx = (double)pick(fx, e)[k], gy = (double)pick(fy, e)[k];
    if (bb != 0.0) gy = gy + bb;
    return -(double)uu[k] * gx - (double)vv[k] * gy;
  }
  __device__ __forceinline__ double2 pair(int b, int v, int j) const {
    const int e = b & 1;
    long long k = (long long)(b >> 1) * ms + (long long)v * n + j;
    const double bb = pick(betab, e);
    const double2 gx = ld2(pick(fx, e) + k);
    double2 gy = ld2(pick(fy, e) + k);
    const double2 u = ld2(uu + k);
    const double2 w = ld2(vv + k);
    if (bb != 0.0) {
      gy.x = gy.x + bb;
      gy.y = gy.y + bb;
    }
    return make_double2(-u.x * gx.x - w.x * gy.x, -u.y * gx.y - w.y * gy.y);
  }
};
using LoadAdvect = LoadAdvectT<double>;

// Store of the source terms after ptospc pass B (evolution.f90:466-487):
// b = 0 -> sqd with damping and the integrating factor, b = 1 -> sqs.
struct StoreSource {
  __host__ double bytes() const { return 8.0 + 0.5 * 24.0; }  // sqd reads qq, pp, epq
  double *sqd, *sqs;
  const double *qq, *pp, *epq;
  double rekman, kdsq, therm;
  int heating, friction, lev, n;
  long long ms = 0;  // ensemble: entry b is term b % 2 of member b / 2
  __device__ __forceinline__ double damped(double x, double p, double q, double e) const {
    double t;
    if (heating) {
      if (friction)
        t = x + therm * (p - 0.0) - rekman * (q + kdsq * p);
      else
        t = x + therm * (p - 0.0);
    } else {
      t = x - rekman * (q + kdsq * p);
    }
    if (lev == 1)
      t = e * t;
    else if (lev == 2)
      t = e * e * t;
    return t;
  }
  __device__ __forceinline__ void operator()(int b, int v /*ky*/, int k /*kx*/, double x) const {
    const long long idx = (long long)(b >> 1) * ms + (long long)v * n + k;
    if (b & 1) {
      sqs[idx] = x;
      return;
    }
    sqd[idx] = damped(x, pp[idx], qq[idx], lev ? epq[idx] : 0.0);
  }
  __device__ __forceinline__ void pair(int b, int v, int k, double2 x) const {
    const long long i = (long long)(b >> 1) * ms + (long long)v * n + k;
    if (b & 1) {
      *reinterpret_cast<double2 *>(sqs + i) = x;
      return;
    }
    const double2 p = *reinterpret_cast<const double2 *>(pp + i);
    const double2 q = *reinterpret_cast<const double2 *>(qq + i);
    const double2 e = lev ? *reinterpret_cast<const double2 *>(epq + i) : make_double2(0.0, 0.0);
    *reinterpret_cast<double2 *>(sqd + i) =
        make_double2(damped(x.x, p.x, q.x, e.x), damped(x.y, p.y, q.y, e.y));
  }
};

// (MB: an ensemble, entry b is entry b % nb of member b / nb, fields ms apart)
template <bool MB>
struct StoreScaledT {
  __host__ double bytes() const { return 8.0; }
  double *p[6];
  double scale[6];
  int n;
  int nb = 6;
  long long ms = 0;
  __device__ __forceinline__ int ent(int b) const { return MB ? b % nb : b; }
  __device__ __forceinline__ long long mof(int b) const { return MB ? (long long)(b / nb) * ms : 0; }
  // last pass of an inverse transform: vector v = ix, element k = iy
  __device__ __forceinline__ void operator()(int b, int v, int k, double x) const {
    const int e = ent(b);
    const double sc = pick(scale, e);
    pick(p, e)[mof(b) + (long long)v * n + k] = sc == 1.0 ? x : sc * x;
  }
  __device__ __forceinline__ void pair(int b, int v, int k, double2 x) const {
    const int e = ent(b);
    const double sc = pick(scale, e);
    if (sc != 1.0) x = make_double2(sc * x.x, sc * x.y);
    *reinterpret_cast<double2 *>(pick(p, e) + mof(b) + (long long)v * n + k) = x;
  }
};
using StoreScaled = StoreScaledT<false>;
template <bool MB>
struct LoadBatchT {
  __host__ double bytes() const { return 8.0; }
  const double *p[6];
  long long vs, es;
  int nb = 6;
  long long ms = 0;
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    const int e = MB ? b % nb : b;
    const long long o = MB ? (long long)(b / nb) * ms : 0;
    return pick(p, e)[o + (long long)v * vs + (long long)j * es];
  }
};
using LoadBatch = LoadBatchT<false>;
// FP32 storage for the inverse transform pair of the FP32-inversion mode:
// the kernel's arithmetic stays FP64 in registers; the intermediate and the
// physical outputs are rounded to FP32 once, when stored.
struct StoreStridedF {
  __host__ double bytes() const { return 4.0; }
  float *p;
  long long bs, vs, es;
  __device__ __forceinline__ void operator()(int b, int v, int k, double x) const {
    p[b * bs + (long long)v * vs + (long long)k * es] = (float)x;
  }
  __device__ __forceinline__ void pair(int b, int v, int k, double2 x) const {
    const long long o = b * bs + (long long)v * vs + (long long)k * es;
    if (es == 1) {
      *reinterpret_cast<float2 *>(p + o) = make_float2((float)x.x, (float)x.y);
    } else {
      p[o] = (float)x.x;
      p[o + es] = (float)x.y;
    }
  }
};
struct LoadBatchF {
  __host__ double bytes() const { return 4.0; }
  const float *p[6];
  long long vs, es;
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    return (double)pick(p, b)[(long long)v * vs + (long long)j * es];
  }
};
struct StoreScaledF {
  __host__ double bytes() const { return 4.0; }
  float *p[6];
  double scale[6];
  int n;
  __device__ __forceinline__ void operator()(int b, int v, int k, double x) const {
    const double sc = pick(scale, b);
    pick(p, b)[(long long)v * n + k] = (float)(sc == 1.0 ? x : sc * x);
  }
  __device__ __forceinline__ void pair(int b, int v, int k, double2 x) const {
    const double sc = pick(scale, b);
    if (sc != 1.0) x = make_double2(sc * x.x, sc * x.y);
    *reinterpret_cast<float2 *>(pick(p, b) + (long long)v * n + k) =
        make_float2((float)x.x, (float)x.y);
  }
};

// Load qq + kdsq*pp (adapt, evolution.f90:541-547).
struct LoadVort {
  __host__ double bytes() const { return btropic ? 8.0 : 16.0; }
  const double *qq, *pp;
  double kdsq;
  int btropic, n;
  long long ms = 0;  // ensemble: entry b = member b, fields ms apart
  // first pass of an inverse transform: vector v = ky, element j = kx
  __device__ __forceinline__ double operator()(int b, int v, int j) const {
    long long k = (long long)b * ms + (long long)v * n + j;
    return btropic ? qq[k] : qq[k] + kdsq * pp[k];
  }
};

// ---------------------------------------------------------------------------
// con2grid (contours.f90:173-346)
// ---------------------------------------------------------------------------
// Packed con2grid.  The coarse cell is C(cx, cy) = sum_b w_b G(4cx-3+b, cy)
// with G(fx, cy) = sum_a w_a L(fx, 4cy-3+a) the 7-tap of fine column fx at
// coarse row cy and L(fx, r) = lbot(fx) + sum_{r' <= r} J(fx, r') (rows and
// columns periodic, 0-based).  The jumps J of the four fine rows 4k..4k+3 of
// a column share one 64-bit word JW(fx, k) as signed 16-bit counts (a
// crossing at row r adds s << 16(r%4)), so a crossing is one atomic and the
// fine grid takes 2 bytes per cell.  A fine edge's net count is at most one
// per contour level crossing it (a level's crossings of a short segment
// alternate in sign), so the counts stay far inside +-32767 for the level
// counts the host allows on this path.  The sum kernel decodes the words
// and forms G from the column's running total and the seven rows around
// each coarse row; integer sums, so the result is the dense scan's to the
// bit in any order.
__device__ __forceinline__ void c2g_decode(unsigned long long w, int &c0, int &c1, int &c2,
                                           int &c3) {
  long long v = (long long)w;
  c0 = (int)(((v & 0xffff) ^ 0x8000) - 0x8000);
  v = (v - c0) >> 16;
  c1 = (int)(((v & 0xffff) ^ 0x8000) - 0x8000);
  v = (v - c1) >> 16;
  c2 = (int)(((v & 0xffff) ^ 0x8000) - 0x8000);
  v = (v - c2) >> 16;
  c3 = (int)v;
}

// Member of node i in an ensemble (mnode[m] <= i < mnode[m+1]; members
// without nodes have equal bounds and are skipped); 0 without an ensemble.
__device__ __forceinline__ int member_of(const int *__restrict__ mnode, int M, int i) {
  if (!mnode) return 0;
  int lo = 0, hi = M;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&mnode[mid]) <= i) lo = mid; else hi = mid;
  }
  return lo;
}
// Per-member strides of con2grid's scratch in an ensemble.
struct C2GMembers {
  const int *mnode;  // nullptr: one simulation
  int M;
  long long jws;     // packed words per member
  int ljs;           // bottom-row jumps per member
  int cs;            // Scalars stride in 64-bit words (member m's csum = csum + m*cs)
};

// Per segment (i, nextq(i)): x fine-grid-line crossings and the crossing of
// y = ymin, counted as +-1 PV jumps (contours.f90:232-270): J += sgn at
// each (PACKED: into the row's 16-bit lane of JW), ljx the bottom-boundary
// jumps.  The FP64 expressions are the reference's, evaluated in its order
// without FMA, so every crossing lands in the same fine cell.
template <bool PACKED>
__global__ void k_c2g_scatter(const double *__restrict__ xq, const double *__restrict__ yq,
                              const int *__restrict__ nextq, const Scalars *__restrict__ s,
                              int *__restrict__ J, unsigned long long *__restrict__ JW,
                              int *__restrict__ ljx,
                              Consts c, int *__restrict__ err,
                              unsigned long long *__restrict__ csum, C2GMembers mb) {
  CASL_PDL_ENTRY();
  // the coarsening that follows accumulates the coarse-cell sum here
  if (blockIdx.x == 0)
    for (int m = threadIdx.x; m < mb.M; m += blockDim.x) csum[(long long)m * mb.cs] = 0;
  const unsigned FULL = 0xffffffffu;
  const int npt = s->nptq, nf = c.nxf, lane = threadIdx.x & 31;
  const int wstride = gridDim.x * blockDim.x;
  // whole warps step through the nodes together (the shuffles below)
  for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < npt; base += wstride) {
    const int i = base + lane;
    int cnt = 0, ixbeg = 0, jump = 0, sgn = 0;
    double xi = 0.0, yi = 0.0, dx = 1.0, dy = 0.0;
    // the segment's far end is almost always the next node, which the next
    // lane has loaded: taken by shuffle, so the loads do not wait on nextq
    int ia = -1;
    double x1 = 0.0, y1 = 0.0;
    if (i < npt) {
      ia = nextq[i];
      x1 = xq[i];
      y1 = yq[i];
    }
    const double xs = __shfl_down_sync(FULL, x1, 1), ys = __shfl_down_sync(FULL, y1, 1);
    int mi = 0;
    if (i < npt) mi = member_of(mb.mnode, mb.M, i);
    if (i < npt) {
      if (ia < 0 || ia >= npt) {
        atomicExch(err, CASL_EINVAL);
      } else {
        xi = x1;
        yi = y1;
        const bool nb = ia == i + 1 && lane < 31;
        const double xa = nb ? xs : xq[ia], ya = nb ? ys : yq[ia];
        // both ends in the domain: an end outside it (or not finite) would
        // give a crossing count without bound; the node itself is reported
        // by its own lane
        if (!(xi >= c.xmin && xi < c.xmax && yi >= c.ymin && yi < c.ymax) ||
            !(xa >= c.xmin && xa < c.xmax && ya >= c.ymin && ya < c.ymax)) {
          atomicExch(err, CASL_EDOMAIN);
        } else {
          const int ixci = 1 + f_int(c.glxfi * (xi - c.xmin));
          const int ixca = 1 + f_int(c.glxfi * (xa - c.xmin));
          const double xx = xa - xi;
          dx = xx - c.ellx * f_dint(xx * c.hlxi);
          const double yy = ya - yi;
          dy = yy - c.elly * f_dint(yy * c.hlyi);
          const int ixdif = ixca - ixci;
          // nxc = ixdif - nf*((2*ixdif)/nf): with |2*ixdif| < 2nf the
          // truncated quotient is -1, 0 or 1
          const int t2 = 2 * ixdif;
          const int nxc = ixdif - nf * (t2 >= nf ? 1 : (t2 <= -nf ? -1 : 0));
          if (fabs(yy) > c.hly) {
            const double cc = f_sign1(dy);
            const double p = -(yi - c.hly * cc) / (dy + c.small);
            int ix = 1 + f_int(c.glxfi * fmod(c.ellx + c.hlx + xi + p * dx, c.ellx));
            ix = ix < 1 ? 1 : (ix > nf ? nf : ix);
            red_add_s32(&ljx[(long long)mi * mb.ljs + ix - 1], -(int)cc);
          }
          if (nxc != 0) {
            jump = f_isign1(nxc);
            ixbeg = ixci + (jump - 1) / 2 + nf;
            sgn = (int)f_sign1(dx);
            cnt = nxc * jump;
          }
        }
      }
    }
    // this lane's own crossings: fine lines ixbeg + k*jump, k < cnt (a few
    // per segment; the lanes' loops diverge but need no exchange)
    for (int k = 0; k < cnt; k++) {
      // (ixbeg + k*jump) mod nf, the argument lying in (nf/2, 5nf/2)
      int m = ixbeg + k * jump;
      m -= m >= nf ? nf : 0;
      m -= m >= nf ? nf : 0;
      const int ix = 1 + m;
      const double xgf = c.xmin + c.glxf * (double)(ix - 1);
      const double x2 = xgf - xi;
      const double px0 = (x2 - c.ellx * f_dint(x2 * c.hlxi)) / dx;
      const double y2 = yi + px0 * dy;
      const int iy = 2 + f_int(c.glyfi * (y2 - c.elly * f_dint(y2 * c.hlyi) - c.ymin));
      if (iy >= 2 && iy <= c.nyf) {
        if (PACKED) {
          const int r = iy - 1;
          red_add_u64(&JW[(long long)mi * mb.jws + (long long)(ix - 1) * c.nx + (r >> 2)],
                      (unsigned long long)((long long)sgn << (16 * (r & 3))));
        } else
          red_add_s32(&J[(long long)(ix - 1) * c.nyf + (iy - 1)], sgn);
      }
    }
  }
}

// qbot: exclusive prefix of the bottom jumps along x -> row 0 of each column.
__global__ void k_c2g_lbot(const int *__restrict__ ljx, int *__restrict__ J, int nxf, int nyf) {
  CASL_PDL_ENTRY();
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nxf; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < nxf ? ljx[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    int incl = x + (wid > 0 ? warp_tot[wid - 1] : 0) + carry;
    if (i < nxf) J[(long long)i * nyf] = incl - v;  // exclusive: lbot(ix)
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = incl;
    __syncthreads();
  }
}

// Inclusive scan down every fine column (contours.f90:272-277), in place:
// J(row, col) -> level L(iy = row+1, ix = col+1).  One warp per column.
__global__ void k_c2g_colscan(int *__restrict__ J, int nxf, int nyf) {
  CASL_PDL_ENTRY();
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nxf) return;
  int *col = J + (long long)warp * nyf;
  int carry = 0;
  for (int base = 0; base < nyf; base += 32) {
    int x = col[base + lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    x += carry;
    col[base + lane] = x;
    carry = __shfl_sync(0xffffffffu, x, 31);
  }
}

// Two nine-point 2:1 averagings (contours.f90:290-327) compose to a 7x7
// stencil with weights [1,2,3,4,3,2,1]^2/256 on fine rows/columns
// 4i-6..4i (1-based, periodic).  Levels are integers, so the coarse cell is
// the exact integer C; the mean is removed exactly from the integer sum.
__global__ void k_c2g_coarsen(const int *__restrict__ L, int *__restrict__ C,
                              unsigned long long *__restrict__ csum, int n, int nf) {
  CASL_PDL_ENTRY();
  const int w7[7] = {1, 2, 3, 4, 3, 2, 1};
  long long local = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    int iy = (int)(t % n) + 1, ix = (int)(t / n) + 1;
    int acc = 0;
#pragma unroll
    for (int b = 0; b < 7; b++) {
      int fx = 4 * ix - 6 + b;
      if (fx <= 0) fx += nf;
      const int *col = L + (long long)(fx - 1) * nf;
      int accy = 0;
#pragma unroll
      for (int a = 0; a < 7; a++) {
        int fy = 4 * iy - 6 + a;
        if (fy <= 0) fy += nf;
        accy += w7[a] * col[fy - 1];
      }
      acc += w7[b] * accy;
    }
    C[t] = acc;
    local += acc;
  }
  // block reduction of the integer sum (order-independent: exact)
  __shared__ long long red[32];
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 32) {
    long long v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(csum, (unsigned long long)v);
  }
}


// Packed con2grid, second half.  A CTA owns CW = 7 coarse columns and their
// 4*CW+3 = 31 fine columns, one warp per column, RPS = 32U coarse rows per
// step with the next step's words in flight.  Lane cy decodes its word,
// the warp scans the word totals (ex = jumps of all rows below 4cy), and
// with the two top counts of the word below (rows 4cy-2, 4cy-1) the seven
// levels L(4cy-3 .. 4cy+3) follow: L(4cy-1) = lbot + ex, one count taken or
// added per row on either side.  G passes through shared memory to the
// 7-tap along x.  Coarse row 0 wraps to the top rows and is formed last.
// Requires n % RPS == 0.
#define C2G_CW 7
#define C2G_FC (4 * C2G_CW + 3)

// The learned closure's sub-cell input: the fine levels at the 3 x 3 points
// (4cx + 2a - 2, 4cy + 2b - 2), a, b = 0..2, of every coarse cell (cx, cy),
// channel-major, F[3a + b][cx][cy].  Warp w of a CTA holds fine column
// 4 cx0 - 3 + w: a column 4k+1 is the a = 0 sample of coarse column k and
// the a = 2 sample of column k - 1, a column 4k+3 the a = 1 sample of k.
// La, Lb, Lc are the levels at fine rows 4cy - 2, 4cy, 4cy + 2.
__device__ __forceinline__ void c2g_feature(int *__restrict__ F, int n, int cx0, int w, int cy,
                                            int La, int Lb, int Lc) {
  const int r = w & 3, k = w >> 2;
  if (r != 1 && r != 3) return;
  const long long nn = (long long)n * n;
  int cxl[2], aa[2], m = 0;
  if (r == 3) {
    cxl[0] = k; aa[0] = 1; m = 1;
  } else {
    if (k < C2G_CW) { cxl[m] = k; aa[m++] = 0; }
    if (k >= 1) { cxl[m] = k - 1; aa[m++] = 2; }
  }
  for (int q = 0; q < m; q++) {
    const int cx = cx0 + cxl[q];
    if (cx >= n) continue;
    int *f = F + (long long)(3 * aa[q]) * nn + (long long)cx * n + cy;
    f[0] = La;
    f[nn] = Lb;
    f[2 * nn] = Lc;
  }
}

template <int U>
__global__ void __launch_bounds__(1024) k_c2g_packed_sum(const unsigned long long *__restrict__ JW,
                                                         const int *__restrict__ ljx,
                                                         int *__restrict__ C,
                                                         unsigned long long *__restrict__ csum,
                                                         int n, int nf, C2GMembers mb,
                                                         int *__restrict__ F) {
  CASL_PDL_ENTRY();
  {  // ensemble member blockIdx.y
    const long long m = blockIdx.y;
    JW += m * mb.jws;
    ljx += m * mb.ljs;
    C += m * (long long)n * n;
    csum += m * mb.cs;
  }
  constexpr int RPS = 32 * U;
  __shared__ int G[RPS][C2G_FC + 2];  // row length 33: conflict-free both ways
  __shared__ int G0[C2G_FC];
  __shared__ long long red[32];
  const unsigned FULL = 0xffffffffu;
  const int w7[7] = {1, 2, 3, 4, 3, 2, 1};
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cx0 = blockIdx.x * C2G_CW;
  int col = 4 * cx0 - 3 + warp;  // this warp's fine column (0-based), wrapped
  if (col < 0) col += nf;
  if (col >= nf) col -= nf;
  const unsigned long long *cp = JW + (long long)col * n + lane;
  const int nsteps = n / RPS;
  unsigned long long v[U];
  if (warp < C2G_FC) {
#pragma unroll
    for (int u = 0; u < U; u++) v[u] = __ldcs(cp + u * 32);
  }
  // lbot(col): the exclusive prefix of the bottom jumps (contours.f90:255-269),
  // scanned by the whole block four entries a thread; the threads whose
  // entries hold one of the block's columns keep that column's prefix
  {
    __shared__ int ptot;
    const int c0 = 4 * cx0 - 3;
    int pcarry = 0;
    for (int base = 0; base < nf; base += 4 * SCAN_BLOCK) {
      const int i0 = base + 4 * threadIdx.x;
      int a[4];
#pragma unroll
      for (int k = 0; k < 4; k++) a[k] = i0 + k < nf ? ljx[i0 + k] : 0;
      int pre = pcarry + block_excl_scan<int>(a[0] + a[1] + a[2] + a[3], &ptot);
      int d = i0 - c0;  // this thread's first entry relative to the block's first column
      d = d < 0 ? d + nf : (d >= nf ? d - nf : d);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        int w = d + k;
        if (w >= nf) w -= nf;
        if (i0 + k < nf && w < C2G_FC) G0[w] = pre;
        pre += a[k];
      }
      pcarry += ptot;
      __syncthreads();
    }
  }
  const int lb = warp < C2G_FC ? G0[warp] : 0;
  __syncthreads();  // G0 is reused for coarse row 0
  int carry = 0, q2 = 0, q3 = 0;       // running total; rows 4cy-2, 4cy-1 below lane 0
  int f0 = 0, f1 = 0, f2 = 0, f3 = 0;  // word 0 (rows 0..3), kept for coarse row 0
  long long local = 0;
  for (int s = 0; s < nsteps; s++) {
    if (warp < C2G_FC) {
#pragma unroll
      for (int u = 0; u < U; u++) {
        int c0, c1, c2, c3;
        c2g_decode(v[u], c0, c1, c2, c3);
        const int tot = c0 + c1 + c2 + c3;
        const int incl = warp_incl_scan(tot) + carry;
        const int ex = incl - tot;
        int p2 = __shfl_up_sync(FULL, c2, 1), p3 = __shfl_up_sync(FULL, c3, 1);
        if (lane == 0) {
          p2 = q2;
          p3 = q3;
        }
        const int L2 = lb + ex, L1 = L2 - p3, L0 = L1 - p2;
        const int L3 = L2 + c0, L4 = L3 + c1, L5 = L4 + c2, L6 = L5 + c3;
        G[u * 32 + lane][warp] =
            w7[0] * L0 + w7[1] * L1 + w7[2] * L2 + w7[3] * L3 + w7[4] * L4 + w7[5] * L5 + w7[6] * L6;
        if (F) {
          const int cy = s * RPS + u * 32 + lane;
          if (cy > 0) c2g_feature(F, n, cx0, warp, cy, L1, L3, L5);
        }
        if (s == 0 && u == 0 && lane == 0) {
          f0 = c0; f1 = c1; f2 = c2; f3 = c3;
        }
        carry = __shfl_sync(FULL, incl, 31);
        q2 = __shfl_sync(FULL, c2, 31);
        q3 = __shfl_sync(FULL, c3, 31);
      }
      if (s + 1 < nsteps) {
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = __ldcs(cp + (s + 1) * RPS + u * 32);
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < C2G_CW * RPS; t += blockDim.x) {
      const int cxl = t / RPS, rl = t % RPS;
      const int cx = cx0 + cxl, cy = s * RPS + rl;
      if (cx < n && cy > 0) {
        int acc = 0;
#pragma unroll
        for (int b = 0; b < 7; b++) acc += w7[b] * G[rl][4 * cxl + b];
        C[(long long)cx * n + cy] = acc;
        local += acc;
      }
    }
    __syncthreads();
  }
  // coarse row 0: fine rows nf-3, nf-2, nf-1 (the top word: q2, q3 are its
  // rows nf-2, nf-1; carry is the column total) and rows 0..3 (word 0)
  if (warp < C2G_FC && lane == 0) {
    const int L2 = lb + carry, L1 = L2 - q3, L0 = L1 - q2;
    const int L3 = lb + f0, L4 = L3 + f1, L5 = L4 + f2, L6 = L5 + f3;
    G0[warp] = w7[0] * L0 + w7[1] * L1 + w7[2] * L2 + w7[3] * L3 + w7[4] * L4 + w7[5] * L5 +
               w7[6] * L6;
    if (F) c2g_feature(F, n, cx0, warp, 0, L1, L3, L5);
  }
  __syncthreads();
  if (threadIdx.x < C2G_CW) {
    const int cx = cx0 + threadIdx.x;
    if (cx < n) {
      int acc = 0;
#pragma unroll
      for (int b = 0; b < 7; b++) acc += w7[b] * G0[4 * threadIdx.x + b];
      C[(long long)cx * n] = acc;
      local += acc;
    }
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(FULL, local, o);
  if (lane == 0) red[warp] = local;
  __syncthreads();
  if (warp == 0) {
    long long x = red[lane];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL, x, o);
    if (lane == 0) atomicAdd(csum, (unsigned long long)x);
  }
}


// c = a * b elementwise
__global__ void k_mul2(const double *__restrict__ a, const double *__restrict__ b,
                       double *__restrict__ c, long long nn) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x)
    c[k] = a[k] * b[k];
}

__global__ void k_c2g_final(const int *__restrict__ C, const Scalars *__restrict__ s,
                            const double *__restrict__ betac, double *__restrict__ qc, int n) {
  CASL_PDL_ENTRY();
  LoadQC ld{C, s, betac, (long long)n * n, 1.0 / (256.0 * (double)n * (double)n), n};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    int iy = (int)(t % n), ix = (int)(t / n);
    qc[t] = ld(0, ix, iy);
  }
}

static int grid_for(long long work, int block = 256) {
  long long g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

int con2grid_dev(casl_handle *h, bool want_levels) {
  const Consts &c = h->c;
  int *err = &h->scal->error;
  unsigned long long *csum = (unsigned long long *)&h->scal->csum;
  const int n = h->n;
  const int U = n % 256 == 0 ? 8 : (n % 128 == 0 ? 4 : (n % 64 == 0 ? 2 : (n % 32 == 0 ? 1 : 0)));
  // packed path while the 16-bit counts cannot overflow (one net crossing
  // per level and fine edge: levels well below 32767)
  // an ensemble always takes the packed path (its scratch holds only that)
  if (h->M > 1 && (want_levels || U == 0 || h->p.ncontq >= 16384)) return CASL_EUNSUPPORTED;
  if (!want_levels && c.nxf == c.nyf && U > 0 && h->p.ncontq < 16384) {
    // four fine rows of a column per 64-bit word, in the first half of the
    // fine-grid buffer (an ensemble: one such block per member)
    unsigned long long *JW = reinterpret_cast<unsigned long long *>(h->fineJ);
    const C2GMembers mb{h->M > 1 ? h->mnode : nullptr, h->M, (long long)c.nxf * n, c.nxf,
                        (int)(sizeof(Scalars) / 8)};
    {
      const FillJob z[2] = {{JW, 2LL * c.nxf * n * h->M, 0u},
                            {h->ljx, (long long)c.nxf * h->M, 0u}};
      if (int rc = fill_words(h->stream, z, 2)) return rc;
    }
    // with no nodes the scatter still runs (its first block clears the sums)
    CASL_K(k_c2g_scatter<true>, grid_for(h->nptq > 0 ? h->nptq : 1), 256, 0, h->stream)(
        h->xq, h->yq, h->nextq, h->scal, nullptr, JW, h->ljx, c, err, csum, mb);
    const dim3 nblk((n + C2G_CW - 1) / C2G_CW, h->M);
    // the learned closure's sub-cell levels, while it is attached (one simulation)
    int *feat = h->M == 1 ? h->c2g_feat : nullptr;
    if (U == 8)
      CASL_K(k_c2g_packed_sum<8>, nblk, 1024, 0, h->stream)(JW, h->ljx, h->coarseC, csum, n, c.nxf, mb, feat);
    else if (U == 4)
      CASL_K(k_c2g_packed_sum<4>, nblk, 1024, 0, h->stream)(JW, h->ljx, h->coarseC, csum, n, c.nxf, mb, feat);
    else if (U == 2)
      CASL_K(k_c2g_packed_sum<2>, nblk, 1024, 0, h->stream)(JW, h->ljx, h->coarseC, csum, n, c.nxf, mb, feat);
    else
      CASL_K(k_c2g_packed_sum<1>, nblk, 1024, 0, h->stream)(JW, h->ljx, h->coarseC, csum, n, c.nxf, mb, feat);
    return check_launch(h);
  }
  // the fine-grid levels themselves are wanted: crossings onto the fine
  // grid, bottom row, scan in place, then coarsen
  size_t fine = (size_t)c.nxf * c.nyf;
  CASL_CUDA_TRY(cudaMemsetAsync(h->fineJ, 0, fine * sizeof(int), h->stream));
  CASL_CUDA_TRY(cudaMemsetAsync(h->ljx, 0, (size_t)c.nxf * sizeof(int), h->stream));
  if (h->nptq > 0) {
    const C2GMembers mb{nullptr, 1, 0, 0, (int)(sizeof(Scalars) / 8)};
    CASL_K(k_c2g_scatter<false>, grid_for(h->nptq), 256, 0, h->stream)(
        h->xq, h->yq, h->nextq, h->scal, h->fineJ, nullptr, h->ljx, c, err, csum, mb);
  } else {
    CASL_CUDA_TRY(cudaMemsetAsync(csum, 0, sizeof(unsigned long long), h->stream));
  }
  CASL_K(k_c2g_lbot, 1, 1024, 0, h->stream)(h->ljx, h->fineJ, c.nxf, c.nyf);
  CASL_K(k_c2g_colscan, (c.nxf * 32 + 255) / 256, 256, 0, h->stream)(h->fineJ, c.nxf, c.nyf);
  CASL_K(k_c2g_coarsen, grid_for((long long)h->n * h->n), 256, 0, h->stream)(
      h->fineJ, h->coarseC, csum, h->n, c.nxf);
  return check_launch(h);
}

// (an ensemble: every member's, spec being M fields long)
int con2grid_to_spec(casl_handle *h, double *spec) {
  long long n = h->n, nn = n * n;
  const int M = h->M;
  if (h->nptq == 0) {
    CASL_CUDA_TRY(cudaMemsetAsync(spec, 0, M * nn * sizeof(double), h->stream));
    return CASL_OK;
  }
  int rc = con2grid_dev(h, false);
  if (rc) return rc;
  LoadQC ld{h->coarseC, h->scal, h->c.beffect ? h->betac : nullptr, nn,
            1.0 / (256.0 * (double)n * (double)n), (int)n};
  rc = RFFT_DISPATCH(true, false, true, ld, (StoreStrided{spec, nn, 1, n}), M);
  if (rc) return rc;
  return RFFT_DISPATCH(true, false, false, (LoadRow{spec, nn, n, (int)n, &h->scal->error}),
                       (StoreStrided{spec, nn, n, 1}), M);
}

int con2grid_to_phys(casl_handle *h, double *phys, bool want_levels) {
  long long nn = (long long)h->n * h->n;
  if (h->nptq == 0) {
    CASL_CUDA_TRY(cudaMemsetAsync(phys, 0, nn * sizeof(double), h->stream));
    return CASL_OK;
  }
  int rc = con2grid_dev(h, want_levels);
  if (rc) return rc;
  CASL_K(k_c2g_final, grid_for(nn), 256, 0, h->stream)(h->coarseC, h->scal,
                                                   h->c.beffect ? h->betac : nullptr, phys, h->n);
  return check_launch(h);
}

// ---------------------------------------------------------------------------
// velint (contours.f90:136-169) and the RK4 node updates (evolution.f90:212-311)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void velint1(double x, double y, const T *__restrict__ uu,
                                        const T *__restrict__ vv, const Consts &c,
                                        double &uq, double &vq) {
  double xx = c.glxi * (x - c.xmin);
  int ix0 = 1 + f_int(xx);
  double pxc = (double)ix0 - xx;
  double px = 1.0 - pxc;
  double yy = c.glyi * (y - c.ymin);
  int iy0 = 1 + f_int(yy);
  double pyc = (double)iy0 - yy;
  double py = 1.0 - pyc;
  // ixp/iyp (contours.f90:58-66); indices clamped so that no input can read
  // outside the field (valid nodes never need the clamp).
  ix0 = ix0 < 1 ? 1 : (ix0 > c.nx ? c.nx : ix0);
  iy0 = iy0 < 1 ? 1 : (iy0 > c.ny ? c.ny : iy0);
  int ix1 = ix0 == c.nx ? 1 : ix0 + 1;
  int iy1 = iy0 == c.ny ? 1 : iy0 + 1;
  long long a00 = (long long)(ix0 - 1) * c.ny + (iy0 - 1);
  long long a01 = (long long)(ix1 - 1) * c.ny + (iy0 - 1);
  long long a10 = (long long)(ix0 - 1) * c.ny + (iy1 - 1);
  long long a11 = (long long)(ix1 - 1) * c.ny + (iy1 - 1);
  uq = pyc * (pxc * (double)__ldg(&uu[a00]) + px * (double)__ldg(&uu[a01])) +
       py * (pxc * (double)__ldg(&uu[a10]) + px * (double)__ldg(&uu[a11]));
  vq = pyc * (pxc * (double)__ldg(&vv[a00]) + px * (double)__ldg(&vv[a01])) +
       py * (pxc * (double)__ldg(&vv[a10]) + px * (double)__ldg(&vv[a11]));
}

__global__ void k_velint(const double *__restrict__ xq, const double *__restrict__ yq, int npt,
                         const double *__restrict__ uu, const double *__restrict__ vv,
                         double *__restrict__ uq, double *__restrict__ vq, Consts c) {
  CASL_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    double u, v;
    velint1(xq[i], yq[i], uu, vv, c, u, v);
    uq[i] = u;
    vq[i] = v;
  }
}

template <int STAGE, class T>
__device__ __forceinline__ void nodes_rk_body(int bid, int nbk, double *__restrict__ xq, double *__restrict__ yq,
                           double *__restrict__ xqi, double *__restrict__ yqi,
                           double *__restrict__ xqf, double *__restrict__ yqf,
                           const T *__restrict__ uu, const T *__restrict__ vv,
                           const Scalars *__restrict__ s, const Consts &c,
                           const int *__restrict__ mnode, int M,
                           const double *__restrict__ du, const double *__restrict__ dv) {
  const int npt = s->nptq;
  const double ex = c.ellx, ey = c.elly, hx = c.hlxi, hy = c.hlyi, oms = c.oms;
  const long long nn = (long long)c.nx * c.ny;
  for (int i = bid * blockDim.x + threadIdx.x; i < npt; i += nbk * blockDim.x) {
    // the node's ensemble member: its time step and velocity field
    const int m = member_of(mnode, M, i);
    const Scalars &sm = s[m];
    const double dt = sm.dt, dt2 = sm.dt2, dt3 = sm.dt3, dt6 = sm.dt6;
    double uq, vq;
    velint1(xq[i], yq[i], uu + m * nn, vv + m * nn, c, uq, vq);
    if (du) {
      uq = uq + du[i];
      vq = vq + dv[i];
    }
    if (STAGE == 1) {
      double x0 = xq[i], y0 = yq[i];
      xqi[i] = x0;
      yqi[i] = y0;
      xq[i] = wrapp(x0 + dt2 * uq, ex, hx, oms);
      yq[i] = wrapp(y0 + dt2 * vq, ey, hy, oms);
      xqf[i] = wrapp(x0 + dt6 * uq, ex, hx, oms);
      yqf[i] = wrapp(y0 + dt6 * vq, ey, hy, oms);
    } else if (STAGE == 2) {
      xq[i] = wrapp(xqi[i] + dt2 * uq, ex, hx, oms);
      yq[i] = wrapp(yqi[i] + dt2 * vq, ey, hy, oms);
      xqf[i] = wrapp(xqf[i] + dt3 * uq, ex, hx, oms);
      yqf[i] = wrapp(yqf[i] + dt3 * vq, ey, hy, oms);
    } else if (STAGE == 3) {
      xq[i] = wrapp(xqi[i] + dt * uq, ex, hx, oms);
      yq[i] = wrapp(yqi[i] + dt * vq, ey, hy, oms);
      xqf[i] = wrapp(xqf[i] + dt3 * uq, ex, hx, oms);
      yqf[i] = wrapp(yqf[i] + dt3 * vq, ey, hy, oms);
    } else {
      xq[i] = wrapp(xqf[i] + dt6 * uq, ex, hx, oms);
      yq[i] = wrapp(yqf[i] + dt6 * vq, ey, hy, oms);
    }
  }
}

// ---------------------------------------------------------------------------
// Spectral pointwise kernels
// ---------------------------------------------------------------------------
// inversion's qq = flo*(qs-qc)+qc+qd and pp = green*qq (evolution.f90:514,
// spectral.f90:321); with reset (evolution.f90:199-200) also qs <- qq and
// qd <- fhi*(qs-qc).
template <bool RESET>
__global__ void k_combine(double *__restrict__ qs, double *__restrict__ qd,
                          const double *__restrict__ qc, double *__restrict__ qq,
                          double *__restrict__ pp, const double *__restrict__ flo,
                          const double *__restrict__ fhi, const double *__restrict__ green,
                          long long nn, long long tot) {
  CASL_PDL_ENTRY();
  // two elements per thread with 16-byte accesses (nn is even); tot = M*nn
  // over the members of an ensemble, whose tables are shared
  for (long long k2 = blockIdx.x * (long long)blockDim.x + threadIdx.x; k2 < tot / 2;
       k2 += (long long)gridDim.x * blockDim.x) {
    const long long k = 2 * k2, kt = k & (nn - 1);  // nn is a power of two
    const double2 s = *reinterpret_cast<const double2 *>(qs + k);
    const double2 c = *reinterpret_cast<const double2 *>(qc + k);
    const double2 d = *reinterpret_cast<const double2 *>(qd + k);
    const double2 f = *reinterpret_cast<const double2 *>(flo + kt);
    const double2 g = *reinterpret_cast<const double2 *>(green + kt);
    const double q0 = f.x * (s.x - c.x) + c.x + d.x, q1 = f.y * (s.y - c.y) + c.y + d.y;
    *reinterpret_cast<double2 *>(qq + k) = make_double2(q0, q1);
    *reinterpret_cast<double2 *>(pp + k) = make_double2(g.x * q0, g.y * q1);
    if (RESET) {
      const double2 h = *reinterpret_cast<const double2 *>(fhi + kt);
      *reinterpret_cast<double2 *>(qs + k) = make_double2(q0, q1);
      *reinterpret_cast<double2 *>(qd + k) = make_double2(h.x * (q0 - c.x), h.y * (q1 - c.y));
    }
  }
}


// ---------------------------------------------------------------------------
// adapt (evolution.f90:524-608): deterministic two-level reductions
// ---------------------------------------------------------------------------
#define RED_BLOCKS 296
template <class T>
__global__ void k_reduce_adapt(const double *__restrict__ zz, const T *__restrict__ uu,
                               const T *__restrict__ vv, double *__restrict__ part,
                               long long nn) {
  CASL_PDL_ENTRY();
  {  // ensemble member blockIdx.y: its fields and its gridDim.x partials
    const long long m = blockIdx.y;
    zz += m * nn;
    uu += m * nn;
    vv += m * nn;
    part += m * 3 * gridDim.x;
  }
  double sum = 0.0, zmax = 0.0, umax = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x) {
    double z = zz[k];
    z = z * z;
    sum += z;
    zmax = fmax(zmax, z);
    const double u = (double)uu[k], v = (double)vv[k];
    double w = u * u + v * v;
    umax = fmax(umax, w);
  }
  __shared__ double s0[256], s1[256], s2[256];
  s0[threadIdx.x] = sum;
  s1[threadIdx.x] = zmax;
  s2[threadIdx.x] = umax;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s0[threadIdx.x] += s0[threadIdx.x + o];
      s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + o]);
      s2[threadIdx.x] = fmax(s2[threadIdx.x], s2[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = s0[0];
    part[3 * blockIdx.x + 1] = s1[0];
    part[3 * blockIdx.x + 2] = s2[0];
  }
}

__global__ void k_adapt_final(const double *__restrict__ part, int nparts, Scalars *s, Consts c,
                              double fixed_dt) {
  CASL_PDL_ENTRY();
  // ensemble member blockIdx.x
  part += (long long)blockIdx.x * 3 * nparts;
  s += blockIdx.x;
  __shared__ double s0[256], s1[256], s2[256];
  double a = 0.0, b = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    a += part[3 * i];
    b = fmax(b, part[3 * i + 1]);
    d = fmax(d, part[3 * i + 2]);
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  s2[threadIdx.x] = d;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s0[threadIdx.x] += s0[threadIdx.x + o];
      s1[threadIdx.x] = fmax(s1[threadIdx.x], s1[threadIdx.x + o]);
      s2[threadIdx.x] = fmax(s2[threadIdx.x], s2[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double dtfac = c.pi / 10.0, cflmax = 0.7;
    double zzrms = sqrt(c.dsumi * s0[0]);
    double zzmax = sqrt(s1[0]) + c.small;
    double uumax = sqrt(s2[0]) + c.small;
    double t1 = c.glx * cflmax / uumax;
    double t2 = dtfac / fmax(zzmax, c.srwfm);
    double dtacc = fmin(t1, t2);
    double dt;
    if (fixed_dt > 0.0)
      dt = fixed_dt;
    else
      dt = fmin(dtacc, s->dtmax);
    s->dt = dt;
    s->dt2 = dt * 0.5;
    s->dt3 = dt * (1.0 / 3.0);
    s->dt6 = dt * (1.0 / 6.0);
    s->twist = s->twist + dt * zzmax;
    s->zzrms = zzrms;
    s->zzmax = zzmax;
    s->uumax = uumax;
  }
}

__global__ void k_epq(const double *__restrict__ qdiss, double *__restrict__ epq,
                      double *__restrict__ emq, const Scalars *__restrict__ s, long long nn,
                      long long tot) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot;
       k += (long long)gridDim.x * blockDim.x) {
    const Scalars &sm = s[k / nn];  // ensemble member of element k
    const double dfac = sm.dt2 * sm.zzrms;
    double e = exp(dfac * qdiss[k & (nn - 1)]);
    epq[k] = e;
    emq[k] = 1.0 / e;
  }
}

// The RK4 update of the spectral fields (evolution.f90:212-311, the qs/qd
// halves of each stage), two elements per thread with 16-byte accesses.
template <int STAGE>
__device__ __forceinline__ void spec_rk_body(int bid, int nbk, double *__restrict__ qs, double *__restrict__ qd,
                          double *__restrict__ qsi, double *__restrict__ qsf,
                          double *__restrict__ qdi, double *__restrict__ qdf,
                          const double *__restrict__ sqs, const double *__restrict__ sqd,
                          double *__restrict__ emq, const Scalars *__restrict__ s, long long nn,
                          long long tot) {
  auto L = [](const double *p, long long k) { return *reinterpret_cast<const double2 *>(p + k); };
  auto S = [](double *p, long long k, double x, double y) {
    *reinterpret_cast<double2 *>(p + k) = make_double2(x, y);
  };
  for (long long k2 = bid * (long long)blockDim.x + threadIdx.x; k2 < tot / 2;
       k2 += (long long)nbk * blockDim.x) {
    const long long k = 2 * k2;
    const Scalars &sm = s[tot == nn ? 0 : k / nn];  // ensemble member of element k
    const double dt = sm.dt, dt2 = sm.dt2, dt3 = sm.dt3, dt6 = sm.dt6;
    const double2 a = L(sqs, k), b = L(sqd, k);
    if (STAGE == 1) {
      const double2 si = L(qs, k), di = L(qd, k), e = L(emq, k);
      S(qsi, k, si.x, si.y);
      S(qs, k, si.x + dt2 * a.x, si.y + dt2 * a.y);
      S(qsf, k, si.x + dt6 * a.x, si.y + dt6 * a.y);
      S(qdi, k, di.x, di.y);
      S(qd, k, e.x * (di.x + dt2 * b.x), e.y * (di.y + dt2 * b.y));
      S(qdf, k, di.x + dt6 * b.x, di.y + dt6 * b.y);
    } else if (STAGE == 2) {
      const double2 si = L(qsi, k), sf = L(qsf, k), di = L(qdi, k), df = L(qdf, k), e = L(emq, k);
      S(qs, k, si.x + dt2 * a.x, si.y + dt2 * a.y);
      S(qsf, k, sf.x + dt3 * a.x, sf.y + dt3 * a.y);
      S(qd, k, e.x * (di.x + dt2 * b.x), e.y * (di.y + dt2 * b.y));
      S(qdf, k, df.x + dt3 * b.x, df.y + dt3 * b.y);
    } else if (STAGE == 3) {
      const double2 si = L(qsi, k), sf = L(qsf, k), di = L(qdi, k), df = L(qdf, k);
      double2 e = L(emq, k);
      e = make_double2(e.x * e.x, e.y * e.y);
      S(emq, k, e.x, e.y);
      S(qs, k, si.x + dt * a.x, si.y + dt * a.y);
      S(qsf, k, sf.x + dt3 * a.x, sf.y + dt3 * a.y);
      S(qd, k, e.x * (di.x + dt * b.x), e.y * (di.y + dt * b.y));
      S(qdf, k, df.x + dt3 * b.x, df.y + dt3 * b.y);
    } else {
      const double2 sf = L(qsf, k), df = L(qdf, k), e = L(emq, k);
      S(qs, k, sf.x + dt6 * a.x, sf.y + dt6 * a.y);
      S(qd, k, e.x * (df.x + dt6 * b.x), e.y * (df.y + dt6 * b.y));
    }
  }
}

// The end of an RK4 stage in one launch: blocks below nbn move the nodes
// (velint + node update), the rest update the spectral fields; the two
// parts touch disjoint data and read only dt from the scalars.
template <class T>
struct NodeRkArgs {
  double *xq, *yq, *xqi, *yqi, *xqf, *yqf;
  const T *uu, *vv;
  const int *mnode;  // ensemble: first node of each member (nullptr: one simulation)
  int M;
  const double *du, *dv;  // learned closure: correction at every node (nullable)
};
struct SpecRkArgs {
  double *qs, *qd, *qsi, *qsf, *qdi, *qdf;
  const double *sqs, *sqd;
  double *emq;
  long long nn, tot;  // tot = M*nn
};
template <int STAGE, class T>
__global__ void k_stage_rk(NodeRkArgs<T> a, SpecRkArgs b, Scalars *__restrict__ s, Consts c,
                           int nbn) {
  CASL_PDL_ENTRY();
  // the half-step time advance that opens stages 2 and 4 (nothing reads t
  // in between)
  if ((STAGE == 1 || STAGE == 3) && blockIdx.x == 0)
    for (int m = threadIdx.x; m < a.M; m += blockDim.x) s[m].t = s[m].t + s[m].dt2;
  if ((int)blockIdx.x < nbn)
    nodes_rk_body<STAGE, T>(blockIdx.x, nbn, a.xq, a.yq, a.xqi, a.yqi, a.xqf, a.yqf, a.uu, a.vv, s, c,
                            a.mnode, a.M, a.du, a.dv);
  else
    spec_rk_body<STAGE>(blockIdx.x - nbn, gridDim.x - nbn, b.qs, b.qd, b.qsi, b.qsf, b.qdi,
                        b.qdf, b.sqs, b.sqd, b.emq, s, b.nn, b.tot);
}


__global__ void k_twist_sub(Scalars *s, double twistmax, int M) {
  CASL_PDL_ENTRY();
  for (int m = threadIdx.x; m < M; m += blockDim.x) s[m].twist = s[m].twist - twistmax;
}
__global__ void k_twist_zero(Scalars *s, int M) {
  CASL_PDL_ENTRY();
  for (int m = threadIdx.x; m < M; m += blockDim.x) s[m].twist = 0.0;
}

// ---------------------------------------------------------------------------
// Stages
// ---------------------------------------------------------------------------
// con2grid + the filter combination that forms qq and pp (evolution.f90:507-514)
static int inversion_qq(casl_handle *h, bool reset) {
  long long nn = (long long)h->n * h->n;
  const int M = h->M;  // ensemble members: one transform batch entry each
  if (h->nptq == 0) {
    CASL_CUDA_TRY(cudaMemsetAsync(h->qc, 0, M * nn * sizeof(double), h->stream));
  } else {
    // con2grid, then its forward transform
    int rc = con2grid_dev(h, false);
    if (rc) return rc;
    long long n = h->n;
    LoadQC ld{h->coarseC, h->scal, h->c.beffect ? h->betac : nullptr, nn,
              1.0 / (256.0 * (double)n * (double)n), (int)n};
    rc = RFFT_DISPATCH(true, false, true, ld, (StoreStrided{h->qc, nn, 1, n}), M);
    if (rc) return rc;
    // The combination runs as its own elementwise pass: inside the batch-1
    // transform's store (about 3.5 warps per SM) its extra loads were
    // exposed and the fused pass took longer than the two apart.
    rc = RFFT_DISPATCH(true, false, false, (LoadRow{h->qc, nn, n, (int)n, &h->scal->error}),
                       (StoreStrided{h->qc, nn, n, 1}), M);
    if (rc) return rc;
  }
  if (reset)
    CASL_K(k_combine<true>, grid_for(M * nn), 256, 0, h->stream)(
        h->qs, h->qd, h->qc, h->qq, h->pp, h->flo, h->fhi, h->green, nn, M * nn);
  else
    CASL_K(k_combine<false>, grid_for(M * nn), 256, 0, h->stream)(
        h->qs, h->qd, h->qc, h->qq, h->pp, h->flo, h->fhi, h->green, nn, M * nn);
  return check_launch(h);
}

// main_invert (spectral.f90:304-342): vv = spctop(xderiv(green*qq)),
// uu = -spctop(yderiv(green*qq))
template <bool MB>
static int main_invert_t(casl_handle *h) {
  long long nn = (long long)h->n * h->n;
  int rc;
  LoadDerivT<MB> ld{};
  ld.f[0] = h->qq; ld.f[1] = h->qq;
  ld.dir[0] = 0; ld.dir[1] = 1;
  ld.wg[0] = 1; ld.wg[1] = 1;
  ld.green = h->green; ld.hrkx = h->hrkx; ld.hrky = h->hrky; ld.n = h->n;
  ld.err = &h->scal->error;
  ld.nb = 2; ld.ms = nn;  // ensemble: two entries per member
  long long n = h->n;
  const int M = h->M;
  // intermediate of entry b at w[0] + b*nn (2M contiguous fields: w[0..1]
  // are 2M fields long)
  rc = RFFT_DISPATCH(false, false, false, ld, (StoreStrided{h->w[0], nn, n, 1}), 2 * M);
  if (rc) return rc;
  StoreScaledT<MB> st{};
  st.p[0] = h->vv; st.p[1] = h->uu;
  st.scale[0] = 1.0; st.scale[1] = -1.0; st.n = h->n;
  st.nb = 2; st.ms = nn;
  // second pass reads tmp[ky*n + ix] (v = ix fastest, j = ky) and writes phys [ix][iy]
  LoadBatchT<MB> lb{};
  lb.p[0] = h->w[0]; lb.p[1] = h->w[0] + nn; lb.vs = 1; lb.es = n;
  lb.nb = 2; lb.ms = 2 * nn;
  return RFFT_DISPATCH(false, true, false, lb, st, 2 * M);
}
static int main_invert_dev(casl_handle *h) {
  return h->M > 1 ? main_invert_t<true>(h) : main_invert_t<false>(h);
}

// main_invert and the four gradients of source (evolution.f90:432-490,
// spectral.f90:304-366) as one batch-6 inverse transform pair: vv, uu from
// green*qq, and the x/y derivatives of qd (into w[4], w[5]) and of qs (into
// sqs, sqd, as scratch for the advection products).  One batch of six fills
// the SMs better than a batch of two beside a batch of four.  Scratch:
// gtmp (6 fields).
template <bool MB>
static int invert_and_gradients_t(casl_handle *h) {
  long long nn = (long long)h->n * h->n, n = h->n;
  const int M = h->M;  // ensemble: six entries per member
  LoadDerivT<MB> ld{};
  const double *src[6] = {h->qq, h->qq, h->qd, h->qd, h->qs, h->qs};
  for (int b = 0; b < 6; b++) {
    ld.f[b] = src[b];
    ld.dir[b] = b & 1;
    ld.wg[b] = b < 2;
  }
  ld.green = h->green; ld.hrkx = h->hrkx; ld.hrky = h->hrky; ld.n = h->n;
  ld.err = &h->scal->error;
  ld.nb = 6; ld.ms = nn;
  double *tmp = h->gtmp;  // 6M contiguous fields
  int rc = RFFT_DISPATCH(false, false, false, ld, (StoreStrided{tmp, nn, n, 1}), 6 * M);
  if (rc) return rc;
  LoadBatchT<MB> lb{};
  for (int b = 0; b < 6; b++) lb.p[b] = tmp + b * nn;
  lb.vs = 1; lb.es = n;
  lb.nb = 6; lb.ms = 6 * nn;
  StoreScaledT<MB> st{};
  double *dst[6] = {h->vv, h->uu, h->w[4], h->w[5], h->sqs, h->sqd};
  for (int b = 0; b < 6; b++) {
    st.p[b] = dst[b];
    st.scale[b] = b == 1 ? -1.0 : 1.0;
  }
  st.n = h->n;
  st.nb = 6; st.ms = nn;
  return RFFT_DISPATCH(false, true, false, lb, st, 6 * M);
}
static int invert_and_gradients(casl_handle *h) {
  return h->M > 1 ? invert_and_gradients_t<true>(h) : invert_and_gradients_t<false>(h);
}

// The same batch-6 inverse pair with FP32 storage (CASL_PREC_FP32_INVERSION):
// the intermediate in gtmp as floats, the outputs in f32 = [u, v, dqd/dx,
// dqd/dy, dqs/dx, dqs/dy].
static int invert_and_gradients32(casl_handle *h) {
  long long nn = (long long)h->n * h->n, n = h->n;
  LoadDeriv ld{};
  const double *src[6] = {h->qq, h->qq, h->qd, h->qd, h->qs, h->qs};
  for (int b = 0; b < 6; b++) {
    ld.f[b] = src[b];
    ld.dir[b] = b & 1;
    ld.wg[b] = b < 2;
  }
  ld.green = h->green; ld.hrkx = h->hrkx; ld.hrky = h->hrky; ld.n = h->n;
  ld.err = &h->scal->error;
  float *tmp = reinterpret_cast<float *>(h->gtmp);  // 6 contiguous FP32 fields
  int rc = RFFT_DISPATCH(false, false, false, ld, (StoreStridedF{tmp, nn, n, 1}), 6);
  if (rc) return rc;
  LoadBatchF lb{};
  for (int b = 0; b < 6; b++) lb.p[b] = tmp + b * nn;
  lb.vs = 1; lb.es = n;
  StoreScaledF st{};
  const int slot[6] = {1, 0, 2, 3, 4, 5};  // b = 0: d/dx of green*qq = v; b = 1: -d/dy = u
  for (int b = 0; b < 6; b++) {
    st.p[b] = h->f32 + slot[b] * nn;
    st.scale[b] = b == 1 ? -1.0 : 1.0;
  }
  st.n = h->n;
  h->uv_fp32 = 1;
  return RFFT_DISPATCH(false, true, false, lb, st, 6);
}

int inversion_dev(casl_handle *h, bool reset) {
  int rc = inversion_qq(h, reset);
  if (rc) return rc;
  h->uv_fp32 = 0;
  return main_invert_dev(h);
}

static int adapt_dev(casl_handle *h) {
  long long nn = (long long)h->n * h->n, n = h->n;
  const int M = h->M;  // ensemble: one entry, one reduction and one dt per member
  LoadVort lv{h->qq, h->pp, h->c.kdsq, h->c.btropic, h->n};
  lv.ms = nn;
  int rc = RFFT_DISPATCH(false, false, false, lv, (StoreStrided{h->w[0], nn, n, 1}), M);
  if (rc) return rc;
  rc = RFFT_DISPATCH(false, true, false, (LoadStrided{h->w[0], nn, 1, n}),
                     (StoreStrided{h->w[1], nn, n, 1}), M);
  if (rc) return rc;
  if (h->prec == CASL_PREC_FP32_INVERSION)
    CASL_K(k_reduce_adapt<float>, RED_BLOCKS, 256, 0, h->stream)(h->w[1], h->f32, h->f32 + nn,
                                                                 h->part, nn);
  else
    CASL_K(k_reduce_adapt<double>, dim3(RED_BLOCKS, M), 256, 0, h->stream)(h->w[1], h->uu, h->vv,
                                                                           h->part, nn);
  CASL_K(k_adapt_final, M, 256, 0, h->stream)(h->part, RED_BLOCKS, h->scal, h->c, h->p.fixed_dt);
  CASL_K(k_epq, grid_for(M * nn), 256, 0, h->stream)(h->qdiss, h->epq, h->emq, h->scal, nn,
                                                     M * nn);
  return check_launch(h);
}

// source (evolution.f90:432-490) after its gradients (invert_and_gradients):
// the advection products fused into ptospc's first pass, damping and the
// integrating factor into its store.
static int source_prod(casl_handle *h, int stage) {
  const int lev = stage == 1 ? 0 : (stage == 4 ? 2 : 1);
  long long nn = (long long)h->n * h->n, n = h->n;
  double *tmp = h->w[0];  // w[0..1]
  int rc;
  // products -> ptospc's first pass into tmp, its second pass with the source store
  if (h->prec == CASL_PREC_FP32_INVERSION) {
    const float *f = h->f32;
    LoadAdvectT<float> la{};
    la.uu = f; la.vv = f + nn;
    la.fx[0] = f + 2 * nn; la.fy[0] = f + 3 * nn;
    la.fx[1] = f + 4 * nn; la.fy[1] = f + 5 * nn;
    la.betab[0] = 0.0; la.betab[1] = h->c.beffect ? h->c.beta : 0.0;
    la.n = h->n;
    rc = RFFT_DISPATCH(true, false, true, la, (StoreStrided{tmp, nn, 1, n}), 2);
  } else {
    LoadAdvect la{};
    la.uu = h->uu; la.vv = h->vv;
    la.fx[0] = h->w[4]; la.fy[0] = h->w[5];
    la.fx[1] = h->sqs; la.fy[1] = h->sqd;
    la.betab[0] = 0.0; la.betab[1] = h->c.beffect ? h->c.beta : 0.0;
    la.n = h->n;
    la.ms = nn;
    // ensemble: two entries per member; tmp (w[0..1]) is 2M fields long
    rc = RFFT_DISPATCH(true, false, true, la, (StoreStrided{tmp, nn, 1, n}), 2 * h->M);
  }
  if (rc) return rc;
  StoreSource ss{};
  ss.sqd = h->sqd; ss.sqs = h->sqs; ss.qq = h->qq; ss.pp = h->pp; ss.epq = h->epq;
  ss.rekman = h->p.rekman; ss.kdsq = h->c.kdsq; ss.therm = h->c.therm;
  ss.heating = h->c.heating; ss.friction = h->c.friction; ss.lev = lev; ss.n = h->n;
  ss.ms = nn;
  return RFFT_DISPATCH(true, false, false, (LoadRow{tmp, nn, n, (int)n, &h->scal->error}), ss, 2 * h->M);
}

}  // namespace casl

// node update and spectral RK update of a stage, one launch; velint reads
// the velocity fields u, v (FP64, or FP32 in the FP32-inversion mode)
template <class T>
static int stage_update(casl_handle *h, int stage, const T *u, const T *v, const double *du,
                        const double *dv) {
  const long long nn = (long long)h->n * h->n, tot = h->M * nn;
  const int nbn = h->contex ? grid_for(h->nptq > 0 ? h->nptq : 1) : 0;
  const int g = nbn + grid_for(tot / 2);
  const NodeRkArgs<T> a{h->xq, h->yq, h->xqi, h->yqi, h->xqf, h->yqf, u, v,
                        h->M > 1 ? h->mnode : nullptr, h->M, du, dv};
  const SpecRkArgs b{h->qs, h->qd, h->qsi, h->qsf, h->qdi, h->qdf, h->sqs, h->sqd, h->emq,
                     nn, tot};
  cudaStream_t st = h->stream;
  switch (stage) {
    case 1: CASL_K((k_stage_rk<1, T>), g, 256, 0, st)(a, b, h->scal, h->c, nbn); break;
    case 2: CASL_K((k_stage_rk<2, T>), g, 256, 0, st)(a, b, h->scal, h->c, nbn); break;
    case 3: CASL_K((k_stage_rk<3, T>), g, 256, 0, st)(a, b, h->scal, h->c, nbn); break;
    default: CASL_K((k_stage_rk<4, T>), g, 256, 0, st)(a, b, h->scal, h->c, nbn); break;
  }
  return check_launch(h);
}

// advance (evolution.f90:166-326): four RK4 stages, each con2grid + the
// filter combination, the batched inversion + source gradients, (stage 1)
// adapt, source, the node update and the spectral RK update.
static int advance_dev(casl_handle *h) {
  int rc;
  Trace tr;
  tr.begin(h->stream, "advance");
  for (int stage = 1; stage <= 4; stage++) {
    // stage 1: the reset inside the filter combination rewrites qs and qd
    // before the gradients read them
    if ((rc = inversion_qq(h, stage == 1))) return rc;
    tr.point("con2grid+qq");
    const bool f32 = h->prec == CASL_PREC_FP32_INVERSION;
    if ((rc = f32 ? invert_and_gradients32(h) : invert_and_gradients(h))) return rc;
    tr.point("invert");
    if (stage == 1 && (rc = adapt_dev(h))) return rc;
    if ((rc = source_prod(h, stage))) return rc;
    tr.point("adapt+source");
    // the learned closure's correction at the nodes (null without it)
    const double *du = nullptr, *dv = nullptr;
    if (f32) {
      const long long nn = (long long)h->n * h->n;
      const float *u = h->f32, *v = h->f32 + nn;
      if (h->closure && (rc = closure_stage32(h, u, v, &du, &dv))) return rc;
      if ((rc = stage_update<float>(h, stage, u, v, du, dv))) return rc;
    } else {
      if (h->closure && (rc = closure_stage(h, &du, &dv))) return rc;
      if ((rc = stage_update<double>(h, stage, h->uu, h->vv, du, dv))) return rc;
    }
    tr.point("stage update");
    static const char *const names[4] = {"RK4 stage 1", "RK4 stage 2", "RK4 stage 3",
                                         "RK4 stage 4"};
    if ((rc = debug_check(h, names[stage - 1]))) return rc;
  }
  tr.flush("advance");
  return CASL_OK;
}

// ---------------------------------------------------------------------------
// Fine-grid judge of node velocities
// ---------------------------------------------------------------------------
namespace casl {
// Stafft-layout spectral coefficient of wavenumber k along an axis of length
// m: index k (cosine, 0 <= k <= m/2) or m - k (sine, 0 < k < m/2).  The same
// band-limited field transformed on grids of n and nf = r n points has
// coefficients in the ratio sqrt(r) per axis, except that the cosine at the
// coarse Nyquist wavenumber n/2 (a regular mode of the fine grid) is in the
// ratio sqrt(r)/2 (stafft.f90:187-287 normalises forward transforms by
// 1/sqrt(n)).
__device__ __forceinline__ bool pad_axis(int idxf, int nf, int n, int &idx, double &fac) {
  const bool sine = idxf > nf / 2;
  const int k = sine ? nf - idxf : idxf;
  if (k > n / 2 || (sine && k == n / 2)) return false;
  idx = sine ? n - k : k;
  const double s = sqrt((double)nf / (double)n);
  fac = (k == n / 2) ? 0.5 * s : s;
  return true;
}

// qqf = qcf + the spectrum of (qq - qc) on the coarse grid, carried to the
// fine grid (spectral arrays [ky][kx], kx fastest).
__global__ void k_pad_add(const double *__restrict__ qq, const double *__restrict__ qc, int n,
                          const double *__restrict__ qcf, double *__restrict__ qqf, int nf) {
  CASL_PDL_ENTRY();
  const long long nnf = (long long)nf * nf;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nnf;
       t += (long long)gridDim.x * blockDim.x) {
    const int kyf = (int)(t / nf), kxf = (int)(t % nf);
    int ix, iy;
    double fx, fy;
    double v = qcf[t];
    if (pad_axis(kxf, nf, n, ix, fx) && pad_axis(kyf, nf, n, iy, fy)) {
      const long long k = (long long)iy * n + ix;
      v += (qq[k] - qc[k]) * (fx * fy);
    }
    qqf[t] = v;
  }
}

int judge_velocity(casl_handle *h, casl_handle *hf, double *uJ, double *vJ, double *uP,
                   double *vP) {
  const int n = h->n, nf = hf->n;
  if (nf != 2 * n && nf != 4 * n && nf != 8 * n) return CASL_EINVAL;
  if (h->c.ellx != hf->c.ellx || h->c.elly != hf->c.elly) return CASL_EINVAL;
  int rc = sync_counts(h);
  if (rc) return rc;
  const int npt = h->nptq, nq = h->nq;
  if (npt > hf->npm || nq > hf->nm) return CASL_ECAPACITY;
  // the coarse inversion: qq, qc (spectral), uu, vv of h
  if ((rc = inversion_dev(h, false))) return rc;
  if (uP && npt)
    CASL_K(k_velint, grid_for(npt), 256, 0, h->stream)(h->xq, h->yq, npt, h->uu, h->vv, uP, vP,
                                                     h->c);
  // contours to the fine handle (internal 0-based links on both)
  cudaEvent_t ev;
  CASL_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CASL_CUDA_TRY(cudaEventRecord(ev, h->stream));
  CASL_CUDA_TRY(cudaStreamWaitEvent(hf->stream, ev, 0));
  cudaStream_t s = hf->stream;
  if (npt) {
    CASL_CUDA_TRY(cudaMemcpyAsync(hf->xq, h->xq, npt * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(hf->yq, h->yq, npt * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(hf->nextq, h->nextq, npt * sizeof(int), cudaMemcpyDeviceToDevice, s));
  }
  if (nq) {
    int *src[4] = {h->i1q, h->i2q, h->npq, h->indq}, *dst[4] = {hf->i1q, hf->i2q, hf->npq, hf->indq};
    for (int i = 0; i < 4; i++)
      CASL_CUDA_TRY(cudaMemcpyAsync(dst[i], src[i], nq * sizeof(int), cudaMemcpyDeviceToDevice, s));
  }
  if ((rc = get_scalars(hf))) return rc;
  hf->hscal->nq = nq;
  hf->hscal->nptq = npt;
  hf->hscal->qjump = h->qjump;
  hf->hscal->error = 0;
  hf->nq = nq;
  hf->nptq = npt;
  hf->qjump = h->qjump;
  hf->contex = npt > 0;
  if ((rc = put_scalars(hf))) return rc;
  // contour PV on the fine grid (its con2grid and forward transform), then
  // the coarse non-contour spectrum added, then the fine inversion
  const long long nnf = (long long)nf * nf;
  if (npt) {
    if ((rc = con2grid_dev(hf, false))) return rc;
    LoadQC ld{hf->coarseC, hf->scal, hf->c.beffect ? hf->betac : nullptr, nnf,
              1.0 / (256.0 * (double)nf * (double)nf), nf};
    casl_handle *hh = hf;
    {
      casl_handle *h = hh;  // RFFT_DISPATCH launches on h's stream at h's size
      if ((rc = RFFT_DISPATCH(true, false, true, ld, (StoreStrided{h->qc, nnf, 1, (long long)nf}), 1)))
        return rc;
      if ((rc = RFFT_DISPATCH(true, false, false, (LoadRow{h->qc, nnf, (long long)nf, nf, &h->scal->error}),
                              (StoreStrided{h->qc, nnf, (long long)nf, 1}), 1)))
        return rc;
    }
  } else {
    CASL_CUDA_TRY(cudaMemsetAsync(hf->qc, 0, nnf * sizeof(double), s));
  }
  CASL_CUDA_TRY(cudaEventRecord(ev, h->stream));
  CASL_CUDA_TRY(cudaStreamWaitEvent(s, ev, 0));
  CASL_K(k_pad_add, grid_for(nnf), 256, 0, s)(h->qq, h->qc, n, hf->qc, hf->qq, nf);
  if ((rc = main_invert_dev(hf))) return rc;
  if (npt)
    CASL_K(k_velint, grid_for(npt), 256, 0, s)(hf->xq, hf->yq, npt, hf->uu, hf->vv, uJ, vJ,
                                             hf->c);
  CASL_CUDA_TRY(cudaEventRecord(ev, s));
  CASL_CUDA_TRY(cudaStreamWaitEvent(h->stream, ev, 0));
  CASL_CUDA_TRY(cudaEventDestroy(ev));
  return check_launch(hf);
}
}  // namespace casl

// ---------------------------------------------------------------------------
// Host-side set-up: constants.f90, spectral.f90:42-158 (same operations and
// order as the reference; computed once and uploaded)
// ---------------------------------------------------------------------------
static double pow_cr(double x, int k) {
#ifdef __SIZEOF_FLOAT128__
  __float128 r = 1, b = x;
  for (int i = 0; i < k; i++) r *= b;
  return (double)r;
#else
  long double r = 1;
  for (int i = 0; i < k; i++) r *= x;
  return (double)r;
#endif
}

static void make_consts(const casl_params &p, Consts &c) {
  memset(&c, 0, sizeof(c));
  c.nx = p.nx; c.ny = p.ny;
  c.nxf = 4 * p.nx; c.nyf = 4 * p.ny;
  c.nxu = 16 * p.nx; c.nyu = 16 * p.ny;
  c.nwx = p.nx / 2; c.nwy = p.ny / 2;
  c.ellx = p.ellx; c.elly = p.elly;
  c.pi = 3.141592653589793238462643383279502884197169399375105820974944592307816;
  c.twopi = 2.0 * c.pi;
  c.small = 1.0e-12;
  c.small3 = c.small * c.small * c.small;
  c.oms = 1.0 - c.small;
  c.hlx = 0.5 * p.ellx; c.hlxi = 1.0 / c.hlx; c.xmin = -c.hlx; c.xmax = c.hlx;
  c.hly = 0.5 * p.elly; c.hlyi = 1.0 / c.hly; c.ymin = -c.hly; c.ymax = c.hly;
  c.kdsq = pow_cr(p.kd, 2);
  c.srwfm = p.beta * p.kd / (1.0 + c.kdsq);
  c.therm = p.rtherm * c.kdsq;
  c.rekman = p.rekman;
  c.beta = p.beta;
  c.aspect = p.ellx / p.elly;
  c.glx = p.ellx / (double)p.nx; c.glxi = (double)p.nx / p.ellx;
  c.gly = p.elly / (double)p.ny; c.glyi = (double)p.ny / p.elly;
  c.garea = c.glx * c.gly;
  c.dsumi = 1.0 / (double)(p.nx * p.ny);
  c.glxf = p.ellx / (double)c.nxf; c.glxfi = (double)c.nxf / p.ellx;
  c.glyf = p.elly / (double)c.nyf; c.glyfi = (double)c.nyf / p.elly;
  c.glxu = p.ellx / (double)c.nxu; c.glxui = (double)c.nxu / p.ellx;
  c.glyu = p.elly / (double)c.nyu; c.glyui = (double)c.nyu / p.elly;
  c.amu = 0.2;
  c.ell = 6.25 * c.glx;
  c.dm = pow_cr(c.amu, 2) * c.ell / 4.0;
  c.dm2 = pow_cr(c.dm, 2);
  c.d4small = c.small * pow_cr(c.glx, 4);
  c.dmsq = 4.0 * c.dm2;
  c.dmi = 2.0 / c.dm;
  c.elf = 1.0 / pow_cr(c.ell, 2);
  c.densf = 1.0 / (c.amu * sqrt(c.ell));
  c.beffect = p.beta != 0.0;
  c.btropic = p.kd == 0.0;
  c.heating = p.rtherm > 0.0;
  c.friction = p.rekman > 0.0;
}

struct HostTables {
  std::vector<double> green, flo, fhi, qdiss, hrkx, hrky, bety, betac, rkxf, rkyf, spmf, alk;
  std::vector<double2> tw;
  std::vector<int> shell_off, shell_idx;
  int kmax = 0, kmaxred = 0;
};

static void make_tables(const casl_params &p, const Consts &c, HostTables &t) {
  int nx = p.nx, ny = p.ny, nwx = nx / 2, nwy = ny / 2;
  size_t nn = (size_t)nx * ny;
  std::vector<double> rkx(nx), rky(ny), rkxf(nx), rkyf(ny);
  t.hrkx.resize(nx); t.hrky.resize(ny);
  double sc = c.pi / p.ellx;
  for (int k = 1; k <= nx; k++) t.hrkx[k - 1] = sc * (double)k;
  sc = c.pi / p.elly;
  for (int k = 1; k <= ny; k++) t.hrky[k - 1] = sc * (double)k;
  rkx[0] = 0.0;
  for (int kx = 1; kx <= nwx - 1; kx++) {
    rkx[kx] = t.hrkx[2 * kx - 1];
    rkx[nx - kx] = t.hrkx[2 * kx - 1];
  }
  rkx[nwx] = t.hrkx[nx - 1];
  double rkxmax = (c.twopi / p.ellx) * (double)nwx;
  for (int kx = 0; kx < nx; kx++) {
    rkxf[kx] = rkx[kx] * exp(-36.0 * pow(rkx[kx] / rkxmax, 36.0));
    t.hrkx[kx] = t.hrkx[kx] * exp(-36.0 * pow(t.hrkx[kx] / rkxmax, 36.0));
  }
  rky[0] = 0.0;
  for (int ky = 1; ky <= nwy - 1; ky++) {
    rky[ky] = t.hrky[2 * ky - 1];
    rky[ny - ky] = t.hrky[2 * ky - 1];
  }
  rky[nwy] = t.hrky[ny - 1];
  double rkymax = (c.twopi / p.elly) * (double)nwy;
  for (int ky = 0; ky < ny; ky++) {
    rkyf[ky] = rky[ky] * exp(-36.0 * pow(rky[ky] / rkymax, 36.0));
    t.hrky[ky] = t.hrky[ky] * exp(-36.0 * pow(t.hrky[ky] / rkymax, 36.0));
  }
  double fac = 36.0 / (double)(nx * ny);
  double a2 = rkxmax * rkxmax, b2 = rkymax * rkymax;
  double rkmsi = 1.0 / (a2 > b2 ? a2 : b2);
  t.green.assign(nn, 0.0); t.flo.assign(nn, 0.0); t.fhi.assign(nn, 0.0); t.qdiss.assign(nn, 0.0);
  for (int ky = 1; ky <= ny; ky++)
    for (int kx = 1; kx <= nx; kx++) {
      double rksqu = rkx[kx - 1] * rkx[kx - 1] + rky[ky - 1] * rky[ky - 1];
      size_t k = (size_t)(ky - 1) * nx + (kx - 1);
      t.qdiss[k] = p.cdamp * pow(rkmsi * rksqu, p.nnu);
      double f = fac * rksqu;
      t.flo[k] = 1.0 / (1.0 + f * f);
      t.fhi[k] = 1.0 - t.flo[k];
    }
  t.green[0] = 0.0;
  for (int kx = 2; kx <= nx; kx++) t.green[kx - 1] = -1.0 / (rkx[kx - 1] * rkx[kx - 1] + c.kdsq);
  for (int ky = 2; ky <= ny; ky++)
    t.green[(size_t)(ky - 1) * nx] = -1.0 / (rky[ky - 1] * rky[ky - 1] + c.kdsq);
  for (int ky = 2; ky <= ny; ky++)
    for (int kx = 2; kx <= nx; kx++)
      t.green[(size_t)(ky - 1) * nx + (kx - 1)] =
          -1.0 / (rkx[kx - 1] * rkx[kx - 1] + rky[ky - 1] * rky[ky - 1] + c.kdsq);
  t.bety.resize(ny);
  for (int iy = 1; iy <= ny; iy++) t.bety[iy - 1] = p.beta * (c.gly * (double)(iy - 1) + c.ymin);
  // con2grid's beta term: the fine-grid -beta*y coarsened by the 7x7 stencil
  // (rows only; columns sum to 16) with its mean removed.
  t.betac.assign(ny, 0.0);
  if (p.beta != 0.0) {
    int nf = c.nyf;
    const int w7[7] = {1, 2, 3, 4, 3, 2, 1};
    double mean = 0.0;
    for (int iy = 1; iy <= ny; iy++) {
      double acc = 0.0;
      for (int a = 0; a < 7; a++) {
        int fy = 4 * iy - 6 + a;
        if (fy <= 0) fy += nf;
        double ygf = c.ymin + c.glyf * (double)(fy - 1);
        acc += w7[a] * (-p.beta * ygf);
      }
      t.betac[iy - 1] = acc / 16.0;
      mean += t.betac[iy - 1];
    }
    mean /= (double)ny;
    for (int iy = 0; iy < ny; iy++) t.betac[iy] -= mean;
  }
  // 1-D spectrum tables (spectral.f90:109-134): shell of every mode, shell
  // population factor spmf, log10 wavenumber alk, the indices of each shell
  {
    double scx = c.twopi / p.ellx, scy = c.twopi / p.elly;
    double delk = sqrt(scx * scx + scy * scy), delki = 1.0 / delk;
    t.kmax = (int)lround(sqrt(rkxmax * rkxmax + rkymax * rkymax) * delki);
    int mx = nx > ny ? nx : ny;
    t.spmf.assign(mx + 1, 0.0);
    t.alk.assign(mx + 1, 0.0);
    std::vector<int> kmag(nn);
    std::vector<int> cnt(t.kmax + 2, 0);
    for (int ky = 0; ky < ny; ky++)
      for (int kx = 0; kx < nx; kx++) {
        int k = (int)lround(sqrt(rkx[kx] * rkx[kx] + rky[ky] * rky[ky]) * delki);
        kmag[(size_t)ky * nx + kx] = k;
        t.spmf[k] = t.spmf[k] + 1.0;
        cnt[k + 1]++;
      }
    double snorm = 4.0 * c.pi / (double)(nx * ny);
    t.spmf[0] = 0.0;
    for (int k = 1; k <= t.kmax; k++) {
      t.spmf[k] = snorm * (double)k / t.spmf[k];
      t.alk[k] = log10(delk * (double)k);
    }
    t.kmaxred = (int)lround(sqrt((rkxmax * rkxmax + rkymax * rkymax) / 2.0) * delki);
    t.shell_off.assign(t.kmax + 2, 0);
    for (int k = 0; k <= t.kmax; k++) t.shell_off[k + 1] = t.shell_off[k] + cnt[k + 1];
    t.shell_idx.resize(nn);
    std::vector<int> pos(t.shell_off.begin(), t.shell_off.end() - 1);
    for (size_t i = 0; i < nn; i++) t.shell_idx[pos[kmag[i]]++] = (int)i;
    t.rkxf = rkxf;
    t.rkyf = rkyf;
  }
  t.tw.resize(nx);
  for (int k = 0; k < nx; k++) {
    double a = c.twopi * (double)k / (double)nx;
    t.tw[k] = make_double2(cos(a), -sin(a));
  }
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace casl {
int sync_counts(casl_handle *h) {
  CASL_CUDA_TRY(cudaMemcpyAsync(h->hscal, h->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->nq = h->hscal->nq;
  h->nptq = h->hscal->nptq;
  h->contex = h->nptq > 0;
  if (h->hscal->error) {
    int e = h->hscal->error;
    return e;
  }
  return CASL_OK;
}

// Opt-in state check (environment variable CASL_CHECK=1), run by casl_step
// after recontouring, after surgery and after each RK4 stage: the first node
// that is not finite, lies outside the domain or links outside the node
// arrays is printed with the phase that left it, and the step returns
// CASL_EDOMAIN there instead of carrying the bad node on.
__global__ void k_first_bad(const double *__restrict__ xq, const double *__restrict__ yq,
                            const int *__restrict__ nextq, int npt, Consts c, int *first) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npt;
       i += (long long)gridDim.x * blockDim.x) {
    const double x = xq[i], y = yq[i];
    const int nx = nextq[i];
    if (!(x >= c.xmin && x < c.xmax && y >= c.ymin && y < c.ymax) || nx < 0 || nx >= npt)
      atomicMin(first, (int)i);
  }
}

int debug_check(casl_handle *h, const char *phase) {
  static int enabled = -1;
  if (enabled < 0) {
    const char *e = getenv("CASL_CHECK");
    enabled = e && e[0] == '1';
  }
  if (!enabled) return CASL_OK;
  int rc = sync_counts(h);
  if (rc) {
    fprintf(stderr, "[casl check] %s: error %d\n", phase, rc);
    return rc;
  }
  const int npt = h->nptq;
  if (npt == 0) return CASL_OK;
  int *d = nullptr, first = INT_MAX;
  CASL_CUDA_TRY(cudaMalloc(&d, sizeof(int)));
  CASL_CUDA_TRY(cudaMemcpyAsync(d, &first, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  k_first_bad<<<148 * 8, 256, 0, h->stream>>>(h->xq, h->yq, h->nextq, npt, h->c, d);
  CASL_CUDA_TRY(cudaMemcpyAsync(&first, d, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  cudaFree(d);
  if (first == INT_MAX) return CASL_OK;
  double x = 0, y = 0;
  int nx = -1;
  cudaMemcpy(&x, h->xq + first, sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(&y, h->yq + first, sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(&nx, h->nextq + first, sizeof(int), cudaMemcpyDeviceToHost);
  fprintf(stderr, "[casl check] %s: node %d of %d at (%.17g, %.17g), next %d\n", phase, first,
          npt, x, y, nx);
  return CASL_EDOMAIN;
}

// Scratch arenas grow with 50% headroom: their sizes follow node and
// crossing counts, which drift from step to step, and re-allocating several
// GB costs far more than the spare memory.
int ensure_scratch(casl_handle *h, size_t bytes) {
  if (h->sx_bytes >= bytes) return CASL_OK;
  if (h->sx) cudaFree(h->sx);
  h->sx = nullptr;
  h->sx_bytes = 0;
  bytes += bytes / 2;
  CASL_CUDA_TRY(cudaMalloc(&h->sx, bytes));
  h->sx_bytes = bytes;
  return CASL_OK;
}

static double wall_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

void Trace::begin(cudaStream_t s, const char *what) {
  static int enabled = -1;
  if (enabled < 0) {
    const char *e = getenv("CASL_TRACE");
    enabled = e ? (e[0] == '1' ? 1 : e[0] == '2' ? 2 : 0) : 0;
  }
  on = enabled >= 1;
  eager = enabled == 2;
  n = 0;
  st = s;
  t_last = wall_ms();
  if (on) point(what);
}

void Trace::point(const char *what) {
  if (!on) return;
  if (eager) {
    cudaError_t e = cudaStreamSynchronize(st);
    const double t = wall_ms();
    fprintf(stderr, "[casl trace] at %s +%.3f ms%s\n", what, t - t_last,
            e == cudaSuccess ? "" : " (stream error)");
    fflush(stderr);
    t_last = t;
    return;
  }
  if (n >= 64) return;
  cudaEventCreate(&ev[n]);
  cudaEventRecord(ev[n], st);
  name[n++] = what;
}

void Trace::flush(const char *title) {
  if (!on || eager) return;
  cudaStreamSynchronize(st);
  fprintf(stderr, "[casl trace] %s:", title);
  for (int i = 1; i < n; i++) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev[i - 1], ev[i]);
    fprintf(stderr, " %s %.3f", name[i], ms);
  }
  float tot = 0.f;
  if (n > 1) cudaEventElapsedTime(&tot, ev[0], ev[n - 1]);
  fprintf(stderr, " | total %.3f ms\n", tot);
  for (int i = 0; i < n; i++) cudaEventDestroy(ev[i]);
  n = 0;
}

int ensure_scratch2(casl_handle *h, size_t bytes) {
  if (h->sx2_bytes >= bytes) return CASL_OK;
  if (h->sx2) cudaFree(h->sx2);
  h->sx2 = nullptr;
  h->sx2_bytes = 0;
  bytes += bytes / 2;
  CASL_CUDA_TRY(cudaMalloc(&h->sx2, bytes));
  h->sx2_bytes = bytes;
  return CASL_OK;
}
}  // namespace casl

// ---------------------------------------------------------------------------
// Diagnostics kernels (deterministic two-level sums)
// ---------------------------------------------------------------------------
__global__ void k_diag_sumsq2(const double *__restrict__ a, const double *__restrict__ b,
                              double *__restrict__ part, long long nn) {
  CASL_PDL_ENTRY();
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x) {
    double v = a[k] * a[k];
    if (b) v = v + b[k] * b[k];
    s += v;
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}
__global__ void k_diag_final(const double *__restrict__ part, int np, double *__restrict__ out) {
  CASL_PDL_ENTRY();
  __shared__ double sh[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += part[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}
__global__ void k_diag_incr(const double *__restrict__ xq, const double *__restrict__ yq,
                            const int *__restrict__ nextq, int npt, double *__restrict__ dx,
                            double *__restrict__ dy, int *__restrict__ head, Consts c) {
  CASL_PDL_ENTRY();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    int a = nextq[i];
    double xx = xq[a] - xq[i];
    dx[i] = xx - c.ellx * f_dint(xx * c.hlxi);
    double yy = yq[a] - yq[i];
    dy[i] = yy - c.elly * f_dint(yy * c.hlyi);
    head[i] = 0;
  }
}
__global__ void k_diag_heads(const int *__restrict__ i1q, int nq, int *__restrict__ head) {
  CASL_PDL_ENTRY();
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += gridDim.x * blockDim.x)
    head[i1q[j]] = 1;
}
// term_i = X_i dy_i - Y_i dx_i with (X_i, Y_i) the exclusive prefix of the
// increments from the contour's first node
// spec1d (spectral.f90:370-424): one warp per shell sums w*ss^2 over the
// shell's modes (lane-strided, then a fixed shuffle tree: deterministic);
// w = 1/4 for the mean, 1/2 for the kx = 0 and ky = 0 modes.
__global__ void k_spec1d(const double *__restrict__ ss, const int *__restrict__ off,
                         const int *__restrict__ idx, int nx, int kmax, double *__restrict__ spec) {
  CASL_PDL_ENTRY();
  const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (k > kmax) return;
  double acc = 0.0;
  for (int i = off[k] + lane; i < off[k + 1]; i += 32) {
    int m = idx[i], kx = m % nx, ky = m / nx;
    double v = ss[m];
    double w = (kx == 0 && ky == 0) ? 0.25 : ((kx == 0 || ky == 0) ? 0.5 : 1.0);
    acc += w * (v * v);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) spec[k] = acc;
}

// ss <- ss * (rkxf^2 + rkyf^2), the filtered K^2 of spec1d's iopt = 1
__global__ void k_mul_rksq(double *__restrict__ ss, const double *__restrict__ rkxf,
                           const double *__restrict__ rkyf, int nx, long long nn) {
  CASL_PDL_ENTRY();
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < nn;
       m += (long long)gridDim.x * blockDim.x) {
    int kx = (int)(m % nx), ky = (int)(m / nx);
    ss[m] = ss[m] * (rkxf[kx] * rkxf[kx] + rkyf[ky] * rkyf[ky]);
  }
}

__global__ void k_diag_shoelace(const double *__restrict__ dx, const double *__restrict__ dy,
                                const double *__restrict__ X, const double *__restrict__ Y,
                                int npt, double *__restrict__ part) {
  CASL_PDL_ENTRY();
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += gridDim.x * blockDim.x) {
    double xe = X[i] - dx[i], ye = Y[i] - dy[i];
    s += xe * dy[i] - ye * dx[i];
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}


extern "C" {

const char *casl_error_string(int code) {
  switch (code) {
    case CASL_OK: return "ok";
    case CASL_EINVAL: return "invalid argument";
    case CASL_ECAPACITY: return "capacity exceeded";
    case CASL_ECUDA: return "CUDA error";
    case CASL_ENOMEM: return "device out of memory";
    case CASL_EDOMAIN: return "node outside the domain or non-finite";
    case CASL_ETIMEOUT: return "bounded device wait timed out";
    case CASL_EUNSUPPORTED: return "unsupported";
    case CASL_EIO: return "file input/output error";
  }
  return "unknown error";
}

int casl_last_cuda_error(casl_handle *h) { return h ? h->last_cuda : 0; }

static int alloc_all(casl_handle *h) {
  long long n = h->n, nn = n * n;
  long long npm = h->npm, nm = h->nm;
  const long long M = h->M;
  double **nodes[] = {&h->xq, &h->yq, &h->xqi, &h->yqi, &h->xqf, &h->yqf, &h->uq, &h->vq};
  for (auto pp : nodes) CASL_CUDA_TRY(cudaMalloc(pp, (size_t)npm * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->nextq, (size_t)npm * sizeof(int)));
  int **cont[] = {&h->i1q, &h->i2q, &h->npq, &h->indq};
  for (auto pp : cont) CASL_CUDA_TRY(cudaMalloc(pp, (size_t)nm * sizeof(int)));
  // per-member fields (M stacked), then the shared tables
  double **fields[] = {&h->qr, &h->qs, &h->qd, &h->qc, &h->qq, &h->pp, &h->uu, &h->vv, &h->emq,
                       &h->epq, &h->qspre, &h->sqs, &h->sqd, &h->qsi, &h->qsf, &h->qdi, &h->qdf};
  for (auto pp : fields) {
    CASL_CUDA_TRY(cudaMalloc(pp, (size_t)(M * nn) * sizeof(double)));
    CASL_CUDA_TRY(cudaMemset(*pp, 0, (size_t)(M * nn) * sizeof(double)));
  }
  double **tables[] = {&h->green, &h->flo, &h->fhi, &h->qdiss};
  for (auto pp : tables) {
    CASL_CUDA_TRY(cudaMalloc(pp, (size_t)nn * sizeof(double)));
    CASL_CUDA_TRY(cudaMemset(*pp, 0, (size_t)nn * sizeof(double)));
  }
  // work fields: w[0..3] contiguous (batched transforms), w[4], w[5]; each
  // M fields wide
  double *wk;
  CASL_CUDA_TRY(cudaMalloc(&wk, (size_t)(6 * M * nn) * sizeof(double)));
  for (int i = 0; i < 6; i++) h->w[i] = wk + i * M * nn;
  CASL_CUDA_TRY(cudaMalloc(&h->hrkx, n * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->hrky, n * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->bety, n * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->betac, n * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->tw, n * sizeof(double2)));
  CASL_CUDA_TRY(cudaMalloc(&h->gtmp, (size_t)(6 * M * nn) * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->shell_idx, (size_t)nn * sizeof(int)));
  CASL_CUDA_TRY(cudaMalloc(&h->shell_off, (size_t)(2 * n + 2) * sizeof(int)));
  CASL_CUDA_TRY(cudaMalloc(&h->rkxf, n * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->rkyf, n * sizeof(double)));
  // one simulation: the dense (4n)^2 levels grid (the packed words use its
  // first half); an ensemble: the packed words of every member (4n x n
  // 64-bit words = 8 n^2 ints each)
  size_t fine = M == 1 ? (size_t)h->c.nxf * h->c.nyf : (size_t)(M * 8 * nn);
  CASL_CUDA_TRY(cudaMalloc(&h->fineJ, fine * sizeof(int)));
  CASL_CUDA_TRY(cudaMalloc(&h->ljx, (size_t)(M * h->c.nxf) * sizeof(int)));
  CASL_CUDA_TRY(cudaMalloc(&h->coarseC, (size_t)(M * nn) * sizeof(int)));
  CASL_CUDA_TRY(cudaMalloc(&h->part, (size_t)(3 * RED_BLOCKS * M) * sizeof(double)));
  CASL_CUDA_TRY(cudaMalloc(&h->scal, (size_t)M * sizeof(Scalars)));
  CASL_CUDA_TRY(cudaMemset(h->scal, 0, (size_t)M * sizeof(Scalars)));
  CASL_CUDA_TRY(cudaMallocHost(&h->hscal, (size_t)M * sizeof(Scalars)));
  memset(h->hscal, 0, (size_t)M * sizeof(Scalars));
  CASL_CUDA_TRY(cudaMalloc(&h->mnode, (size_t)(M + 1) * sizeof(int)));
  CASL_CUDA_TRY(cudaMalloc(&h->mcont, (size_t)(M + 1) * sizeof(int)));
  CASL_CUDA_TRY(cudaMemset(h->mnode, 0, (size_t)(M + 1) * sizeof(int)));
  CASL_CUDA_TRY(cudaMemset(h->mcont, 0, (size_t)(M + 1) * sizeof(int)));
  CASL_CUDA_TRY(cudaMallocHost(&h->hmnode, (size_t)(M + 1) * sizeof(int)));
  CASL_CUDA_TRY(cudaMallocHost(&h->hmcont, (size_t)(M + 1) * sizeof(int)));
  memset(h->hmnode, 0, (size_t)(M + 1) * sizeof(int));
  memset(h->hmcont, 0, (size_t)(M + 1) * sizeof(int));
  h->mqjump = (double *)calloc((size_t)M, sizeof(double));
  if (!h->mqjump) return CASL_ENOMEM;
  return CASL_OK;
}

static void free_all(casl_handle *h) {
  void *ptrs[] = {h->xq, h->yq, h->xqi, h->yqi, h->xqf, h->yqf, h->uq, h->vq, h->nextq, h->i1q,
                  h->i2q, h->npq, h->indq, h->qr, h->qs, h->qd, h->qc, h->qq, h->pp, h->uu,
                  h->vv, h->emq, h->epq, h->qspre, h->sqs, h->sqd, h->qsi, h->qsf, h->qdi,
                  h->qdf, h->green, h->flo, h->fhi, h->qdiss, h->w[0], h->hrkx, h->hrky,
                  h->bety, h->betac, h->tw, h->fineJ, h->ljx, h->coarseC, h->part, h->scal,
                  h->sx, h->sx2, h->sxe, h->shell_idx, h->shell_off, h->rkxf, h->rkyf, h->gtmp};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (h->mnode) cudaFree(h->mnode);
  if (h->mcont) cudaFree(h->mcont);
  if (h->hmnode) cudaFreeHost(h->hmnode);
  if (h->hmcont) cudaFreeHost(h->hmcont);
  free(h->mqjump);
  free(h->spmf_h);
  free(h->alk_h);
  if (h->hscal) cudaFreeHost(h->hscal);
}

int casl_create(const casl_params *p, int device, casl_handle **out) {
  return casl::create_handle_members(p, device, 1, out);
}

}  // extern "C"

// A handle of M ensemble members (M = 1: one simulation).
int casl::create_handle_members(const casl_params *p, int device, int M, casl_handle **out) {
  if (!p || !out || M < 1) return CASL_EINVAL;
  *out = nullptr;
  int n = p->nx;
  if (p->nx != p->ny || n < 32 || n > 2048 || (n & (n - 1)) || p->ellx <= 0 || p->elly <= 0 ||
      p->ncontq <= 0)
    return CASL_EINVAL;
  casl_handle *h = (casl_handle *)calloc(1, sizeof(casl_handle));
  if (!h) return CASL_ENOMEM;
  h->p = *p;
  if (h->p.nlevm <= 0) h->p.nlevm = 2000;
  if (h->p.npm <= 0) h->p.npm = 500LL * n * n;
  if (h->p.nm <= 0) h->p.nm = h->p.npm / 20 + h->p.npm / 200;
  if (h->p.nregmax <= 0) h->p.nregmax = 20;
  if (h->p.twistmax <= 0) h->p.twistmax = 2.5;
  h->n = n;
  h->M = M;
  h->npm = h->p.npm;
  h->nm = h->p.nm;
  h->device = device;
  make_consts(h->p, h->c);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    free(h);
    return CASL_ECUDA;
  }
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    free(h);
    return CASL_ECUDA;
  }
  int rc = alloc_all(h);
  if (rc) {
    free_all(h);
    cudaStreamDestroy(h->stream);
    free(h);
    return rc;
  }
  HostTables t;
  make_tables(h->p, h->c, t);
  size_t nn = (size_t)n * n;
  cudaMemcpy(h->green, t.green.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->flo, t.flo.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->fhi, t.fhi.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->qdiss, t.qdiss.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->hrkx, t.hrkx.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->hrky, t.hrky.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->bety, t.bety.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->betac, t.betac.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->shell_idx, t.shell_idx.data(), nn * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(h->shell_off, t.shell_off.data(), t.shell_off.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(h->rkxf, t.rkxf.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(h->rkyf, t.rkyf.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  h->kmax = t.kmax;
  h->kmaxred = t.kmaxred;
  h->spmf_h = (double *)malloc((n + 1) * sizeof(double));
  h->alk_h = (double *)malloc((n + 1) * sizeof(double));
  if (h->spmf_h && h->alk_h) {
    memcpy(h->spmf_h, t.spmf.data(), (n + 1) * sizeof(double));
    memcpy(h->alk_h, t.alk.data(), (n + 1) * sizeof(double));
  }
  e = cudaMemcpy(h->tw, t.tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
  if (e != cudaSuccess || !h->spmf_h || !h->alk_h) {
    free_all(h);
    cudaStreamDestroy(h->stream);
    free(h);
    return CASL_ECUDA;
  }
  for (int m = 0; m < M; m++) h->hscal[m].dtmax = h->p.dtmax > 0 ? h->p.dtmax : 1.0e30;
  cudaMemcpy(h->scal, h->hscal, (size_t)M * sizeof(Scalars), cudaMemcpyHostToDevice);
  *out = h;
  return CASL_OK;
}

extern "C" {

void casl_destroy(casl_handle *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  io_release(h);
  cudaStreamSynchronize(h->stream);
  closure_release(h);
  forcing_release(h);
  ensemble_release(h);
  cudaFree(h->f32);
  free_all(h);
  if (h->prof_ev) {
    for (int i = 0; i < 2 * CASL_PROF_MAX; i++) cudaEventDestroy(h->prof_ev[i]);
    free(h->prof_ev);
  }
  cudaStreamDestroy(h->stream);
  free(h);
}

int casl_synchronize(casl_handle *h) {
  if (!h) return CASL_EINVAL;
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CASL_OK;
}

}  // extern "C"

namespace casl {
int put_scalars(casl_handle *h) {
  CASL_CUDA_TRY(cudaMemcpyAsync(h->scal, h->hscal, sizeof(Scalars), cudaMemcpyHostToDevice, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CASL_OK;
}
}  // namespace casl

extern "C" {
}  // extern "C"

namespace casl {
int get_scalars(casl_handle *h) {
  CASL_CUDA_TRY(cudaMemcpyAsync(h->hscal, h->scal, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CASL_OK;
}
}  // namespace casl

extern "C" {

__global__ void k_to0(int *a, long long m, int off) {
  CASL_PDL_ENTRY();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x)
    a[i] += off;
}

// The checks casl_set_contours makes on the uploaded state, reported through
// the sticky error word: every node finite and inside the domain
// [xmin,xmax) x [ymin,ymax) that con2grid and the box searches index with
// (CASL_EDOMAIN); every successor, and every contour's node range, inside the
// node arrays (CASL_EINVAL).  Links are 0-based here.
__global__ void k_validate(const double *__restrict__ xq, const double *__restrict__ yq,
                           const int *__restrict__ nextq, int npt, const int *__restrict__ i1q,
                           const int *__restrict__ i2q, const int *__restrict__ npq, int nq,
                           Consts c, Scalars *__restrict__ s) {
  CASL_PDL_ENTRY();
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < npt; i += stride) {
    double x = xq[i], y = yq[i];
    if (!(x >= c.xmin && x < c.xmax && y >= c.ymin && y < c.ymax)) atomicExch(&s->error, CASL_EDOMAIN);
    int nx = nextq[i];
    if (nx < 0 || nx >= npt) atomicExch(&s->error, CASL_EINVAL);
  }
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nq; j += stride) {
    int a = i1q[j], b = i2q[j];
    if (a < 0 || b >= npt || b < a || npq[j] != b - a + 1) atomicExch(&s->error, CASL_EINVAL);
  }
}

int casl_set_contours(casl_handle *h, int nq, int nptq, double qjump, const double *xq,
                      const double *yq, const int *nextq, const int *indq, const int *npq,
                      const int *i1q, const int *i2q) {
  if (!h || nq < 0 || nptq < 0) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // ensembles: casl_ensemble_initialise
  if (nptq > h->npm || nq > h->nm) return CASL_ECAPACITY;
  if (nptq > 0 && (!xq || !yq || !nextq)) return CASL_EINVAL;
  if (nq > 0 && (!indq || !npq || !i1q || !i2q)) return CASL_EINVAL;
  cudaStream_t s = h->stream;
  if (nptq) {
    CASL_CUDA_TRY(cudaMemcpyAsync(h->xq, xq, nptq * sizeof(double), cudaMemcpyHostToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(h->yq, yq, nptq * sizeof(double), cudaMemcpyHostToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(h->nextq, nextq, nptq * sizeof(int), cudaMemcpyHostToDevice, s));
    CASL_K(k_to0, grid_for(nptq), 256, 0, s)(h->nextq, nptq, -1);
  }
  if (nq) {
    CASL_CUDA_TRY(cudaMemcpyAsync(h->indq, indq, nq * sizeof(int), cudaMemcpyHostToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(h->npq, npq, nq * sizeof(int), cudaMemcpyHostToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(h->i1q, i1q, nq * sizeof(int), cudaMemcpyHostToDevice, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(h->i2q, i2q, nq * sizeof(int), cudaMemcpyHostToDevice, s));
    CASL_K(k_to0, grid_for(nq), 256, 0, s)(h->i1q, nq, -1);
    CASL_K(k_to0, grid_for(nq), 256, 0, s)(h->i2q, nq, -1);
  }
  // a new state replaces the old one, and with it any error the old one left
  const FillJob z[1] = {{&h->scal->error, 1, 0u}};
  if (int rc = fill_words(s, z, 1)) return rc;
  if (nptq || nq)
    CASL_K(k_validate, grid_for(nptq > nq ? nptq : nq), 256, 0, s)(
        h->xq, h->yq, h->nextq, nptq, h->i1q, h->i2q, h->npq, nq, h->c, h->scal);
  int rc = get_scalars(h);
  if (rc) return rc;
  if (int bad = h->hscal->error) {
    // rejected: leave an empty state rather than one that would fault later
    h->hscal->error = 0;
    h->hscal->nq = h->hscal->nptq = 0;
    h->nq = h->nptq = 0;
    h->contex = 0;
    if ((rc = put_scalars(h))) return rc;
    return bad;
  }
  h->hscal->nq = nq;
  h->hscal->nptq = nptq;
  h->hscal->qjump = qjump;
  h->nq = nq;
  h->nptq = nptq;
  h->qjump = qjump;
  h->contex = nptq > 0;
  return put_scalars(h);
}

int casl_get_counts(casl_handle *h, int *nq, int *nptq, double *qjump) {
  if (!h) return CASL_EINVAL;
  int rc = get_scalars(h);
  if (rc) return rc;
  if (nq) *nq = h->hscal->nq;
  if (nptq) *nptq = h->hscal->nptq;
  if (qjump) *qjump = h->hscal->qjump;
  return CASL_OK;
}

int casl_get_contours(casl_handle *h, double *xq, double *yq, int *nextq, int *indq, int *npq,
                      int *i1q, int *i2q) {
  if (!h) return CASL_EINVAL;
  int rc = sync_counts(h);
  if (rc) return rc;
  cudaStream_t s = h->stream;
  int npt = h->nptq, nq = h->nq;
  if (npt) {
    CASL_K(k_to0, grid_for(npt), 256, 0, s)(h->nextq, npt, 1);
    if (xq) CASL_CUDA_TRY(cudaMemcpyAsync(xq, h->xq, npt * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (yq) CASL_CUDA_TRY(cudaMemcpyAsync(yq, h->yq, npt * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (nextq) CASL_CUDA_TRY(cudaMemcpyAsync(nextq, h->nextq, npt * sizeof(int), cudaMemcpyDeviceToHost, s));
    CASL_K(k_to0, grid_for(npt), 256, 0, s)(h->nextq, npt, -1);
  }
  if (nq) {
    CASL_K(k_to0, grid_for(nq), 256, 0, s)(h->i1q, nq, 1);
    CASL_K(k_to0, grid_for(nq), 256, 0, s)(h->i2q, nq, 1);
    if (indq) CASL_CUDA_TRY(cudaMemcpyAsync(indq, h->indq, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (npq) CASL_CUDA_TRY(cudaMemcpyAsync(npq, h->npq, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (i1q) CASL_CUDA_TRY(cudaMemcpyAsync(i1q, h->i1q, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (i2q) CASL_CUDA_TRY(cudaMemcpyAsync(i2q, h->i2q, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    CASL_K(k_to0, grid_for(nq), 256, 0, s)(h->i1q, nq, -1);
    CASL_K(k_to0, grid_for(nq), 256, 0, s)(h->i2q, nq, -1);
  }
  CASL_CUDA_TRY(cudaStreamSynchronize(s));
  return check_launch(h);
}

static double *field_ptr(casl_handle *h, int which) {
  switch (which) {
    case CASL_QS: return h->qs;
    case CASL_QD: return h->qd;
    case CASL_QC: return h->qc;
    case CASL_QQ: return h->qq;
    case CASL_PP: return h->pp;
    case CASL_QSPRE: return h->qspre;
    case CASL_EMQ: return h->emq;
    case CASL_EPQ: return h->epq;
    case CASL_UU: return h->uu;
    case CASL_VV: return h->vv;
    case CASL_QR: return h->qr;
  }
  return nullptr;
}

int casl_set_field(casl_handle *h, int which, const double *host) {
  if (!h || !host) return CASL_EINVAL;
  double *d = field_ptr(h, which);
  if (!d) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  CASL_CUDA_TRY(cudaMemcpyAsync(d, host, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CASL_OK;
}

__global__ void k_widen(const float *__restrict__ a, double *__restrict__ b, long long nn) {
  CASL_PDL_ENTRY();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x)
    b[t] = (double)a[t];
}

int casl_get_field(casl_handle *h, int which, double *host) {
  if (!h || !host) return CASL_EINVAL;
  double *d = field_ptr(h, which);
  if (!d) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  if (h->uv_fp32 && (which == CASL_UU || which == CASL_VV)) {
    // the last stage's FP32 velocity, widened (FP32-inversion mode)
    d = h->w[5];
    CASL_K(k_widen, grid_for((long long)nn), 256, 0, h->stream)(
        h->f32 + (which == CASL_UU ? 0 : nn), d, (long long)nn);
  }
  CASL_CUDA_TRY(cudaMemcpyAsync(host, d, nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CASL_OK;
}

int casl_get_scalar(casl_handle *h, int which, double *value) {
  if (!h || !value) return CASL_EINVAL;
  int rc = get_scalars(h);
  if (rc) return rc;
  Scalars &s = *h->hscal;
  switch (which) {
    case CASL_T: *value = s.t; break;
    case CASL_DT: *value = s.dt; break;
    case CASL_TWIST: *value = s.twist; break;
    case CASL_IREG: *value = h->ireg; break;
    case CASL_ZZRMS: *value = s.zzrms; break;
    case CASL_ZZMAX: *value = s.zzmax; break;
    case CASL_UUMAX: *value = s.uumax; break;
    case CASL_QJUMP: *value = s.qjump; break;
    case CASL_NODESTEPS: *value = h->node_steps; break;
    default: return CASL_EINVAL;
  }
  return CASL_OK;
}

int casl_set_scalar(casl_handle *h, int which, double value) {
  if (!h) return CASL_EINVAL;
  int rc = get_scalars(h);
  if (rc) return rc;
  Scalars &s = *h->hscal;
  switch (which) {
    case CASL_T: s.t = value; break;
    case CASL_DT:
      s.dt = value; s.dt2 = value * 0.5; s.dt3 = value * (1.0 / 3.0); s.dt6 = value * (1.0 / 6.0);
      break;
    case CASL_TWIST: s.twist = value; break;
    case CASL_IREG: h->ireg = (int)value; break;
    case CASL_QJUMP: s.qjump = value; h->qjump = value; break;
    case CASL_NODESTEPS: h->node_steps = value; return CASL_OK;
    default: return CASL_EINVAL;
  }
  return put_scalars(h);
}

int casl_ptospc(casl_handle *h, const double *rvar, double *svar) {
  if (!h || !rvar || !svar) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->w[4], rvar, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  int rc = ptospc_dev(h, h->w[4], h->w[5]);
  if (rc) return rc;
  CASL_CUDA_TRY(cudaMemcpyAsync(svar, h->w[5], nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return check_launch(h);
}

int casl_spctop(casl_handle *h, const double *svar, double *rvar) {
  if (!h || !rvar || !svar) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->w[4], svar, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  int rc = spctop_dev(h, h->w[4], h->w[5], h->w[0]);
  if (rc) return rc;
  CASL_CUDA_TRY(cudaMemcpyAsync(rvar, h->w[5], nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return check_launch(h);
}

int casl_con2grid(casl_handle *h, double *qc, int *levels) {
  if (h && h->M > 1) return CASL_EUNSUPPORTED;
  if (!h) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  int rc = con2grid_to_phys(h, h->w[5], levels != nullptr);
  if (rc) return rc;
  if (qc) CASL_CUDA_TRY(cudaMemcpyAsync(qc, h->w[5], nn * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (levels) {
    size_t fine = (size_t)h->c.nxf * h->c.nyf;
    if (h->nptq == 0)
      memset(levels, 0, fine * sizeof(int));
    else
      CASL_CUDA_TRY(cudaMemcpyAsync(levels, h->fineJ, fine * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  }
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  rc = get_scalars(h);
  if (rc) return rc;
  if (h->hscal->error) {
    int e = h->hscal->error;
    h->hscal->error = 0;
    put_scalars(h);
    return e;
  }
  return CASL_OK;
}

int casl_velint(casl_handle *h, const double *uu, const double *vv, double *uq, double *vq) {
  if (!h || !uu || !vv || !uq || !vq) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  cudaStream_t s = h->stream;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->w[4], uu, nn * sizeof(double), cudaMemcpyHostToDevice, s));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->w[5], vv, nn * sizeof(double), cudaMemcpyHostToDevice, s));
  int npt = h->nptq;
  if (npt > 0) {
    CASL_K(k_velint, grid_for(npt), 256, 0, s)(h->xq, h->yq, npt, h->w[4], h->w[5], h->uq, h->vq, h->c);
    CASL_CUDA_TRY(cudaMemcpyAsync(uq, h->uq, npt * sizeof(double), cudaMemcpyDeviceToHost, s));
    CASL_CUDA_TRY(cudaMemcpyAsync(vq, h->vq, npt * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CASL_CUDA_TRY(cudaStreamSynchronize(s));
  return check_launch(h);
}

int casl_main_invert(casl_handle *h, const double *qq, double *uu, double *vv, double *pp) {
  if (!h || !qq) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  cudaStream_t s = h->stream;
  // Runs on scratch copies so that the simulation state is untouched.
  double *q = h->w[4], *p = h->w[5];
  CASL_CUDA_TRY(cudaMemcpyAsync(q, qq, nn * sizeof(double), cudaMemcpyHostToDevice, s));
  long long n = h->n;
  LoadDeriv ld{};
  ld.f[0] = q; ld.f[1] = q; ld.dir[0] = 0; ld.dir[1] = 1;
  ld.wg[0] = 1; ld.wg[1] = 1;
  ld.green = h->green; ld.hrkx = h->hrkx; ld.hrky = h->hrky; ld.n = h->n;
  ld.err = &h->scal->error;
  int rc = RFFT_DISPATCH(false, false, false, ld, (StoreStrided{h->w[0], (long long)nn, n, 1}), 2);
  if (rc) return rc;
  StoreScaled st{};
  st.p[0] = h->w[2]; st.p[1] = h->w[3]; st.scale[0] = 1.0; st.scale[1] = -1.0; st.n = h->n;
  LoadBatch lb{};
  lb.p[0] = h->w[0]; lb.p[1] = h->w[1]; lb.vs = 1; lb.es = n;
  rc = RFFT_DISPATCH(false, true, false, lb, st, 2);
  if (rc) return rc;
  if (uu) CASL_CUDA_TRY(cudaMemcpyAsync(uu, h->w[3], nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (vv) CASL_CUDA_TRY(cudaMemcpyAsync(vv, h->w[2], nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (pp) {
    // pp = green*qq (spectral.f90:321)
    CASL_K(k_mul2, grid_for((long long)nn), 256, 0, s)(h->green, q, p, (long long)nn);
    CASL_CUDA_TRY(cudaMemcpyAsync(pp, p, nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CASL_CUDA_TRY(cudaStreamSynchronize(s));
  return check_launch(h);
}

int casl_gradient(casl_handle *h, const double *ff, double *ffx, double *ffy) {
  if (!h || !ff) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  cudaStream_t s = h->stream;
  double *f = h->w[4];
  CASL_CUDA_TRY(cudaMemcpyAsync(f, ff, nn * sizeof(double), cudaMemcpyHostToDevice, s));
  long long n = h->n;
  LoadDeriv ld{};
  ld.f[0] = f; ld.f[1] = f; ld.dir[0] = 0; ld.dir[1] = 1;
  ld.green = nullptr; ld.hrkx = h->hrkx; ld.hrky = h->hrky; ld.n = h->n;
  ld.err = &h->scal->error;
  int rc = RFFT_DISPATCH(false, false, false, ld, (StoreStrided{h->w[0], (long long)nn, n, 1}), 2);
  if (rc) return rc;
  StoreScaled st{};
  st.p[0] = h->w[2]; st.p[1] = h->w[3]; st.scale[0] = 1.0; st.scale[1] = 1.0; st.n = h->n;
  LoadBatch lb{};
  lb.p[0] = h->w[0]; lb.p[1] = h->w[1]; lb.vs = 1; lb.es = n;
  rc = RFFT_DISPATCH(false, true, false, lb, st, 2);
  if (rc) return rc;
  if (ffx) CASL_CUDA_TRY(cudaMemcpyAsync(ffx, h->w[2], nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (ffy) CASL_CUDA_TRY(cudaMemcpyAsync(ffy, h->w[3], nn * sizeof(double), cudaMemcpyDeviceToHost, s));
  CASL_CUDA_TRY(cudaStreamSynchronize(s));
  return check_launch(h);
}

int casl_inversion(casl_handle *h) {
  if (!h) return CASL_EINVAL;
  int rc = inversion_dev(h, false);
  if (rc) return rc;
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return sync_counts(h);
}

int casl_advance(casl_handle *h) {
  if (!h) return CASL_EINVAL;
  int rc = advance_dev(h);
  if (rc) return rc;
  return sync_counts(h);
}

int casl_surgery(casl_handle *h) {
  if (h && h->M > 1) {  // an ensemble: surgery on every member, then the member ranges
    int rc = sync_counts(h);
    if (rc) return rc;
    if ((rc = surgery_dev(h))) return rc;
    if ((rc = member_ranges(h))) return rc;
    return sync_counts(h);
  }
  if (!h) return CASL_EINVAL;
  int rc = surgery_dev(h);
  if (rc) return rc;
  return sync_counts(h);
}

int casl_renode(casl_handle *h, const double *xd, const double *yd, int npd, double *xr,
                double *yr, int cap, int *npr) {
  if (!h || !xd || !yd || !xr || !yr || !npr || npd < 1 || cap < 0) return CASL_EINVAL;
  return renode_host(h, xd, yd, npd, xr, yr, cap, npr);
}

int casl_recontour(casl_handle *h, const double *qq) {
  if (h && h->M > 1) return CASL_EUNSUPPORTED;  // ensembles recontour inside casl_step
  if (!h || !qq) return CASL_EINVAL;
  size_t nn = (size_t)h->n * h->n;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->qr, qq, nn * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  int rc = recontour_dev(h, h->qr);
  if (rc) return rc;
  return sync_counts(h);
}

// init (evolution.f90:96-131)
// (tot = M*nn over an ensemble's members; the tables are shared)
__global__ void k_evo_init(double *qd, double *qspre, const double *qs, const double *qc,
                           const double *fhi, long long nn, long long tot) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot;
       k += (long long)gridDim.x * blockDim.x) {
    qd[k] = fhi[k & (nn - 1)] * (qs[k] - qc[k]);
    qspre[k] = qs[k];
  }
}
// prepare (evolution.f90:135-162), spectral part
__global__ void k_prepare(double *qs, double *qd, const double *qc, const double *flo,
                          long long nn, long long tot) {
  CASL_PDL_ENTRY();
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < tot;
       k += (long long)gridDim.x * blockDim.x) {
    double s = flo[k & (nn - 1)] * (qs[k] - qc[k]) + qc[k] + qd[k];
    qs[k] = s;
    qd[k] = s - qc[k];
  }
}

}  // extern "C"

namespace casl {
int evo_init(casl_handle *h) {
  long long nn = (long long)h->n * h->n;
  h->contex = h->nptq > 0;
  int rc = con2grid_to_spec(h, h->qc);
  if (rc) return rc;
  CASL_K(k_evo_init, grid_for(h->M * nn), 256, 0, h->stream)(h->qd, h->qspre, h->qs, h->qc,
                                                             h->fhi, nn, h->M * nn);
  // init also clears the save flags (evolution.f90:113-116)
  saves_clear_flags(h);
  return check_launch(h);
}
}  // namespace casl

extern "C" {

static int evo_prepare(casl_handle *h) {
  long long nn = (long long)h->n * h->n;
  int rc = con2grid_to_spec(h, h->qc);
  if (rc) return rc;
  CASL_K(k_prepare, grid_for(h->M * nn), 256, 0, h->stream)(h->qs, h->qd, h->qc, h->flo, nn,
                                                            h->M * nn);
  if ((rc = check_launch(h))) return rc;
  return spctop_dev(h, h->qd, h->qr, h->w[0], h->M);
}

__global__ void k_sub_bety(double *q, const double *bety, int n) {
  CASL_PDL_ENTRY();
  long long nn = (long long)n * n;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x)
    q[k] -= bety[k % n];
}

__global__ void k_minmax(const double *q, long long nn, double *part) {
  CASL_PDL_ENTRY();
  double mx = -1e308, mn = 1e308;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nn;
       k += (long long)gridDim.x * blockDim.x) {
    mx = fmax(mx, q[k]);
    mn = fmin(mn, q[k]);
  }
  __shared__ double a[256], b[256];
  a[threadIdx.x] = mx;
  b[threadIdx.x] = mn;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      a[threadIdx.x] = fmax(a[threadIdx.x], a[threadIdx.x + o]);
      b[threadIdx.x] = fmin(b[threadIdx.x], b[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = a[0];
    part[2 * blockIdx.x + 1] = b[0];
  }
}

int casl_initialise(casl_handle *h, const double *qq_init) {
  if (!h || !qq_init) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // casl_ensemble_initialise
  long long nn = (long long)h->n * h->n;
  cudaStream_t s = h->stream;
  int rc = get_scalars(h);
  if (rc) return rc;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->qr, qq_init, nn * sizeof(double), cudaMemcpyHostToDevice, s));
  double qjump;
  if (h->c.beffect) {
    CASL_K(k_sub_bety, grid_for(nn), 256, 0, s)(h->qr, h->bety, h->n);
    qjump = h->p.beta * h->p.elly / (double)h->p.ncontq;
  } else {
    // contint (generic.f90:216-229)
    CASL_K(k_minmax, RED_BLOCKS, 256, 0, s)(h->qr, nn, h->part);
    std::vector<double> part(2 * RED_BLOCKS);
    CASL_CUDA_TRY(cudaMemcpyAsync(part.data(), h->part, part.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
    CASL_CUDA_TRY(cudaStreamSynchronize(s));
    double mx = part[0], mn = part[1];
    for (int i = 1; i < RED_BLOCKS; i++) {
      mx = fmax(mx, part[2 * i]);
      mn = fmin(mn, part[2 * i + 1]);
    }
    qjump = (mx - mn) / (double)h->p.ncontq;
  }
  rc = ptospc_dev(h, h->qr, h->qs);
  if (rc) return rc;
  Scalars &sc = *h->hscal;
  sc.t = 0.0; sc.dt = 0.0; sc.twist = 0.0; sc.qjump = qjump; sc.nq = 0; sc.nptq = 0;
  sc.error = 0;
  sc.dtmax = h->p.dtmax > 0 ? h->p.dtmax : 1.0e30;
  h->qjump = qjump;
  h->nq = 0;
  h->nptq = 0;
  if ((rc = put_scalars(h))) return rc;
  if ((rc = recontour_dev(h, h->qr))) return rc;
  if ((rc = sync_counts(h))) return rc;
  if ((rc = evo_init(h))) return rc;
  h->ireg = 0;
  return sync_counts(h);
}

int casl_step(casl_handle *h, int nsteps) {
  if (!h || nsteps < 0) return CASL_EINVAL;
  int rc;
  for (int it = 0; it < nsteps; it++) {
    // exact counts for this step's regularisation (one small copy per step)
    if ((rc = sync_counts(h))) return rc;
    bool force = h->p.force_surgery != 0;
    bool reg = force;
    if (!force) {
      if ((rc = get_scalars(h))) return rc;
      reg = h->hscal->twist > h->p.twistmax;
    }
    if (reg) {
      h->ireg++;
      if (h->ireg == h->p.nregmax) {
        // prepare + recontour + init (evolution.f90:62-66; caps.f90:83-91);
        // an ensemble recontours member by member
        if ((rc = evo_prepare(h))) return rc;
        if ((rc = h->M > 1 ? ensemble_recontour(h) : recontour_dev(h, h->qr))) return rc;
        if ((rc = debug_check(h, "recontour"))) return rc;
        if ((rc = sync_counts(h))) return rc;
        if ((rc = evo_init(h))) return rc;
        CASL_K(k_twist_zero, 1, 256, 0, h->stream)(h->scal, h->M);
        h->ireg = 0;
        if (force) {
          h->ireg = 1;
          if ((rc = surgery_dev(h))) return rc;
          if ((rc = debug_check(h, "surgery after recontouring"))) return rc;
          if (h->M > 1 && (rc = member_ranges(h))) return rc;
          CASL_K(k_twist_sub, 1, 256, 0, h->stream)(h->scal, h->p.twistmax, h->M);
        }
      } else {
        if ((rc = surgery_dev(h))) return rc;
        if ((rc = debug_check(h, "surgery"))) return rc;
        if (h->M > 1 && (rc = member_ranges(h))) return rc;
        CASL_K(k_twist_sub, 1, 256, 0, h->stream)(h->scal, h->p.twistmax, h->M);
      }
    }
    if ((rc = saves_before_advance(h))) return rc;
    if (h->closure && (rc = closure_step_check(h))) return rc;
    h->node_steps += (double)h->nptq;
    if ((rc = advance_dev(h))) return rc;
    if ((rc = saves_after_advance(h))) return rc;
  }
  return sync_counts(h);
}

int casl_set_precision(casl_handle *h, int mode) {
  if (!h || (mode != CASL_PREC_FP64 && mode != CASL_PREC_FP32_INVERSION)) return CASL_EINVAL;
  if (h->M > 1 && mode != CASL_PREC_FP64) return CASL_EUNSUPPORTED;
  cudaSetDevice(h->device);
  if (mode == CASL_PREC_FP32_INVERSION && !h->f32) {
    const size_t bytes = (size_t)6 * h->n * h->n * sizeof(float);
    CASL_CUDA_TRY(cudaMalloc(&h->f32, bytes));
    CASL_CUDA_TRY(cudaMemset(h->f32, 0, bytes));
  }
  h->prec = mode;
  return CASL_OK;
}

int casl_get_precision(casl_handle *h, int *mode) {
  if (!h || !mode) return CASL_EINVAL;
  *mode = h->prec;
  return CASL_OK;
}

int casl_get_stream(casl_handle *h, void **stream) {
  if (!h || !stream) return CASL_EINVAL;
  *stream = (void *)h->stream;
  return CASL_OK;
}

int casl_launch_count(long long *count) {
  if (!count) return CASL_EINVAL;
  *count = (long long)casl::g_launches;
  return CASL_OK;
}

int casl_kernel_times(int mode, char *buf, long long cap) {
  using namespace casl;
  casl_handle *h = nullptr;  // process-wide: no handle records the error
  if (mode < 0 || mode > 2) return CASL_EINVAL;
  if (mode == 1 && !g_kt.ev) {
    g_kt.ev = (cudaEvent_t *)calloc(2 * KT_MAX, sizeof(cudaEvent_t));
    g_kt.name = (const char **)calloc(KT_MAX, sizeof(const char *));
    if (!g_kt.ev || !g_kt.name) return CASL_ENOMEM;
    for (int i = 0; i < 2 * KT_MAX; i++) CASL_CUDA_TRY(cudaEventCreate(&g_kt.ev[i]));
  }
  if (mode == 2) {
    // report: per kernel name, launches / total ms / mean us, by total
    if (!buf || cap <= 0) return CASL_EINVAL;
    CASL_CUDA_TRY(cudaDeviceSynchronize());
    std::vector<std::pair<std::string, std::pair<long long, double>>> rows;
    std::map<std::string, size_t> at;
    for (int i = 0; i < g_kt.n; i++) {
      float ms = 0.f;
      CASL_CUDA_TRY(cudaEventElapsedTime(&ms, g_kt.ev[2 * i], g_kt.ev[2 * i + 1]));
      auto it = at.find(g_kt.name[i]);
      if (it == at.end()) {
        it = at.emplace(g_kt.name[i], rows.size()).first;
        rows.push_back({g_kt.name[i], {0, 0.0}});
      }
      rows[it->second].second.first++;
      rows[it->second].second.second += ms;
    }
    std::sort(rows.begin(), rows.end(),
              [](const auto &a, const auto &b) { return a.second.second > b.second.second; });
    std::string out;
    char line[256];
    for (auto &r : rows) {
      snprintf(line, sizeof line, "%-40s %7lld %10.3f ms %9.2f us\n", r.first.c_str(),
               r.second.first, r.second.second, 1e3 * r.second.second / r.second.first);
      out += line;
    }
    snprintf(buf, (size_t)cap, "%s", out.c_str());
    g_kt.n = 0;
    return CASL_OK;
  }
  g_kt.on = mode == 1;
  g_kt.n = 0;
  return CASL_OK;
}

int casl_profile(casl_handle *h, int kernel_class) {
  if (!h || kernel_class < 0 || kernel_class > CASL_PROF_FFT) return CASL_EINVAL;
  if (!h->prof_ev && kernel_class) {
    h->prof_ev = (cudaEvent_t *)calloc(2 * CASL_PROF_MAX, sizeof(cudaEvent_t));
    if (!h->prof_ev) return CASL_ENOMEM;
    for (int i = 0; i < 2 * CASL_PROF_MAX; i++) CASL_CUDA_TRY(cudaEventCreate(&h->prof_ev[i]));
  }
  h->prof_class = kernel_class;
  h->prof_n = 0;
  h->prof_bytes = 0.0;
  return CASL_OK;
}

int casl_profile_read(casl_handle *h, double *total_ms, long long *launches, double *bytes) {
  if (!h || !total_ms || !launches || !bytes) return CASL_EINVAL;
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  double tot = 0.0;
  for (int i = 0; i < h->prof_n; i++) {
    float ms = 0.f;
    CASL_CUDA_TRY(cudaEventElapsedTime(&ms, h->prof_ev[2 * i], h->prof_ev[2 * i + 1]));
    tot += ms;
  }
  *total_ms = tot;
  *launches = h->prof_n;
  *bytes = h->prof_bytes;
  h->prof_n = 0;
  h->prof_bytes = 0.0;
  return CASL_OK;
}

int casl_diagnostics(casl_handle *h, double out[4]) {
  if (!h || !out) return CASL_EINVAL;
  if (h->M > 1) return CASL_EUNSUPPORTED;  // one simulation's energies and circulation
  cudaStream_t st = h->stream;
  const long long nn = (long long)h->n * h->n;
  if (h->uv_fp32) {
    // FP32-inversion mode: the energies from the FP64 velocity of qq
    int rc = main_invert_dev(h);
    if (rc) return rc;
    h->uv_fp32 = 0;
  }
  // ekin = 1/2 garea sum(u^2+v^2) (evolution.f90:628-629)
  CASL_K(k_diag_sumsq2, RED_BLOCKS, 256, 0, st)(h->uu, h->vv, h->part, nn);
  CASL_K(k_diag_final, 1, 256, 0, st)(h->part, RED_BLOCKS, h->part + 2 * RED_BLOCKS);
  // epot = 1/2 garea kd^2 sum(psi^2) (evolution.f90:636-640)
  if (!h->c.btropic) {
    int rc = spctop_dev(h, h->pp, h->w[5], h->w[0]);
    if (rc) return rc;
    CASL_K(k_diag_sumsq2, RED_BLOCKS, 256, 0, st)(h->w[5], nullptr, h->part, nn);
    CASL_K(k_diag_final, 1, 256, 0, st)(h->part, RED_BLOCKS, h->part + 2 * RED_BLOCKS + 1);
  }
  // integral of (q - beta y)^2 (generic.f90:198-212 on spctop(qq))
  int rc = spctop_dev(h, h->qq, h->w[5], h->w[0]);
  if (rc) return rc;
  CASL_K(k_diag_sumsq2, RED_BLOCKS, 256, 0, st)(h->w[5], nullptr, h->part, nn);
  CASL_K(k_diag_final, 1, 256, 0, st)(h->part, RED_BLOCKS, h->part + 2 * RED_BLOCKS + 2);
  // contour circulation: qjump * sum of signed areas (shoelace on unwrapped
  // increments along each contour)
  double hs[3] = {0, 0, 0}, circ = 0.0;
  int npt = h->nptq;
  if (npt > 0) {
    size_t need = (size_t)npt * 48 + ((size_t)16 << 20);
    rc = ensure_scratch(h, need);
    if (rc) return rc;
    Arena ar{(char *)h->sx, h->sx_bytes, 0};
    double *dx = ar.get<double>(npt), *dy = ar.get<double>(npt);
    double *X = ar.get<double>(npt), *Y = ar.get<double>(npt);
    int *head = ar.get<int>(npt);
    SegPair *tmps = ar.get<SegPair>(scan_tmp_elems(npt) + 4);
    double *cpart = ar.get<double>(RED_BLOCKS + 4);
    if (ar.failed) return CASL_ENOMEM;
    CASL_K(k_diag_incr, grid_for(npt), 256, 0, st)(h->xq, h->yq, h->nextq, npt, dx, dy, head, h->c);
    CASL_K(k_diag_heads, grid_for(h->nq), 256, 0, st)(h->i1q, h->nq, head);
    segmented_scan(st, dx, head, X, npt, tmps);
    segmented_scan(st, dy, head, Y, npt, tmps);
    CASL_K(k_diag_shoelace, RED_BLOCKS, 256, 0, st)(dx, dy, X, Y, npt, cpart);
    CASL_K(k_diag_final, 1, 256, 0, st)(cpart, RED_BLOCKS, cpart + RED_BLOCKS);
    CASL_CUDA_TRY(cudaMemcpyAsync(&circ, cpart + RED_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, st));
  }
  CASL_CUDA_TRY(cudaMemcpyAsync(hs, h->part + 2 * RED_BLOCKS, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  rc = check_launch(h);
  if (rc) return rc;
  out[0] = 0.5 * h->c.garea * hs[0];
  out[1] = h->c.btropic ? 0.0 : 0.5 * h->c.garea * h->c.kdsq * hs[1];
  out[2] = h->c.garea * hs[2];
  out[3] = h->hscal->qjump * (0.5 * circ);
  if (npt > 0) {
    rc = get_scalars(h);
    if (rc) return rc;
    out[3] = h->hscal->qjump * (0.5 * circ);
  }
  return CASL_OK;
}

}  // extern "C"

namespace casl {
// Shell sums of the spectral field ss (device) into dspec[0..n] (device).
int spec1d_dev(casl_handle *h, const double *ss, double *dspec) {
  CASL_CUDA_TRY(cudaMemsetAsync(dspec, 0, (h->n + 1) * sizeof(double), h->stream));
  CASL_K(k_spec1d, (32 * (h->kmax + 1) + 255) / 256, 256, 0, h->stream)(
      ss, h->shell_off, h->shell_idx, h->n, h->kmax, dspec);
  return check_launch(h);
}
}  // namespace casl

extern "C" {
int casl_spec1d(casl_handle *h, double *ss, double *spec, int iopt) {
  if (!h || !ss || !spec || (iopt != 0 && iopt != 1)) return CASL_EINVAL;
  cudaStream_t st = h->stream;
  const long long nn = (long long)h->n * h->n;
  double *d = h->w[5], *dspec = h->w[4];
  CASL_CUDA_TRY(cudaMemcpyAsync(d, ss, nn * sizeof(double), cudaMemcpyHostToDevice, st));
  if (iopt == 1)
    CASL_K(k_mul_rksq, grid_for(nn), 256, 0, st)(d, h->rkxf, h->rkyf, h->n, nn);
  int rc = spec1d_dev(h, d, dspec);
  if (rc) return rc;
  CASL_CUDA_TRY(cudaMemcpyAsync(spec, dspec, (h->n + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
  if (iopt == 1)
    CASL_CUDA_TRY(cudaMemcpyAsync(ss, d, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  return check_launch(h);
}

int casl_spec_tables(casl_handle *h, int *kmax, int *kmaxred, double *spmf, double *alk) {
  if (!h || !kmax || !kmaxred) return CASL_EINVAL;
  *kmax = h->kmax;
  *kmaxred = h->kmaxred;
  if (spmf) memcpy(spmf, h->spmf_h, (h->n + 1) * sizeof(double));
  if (alk) memcpy(alk, h->alk_h, (h->n + 1) * sizeof(double));
  return CASL_OK;
}

}  // extern "C"
