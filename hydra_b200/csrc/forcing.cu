// Forcing of the residual PV qd: the stochastic point-vortex / dipole
// forcing pvforce (evolution.f90:330-428) and the narrow-band spectral
// forcing init_forcing / nb_forcing (spectral.f90:160-285), both added to qd
// at the end of a time step as advance does (evolution.f90:316-323).
//
// The reference draws its random numbers from GNU rand() inside these
// procedures; here the caller passes them in, in the reference's draw order,
// so a run is reproducible from any generator (the configurations of this
// path have both forcings off).
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>

#include <unordered_map>
#include <vector>

#include "state.cuh"

namespace casl {

struct ForcingState {
  std::vector<int> kxfxo, kyfyo, kxf, kyf;  // 1-based spectral indices of the band
  std::vector<double> rkx, rky;             // unfiltered wavenumbers (spectral.f90:57-78)
  double forfac;
  long long *d_idx;                         // dqdt entries: spectral index, value
  double *d_val;
  long long cap;
};

// pvforce's scatter: vortex k adds its circulation to the four corners of
// its grid box (inverse bilinear interpolation), into the physical field w.
__global__ void k_pv_scatter(const double *__restrict__ rnd, int nvor, int ivor, double vorvor,
                             double twopi, int nx, int ny, double *__restrict__ w) {
  CASL_PDL_ENTRY();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nvor; k += gridDim.x * blockDim.x) {
    const double dnx = (double)nx, dny = (double)ny;
    const int m = ivor == 1 ? 2 : 3;
    const double *r = rnd + (long long)m * k;
    double xx = dnx * r[m - 2], yy = dny * r[m - 1];
    int ix0 = 1 + f_int(xx);
    double pxc = (double)ix0 - xx, px = 1.0 - pxc;
    int iy0 = 1 + f_int(yy);
    double pyc = (double)iy0 - yy, py = 1.0 - pyc;
    ix0 = ix0 < 1 ? 1 : (ix0 > nx ? nx : ix0);
    iy0 = iy0 < 1 ? 1 : (iy0 > ny ? ny : iy0);
    const int ix1 = ix0 == nx ? 1 : ix0 + 1, iy1 = iy0 == ny ? 1 : iy0 + 1;
    double a00, a01, a10, a11;  // (iy0,ix0), (iy0,ix1), (iy1,ix0), (iy1,ix1)
    if (ivor == 1) {
      const double svor = (k & 1) ? -vorvor : vorvor;  // +, -, +, ... (svor flips first)
      a00 = svor * pyc * pxc;
      a01 = svor * pyc * px;
      a10 = svor * py * pxc;
      a11 = svor * py * px;
    } else {
      const double theta = twopi * r[0];
      const double cth = cos(theta), sth = sin(theta);
      a00 = -(vorvor * (pyc * cth + pxc * sth));
      a01 = vorvor * (pyc * cth - px * sth);
      a10 = vorvor * (pxc * sth - py * cth);
      a11 = vorvor * (px * sth + py * cth);
    }
    atomicAdd(&w[(long long)(ix0 - 1) * ny + (iy0 - 1)], a00);
    atomicAdd(&w[(long long)(ix1 - 1) * ny + (iy0 - 1)], a01);
    atomicAdd(&w[(long long)(ix0 - 1) * ny + (iy1 - 1)], a10);
    atomicAdd(&w[(long long)(ix1 - 1) * ny + (iy1 - 1)], a11);
  }
}

__global__ void k_add_into(double *__restrict__ qd, const double *__restrict__ a, long long nn) {
  CASL_PDL_ENTRY();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nn;
       t += (long long)gridDim.x * blockDim.x)
    qd[t] = qd[t] + a[t];
}

__global__ void k_add_sparse(double *__restrict__ qd, const long long *__restrict__ idx,
                             const double *__restrict__ val, int m) {
  CASL_PDL_ENTRY();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x)
    qd[idx[t]] = qd[idx[t]] + val[t];
}

void forcing_release(casl_handle *h) {
  ForcingState *f = h->forcing;
  if (!f) return;
  cudaFree(f->d_idx);
  cudaFree(f->d_val);
  delete f;
  h->forcing = nullptr;
}

static int gsz(long long w) {
  long long g = (w + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace casl

using namespace casl;

extern "C" {

int casl_pvforce(casl_handle *h, int ivor, double vorvor, int nvor, const double *rnd) {
  if (!h || nvor < 0 || (nvor > 0 && !rnd)) return CASL_EINVAL;
  if (nvor == 0) return CASL_OK;
  cudaSetDevice(h->device);
  const int m = ivor == 1 ? 2 : 3;
  for (long long i = 0; i < (long long)m * nvor; i++)
    if (!(rnd[i] >= 0.0 && rnd[i] < 1.0)) return CASL_EINVAL;
  const long long nn = (long long)h->n * h->n;
  cudaStream_t st = h->stream;
  // the uniforms go through the last work field's tail (w[5] is n^2 doubles;
  // larger draws are refused)
  if ((long long)m * nvor > nn) return CASL_EINVAL;
  double *w = h->w[4], *ws = h->w[5], *dr = h->w[3];
  CASL_CUDA_TRY(cudaMemcpyAsync(dr, rnd, (size_t)m * nvor * sizeof(double), cudaMemcpyHostToDevice,
                                st));
  const FillJob z[1] = {{w, 2 * nn, 0u}};
  if (int rc = fill_words(st, z, 1)) return rc;
  CASL_K(k_pv_scatter, gsz(nvor), 256, 0, st)(dr, nvor, ivor, vorvor, h->c.twopi, h->n, h->n, w);
  int rc = ptospc_dev(h, w, ws);
  if (rc) return rc;
  CASL_K(k_add_into, gsz(nn), 256, 0, st)(h->qd, ws, nn);
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  return check_launch(h);
}

int casl_nb_forcing_init(casl_handle *h, double kfmid, double fwid, double famp, int *nrand) {
  if (!h || !nrand || !(fwid > 0.0)) return CASL_EINVAL;
  const int nx = h->n, ny = h->n, nwx = nx / 2, nwy = ny / 2;
  // the reference stops on a band reaching wavenumber 0 or the Nyquist one
  if (fwid >= kfmid) return CASL_EINVAL;
  const int lim = (nwx - (int)kfmid) < (nwy - (int)kfmid) ? (nwx - (int)kfmid) : (nwy - (int)kfmid);
  if (fwid >= (double)lim) return CASL_EINVAL;
  cudaSetDevice(h->device);
  forcing_release(h);
  ForcingState *f = new ForcingState();
  // wavenumbers as init_spectral forms them (spectral.f90:57-78)
  f->rkx.assign(nx, 0.0);
  f->rky.assign(ny, 0.0);
  const double scx = h->c.pi / h->p.ellx, scy = h->c.pi / h->p.elly;
  for (int kx = 1; kx <= nwx - 1; kx++) f->rkx[kx] = f->rkx[nx - kx] = scx * (double)(2 * kx);
  f->rkx[nwx] = scx * (double)nx;
  for (int ky = 1; ky <= nwy - 1; ky++) f->rky[ky] = f->rky[ny - ky] = scy * (double)(2 * ky);
  f->rky[nwy] = scy * (double)ny;
  const double small = h->c.small;
  for (int kx = 1; kx <= nx; kx++)
    if (fabs(f->rkx[kx - 1] - kfmid) <= fwid + small) f->kxfxo.push_back(kx);
  for (int ky = 1; ky <= ny; ky++)
    if (fabs(f->rky[ky - 1] - kfmid) <= fwid + small) f->kyfyo.push_back(ky);
  for (int ky = 2; ky <= nwy; ky++)
    for (int kx = 2; kx <= nwx; kx++) {
      const double rk = sqrt(f->rkx[kx - 1] * f->rkx[kx - 1] + f->rky[ky - 1] * f->rky[ky - 1]);
      if (fabs(rk - kfmid) <= fwid + small) {
        f->kxf.push_back(kx);
        f->kyf.push_back(ky);
      }
    }
  f->forfac = (double)(nx * ny / 2) * famp / (h->c.twopi * fwid);
  f->cap = 2LL * f->kxfxo.size() + 2LL * f->kyfyo.size() + 4LL * f->kxf.size() + 1;
  if (cudaMalloc(&f->d_idx, f->cap * sizeof(long long)) != cudaSuccess ||
      cudaMalloc(&f->d_val, f->cap * sizeof(double)) != cudaSuccess) {
    cudaFree(f->d_idx);
    delete f;
    return CASL_ENOMEM;
  }
  h->forcing = f;
  *nrand = (int)(f->cap - 1);
  return CASL_OK;
}

int casl_nb_forcing(casl_handle *h, double dt, const double *rnd) {
  if (!h || !h->forcing || !rnd) return CASL_EINVAL;
  cudaSetDevice(h->device);
  ForcingState *f = h->forcing;
  const long long nx = h->n, ny = h->n, nx2 = nx + 2, ny2 = ny + 2;
  auto spc = [&](long long kx, long long ky) { return (ky - 1) * nx + (kx - 1); };
  // dqdt's band entries in the reference's order; a later write to the same
  // entry replaces the earlier one, as in the reference
  std::unordered_map<long long, double> dq;
  std::vector<long long> order;
  auto put = [&](long long k, double v) {
    if (dq.find(k) == dq.end()) order.push_back(k);
    dq[k] = v;
  };
  const double ffac = f->forfac * dt;
  long long r = 0;
  for (int kxfl : f->kxfxo) {
    const double f1 = rnd[r++], f2 = rnd[r++];
    const double fmag = sqrt(2.0 * ffac * f->rkx[kxfl - 1] / (f1 * f1 + f2 * f2));
    put(spc(kxfl, 1), fmag * f1);
    put(spc(nx2 - kxfl, 1), fmag * f2);
  }
  for (int kyfl : f->kyfyo) {
    const double f1 = rnd[r++], f2 = rnd[r++];
    const double fmag = sqrt(2.0 * ffac * f->rky[kyfl - 1] / (f1 * f1 + f2 * f2));
    put(spc(1, kyfl), fmag * f1);
    put(spc(1, ny2 - kyfl), fmag * f2);
  }
  for (size_t k = 0; k < f->kxf.size(); k++) {
    const int kxfl = f->kxf[k], kyfl = f->kyf[k];
    const double rk = sqrt(f->rkx[kxfl - 1] * f->rkx[kxfl - 1] + f->rky[kyfl - 1] * f->rky[kyfl - 1]);
    double f1 = rnd[r++], f2 = rnd[r++];
    double fmag = sqrt(ffac * rk / (f1 * f1 + f2 * f2));
    put(spc(kxfl, kyfl), fmag * f1);
    put(spc(nx2 - kxfl, kyfl), fmag * f2);
    f1 = rnd[r++];
    f2 = rnd[r++];
    fmag = sqrt(ffac * rk / (f1 * f1 + f2 * f2));
    put(spc(kxfl, ny2 - kyfl), fmag * f2);
    put(spc(nx2 - kxfl, ny2 - kyfl), -fmag * f1);
  }
  const int m = (int)order.size();
  if (m == 0) return CASL_OK;
  std::vector<double> val(m);
  for (int i = 0; i < m; i++) val[i] = dq[order[i]];
  cudaStream_t st = h->stream;
  CASL_CUDA_TRY(cudaMemcpyAsync(f->d_idx, order.data(), m * sizeof(long long),
                                cudaMemcpyHostToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(f->d_val, val.data(), m * sizeof(double), cudaMemcpyHostToDevice,
                                st));
  CASL_K(k_add_sparse, gsz(m), 256, 0, st)(h->qd, f->d_idx, f->d_val, m);
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  return check_launch(h);
}

}  // extern "C"
