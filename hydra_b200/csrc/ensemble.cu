// Batched ensembles: M independent simulations of one grid size in one
// handle (casl_ensemble_*), stepped together.
//
// Layout.  Member m's fields are the m-th n*n block of every field; its
// contours follow member m-1's in the node and contour arrays, and its
// levels are stored offset by m*CASL_LSTRIDE, so that the contours stay
// sorted by level across the whole ensemble.  Surgery and renode, which work
// level by level and contour by contour, then run on all members in one
// pass each; con2grid, the transforms, adapt and the RK4 updates take the
// member from the node (mnode ranges) or the batch index.  Recontouring is
// done member by member through a one-member view handle, whose output is
// appended to the new ensemble arrays.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "state.cuh"

namespace casl {

int recontour_dev(casl_handle *h, const double *qq_dev);

// Each member's first contour and node from the level offsets (contours are
// sorted by level, so by member); members without contours get the next
// member's start.  One block; counts from the device scalars.
__global__ void k_member_ranges(const int *__restrict__ indq, const int *__restrict__ i1q,
                                const Scalars *__restrict__ s, int M, int *__restrict__ mnode,
                                int *__restrict__ mcont) {
  CASL_PDL_ENTRY();
  const int nq = s->nq, npt = s->nptq;
  for (int m = threadIdx.x; m < M; m += blockDim.x) mcont[m] = -1;
  __syncthreads();
  auto member = [&](int j) {
    int m = (indq[j] + CASL_LBIAS) / CASL_LSTRIDE;
    return m < 0 ? 0 : (m >= M ? M - 1 : m);
  };
  for (int j = threadIdx.x; j < nq; j += blockDim.x) {
    const int m = member(j);
    if (j == 0 || member(j - 1) != m) {
      mcont[m] = j;
      mnode[m] = i1q[j];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int nc = nq, nn = npt;
    for (int m = M - 1; m >= 0; m--) {
      if (mcont[m] < 0) {
        mcont[m] = nc;
        mnode[m] = nn;
      } else {
        nc = mcont[m];
        nn = mnode[m];
      }
    }
    mcont[M] = nq;
    mnode[M] = npt;
  }
}

// Member m's contours into the view's arrays, renumbered from 0 and with
// the member's level offset removed.
__global__ void k_slice_member(const double *__restrict__ xq, const double *__restrict__ yq,
                               const int *__restrict__ nextq, const int *__restrict__ i1q,
                               const int *__restrict__ i2q, const int *__restrict__ npq,
                               const int *__restrict__ indq, int a, int npt, int ca, int nq,
                               int loff, double *__restrict__ vx, double *__restrict__ vy,
                               int *__restrict__ vnext, int *__restrict__ vi1,
                               int *__restrict__ vi2, int *__restrict__ vnp,
                               int *__restrict__ vind) {
  CASL_PDL_ENTRY();
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += stride) {
    vx[i] = xq[a + i];
    vy[i] = yq[a + i];
    vnext[i] = nextq[a + i] - a;
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += stride) {
    vi1[j] = i1q[ca + j] - a;
    vi2[j] = i2q[ca + j] - a;
    vnp[j] = npq[ca + j];
    vind[j] = indq[ca + j] - loff;
  }
}

// A view's contours appended at node offset No and contour offset Co.
__global__ void k_append_member(const double *__restrict__ vx, const double *__restrict__ vy,
                                const int *__restrict__ vnext, const int *__restrict__ vi1,
                                const int *__restrict__ vi2, const int *__restrict__ vnp,
                                const int *__restrict__ vind, int npt, int nq, int No, int Co,
                                int loff, double *__restrict__ xq, double *__restrict__ yq,
                                int *__restrict__ nextq, int *__restrict__ i1q,
                                int *__restrict__ i2q, int *__restrict__ npq,
                                int *__restrict__ indq) {
  CASL_PDL_ENTRY();
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npt; i += stride) {
    xq[No + i] = vx[i];
    yq[No + i] = vy[i];
    nextq[No + i] = vnext[i] + No;
  }
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nq; j += stride) {
    i1q[Co + j] = vi1[j] + No;
    i2q[Co + j] = vi2[j] + No;
    npq[Co + j] = vnp[j];
    indq[Co + j] = vind[j] + loff;
  }
}

__global__ void k_set_total_counts(Scalars *s, int nq, int npt) {
  CASL_PDL_ENTRY();
  s->nq = nq;
  s->nptq = npt;
}

static int gsz(long long w) {
  long long g = (w + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

int member_ranges(casl_handle *h) {
  CASL_K(k_member_ranges, 1, 1024, 0, h->stream)(h->indq, h->i1q, h->scal, h->M, h->mnode,
                                                  h->mcont);
  return check_launch(h);
}

static int member_ranges_host(casl_handle *h) {
  int rc = member_ranges(h);
  if (rc) return rc;
  CASL_CUDA_TRY(cudaMemcpyAsync(h->hmnode, h->mnode, (h->M + 1) * sizeof(int),
                                cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->hmcont, h->mcont, (h->M + 1) * sizeof(int),
                                cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return CASL_OK;
}

// The one-member view: the ensemble's constants and stream, node arrays and
// scratch of its own, sized for the largest member seen so far.
static void view_free(casl_handle *v) {
  if (!v) return;
  void *ps[] = {v->xq, v->yq, v->nextq, v->i1q, v->i2q, v->npq, v->indq, v->scal, v->sx, v->sx2, v->sxe};
  for (void *p : ps) cudaFree(p);
  if (v->hscal) cudaFreeHost(v->hscal);
  free(v);
}

static int view_get(casl_handle *h, long long npm, long long nm, casl_handle **out) {
  casl_handle *v = h->view;
  if (v && v->npm >= npm && v->nm >= nm) {
    *out = v;
    return CASL_OK;
  }
  if (v) {
    // keep the grown scratch arenas; replace the node arrays
    void *ps[] = {v->xq, v->yq, v->nextq, v->i1q, v->i2q, v->npq, v->indq};
    for (void *p : ps) cudaFree(p);
  } else {
    v = (casl_handle *)calloc(1, sizeof(casl_handle));
    if (!v) return CASL_ENOMEM;
    v->p = h->p;
    v->c = h->c;
    v->n = h->n;
    v->M = 1;
    v->device = h->device;
    v->stream = h->stream;
    if (cudaMalloc(&v->scal, sizeof(Scalars)) != cudaSuccess ||
        cudaMallocHost(&v->hscal, sizeof(Scalars)) != cudaSuccess) {
      view_free(v);
      return CASL_ENOMEM;
    }
    memset(v->hscal, 0, sizeof(Scalars));
    h->view = v;
  }
  v->npm = npm;
  v->nm = nm;
  v->p.npm = npm;
  v->p.nm = nm;
  bool ok = cudaMalloc(&v->xq, npm * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&v->yq, npm * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&v->nextq, npm * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&v->i1q, nm * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&v->i2q, nm * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&v->npq, nm * sizeof(int)) == cudaSuccess &&
            cudaMalloc(&v->indq, nm * sizeof(int)) == cudaSuccess;
  if (!ok) return CASL_ENOMEM;
  *out = v;
  return CASL_OK;
}

void ensemble_release(casl_handle *h) {
  view_free(h->view);
  h->view = nullptr;
}

// recontour (congen.f90:24-128) of every member from its residual qr
// (prepare has run on all members): member by member through the view,
// appended to the ensemble's new arrays.  The RK4 temporaries hold the new
// arrays meanwhile (xqi, yqi the nodes, uq the links, vq the contour data).
int ensemble_recontour(casl_handle *h) {
  const int M = h->M;
  const long long nn = (long long)h->n * h->n;
  int rc = sync_counts(h);
  if (rc) return rc;
  if ((rc = member_ranges_host(h))) return rc;
  int maxn = 0, maxc = 0;
  for (int m = 0; m < M; m++) {
    maxn = h->hmnode[m + 1] - h->hmnode[m] > maxn ? h->hmnode[m + 1] - h->hmnode[m] : maxn;
    maxc = h->hmcont[m + 1] - h->hmcont[m] > maxc ? h->hmcont[m + 1] - h->hmcont[m] : maxc;
  }
  // a member's recontoured nodes: capacity 4x its largest node count (at
  // least 64k), never more than the ensemble's
  long long vn = 4LL * maxn + 65536, vc = 4LL * maxc + 4096;
  if (vn > h->npm) vn = h->npm;
  if (vc > h->nm) vc = h->nm;
  casl_handle *v;
  if ((rc = view_get(h, vn, vc, &v))) return rc;
  double *nx = h->xqi, *ny = h->yqi;
  int *nnext = reinterpret_cast<int *>(h->uq);
  int *ci = reinterpret_cast<int *>(h->vq);  // i1q, i2q, npq, indq: 4 * nm ints
  int *ni1 = ci, *ni2 = ci + h->nm, *nnp = ci + 2 * h->nm, *nind = ci + 3 * h->nm;
  if (4 * h->nm > 2 * h->npm) return CASL_ECAPACITY;
  cudaStream_t st = h->stream;
  long long No = 0, Co = 0;
  for (int m = 0; m < M; m++) {
    const int a = h->hmnode[m], npt = h->hmnode[m + 1] - a;
    const int ca = h->hmcont[m], nq = h->hmcont[m + 1] - ca;
    const int loff = m * CASL_LSTRIDE;
    // a member whose new contours do not fit the view is recontoured again
    // with a view four times larger (up to the ensemble's capacities)
    for (;;) {
      if (npt > 0 || nq > 0)
        CASL_K(k_slice_member, gsz(npt > nq ? npt : nq), 256, 0, st)(
            h->xq, h->yq, h->nextq, h->i1q, h->i2q, h->npq, h->indq, a, npt, ca, nq, loff, v->xq,
            v->yq, v->nextq, v->i1q, v->i2q, v->npq, v->indq);
      Scalars &vs = *v->hscal;
      memset(&vs, 0, sizeof(Scalars));
      vs.nq = nq;
      vs.nptq = npt;
      vs.qjump = h->mqjump[m];
      v->nq = nq;
      v->nptq = npt;
      v->qjump = h->mqjump[m];
      v->contex = npt > 0;
      if ((rc = put_scalars(v))) return rc;
      rc = recontour_dev(v, h->qr + m * nn);
      if (rc == CASL_OK) rc = sync_counts(v);
      if (rc != CASL_ECAPACITY || (v->npm >= h->npm && v->nm >= h->nm)) break;
      long long gn = 4 * v->npm < h->npm ? 4 * v->npm : h->npm;
      long long gc = 4 * v->nm < h->nm ? 4 * v->nm : h->nm;
      if ((rc = view_get(h, gn, gc, &v))) return rc;
    }
    if (rc) return rc;
    const int onpt = v->nptq, onq = v->nq;
    if (No + onpt > h->npm || Co + onq > h->nm) return CASL_ECAPACITY;
    if (onpt > 0 || onq > 0)
      CASL_K(k_append_member, gsz(onpt > onq ? onpt : onq), 256, 0, st)(
          v->xq, v->yq, v->nextq, v->i1q, v->i2q, v->npq, v->indq, onpt, onq, (int)No, (int)Co,
          loff, nx, ny, nnext, ni1, ni2, nnp, nind);
    No += onpt;
    Co += onq;
  }
  // the new arrays in place of the old ones
  CASL_CUDA_TRY(cudaMemcpyAsync(h->xq, nx, No * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->yq, ny, No * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->nextq, nnext, No * sizeof(int), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->i1q, ni1, Co * sizeof(int), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->i2q, ni2, Co * sizeof(int), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->npq, nnp, Co * sizeof(int), cudaMemcpyDeviceToDevice, st));
  CASL_CUDA_TRY(cudaMemcpyAsync(h->indq, nind, Co * sizeof(int), cudaMemcpyDeviceToDevice, st));
  CASL_K(k_set_total_counts, 1, 1, 0, st)(h->scal, (int)Co, (int)No);
  if ((rc = sync_counts(h))) return rc;
  return member_ranges(h);
}

}  // namespace casl

using namespace casl;


extern "C" {

int casl_ensemble_create(const casl_params *p, int members, int device, casl_handle **out) {
  if (!p || !out || members < 1 || members > 4096) return CASL_EINVAL;
  // the step regularises every member every step, so that all members
  // recontour at the same step
  casl_params q = *p;
  q.force_surgery = 1;
  return create_handle_members(&q, device, members, out);
}

int casl_ensemble_members(casl_handle *h, int *members) {
  if (!h || !members) return CASL_EINVAL;
  *members = h->M;
  return CASL_OK;
}

// initialise (caps.f90:106-361, loopinit = 0) of every member: q_all holds
// the M initial fields one after the other, ncontq (nullable) each member's
// number of PV jumps.
int casl_ensemble_initialise(casl_handle *h, const double *q_all, const int *ncontq) {
  if (!h || !q_all) return CASL_EINVAL;
  cudaSetDevice(h->device);
  const int M = h->M, n = h->n;
  const long long nn = (long long)n * n;
  cudaStream_t st = h->stream;
  if (h->c.beffect) {
    // PV anomaly q - beta*y of every member and qjump = beta*Ly/ncontq
    // (caps.f90:149-163), with the same bety values one simulation subtracts
    std::vector<double> bety(n), qa((size_t)(M * nn));
    CASL_CUDA_TRY(cudaMemcpy(bety.data(), h->bety, n * sizeof(double), cudaMemcpyDeviceToHost));
    for (long long k = 0; k < M * nn; k++) qa[k] = q_all[k] - bety[k % n];
    CASL_CUDA_TRY(cudaMemcpyAsync(h->qr, qa.data(), M * nn * sizeof(double), cudaMemcpyHostToDevice, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    for (int m = 0; m < M; m++) {
      const int nc = ncontq ? ncontq[m] : h->p.ncontq;
      if (nc <= 0) return CASL_EINVAL;
      h->mqjump[m] = h->p.beta * h->p.elly / (double)nc;
    }
  } else {
    CASL_CUDA_TRY(cudaMemcpyAsync(h->qr, q_all, M * nn * sizeof(double), cudaMemcpyHostToDevice, st));
    // qjump of each member from its range (contint, generic.f90:216-229)
    for (int m = 0; m < M; m++) {
      const double *q = q_all + m * nn;
      double mx = q[0], mn = q[0];
      for (long long k = 1; k < nn; k++) {
        mx = q[k] > mx ? q[k] : mx;
        mn = q[k] < mn ? q[k] : mn;
      }
      const int nc = ncontq ? ncontq[m] : h->p.ncontq;
      if (nc <= 0) return CASL_EINVAL;
      h->mqjump[m] = (mx - mn) / (double)nc;
    }
  }
  // qs = ptospc(q) for every member
  int rc = ptospc_dev(h, h->qr, h->qs, M);
  if (rc) return rc;
  for (int m = 0; m < M; m++) {
    Scalars &s = h->hscal[m];
    memset(&s, 0, sizeof(Scalars));
    s.qjump = h->mqjump[m];
    s.dtmax = h->p.dtmax > 0 ? h->p.dtmax : 1.0e30;
  }
  h->qjump = h->mqjump[0];
  CASL_CUDA_TRY(cudaMemcpyAsync(h->scal, h->hscal, M * sizeof(Scalars), cudaMemcpyHostToDevice, st));
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  h->nq = h->nptq = 0;
  // no contours yet: every member is recontoured from its field alone
  if ((rc = member_ranges(h))) return rc;
  if ((rc = ensemble_recontour(h))) return rc;
  if ((rc = evo_init(h))) return rc;
  h->ireg = 0;
  return sync_counts(h);
}

// Member m's counts, contours (1-based, its own numbering and levels, as
// casl_get_contours gives them for one simulation; any array may be NULL)
// and scalars.
int casl_ensemble_member_counts(casl_handle *h, int m, int *nq, int *nptq, double *qjump) {
  if (!h || m < 0 || m >= h->M) return CASL_EINVAL;
  int rc = sync_counts(h);
  if (rc) return rc;
  if ((rc = member_ranges_host(h))) return rc;
  if (nq) *nq = h->hmcont[m + 1] - h->hmcont[m];
  if (nptq) *nptq = h->hmnode[m + 1] - h->hmnode[m];
  if (qjump) *qjump = h->mqjump[m];
  return CASL_OK;
}

int casl_ensemble_member_contours(casl_handle *h, int m, double *xq, double *yq, int *nextq,
                                  int *indq, int *npq, int *i1q, int *i2q) {
  int nq, npt;
  int rc = casl_ensemble_member_counts(h, m, &nq, &npt, nullptr);
  if (rc) return rc;
  const int a = h->hmnode[m], ca = h->hmcont[m];
  cudaStream_t st = h->stream;
  std::vector<int> t;
  auto get_d = [&](double *dst, const double *src, int k) -> int {
    if (dst && k) CASL_CUDA_TRY(cudaMemcpyAsync(dst, src, k * sizeof(double), cudaMemcpyDeviceToHost, st));
    return CASL_OK;
  };
  auto get_i = [&](int *dst, const int *src, int k, int off) -> int {
    if (!dst || !k) return CASL_OK;
    CASL_CUDA_TRY(cudaMemcpyAsync(dst, src, k * sizeof(int), cudaMemcpyDeviceToHost, st));
    CASL_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < k; i++) dst[i] += off;
    return CASL_OK;
  };
  if ((rc = get_d(xq, h->xq + a, npt))) return rc;
  if ((rc = get_d(yq, h->yq + a, npt))) return rc;
  if ((rc = get_i(nextq, h->nextq + a, npt, 1 - a))) return rc;
  if ((rc = get_i(i1q, h->i1q + ca, nq, 1 - a))) return rc;
  if ((rc = get_i(i2q, h->i2q + ca, nq, 1 - a))) return rc;
  if ((rc = get_i(npq, h->npq + ca, nq, 0))) return rc;
  if ((rc = get_i(indq, h->indq + ca, nq, -m * CASL_LSTRIDE))) return rc;
  CASL_CUDA_TRY(cudaStreamSynchronize(st));
  return CASL_OK;
}

int casl_ensemble_member_scalar(casl_handle *h, int m, int which, double *value) {
  if (!h || !value || m < 0 || m >= h->M) return CASL_EINVAL;
  Scalars s;
  CASL_CUDA_TRY(cudaMemcpyAsync(&s, h->scal + m, sizeof(Scalars), cudaMemcpyDeviceToHost, h->stream));
  CASL_CUDA_TRY(cudaStreamSynchronize(h->stream));
  switch (which) {
    case CASL_T: *value = s.t; break;
    case CASL_DT: *value = s.dt; break;
    case CASL_TWIST: *value = s.twist; break;
    case CASL_ZZRMS: *value = s.zzrms; break;
    case CASL_ZZMAX: *value = s.zzmax; break;
    case CASL_UUMAX: *value = s.uumax; break;
    case CASL_QJUMP: *value = h->mqjump[m]; break;
    default: return CASL_EINVAL;
  }
  return CASL_OK;
}

}  // extern "C"
